"""Build recipe for the oracle's C restatement (test infrastructure only).

Compiles ``oracle/tse_oracle.c`` into ``oracle/_build/libtseoracle.so`` with
gcc, OpenMP and ``-ffp-contract=off`` (no FMA contraction, matching numba's
``fastmath=False`` code generation of the reference).

The reference itself is Python/numba, so there is no C source of it to
compile into ``oracle/_ref``; its outputs are pinned through the golden
fixtures under ``tests/golden/``.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "tse_oracle.c")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libtseoracle.so")


def build(force=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= os.path.getmtime(SRC)):
        return LIB
    cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
           "-fPIC", "-shared", "-std=c11", SRC, "-o", LIB + ".tmp", "-lm"]
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
