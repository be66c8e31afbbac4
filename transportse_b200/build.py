"""Build libtsecuda.so in-tree with nvcc for sm_100a.

FP64 kernels that must reproduce the reference's arithmetic bit for bit are
compiled with ``--fmad=false`` (no FMA contraction); the FP32
defect-correction kernels keep FMA contraction.  The CUDA runtime is linked
statically, so the library depends on the driver only.

Output: ``transportse_b200/_build/libtsecuda.so`` (and ``ptxas.log`` with the
register / spill report of every kernel).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libtsecuda.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
          "-I", os.path.join(os.path.dirname(HERE), "include")]
# source -> extra flags
SOURCES = {
    "tse_pressure.cu": ["--fmad=false"],
    "tse_transport.cu": ["--fmad=false"],
    "tse_flow.cu": ["--fmad=false"],
    "tse_capi.cu": ["--fmad=false"],
    "tse_dc.cu": [],
    "tse_batch.cu": [],
    "tse_selftest.cu": [],
}


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_source_mtime():
    t = 0.0
    for f in os.listdir(CSRC):
        t = max(t, os.path.getmtime(os.path.join(CSRC, f)))
    hdr = os.path.join(os.path.dirname(HERE), "include")
    for f in os.listdir(hdr):
        t = max(t, os.path.getmtime(os.path.join(hdr, f)))
    return max(t, os.path.getmtime(__file__))


def build(force=False, verbose=False):
    os.makedirs(OUT, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_source_mtime():
        return LIB
    cc = nvcc()

    def compile_one(src):
        obj = os.path.join(OUT, src.replace(".cu", ".o"))
        cmd = [cc, "-c", os.path.join(CSRC, src), "-o", obj] + ARCH + COMMON + SOURCES[src]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, p.stdout, p.stderr))
        return obj, p.stderr

    with cf.ThreadPoolExecutor(max_workers=min(8, len(SOURCES))) as ex:
        results = list(ex.map(compile_one, sorted(SOURCES)))
    with open(os.path.join(OUT, "ptxas.log"), "w") as f:
        for obj, log in results:
            f.write("== %s\n%s\n" % (os.path.basename(obj), log))
    tmp = LIB + ".tmp"
    cmd = [cc, "-shared", "-o", tmp] + ARCH + [o for o, _ in results] + ["-Xcompiler", "-fPIC"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
