"""The C-ABI library builds for sm_100a, loads, and exports every entry point
include/tse_cuda.h declares; the ctypes structs match the C structs field by
field.  No compute calls (these run without a GPU)."""
import ctypes as ct
import os
import re
import subprocess

import pytest

from tests.conftest import ROOT
from transportse_b200 import _native as N
from transportse_b200 import build

HEADER = os.path.join(ROOT, "include", "tse_cuda.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tse_[a-zA-Z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    path = build.build()
    lib = ct.CDLL(path)
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
        assert s in N.SIGNATURES, "ctypes signature missing for " + s


def test_version_string_without_gpu():
    assert b"sm_100a" in N.lib().tse_version()


def test_workspace_sizes_without_gpu():
    g = N.TseGrid(60, 1, 30, 0, None, None, None, 9.81, 0.0, 1.0)
    for kind in (N.TSE_WS_PRESSURE, N.TSE_WS_TRANSPORT, N.TSE_WS_REDUCE):
        assert N.lib().tse_workspace_bytes(ct.byref(g), kind) > 0
    g.nx = 0
    assert N.lib().tse_workspace_bytes(ct.byref(g), N.TSE_WS_PRESSURE) == 0


STRUCTS = {
    "TseGrid": N.TseGrid, "TseSolveStatus": N.TseSolveStatus,
    "TsePressureArgs": N.TsePressureArgs, "TseSpeciesArgs": N.TseSpeciesArgs,
    "TseHeatArgs": N.TseHeatArgs, "TseDcOptions": N.TseDcOptions,
    "TseBatchPressure": N.TseBatchPressure, "TseBatchSpecies": N.TseBatchSpecies,
    "TseBatchHeat": N.TseBatchHeat,
}


def test_struct_layout_matches_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "%s"' % HEADER,
             "int main(void) {"]
    for sname, cls in STRUCTS.items():
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (sname, sname))
        for fname, _ in cls._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (sname, fname, sname, fname))
    lines.append("return 0; }")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", str(c), "-o", str(exe)])
    out = dict(l.rsplit(" ", 1) for l in subprocess.check_output([str(exe)]).decode().split("\n") if l)
    for sname, cls in STRUCTS.items():
        assert int(out[sname]) == ct.sizeof(cls), sname
        for fname, _ in cls._fields_:
            assert int(out["%s.%s" % (sname, fname)]) == getattr(cls, fname).offset, (sname, fname)


def test_ops_fail_loudly_without_library(monkeypatch):
    monkeypatch.setattr(N, "_lib", None)
    monkeypatch.setattr(N, "LIB_PATH", "/nonexistent/libtsecuda.so")
    with pytest.raises(RuntimeError):
        N.lib()


def test_batch_entry_points_validate_without_gpu():
    """Argument errors return TSE_ERR_ARG before any device call."""
    L = N.lib()
    assert L.tse_batch_workspace_bytes(4, 4096) >= 256
    opts = N.TseDcOptions(128, 8, 0)
    g = N.TseGrid(8, 8, 8, 0, None, None, None, 9.81, 0.0, 1.0)
    ws = ct.c_void_p(4096)   # never dereferenced: validation fails first
    for name, args_t in (("P", N.TsePressureArgs), ("C", N.TseSpeciesArgs), ("T", N.TseHeatArgs)):
        fn = getattr(L, "tse_compute_%s_dc_batch" % name)
        Item = N.BATCH_ITEM["compute_" + name]
        assert fn(None, 1, ct.byref(opts), ws, 1 << 20, None) == -1
        a = args_t()
        a.max_it = 10
        if name == "P":
            a.dt_P = float("nan")
        else:
            a.dt = float("nan")
        a.min_dt = 1.0
        items = (Item * 1)(Item(ct.pointer(g), ct.pointer(a), ws, ws, 1 << 20))
        assert fn(items, 0, ct.byref(opts), ws, 1 << 20, None) == -1
        # NaN dt would halve forever: refused
        assert fn(items, 1, ct.byref(opts), ws, 1 << 20, None) == -1


def test_selftest_validates_without_gpu():
    L = N.lib()
    assert L.tse_selftest_bounded_waits(None, 0.1, None, 0, None) == -1
    assert L.tse_selftest_bounded_waits(ct.c_void_p(16), 0.1, ct.c_void_p(4096), 100, None) == -1
    assert L.tse_selftest_bounded_waits(ct.c_void_p(16), 0.0, ct.c_void_p(4096), 512, None) == -1


def test_per_call_selectors_match_the_header_layout():
    """The sweep and loop selectors are fields of each call's structs (no
    process-wide switch): their offsets follow the header's layout."""
    assert N.TsePressureArgs.sweep.offset == 12 * 8 + 6 * 8 + 4
    assert ct.sizeof(N.TsePressureArgs) == 12 * 8 + 6 * 8 + 8
    for T, nptr in ((N.TseSpeciesArgs, 15), (N.TseHeatArgs, 16)):
        assert T.sweep.offset == nptr * 8 + 7 * 8 + 8
        assert ct.sizeof(T) == nptr * 8 + 7 * 8 + 16
    assert N.TseDcOptions.host_loop.offset == 32 and N.TseDcOptions.loop_ms.offset == 40
    assert N.TseDcOptions.chunk.offset == 48 and N.TseDcOptions.graph_runs.offset == 60
    assert N.TseDcOptions.active_cells.offset == 64
    assert ct.sizeof(N.TseDcOptions) == 72
    L = N.lib()
    for name in ("tse_set_exact_sweep", "tse_set_batch_loop"):
        assert not hasattr(L, name)


def test_batch_loop_stats_without_gpu():
    """The batched form's loop statistics read without a device call."""
    L = N.lib()
    g, h = ct.c_int64(-1), ct.c_int64(-1)
    assert L.tse_batch_loop_stats(ct.byref(g), ct.byref(h)) == 0
    assert g.value >= 0 and h.value >= 0
    assert L.tse_batch_loop_stats(None, ct.byref(h)) == -1
