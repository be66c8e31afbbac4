"""The pressure solve that allocates nothing (tse_compute_P_noalloc).

Callers that cannot allocate device memory -- a host program that can only
hand over its field buffers because another allocator owns the GPU's memory,
or a time loop that must not stall on cudaMalloc -- use this entry point; its
scratch is a fixed array inside the library.  This test calls it through the
C-ABI and checks it against the workspace entry point tse_compute_P on the
same inputs, twice in a row (the second solve starts from the first one's
result, so stale scratch from the first call would show), within the 1e-9
relative tolerance of the FP64 path and with identical iteration counts and
time steps.  It also checks that a grid too large for the fixed scratch is
refused.  The file is named so that pytest collects it last.
"""
import ctypes as ct

import numpy
import pytest
import torch

from transportse_b200 import _native as N
from transportse_b200 import workloads

pytestmark = pytest.mark.gpu
TOL = 1e-9


def _inputs(shape, seed, dev):
    nx, ny, nz = shape
    rng = numpy.random.default_rng(seed)
    cfg = workloads.base_config("noalloc", nx, ny, nz, rng.uniform(0.5, 2, nx),
                                rng.uniform(0.5, 2, ny), rng.uniform(0.5, 2, nz))
    cfg.beta = 4.0
    K = 1e-12 * numpy.exp(rng.standard_normal(shape))
    f = {"c_f": 4.5e-10 * rng.uniform(0.5, 1.5, shape), "nue": rng.uniform(8e-4, 1.2e-3, shape),
         "rho_f": rng.uniform(995, 1150, shape), "phi": rng.uniform(0.05, 0.3, shape),
         "Kx": K, "Ky": 0.8 * K, "Kz": 0.2 * K, "c_r": 1e-10 * rng.uniform(0.5, 1.5, shape)}
    BP = (rng.uniform(size=shape) < 0.1).astype(float)
    BP[:, :, -1] = 1.0
    f["BP"] = BP
    f["WP"] = numpy.where(rng.uniform(size=shape) < 0.2, rng.uniform(-1e-4, 1e-4, shape), 0.0)
    P = workloads.hydrostatic(cfg) + rng.uniform(-300, 300, shape)
    t = {k: torch.as_tensor(v, dtype=torch.float64, device=dev) for k, v in f.items()}
    g = {k: torch.as_tensor(numpy.asarray(getattr(cfg, k), dtype=numpy.float64), device=dev)
         for k in ("dx", "dy", "dz")}
    b = numpy.radians(cfg.beta)
    import math
    grid = N.TseGrid(nx, ny, nz, 0, g["dx"].data_ptr(), g["dy"].data_ptr(), g["dz"].data_ptr(),
                     9.81, math.sin(b), math.cos(b))
    return grid, t, g, torch.as_tensor(P, device=dev)


def _args(t, P, Pn, dt):
    a = N.TsePressureArgs()
    a.P, a.Pn = P.data_ptr(), Pn.data_ptr()
    for k in ("c_f", "nue", "rho_f", "phi", "Kx", "Ky", "Kz", "c_r", "BP", "WP"):
        setattr(a, k, t[k].data_ptr())
    a.dt_P, a.SOR, a.inc_it, a.max_dt, a.min_dt, a.P_conv = dt, 1.6, 1.25, 1e5, 1e-8, 1e-11
    a.max_it = 20000
    return a


def _status(buf):
    return N.TseSolveStatus.from_buffer_copy(buf.cpu().numpy().tobytes())


def _rel(a, b):
    a, b = a.cpu().numpy(), b.cpu().numpy()
    return float(numpy.max(numpy.abs(a - b)) / max(numpy.max(numpy.abs(b)), 1e-300))


def test_noalloc_matches_workspace_solve_twice(cuda_device):
    lib = N.lib()
    dev = cuda_device
    grid, t, g, P0 = _inputs((21, 9, 13), 7, dev)   # odd nz: padded colour layout
    stream = ct.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    ws_bytes = lib.tse_workspace_bytes(ct.byref(grid), N.TSE_WS_PRESSURE)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    st_ref = torch.zeros(ct.sizeof(N.TseSolveStatus), dtype=torch.uint8, device=dev)
    st_new = torch.zeros_like(st_ref)
    P_ref, P_new = P0.clone(), P0.clone()
    dt_ref = dt_new = 3600.0
    for call in range(2):
        Pn_ref, Pn_new = torch.empty_like(P0), torch.empty_like(P0)
        rc = lib.tse_compute_P(ct.byref(grid), ct.byref(_args(t, P_ref, Pn_ref, dt_ref)),
                               ct.c_void_p(st_ref.data_ptr()), ct.c_void_p(ws.data_ptr()),
                               ws_bytes, stream)
        assert rc == 0
        rc = lib.tse_compute_P_noalloc(ct.byref(grid), ct.byref(_args(t, P_new, Pn_new, dt_new)),
                                       ct.c_void_p(st_new.data_ptr()), stream)
        assert rc == 0
        torch.cuda.synchronize(dev)
        s_ref, s_new = _status(st_ref), _status(st_new)
        assert s_new.error == 0 and s_ref.error == 0
        assert (s_new.converged, s_new.num_it, s_new.halvings) == \
               (s_ref.converged, s_ref.num_it, s_ref.halvings), call
        assert s_new.t == s_ref.t and s_new.dt == s_ref.dt, call
        assert _rel(P_new, P_ref) <= TOL, call
        assert _rel(Pn_new, Pn_ref) <= TOL, call
        # the same kernels on the same inputs: equal bit for bit, which would
        # also show anything left over in the shared scratch
        assert torch.equal(P_new, P_ref) and torch.equal(Pn_new, Pn_ref), call
        dt_ref, dt_new = s_ref.dt, s_new.dt


def test_noalloc_refuses_grids_beyond_its_scratch(cuda_device):
    lib = N.lib()
    dev = cuda_device
    grid, t, g, P0 = _inputs((40, 40, 40), 3, dev)
    st = torch.zeros(ct.sizeof(N.TseSolveStatus), dtype=torch.uint8, device=dev)
    Pn = torch.empty_like(P0)
    stream = ct.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    rc = lib.tse_compute_P_noalloc(ct.byref(grid), ct.byref(_args(t, P0, Pn, 3600.0)),
                                   ct.c_void_p(st.data_ptr()), stream)
    assert rc == -2   # TSE_ERR_WORKSPACE: nothing launched
