"""Failure detection on the GPU without a fault: every kind of bounded wait
the persistent kernels use (generation grid barrier, counter grid barrier,
mbarrier wait of the staged sweeps) is made to run out -- its condition never
comes true -- and must give up after its time limit with its error flag
raised, leaving the context usable."""
import ctypes as ct
import time

import pytest
import torch

from transportse_b200 import _native as N

pytestmark = pytest.mark.gpu


def test_bounded_waits_give_up_and_report(cuda_device):
    L = N.lib()
    res = torch.full((3,), -1, dtype=torch.int32, device=cuda_device)
    ws = torch.empty(512, dtype=torch.uint8, device=cuda_device)
    stream = torch.cuda.current_stream(cuda_device)
    t0 = time.perf_counter()
    rc = L.tse_selftest_bounded_waits(ct.c_void_p(res.data_ptr()), 0.2,
                                      ct.c_void_p(ws.data_ptr()), ws.numel(),
                                      ct.c_void_p(stream.cuda_stream))
    assert rc == 0
    got = res.cpu().tolist()
    elapsed = time.perf_counter() - t0
    assert got == [1, 1, 1], got
    assert elapsed >= 0.5            # each wait held for its limit before giving up
    # the context is still usable: a solve right after succeeds
    x = torch.arange(1000, dtype=torch.float64, device=cuda_device)
    assert float((x * 2).sum().item()) == 999000.0
