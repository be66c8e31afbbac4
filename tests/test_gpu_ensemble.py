"""Ensembles and serving: each model's result is the same alone and in the mix.

FP64 form: identical bit for bit (the FP64 solves do not depend on how many
blocks they get).  FP32+DC form: within 1e-6 (its sums are grouped by block
count, which changes with the number of concurrent models).  The ensemble
member that has a reference fixture is also checked against the reference's
own run."""
import numpy
import pytest

from tests.golden.make_golden import E2E
from tests.helpers import load, rel_err
from transportse_b200 import workloads

pytestmark = pytest.mark.gpu

SHAPES = [(9, 7, 8), (12, 10, 9), (16, 8, 12), (20, 12, 10), (7, 15, 6)]


def _configs():
    return [workloads.ensemble_member(seed=3 if s == (9, 7, 8) else 100 + i, shape=s)
            for i, s in enumerate(SHAPES)]


@pytest.mark.parametrize("precision,mode,tol", [("fp64", "streams", 0.0),
                                                 ("fp32dc", "streams", 1e-6),
                                                 ("fp32dc", "cluster", 1e-6),
                                                 ("fp32dc", "batched", 1e-6)])
def test_ensemble_alone_equals_mixed(precision, mode, tol, cuda_device):
    """alone: one model at a time, whole-GPU solves; mixed: four at a time
    (streams), four at a time with every solve a single-cluster launch
    (cluster), or all in lock step through the batch gate (batched)."""
    from transportse_b200.ensemble import Ensemble
    steps = 3
    batched = mode == "batched"
    alone, _ = Ensemble(_configs(), device=cuda_device, precision=precision,
                        concurrency=1, batched=False, cluster_cells=0).run(steps)
    mixed, stats = Ensemble(_configs(), device=cuda_device, precision=precision,
                            concurrency=None if batched else 4, batched=batched,
                            cluster_cells=(1 << 30) if mode == "cluster" else 0).run(steps)
    assert stats["models"] == len(SHAPES) and stats["cell_updates"] > 0
    if batched:
        b = stats["batch"]
        assert b["solves"]["compute_P"] >= len(SHAPES) * steps
        assert b["launches"]["compute_P"] < b["solves"]["compute_P"]
    for a, b in zip(alone, mixed):
        for k in ("P", "C", "T"):
            e = rel_err(b[k], a[k])
            assert e <= tol, (precision, k, e)
        if precision == "fp64":
            assert a["iterations"] == b["iterations"]


def test_ensemble_member_matches_reference(cuda_device):
    from transportse_b200.ensemble import Ensemble
    builder, kw, steps, keep, fields = E2E["ensemble_member"]
    fx = load("e2e_ensemble_member")
    res, _ = Ensemble([builder(**kw)], device=cuda_device, precision="fp64",
                      concurrency=1).run(steps, keep=("P", "C", "T", "qx", "qy", "qz"))
    for f in ("P", "C", "T", "qx", "qy", "qz"):
        assert rel_err(res[0][f], fx["%s@%d" % (f, steps)]) <= 1e-9, f


def test_serving_results_alone_and_in_the_mix(cuda_device):
    from transportse_b200.serving import Server, poisson_trace
    trace = poisson_trace(6, rate=40.0, seed=9, builder=workloads.serving_request, steps=2,
                          n_min=8, n_max=20)
    reqs, stats = Server(device=cuda_device, slots=3).replay(trace)
    assert stats["requests"] == 6 and stats["p99_s"] >= stats["p50_s"] > 0
    for r in reqs:
        cfg = workloads.serving_request(9 * 1000 + r.rid, n_min=8, n_max=20)
        from transportse_b200.ensemble import run_model
        alone = run_model(cfg, 2, cuda_device, "fp32dc", max_blocks=0)
        for k in ("P", "C", "T"):
            assert rel_err(r.result[k], alone[k]) <= 1e-6, (r.rid, k)


@pytest.mark.parametrize("slots", [12, 0])
def test_serving_with_a_slot_per_request(slots, cuda_device):
    """Every request starts on arrival (a slot each, or no slot limit):
    new models upload their state from pageable host memory while the
    running ones' batched calls -- of varying model counts, so their loop
    graphs are built -- are in flight.  Every request completes with its
    alone result; without a limit, no more workers than requests."""
    from transportse_b200.ensemble import run_model
    from transportse_b200.serving import Server, poisson_trace
    trace = poisson_trace(12, rate=60.0, seed=11, builder=workloads.serving_request, steps=2,
                          n_min=8, n_max=24)
    srv = Server(device=cuda_device, slots=slots)
    reqs, stats = srv.replay(trace)
    assert stats["requests"] == 12 and all(r.error is None for r in reqs)
    assert len(srv.workers) <= 12
    for r in reqs[:4]:
        cfg = workloads.serving_request(11 * 1000 + r.rid, n_min=8, n_max=24)
        alone = run_model(cfg, 2, cuda_device, "fp32dc", max_blocks=0)
        for k in ("P", "C", "T"):
            assert rel_err(r.result[k], alone[k]) <= 1e-6, (r.rid, k)


def test_serving_rejects_requests_beyond_the_budget(cuda_device):
    from transportse_b200.serving import Request, Server
    s = Server(device=cuda_device, slots=1, hbm_budget=1 << 20)
    with pytest.raises(MemoryError):
        s.submit(Request(0, workloads.serving_request(1, n=16), 1, 0.0))
