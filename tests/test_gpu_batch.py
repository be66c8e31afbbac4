"""Batched mixed-precision solves (tse_compute_*_dc_batch through BatchGate):
every model's result in a batch equals its single-model mixed-precision
solve to 1e-6 and the reference to the same bound; the dt-halving and stop
paths give the same t / dt / event sequence; cluster sizes 1-16 agree."""
import threading

import numpy
import pytest
import torch

from oracle.oracle import OracleModel
from tests.golden import cases
from tests.helpers import NumpyKernels, load, model_for, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _run_members(fns, device, cluster=0, host_loop=False, batch_cells=None, graph_runs=0):
    """Run fns[i](gate) on threads of their own, each on its own stream, all
    joined to one gate before any starts (so the first solves batch)."""
    from transportse_b200.batch import BatchGate
    gate = BatchGate(device, cluster=cluster, host_loop=host_loop, batch_cells=batch_cells)
    gate.graph_runs = graph_runs
    out = [None] * len(fns)
    errs = []
    for _ in fns:
        gate.join()

    def work(i):
        s = torch.cuda.Stream(device=device)
        try:
            with torch.cuda.device(device), torch.cuda.stream(s):
                out[i] = fns[i](gate)
                s.synchronize()
        except Exception as e:  # reported below
            errs.append(e)
        finally:
            gate.leave()

    th = [threading.Thread(target=work, args=(i,)) for i in range(len(fns))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if errs:
        raise errs[0]
    return out, gate


def _pressure_case(shape, seed):
    from transportse_b200 import workloads
    nx, ny, nz = shape
    rng = numpy.random.default_rng(seed)
    cfg = workloads.base_config("batch", nx, ny, nz, rng.uniform(0.5, 2, nx),
                                rng.uniform(0.5, 2, ny), rng.uniform(0.5, 2, nz))
    cfg.beta = 2.0
    cfg.c_r[:] = 1e-10
    K = 1e-12 * numpy.exp(rng.standard_normal(shape))
    args = (4.5e-10 * numpy.ones(shape), rng.uniform(8e-4, 1.2e-3, shape),
            rng.uniform(995, 1150, shape), rng.uniform(0.05, 0.3, shape), K, K, 0.3 * K)
    z = numpy.zeros(shape)
    P = workloads.hydrostatic(cfg) + rng.uniform(-300, 300, shape)
    BP = numpy.zeros(shape)
    BP[:, :, -1] = 1
    WP = numpy.where(rng.uniform(size=shape) < 0.2, rng.uniform(-1e-4, 1e-4, shape), 0.0)
    return cfg, P, args + (z, z, z, 3600.0, BP, WP)


SHAPES = [(33, 17, 21), (1, 1, 40), (16, 16, 16), (9, 1, 31), (40, 30, 24), (5, 7, 3)]
# column heights far apart in one batch: the stage layout is sized for the
# tallest column, each model's windows for its own
# column heights from 2 to 1600: the fused sweep sizes its stages for the
# tallest, whose stages leave room for rings of 3
MIXED_H = [(2, 2, 600), (60, 40, 2), (12, 9, 7), (1, 2, 1600)]


@pytest.mark.parametrize("cluster", [0, 1, 4, 16])
def test_batched_pressure_equals_single_solves(cluster, cuda_device):
    kw = dict(SOR=1.7, max_it=20000, inc_it=1.25, max_dt=1e5, min_dt=1e-8, P_conv=1e-10)
    cases_ = [_pressure_case(s, 7 + i) for i, s in enumerate(SHAPES)]
    single = []
    for cfg, P, rest in cases_:
        single.append(NumpyKernels(model_for(cfg, cuda_device, "fp32dc")).compute_P(
            P.copy(), *rest, **kw))

    def member(i):
        cfg, P, rest = cases_[i]

        def fn(gate):
            m = model_for(cfg, cuda_device, "fp32dc")
            m.batch_gate = gate
            return NumpyKernels(m).compute_P(P.copy(), *rest, **kw)
        return fn

    got, gate = _run_members([member(i) for i in range(len(SHAPES))], cuda_device, cluster)
    st = gate.stats()
    assert st["solves"]["compute_P"] == len(SHAPES)
    assert st["launches"]["compute_P"] == 1
    for i, (g, s) in enumerate(zip(got, single)):
        cfg, P, rest = cases_[i]
        assert g[4] == s[4] and g[0] == s[0] and g[1] == s[1], SHAPES[i]
        assert abs(g[5] - s[5]) <= max(10, 0.05 * s[5]), (SHAPES[i], g[5], s[5])
        assert rel_err(g[2], s[2]) <= TOL, SHAPES[i]
        ro = OracleModel(cfg).compute_P(P.copy(), *rest, **kw)
        assert rel_err(g[2], ro[2]) <= TOL, SHAPES[i]


@pytest.mark.parametrize("kw", [
    dict(SOR=1.7, max_it=20000, inc_it=1.25, max_dt=1e5, min_dt=1e-8, P_conv=1e-10),
    dict(SOR=1.7, max_it=25, inc_it=1.25, max_dt=1e5, min_dt=400.0, P_conv=1e-12)])
def test_device_loop_equals_host_loop(kw, cuda_device):
    """The fused form's device-driven loop (one CUDA graph: a conditional WHILE
    node around plan, sweep, events and residual kernels) and its host loop
    take the same steps: every model's pressure, t, dt, convergence flag and
    iteration count agree bit for bit -- through cycle ends and refreshes
    (first case) and through dt halvings down to min_dt (second)."""
    import ctypes as ct
    from transportse_b200 import _native
    lib = _native.lib()
    cases_ = [_pressure_case(s, 7 + i) for i, s in enumerate(SHAPES)]

    def member(i):
        cfg, P, rest = cases_[i]

        def fn(gate):
            m = model_for(cfg, cuda_device, "fp32dc")
            m.batch_gate = gate
            return NumpyKernels(m).compute_P(P.copy(), *rest, **kw)
        return fn

    out, used = {}, {}
    for mode in (1, 0):
        g0, h0 = ct.c_int64(), ct.c_int64()
        lib.tse_batch_loop_stats(ct.byref(g0), ct.byref(h0))
        # per call: TseDcOptions.host_loop = 0 device-driven, 1 host loop
        out[mode], _ = _run_members([member(i) for i in range(len(SHAPES))], cuda_device,
                                    host_loop=mode == 0)
        g1, h1 = ct.c_int64(), ct.c_int64()
        lib.tse_batch_loop_stats(ct.byref(g1), ct.byref(h1))
        used[mode] = (g1.value - g0.value, h1.value - h0.value)
    assert used[1] == (1, 0) and used[0] == (0, 1), used
    for i, (a, b) in enumerate(zip(out[1], out[0])):
        assert (a[0], a[1], a[4], a[5]) == (b[0], b[1], b[4], b[5]), SHAPES[i]
        assert numpy.array_equal(a[2], b[2]), SHAPES[i]


@pytest.mark.parametrize("kw", [
    dict(SOR=1.7, max_it=20000, inc_it=1.25, max_dt=1e5, min_dt=1e-8, P_conv=1e-10),
    dict(SOR=1.7, max_it=25, inc_it=1.25, max_dt=1e5, min_dt=400.0, P_conv=1e-12)])
def test_device_loop_admitting_models_equals_host_loop(kw, cuda_device):
    """A cell budget below the batch's total (TseDcOptions.active_cells): the
    device-driven loop starts with the largest models and admits the others
    into the running loop as earlier ones finish; each admitted model counts
    its own iterations and checks from its admission.  Every model's
    pressure, t, dt, convergence flag and iteration count equal the host
    loop's (all models at once, no budget) bit for bit -- through cycle ends,
    refreshes and dt halvings -- and the batch still goes out as one call."""
    cases_ = [_pressure_case(s, 7 + i) for i, s in enumerate(SHAPES)]

    def member(i):
        cfg, P, rest = cases_[i]

        def fn(gate):
            m = model_for(cfg, cuda_device, "fp32dc")
            m.batch_gate = gate
            return NumpyKernels(m).compute_P(P.copy(), *rest, **kw)
        return fn

    ref, _ = _run_members([member(i) for i in range(len(SHAPES))], cuda_device, host_loop=True,
                          batch_cells=0)
    # 5,000 cells: the 28,800- and 11,781-cell models run alone, the rest in
    # waves behind them; then the same with the graph relaunched by the host
    # every 3 loop-body runs (TseDcOptions.graph_runs), which a solve of more
    # than 4,096 sweep launches would do
    for runs in (0, 3):
        got, gate = _run_members([member(i) for i in range(len(SHAPES))], cuda_device,
                                 batch_cells=5000, graph_runs=runs)
        st = gate.stats()
        assert st["launches"]["compute_P"] == 1 and st["solves"]["compute_P"] == len(SHAPES)
        assert (st["graph_launches"] > 3) == (runs == 3), st["graph_launches"]
        for i, (a, b) in enumerate(zip(got, ref)):
            assert (a[0], a[1], a[4], a[5]) == (b[0], b[1], b[4], b[5]), (SHAPES[i], runs)
            assert numpy.array_equal(a[2], b[2]), (SHAPES[i], runs)


def test_batched_halving_and_stop_follow_the_reference(cuda_device):
    # unreachable tolerance: every solve halves dt max_it by max_it until it
    # reaches min_dt, then stops unconverged (tse.py:724-740)
    kw = dict(SOR=1.7, max_it=25, inc_it=1.25, max_dt=1e5, min_dt=400.0, P_conv=1e-12)
    cases_ = [_pressure_case(s, 50 + i) for i, s in enumerate(SHAPES[:4])]
    ref = [OracleModel(cfg).compute_P(P.copy(), *rest, **kw) for cfg, P, rest in cases_]

    def member(i):
        cfg, P, rest = cases_[i]

        def fn(gate):
            m = model_for(cfg, cuda_device, "fp32dc")
            m.batch_gate = gate
            return NumpyKernels(m).compute_P(P.copy(), *rest, **kw)
        return fn

    got, _ = _run_members([member(i) for i in range(len(cases_))], cuda_device)
    for g, r in zip(got, ref):
        assert not r[4] and not g[4]
        assert g[0] == r[0] and g[1] == r[1] and g[5] == r[5]
        assert rel_err(g[2], r[2]) <= TOL


def test_batched_unit_calls_match_reference_fixtures(cuda_device):
    """Both reference unit cases (pressure, fluxes, species, heat, Smolarkiewicz
    calls) on two threads whose solves batch together."""
    variants = ["a", "b"]

    def member(v):
        def fn(gate):
            cfg, inp = cases.unit_inputs_with_cfg(v)
            m = model_for(cfg, cuda_device, "fp32dc")
            m.batch_gate = gate
            return cases.run_unit_calls(NumpyKernels(m), inp, v)
        return fn

    got, gate = _run_members([member(v) for v in variants], cuda_device)
    assert sum(gate.stats()["solves"].values()) > sum(gate.stats()["launches"].values())
    for v, out in zip(variants, got):
        fx = load("unit_" + v)
        for k in fx.files:
            if not k.startswith("out_"):
                continue
            name = k[4:]
            ref, g = fx[k], out[name]
            if name.endswith("_scal"):
                t, dt, conv, nit = g
                assert conv == ref[2], name
                assert abs(nit - ref[3]) <= max(10, 0.05 * max(nit, ref[3])), (name, nit, ref[3])
                if conv:
                    assert abs(t - ref[0]) <= 1e-12 * abs(ref[0]), name
            else:
                assert rel_err(g, ref) <= TOL, (v, name, rel_err(g, ref))


def test_fused_batch_with_far_apart_column_heights(cuda_device):
    kw = dict(SOR=1.7, max_it=20000, inc_it=1.25, max_dt=1e5, min_dt=1e-8, P_conv=1e-10)
    cases_ = [_pressure_case(s, 90 + i) for i, s in enumerate(MIXED_H)]

    def member(i):
        cfg, P, rest = cases_[i]

        def fn(gate):
            m = model_for(cfg, cuda_device, "fp32dc")
            m.batch_gate = gate
            return NumpyKernels(m).compute_P(P.copy(), *rest, **kw)
        return fn

    got, gate = _run_members([member(i) for i in range(len(MIXED_H))], cuda_device, 0)
    assert gate.stats()["launches"]["compute_P"] == 1
    for i, g in enumerate(got):
        cfg, P, rest = cases_[i]
        ro = OracleModel(cfg).compute_P(P.copy(), *rest, **kw)
        assert g[4] == ro[4] and g[0] == ro[0] and g[1] == ro[1], MIXED_H[i]
        assert abs(g[5] - ro[5]) <= max(10, 0.05 * ro[5]), (MIXED_H[i], g[5], ro[5])
        assert rel_err(g[2], ro[2]) <= TOL, MIXED_H[i]


@pytest.mark.parametrize("precision", ["fp64", "fp32dc"])
@pytest.mark.parametrize("case", ["nan_input", "max_it_1"])
def test_failure_paths_follow_the_reference(precision, case, cuda_device):
    """Non-convergence as the reference handles it: a NaN in the pressure (the
    L2 change is NaN and counts as 1) or max_it = 1 makes every attempt fail,
    dt is halved until it drops below min_dt, and the solve returns
    unconverged -- same t, dt and iteration count as the oracle, no hang."""
    cfg, P, rest = _pressure_case((9, 1, 31), 123)
    if case == "nan_input":
        P[4, 0, 10] = float("nan")
        kw = dict(SOR=1.7, max_it=30, inc_it=1.25, max_dt=1e5, min_dt=400.0, P_conv=1e-10)
    else:
        kw = dict(SOR=1.7, max_it=1, inc_it=1.25, max_dt=1e5, min_dt=1.0, P_conv=1e-10)
    ro = OracleModel(cfg).compute_P(P.copy(), *rest, **kw)
    g = NumpyKernels(model_for(cfg, cuda_device, precision)).compute_P(P.copy(), *rest, **kw)
    assert not ro[4] and not g[4]
    assert g[0] == ro[0] and g[1] == ro[1] and g[5] == ro[5], (g[:2], g[5], ro[:2], ro[5])


def test_batched_driver_runs_match_reference_runs(cuda_device, tmp_path):
    """Every reference end-to-end run at once, each model on its own thread
    with its own number of steps, all mixed-precision solves batched through
    one gate (models leave the batch as they finish): each matches its
    reference run within 1e-6, dt sequence included."""
    from tests.golden.make_golden import E2E
    from transportse_b200.driver import Simulation
    names = sorted(E2E)

    def member(name):
        def fn(gate):
            builder, kw, steps, keep, fields = E2E[name]
            sim = Simulation(builder(**kw), device=cuda_device, precision="fp32dc",
                             plot_prefix=str(tmp_path / name))
            sim.M.batch_gate = gate
            got, dts = {}, []

            def tap(rec, s):
                dts.append(rec["dt"])
                if rec["step"] in keep:
                    for f in fields:
                        got["%s@%d" % (f, rec["step"])] = s.field(f)
            sim.run(max_steps=steps, on_step=tap)
            return got, dts
        return fn

    out, gate = _run_members([member(n) for n in names], cuda_device)
    st = gate.stats()
    assert sum(st["solves"].values()) > sum(st["launches"].values())
    for name, (got, dts) in zip(names, out):
        fx = load("e2e_" + name)
        # CFL-limited steps take dt from the fluxes, which carry the form's error
        assert rel_err(numpy.array(dts), fx["s_dt"]) <= TOL, name
        for k in fx.files:
            if "@" in k and k.split("@")[0] in ("P", "C", "T"):
                assert rel_err(got[k], fx[k]) <= TOL, (name, k, rel_err(got[k], fx[k]))
