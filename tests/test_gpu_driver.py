"""End-to-end: the GPU driver (transportse_b200.driver.Simulation) against
the reference's own multi-step runs (tests/golden/e2e_*.npz, recorded from
tse.py).  Fields within 1e-9 relative; per-step dt, t_sim and cumulative
iteration counts must match exactly."""
import numpy
import pytest

from tests.golden import cases
from tests.golden.make_golden import COURSE, E2E
from tests.helpers import (check_snapshots, dynamic_pressure_err, load, rel_err,
                           run_fixture_case)

pytestmark = pytest.mark.gpu
TOL = 1e-9


@pytest.mark.parametrize("name", sorted(E2E))
def test_driver_matches_reference_run(name, cuda_device, tmp_path):
    from transportse_b200.driver import Simulation
    builder, kw, steps, keep, fields = E2E[name]
    fx = load("e2e_" + name)
    cfg = builder(**kw)
    assert cases.config_checksum(cfg) == str(fx["config_checksum"])
    got = {}
    scal = {k: [] for k in ("dt", "t_sim", "numitP", "numitC", "numitT", "num_CFL")}

    def tap(rec, sim):
        for k in scal:
            scal[k].append(rec[k])
        if rec["step"] in keep:
            for f in fields:
                got["%s@%d" % (f, rec["step"])] = sim.field(f)

    sim = Simulation(cfg, device=cuda_device, plot_prefix=str(tmp_path / "snap"))
    sim.run(max_steps=steps, on_step=tap)
    if "n_plots" in fx.files:
        check_snapshots(sim.plots.written, fx, TOL)
    for k in ("numitP", "numitC", "numitT", "num_CFL"):
        assert numpy.array_equal(numpy.array(scal[k]), fx["s_" + k]), k
    for k in ("dt", "t_sim"):
        assert rel_err(numpy.array(scal[k]), fx["s_" + k]) <= TOL, k
    worst = 0.0
    for k in fx.files:
        if "@" in k:
            e = rel_err(got[k], fx[k])
            worst = max(worst, e)
            assert e <= TOL, (k, e)


@pytest.mark.parametrize("name", sorted(COURSE))
def test_driver_matches_reference_course_models(name, cuda_device, tmp_path):
    """The reference's own example models (course/01..04: flow; heat; heat and
    tracer; the polynomial EOS declared for the device), run to their end time
    (649-852 steps, snapshot times landed on): every step's dt and t within
    1e-9 and its iteration counts exact, fields within 1e-9, the snapshot
    count equal."""
    fx = load(name)
    cfg = cases.config_from_fixture(fx, name)
    assert cases.config_checksum(cfg) == str(fx["config_checksum"])
    scal, got, sim = run_fixture_case(cfg, fx, cuda_device, "fp64", tmp_path)
    assert len(sim.plots.written) == int(fx["n_plot_files"])
    for k in ("numitP", "numitC", "numitT", "num_CFL"):
        assert numpy.array_equal(numpy.array(scal[k]), fx["s_" + k]), k
    for k in ("dt", "t_sim"):
        assert rel_err(numpy.array(scal[k]), fx["s_" + k]) <= TOL, k
    P0 = numpy.asarray(cfg.P)
    for k in fx.files:
        if "@" in k:
            assert rel_err(got[k], fx[k]) <= TOL, (k, rel_err(got[k], fx[k]))
            if k.startswith("P@"):
                assert dynamic_pressure_err(got[k], fx[k], P0) <= TOL, k


def test_swap_state_continues_the_run(cuda_device):
    """A run whose state moves into another set of buffers between steps
    (Simulation.swap_state, as a caller streaming host inputs does) gives the
    same fields bit for bit as the run that never swaps."""
    import torch
    from transportse_b200 import workloads
    from transportse_b200.driver import Simulation
    make = lambda: workloads.reservoir_3d(12, 10, 8, seed=3)   # noqa: E731
    ref = Simulation(make(), device=cuda_device, precision="fp64")
    ref.run(max_steps=3)
    sim = Simulation(make(), device=cuda_device, precision="fp64")
    sim.run(max_steps=1)
    for _ in range(2):
        other = {n: t.clone() for n, t in sim.S.items()}
        old = sim.swap_state(other)
        assert sim.S is other and old is not other
        sim.run(max_steps=1)
    for f in ("P", "C", "T", "qx", "qy", "qz", "rho_f"):
        assert numpy.array_equal(sim.field(f), ref.field(f)), f
    bad = {n: t.clone() for n, t in sim.S.items()}
    bad["P"] = torch.zeros(3, device=sim.S["P"].device, dtype=torch.float64)
    with pytest.raises(ValueError):
        sim.swap_state(bad)
