"""End-to-end: the GPU driver (transportse_b200.driver.Simulation) against
the reference's own multi-step runs (tests/golden/e2e_*.npz, recorded from
tse.py).  Fields within 1e-9 relative; per-step dt, t_sim and cumulative
iteration counts must match exactly."""
import numpy
import pytest

from tests.golden import cases
from tests.golden.make_golden import E2E
from tests.helpers import check_snapshots, load, rel_err

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
