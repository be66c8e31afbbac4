"""FP32 sweeps with FP64 defect correction (precision 'fp32dc') against the
reference: the golden unit fixtures (outputs of tse.py's numba kernels), the
oracle on further shapes, and the reference's end-to-end runs.

Tolerance: 1e-6 relative to each field's scale (the FP32+refinement bound),
for every field the fixtures hold -- pressure, concentrations, temperature,
the Darcy fluxes it drives, density -- and for the pressure change since the
start (P - P0) on its own scale, so the flow-driven part of the pressure is
not hidden under the hydrostatic head; convergence flags and the dt sequence
must match; iteration counts may differ by a few check intervals because the
change of the FP32 correction is measured in FP32."""
import numpy
import pytest

from oracle.oracle import OracleModel
from tests.golden import cases
from tests.golden.make_golden import COURSE, E2E
from tests.helpers import (NumpyKernels, check_snapshots, dynamic_pressure_err, load, model_for,
                           rel_err, run_fixture_case)

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _its_close(a, b):
    return abs(a - b) <= max(10, 0.05 * max(a, b))


@pytest.mark.parametrize("variant", ["a", "b"])
def test_dc_unit_kernels_match_reference_fixtures(variant, cuda_device):
    fx = load("unit_" + variant)
    cfg, inp = cases.unit_inputs_with_cfg(variant)
    m = model_for(cfg, cuda_device, precision="fp32dc")
    out = cases.run_unit_calls(NumpyKernels(m), inp, variant)
    for k in fx.files:
        if not k.startswith("out_"):
            continue
        name = k[4:]
        ref, got = fx[k], out[name]
        if name.endswith("_scal"):
            t, dt, conv, nit = got
            assert conv == ref[2], name
            assert _its_close(nit, ref[3]), (name, nit, ref[3])
            if conv:
                assert abs(t - ref[0]) <= 1e-12 * abs(ref[0]), name
        else:
            assert rel_err(got, ref) <= TOL, (name, rel_err(got, ref))


# the last two are tall columns: the staged sweep's stages grow with the
# column, so fewer fit (rings of 3 and of 2 stages instead of 4)
@pytest.mark.parametrize("shape", [(33, 17, 21), (1, 1, 40), (16, 16, 16), (9, 1, 31), (2, 2, 1600),
                                   (1, 2, 4000)])
def test_dc_pressure_vs_oracle(shape, cuda_device):
    from transportse_b200 import workloads
    nx, ny, nz = shape
    rng = numpy.random.default_rng(sum(shape))
    cfg = workloads.base_config("dc", nx, ny, nz, rng.uniform(0.5, 2, nx), rng.uniform(0.5, 2, ny),
                                rng.uniform(0.5, 2, nz))
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
    kw = dict(SOR=1.7, max_it=20000, inc_it=1.25, max_dt=1e5, min_dt=1e-8, P_conv=1e-10)
    ro = OracleModel(cfg).compute_P(P.copy(), *args, z, z, z, 3600.0, BP, WP, **kw)
    rg = NumpyKernels(model_for(cfg, cuda_device, "fp32dc")).compute_P(
        P.copy(), *args, z, z, z, 3600.0, BP, WP, **kw)
    assert rg[4] == ro[4] and rg[0] == ro[0] and rg[1] == ro[1]
    assert _its_close(rg[5], ro[5]), (rg[5], ro[5])
    assert rel_err(rg[2], ro[2]) <= TOL
    # pressure differences drive the flow: check them at the same tolerance
    assert rel_err(rg[2] - rg[3], ro[2] - ro[3]) <= 1e-4


@pytest.mark.parametrize("name", sorted(E2E))
def test_dc_driver_matches_reference_run(name, cuda_device, tmp_path):
    from transportse_b200.driver import Simulation
    builder, kw, steps, keep, fields = E2E[name]
    fx = load("e2e_" + name)
    cfg = builder(**kw)
    got = {}

    def tap(rec, sim):
        if rec["step"] in keep:
            for f in fields:
                got["%s@%d" % (f, rec["step"])] = sim.field(f)

    sim = Simulation(cfg, device=cuda_device, precision="fp32dc",
                     plot_prefix=str(tmp_path / "snap"))
    sim.run(max_steps=steps, on_step=tap)
    if "n_plots" in fx.files:
        check_snapshots(sim.plots.written, fx, TOL)
    P0 = numpy.asarray(cfg.P)
    for k in fx.files:
        if "@" in k:
            e = rel_err(got[k], fx[k])
            assert e <= TOL, (k, e)
            if k.startswith("P@"):
                assert dynamic_pressure_err(got[k], fx[k], P0) <= TOL, k


@pytest.mark.parametrize("name", sorted(COURSE))
def test_dc_driver_matches_reference_course_models(name, cuda_device, tmp_path):
    """The reference's example models (course/01..04) to their end time in the
    mixed-precision form: every field and the pressure change within 1e-6, the
    step count and snapshot count equal, the time within 1e-6 at every step."""
    fx = load(name)
    cfg = cases.config_from_fixture(fx, name)
    scal, got, sim = run_fixture_case(cfg, fx, cuda_device, "fp32dc", tmp_path)
    assert len(scal["dt"]) == len(fx["s_dt"])
    assert len(sim.plots.written) == int(fx["n_plot_files"])
    assert rel_err(numpy.array(scal["t_sim"]), fx["s_t_sim"]) <= TOL
    P0 = numpy.asarray(cfg.P)
    for k in fx.files:
        if "@" in k:
            assert rel_err(got[k], fx[k]) <= TOL, (k, rel_err(got[k], fx[k]))
            if k.startswith("P@"):
                assert dynamic_pressure_err(got[k], fx[k], P0) <= TOL, k
