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


def test_sweep_variants_give_identical_results(cuda_device):
    """The staged sweep's compiled variants (chunk of 256/512/1024 cells, ring
    of 2-4 stages, 1 or 2 pipelines) only reschedule the same cell updates:
    a mixed-precision pressure solve and a species solve give the same fields,
    iteration counts and dt bit for bit under each (the check sums are
    grouped by chunk, but no norm of these solves lies within rounding of its
    tolerance), and the call reports the variant that ran."""
    from transportse_b200 import workloads
    shape = (40, 36, 50)
    rng = numpy.random.default_rng(17)
    cfg = workloads.base_config("var", *shape, rng.uniform(0.5, 2, shape[0]),
                                rng.uniform(0.5, 2, shape[1]), rng.uniform(0.5, 2, shape[2]))
    cfg.beta = 3.0
    cfg.c_r[:] = 1e-10
    K = 1e-12 * numpy.exp(rng.standard_normal(shape))
    pargs = (4.5e-10 * numpy.ones(shape), rng.uniform(8e-4, 1.2e-3, shape),
             rng.uniform(995, 1150, shape), rng.uniform(0.05, 0.3, shape), K, K, 0.3 * K)
    z = numpy.zeros(shape)
    P = workloads.hydrostatic(cfg) + rng.uniform(-300, 300, shape)
    BP = numpy.zeros(shape)
    BP[:, :, -1] = 1
    WP = numpy.where(rng.uniform(size=shape) < 0.2, rng.uniform(-1e-4, 1e-4, shape), 0.0)
    C = rng.uniform(0, 1, shape)
    D = 1e-6 * rng.uniform(0.5, 1.5, shape)
    BC = (rng.uniform(size=shape) < 0.05).astype(float)
    q = [rng.uniform(-1e-4, 1e-4, shape) for _ in range(3)]
    out = {}
    for variant in ((512, 4, 2), (256, 3, 2), (1024, 2, 2), (512, 2, 1), (256, 4, 1)):
        m = model_for(cfg, cuda_device, "fp32dc")
        m.sweep_variant = variant
        nk = NumpyKernels(m)
        rp = nk.compute_P(P.copy(), *pargs, z, z, z, 3600.0, BP, WP, SOR=1.7, max_it=20000,
                          inc_it=1.25, max_dt=1e5, min_dt=1e-8, P_conv=1e-10)
        ran = m.last_variant
        rc = nk.compute_C(C.copy(), D, D, D, pargs[3], pargs[2], *q, 3600.0, BC, z, numpy.ones(shape),
                          z, omega=1, SOR=1.1, max_it=100, inc_it=1.05, max_dt=1e5, min_dt=1e-8,
                          C_conv=1e-10)
        assert ran == variant, (ran, variant)
        out[variant] = (rp, rc)
    ref_p, ref_c = out[(512, 4, 2)]
    assert ref_p[5] > 50
    for v, (p, c) in out.items():
        assert (p[0], p[1], p[4], p[5]) == (ref_p[0], ref_p[1], ref_p[4], ref_p[5]), v
        assert numpy.array_equal(p[2], ref_p[2]), v
        assert (c[0], c[1], c[3], c[4]) == (ref_c[0], ref_c[1], ref_c[3], ref_c[4]), v
        assert numpy.array_equal(c[2], ref_c[2]), v
