"""CUDA kernels against the reference: the golden unit fixtures (outputs of
tse.py's own numba kernels) and the oracle on further grid shapes.

Tolerance: 1e-9 relative (to the field's max magnitude) for FP64 fields; the
iteration counts, convergence flags and dt values must match exactly.  The
kernels keep the reference's operation order, so most fields agree bit for
bit; only the L2 sums are reduced in a different order (tree vs sequential)."""
import numpy
import pytest

from oracle.oracle import OracleModel
from tests.golden import cases
from tests.helpers import NumpyKernels, load, model_for, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-9


def _compare(out, ref, keys=None):
    worst = {}
    for k in (keys or ref):
        r = ref[k]
        g = out[k]
        if k.endswith("_scal"):
            # t, dt, converged, num_it: exact
            assert numpy.array_equal(numpy.asarray(g), numpy.asarray(r)), (k, g, r)
        else:
            e = rel_err(g, r)
            worst[k] = e
            assert e <= TOL, (k, e)
    return worst


@pytest.mark.parametrize("variant", ["a", "b"])
def test_unit_kernels_match_reference_fixtures(variant, cuda_device):
    fx = load("unit_" + variant)
    cfg, inp = cases.unit_inputs_with_cfg(variant)
    m = model_for(cfg, cuda_device)
    out = cases.run_unit_calls(NumpyKernels(m), inp, variant)
    ref = {k[4:]: fx[k] for k in fx.files if k.startswith("out_")}
    worst = _compare(out, ref)
    exact = [k for k in ref if not k.endswith("_scal")
             and numpy.array_equal(numpy.asarray(out[k]), ref[k], equal_nan=True)]
    # every kernel except the reductions is bit-exact
    for k in ("qx", "qy", "qz", "e", "vx", "vy", "vz", "p1_P", "p1_Pn"):
        assert k in exact, (k, worst.get(k))


SHAPES = [(33, 17, 21), (1, 1, 40), (40, 1, 1), (5, 7, 2), (16, 16, 16), (9, 1, 31)]


def _random_case(shape, seed):
    nx, ny, nz = shape
    rng = numpy.random.default_rng(seed)
    from transportse_b200 import workloads
    cfg = workloads.base_config("rnd", nx, ny, nz, rng.uniform(0.5, 2, nx), rng.uniform(0.5, 2, ny),
                                rng.uniform(0.5, 2, nz), species=1)
    cfg.beta = 3.0
    shp = shape
    cfg.c_r[:] = 1e-10 * rng.uniform(0.5, 1.5, shp)
    cfg.l_r[:] = rng.uniform(1.5, 3.5, shp)
    cfg.rho_r[:] = 2650.0
    cfg.cp_r[:] = 900.0
    cfg.lf_l[:] = rng.uniform(0, 1, shp)
    cfg.lf_t[:] = rng.uniform(0, 0.3, shp)
    cfg.C_IMBLFLO = True
    return cfg, rng


@pytest.mark.parametrize("shape", SHAPES)
def test_pressure_and_species_vs_oracle_shapes(shape, cuda_device):
    cfg, rng = _random_case(shape, hash(shape) % 1000)
    shp = shape
    K = 1e-12 * numpy.exp(rng.standard_normal(shp))
    f = dict(c_f=4.5e-10 * rng.uniform(0.5, 1.5, shp), nue=rng.uniform(8e-4, 1.2e-3, shp),
             rho_f=rng.uniform(995, 1150, shp), phi=rng.uniform(0.05, 0.3, shp), Kx=K,
             Ky=K * 0.7, Kz=K * 0.2)
    from transportse_b200 import workloads
    P = workloads.hydrostatic(cfg) + rng.uniform(-300, 300, shp)
    BP = (rng.uniform(size=shp) < 0.1).astype(float)
    BP.reshape(-1)[0] = 1.0
    WP = numpy.where(rng.uniform(size=shp) < 0.2, rng.uniform(-1e-4, 1e-4, shp), 0.0)
    z = numpy.zeros(shp)
    orc = OracleModel(cfg)
    m = model_for(cfg, cuda_device)
    nk = NumpyKernels(m)
    args = (f["c_f"], f["nue"], f["rho_f"], f["phi"], f["Kx"], f["Ky"], f["Kz"], z, z, z)
    kw = dict(SOR=1.6, max_it=20000, inc_it=1.25, max_dt=1e5, min_dt=1e-8, P_conv=1e-11)
    r_o = orc.compute_P(P.copy(), *args, 3600.0, BP, WP, **kw)
    r_g = nk.compute_P(P.copy(), *args, 3600.0, BP, WP, **kw)
    assert r_o[0] == r_g[0] and r_o[1] == r_g[1] and r_o[4] == r_g[4] and r_o[5] == r_g[5]
    assert rel_err(r_g[2], r_o[2]) <= TOL
    assert numpy.array_equal(r_g[3], r_o[3])
    q0 = [rng.uniform(-1e-5, 1e-5, shp) for _ in range(3)]
    qo = orc.compute_q(r_o[2], BP, f["Kx"], f["Ky"], f["Kz"], *[x.copy() for x in q0], f["nue"], f["rho_f"])
    qg = nk.compute_q(r_o[2], BP, f["Kx"], f["Ky"], f["Kz"], *[x.copy() for x in q0], f["nue"], f["rho_f"])
    for a, b in zip(qo, qg):
        assert numpy.array_equal(a, b)
    C = rng.uniform(0, 1, shp)
    D = 1e-6 * rng.uniform(0.5, 1.5, shp)
    BC = (rng.uniform(size=shp) < 0.1).astype(float)
    WC = numpy.where(rng.uniform(size=shp) < 0.2, 1e-5, 0.0)
    e = rng.uniform(-1e-6, 1e-6, shp)
    q = [rng.uniform(-1e-4, 1e-4, shp) for _ in range(3)]
    for omega in (1, 0.5):
        kwc = dict(omega=omega, SOR=1.1, max_it=100, inc_it=1.05, max_dt=1e5, min_dt=1e-8, C_conv=1e-11)
        co = orc.compute_C(C.copy(), D, D, D, f["phi"], f["rho_f"], *q, 3600.0, BC, WC, numpy.ones(shp), e, **kwc)
        cg = nk.compute_C(C.copy(), D, D, D, f["phi"], f["rho_f"], *q, 3600.0, BC, WC, numpy.ones(shp), e, **kwc)
        assert co[0] == cg[0] and co[1] == cg[1] and co[3] == cg[3] and co[4] == cg[4]
        assert rel_err(cg[2], co[2]) <= TOL


def test_reductions_vs_oracle(cuda_device):
    cfg, rng = _random_case((23, 11, 13), 5)
    shp = (23, 11, 13)
    orc = OracleModel(cfg)
    m = model_for(cfg, cuda_device)
    a, b = rng.standard_normal(shp), rng.standard_normal(shp)
    assert abs(m.l2_norm(a, b) - orc.l2_norm(a, b)) <= 1e-13 * orc.l2_norm(a, b)
    bad = a.copy()
    bad[3, 2, 1] = numpy.nan
    assert m.l2_norm(bad, b) == 1.0
    qx, qy, qz = (rng.uniform(-1e-5, 1e-5, shp) for _ in range(3))
    phi = rng.uniform(0.05, 0.3, shp)
    assert m.dt_cfl(qx, qy, qz, phi) == orc.dt_cfl(qx, qy, qz, phi)
    D4 = rng.uniform(1e-10, 1e-8, shp + (3,))
    assert m.explicit_C(D4, phi) == orc.explicit_C(D4, phi)
    s, mx, mn = m.field_stats(a)
    assert mx == a.max() and mn == a.min() and abs(s - a.sum()) <= 1e-12 * numpy.abs(a).sum()


def test_mass_totals_vs_numpy(cuda_device):
    """FP64 device mass-balance totals against a NumPy FP64 evaluation."""
    from transportse_b200 import workloads
    from transportse_b200.driver import Simulation
    cfg = workloads.reservoir_3d(14, 9, 11, seed=3)
    cfg.GPU_MASSBAL = True
    sim = Simulation(cfg, device=cuda_device).run(max_steps=2)
    last = sim.mass_log[-1]
    f = sim.field
    V = (cfg.dx[:, None, None] * cfg.dy[None, :, None] * cfg.dz[None, None, :])
    phi, rho = f("phi"), f("rho_f")
    water = numpy.sum(phi * rho * V)
    C = f("C")
    species = [numpy.sum(f("R") * phi * C[..., s] * V) for s in range(C.shape[-1])]
    heat = numpy.sum((phi * rho * f("cp_f") + (1 - phi) * f("rho_r") * f("cp_r")) * f("T") * V)
    assert abs(last["water"] - water) <= 1e-12 * abs(water)
    for s in range(C.shape[-1]):
        assert abs(last["species"][s] - species[s]) <= 1e-12 * abs(species[s])
    assert abs(last["heat"] - heat) <= 1e-12 * abs(heat)
    assert len(sim.mass_log) == 2


# (3, 2, 1000): stages big enough that the rings hold 2 stages; (1, 2, 3000):
# the pressure solve's stages fit no ring (the plain kernel runs in both modes),
# the species solve's rings hold 2
@pytest.mark.parametrize("shape", [(64, 48, 40), (37, 23, 51), (96, 96, 64), (3, 2, 1000), (1, 2, 3000)])
def test_staged_and_plain_exact_solves_agree(shape, cuda_device):
    """The staged FP64 sweep (bulk copies into shared-memory stages) and the
    plain-load sweep compute every cell with the same operations: over whole
    pressure and species solves (x and z buoyancy, omega < 1, the IMBLFLO
    term) their fields agree bit for bit and their iteration counts and dt
    match."""
    from transportse_b200 import _native
    lib = _native.lib()
    cfg, rng = _random_case(shape, 7)
    shp = shape
    K = 1e-12 * numpy.exp(rng.standard_normal(shp))
    f = dict(c_f=4.5e-10 * rng.uniform(0.5, 1.5, shp), nue=rng.uniform(8e-4, 1.2e-3, shp),
             rho_f=rng.uniform(995, 1150, shp), phi=rng.uniform(0.05, 0.3, shp))
    from transportse_b200 import workloads
    P = workloads.hydrostatic(cfg) + rng.uniform(-300, 300, shp)
    BP = (rng.uniform(size=shp) < 0.05).astype(float)
    WP = numpy.where(rng.uniform(size=shp) < 0.2, rng.uniform(-1e-4, 1e-4, shp), 0.0)
    z = numpy.zeros(shp)
    C = rng.uniform(0, 1, shp)
    D = 1e-6 * rng.uniform(0.5, 1.5, shp)
    BC = (rng.uniform(size=shp) < 0.05).astype(float)
    WC = numpy.where(rng.uniform(size=shp) < 0.2, 1e-5, 0.0)
    e = rng.uniform(-1e-6, 1e-6, shp)
    q = [rng.uniform(-1e-4, 1e-4, shp) for _ in range(3)]
    m = model_for(cfg, cuda_device)
    nk = NumpyKernels(m)
    out = {}
    for mode in (0, 1):
        m.sweep = mode   # per call: 0 staged bulk-copy kernel, 1 plain loads
        rp = nk.compute_P(P.copy(), f["c_f"], f["nue"], f["rho_f"], f["phi"], K, K * 0.7, K * 0.2,
                          z, z, z, 3600.0, BP, WP, SOR=1.7, max_it=20000, inc_it=1.25,
                          max_dt=1e5, min_dt=1e-8, P_conv=1e-10)
        rc = [nk.compute_C(C.copy(), D, D, D, f["phi"], f["rho_f"], *q, 3600.0, BC, WC,
                           numpy.ones(shp), e, omega=om, SOR=1.1, max_it=100, inc_it=1.05,
                           max_dt=1e5, min_dt=1e-8, C_conv=1e-12) for om in (1, 0.5)]
        out[mode] = (rp, rc)
    (p1, c1), (p0, c0) = out[0], out[1]
    assert p1[5] > 20 and (p1[0], p1[1], p1[4], p1[5]) == (p0[0], p0[1], p0[4], p0[5])
    assert numpy.array_equal(p1[2], p0[2])
    for a, b in zip(c1, c0):
        assert (a[0], a[1], a[3], a[4]) == (b[0], b[1], b[3], b[4])
        assert numpy.array_equal(a[2], b[2])


def test_declared_eos_forms_bit_exact(cuda_device):
    """tse_eos_form (constant; fourth-order polynomial in T, guarded by a
    species) against the host evaluation the declaration is validated with,
    bit for bit, including the guarded cells, which keep their value."""
    import torch
    from transportse_b200 import eos, workloads
    cfg = workloads.base_config("eos", 17, 5, 9, 1.0, 1.0, 1.0, species=3)
    m = model_for(cfg, cuda_device)
    rng = numpy.random.default_rng(12)
    shp = (17, 5, 9)
    T = rng.uniform(-5.0, 160.0, shp)
    guard = numpy.where(rng.uniform(size=shp) < 0.3, 1.0, rng.uniform(0, 2, shp))
    old = rng.uniform(900.0, 1100.0, shp)
    coef = [2.1e-8, -7.3e-6, -3.7e-3, 0.05, 999.8]
    forms = [{"kind": "poly4_T", "coef": coef, "unless": (2, 1.0)},
             {"kind": "poly4_T", "coef": coef},
             {"kind": "constant", "value": 1.234e-3, "unless": (2, 1.0)}]
    dev = lambda a: torch.as_tensor(a, device=cuda_device)
    for d in forms:
        out = dev(old.copy())
        g = dev(guard) if "unless" in d else None
        m.eos_form(d["kind"], d.get("coef", d.get("value")), dev(T), out, g,
                   d.get("unless", (0, 0.0))[1])
        got = out.cpu().numpy()
        want = numpy.empty(shp)
        for c in numpy.ndindex(shp):
            want[c] = eos.eval_form_host(d, [0.0, 0.0, guard[c]], T[c], old[c])
        assert numpy.array_equal(got, want), d
