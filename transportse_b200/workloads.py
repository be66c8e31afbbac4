"""Synthetic TRANSPORTSE config modules for the benchmark shapes.

Every builder returns a ``types.ModuleType`` that carries the same attribute
set as a TRANSPORTSE config file (grid, fields, process flags, solver
parameters, callbacks), i.e. the attributes tse.py reads at tse.py:48-50,
82-151, 202, 228, 232-245, 1120-1125 and 1151-1172.  The modules can be run by
the reference driver (`python tse.py <config.py>` style) and by
``transportse_b200.driver`` alike.

Inputs are seeded (``numpy.random.default_rng(seed)``); no dataset is read.

Shapes (named by what they are):

* ``slice_2d``       60 x 1 x 30 vertical slice, density-driven sinking of a
                     dense plume below a Dirichlet patch (one species).
* ``reservoir_3d``   geometric node spacing, Gaussian-random-field log10 K,
                     two species plus heat, linear EOS, SIA Picard loop.
* ``ensemble_member`` one model of an ensemble: log-uniform grid size per axis,
                     lognormal K, one source/sink cell, one species plus heat.
* ``sloped_3d``      sloped domain, anisotropic lognormal K, three species with
                     dispersivity, Smolarkiewicz correction, NLTE heat.
* ``serving_request`` cubic grid of log-uniform size, flow/heat/one species,
                     Dirichlet concentration patch on top.
"""
from __future__ import annotations

import math
import types

import numpy

G = 9.81

# Linear equation of state rho = rho0 + sum_s a_s * C_s - b * (T - T0), written
# as generated source so that the callback is a plain function of the cell
# values that numba can also compile (tse.py:202-205 compiles it when
# JITFLUPRO is set).  The declared GPU_EOS block carries the same numbers; the
# device kernel evaluates the expression in the same order.
_EOS_ARGS = ("C, T, P, nue, rho_f, c_f, cp_f, l_f, cp_r, l_r, phi, "
             "Kx, Ky, Kz, D_fx, D_fy, D_fz, rho_r")


def make_linear_eos(rho0, species_coeffs, tcoef, T0):
    """Return (callback, GPU_EOS declaration) for the linear density law."""
    expr = repr(float(rho0))
    for s, a in species_coeffs:
        expr += " + %r * C[%d]" % (float(a), int(s))
    expr += " - %r * (T - %r)" % (float(tcoef), float(T0))
    src = ("def fluid_properties(%s):\n"
           "    rho_f = %s\n"
           "    return %s\n") % (_EOS_ARGS, expr, _EOS_ARGS)
    ns = {}
    exec(compile(src, "<linear_eos>", "exec"), ns)
    fn = ns["fluid_properties"]
    fn.__doc__ = "rho_f = " + expr
    decl = {"rho": {"kind": "linear", "rho0": float(rho0),
                    "species": [(int(s), float(a)) for s, a in species_coeffs],
                    "tcoef": float(tcoef), "T0": float(T0)},
            "nue": {"kind": "keep"}}
    return fn, decl


def _identity_fluid_properties(C, T, P, nue, rho_f, c_f, cp_f, l_f, cp_r, l_r,
                               phi, Kx, Ky, Kz, D_fx, D_fy, D_fz, rho_r):
    return (C, T, P, nue, rho_f, c_f, cp_f, l_f, cp_r, l_r, phi, Kx, Ky, Kz,
            D_fx, D_fy, D_fz, rho_r)


def _noop_chemistry(C, P, T, rho_f, phi, Kx, Ky, Kz, dt_chem, i, j, k):
    return C, P, T, rho_f, phi, Kx, Ky, Kz


def base_config(name, nx, ny, nz, dx, dy, dz, species=1, nlte=False):
    """Config module with every attribute tse.py reads, all fields zero."""
    m = types.ModuleType(name)
    m.__file__ = name + ".py"
    m.parallel_processes = 1
    m.parallel_chemistry = 1
    m.numba_fastmath = False
    m.numba_tl = "omp"
    m.nx, m.ny, m.nz = int(nx), int(ny), int(nz)
    m.dx = numpy.ascontiguousarray(numpy.broadcast_to(numpy.asarray(dx, dtype=numpy.float64), (nx,)))
    m.dy = numpy.ascontiguousarray(numpy.broadcast_to(numpy.asarray(dy, dtype=numpy.float64), (ny,)))
    m.dz = numpy.ascontiguousarray(numpy.broadcast_to(numpy.asarray(dz, dtype=numpy.float64), (nz,)))
    m.lx, m.ly, m.lz = float(m.dx.sum()), float(m.dy.sum()), float(m.dz.sum())
    m.g = G
    m.beta = 0.0
    m.t = 1e12
    m.FLUIDFLOW = True
    m.SPECTRANS = False
    m.HEATTRANS = False
    m.FLUIDPROP = False
    m.CHEMREACT = False
    m.DYNAMICBC = False
    m.MASSBALAN = False
    m.DTCHEM = 1
    m.C_IMBLFLO = False
    m.T_IMBLFLO = False
    m.SIA = False
    m.SIA_maxit = 1
    m.SIA_conv = 1e-6
    m.SMOLAR_C = False
    m.SMOLAR_T = False
    m.NLTE_SOLV = bool(nlte)
    m.SPECIES = int(species)
    m.SPTRANS = numpy.arange(species)
    shp = (nx, ny, nz)
    z = lambda: numpy.zeros(shp)
    for a in ("phi", "Kx", "Ky", "Kz", "c_r", "cp_r", "l_r", "rho_r", "lf_l",
              "lf_t", "lt_l", "lt_t", "L", "c_f", "cp_f", "l_f", "rho_f",
              "nue", "P", "BP", "BC", "BT", "WP", "WT", "qx", "qy", "qz"):
        setattr(m, a, z())
    m.R = numpy.ones(shp)
    m.mass = numpy.zeros(3)
    for a in ("D_fx", "D_fy", "D_fz", "C", "WC"):
        setattr(m, a, numpy.zeros(shp + (species,)))
    m.T = numpy.zeros(shp + (2,)) if nlte else numpy.zeros(shp)
    m.fluid_properties = _identity_fluid_properties
    m.chemical_reactions = _noop_chemistry
    m.dt = 1.0
    m.dt_max = 1e6
    m.OMEGA_C = 1
    m.OMEGA_T = 1
    m.SOR_P = 1.8
    m.SOR_C = 1.0
    m.SOR_T = 1.0
    m.CONV_P = 1e-10
    m.CONV_C = 1e-10
    m.CONV_T = 1e-10
    m.PRINTOUT = 1
    m.PLOTSAVE = False
    m.PLOTTIME = numpy.zeros(0)
    return m


def hydrostatic(m, rho=1000.0, p_top=1.0e5):
    """P(k) for a column whose top cell (k = nz-1) holds p_top (cos(beta) factor)."""
    cb = math.cos(math.radians(m.beta))
    dz = m.dz
    p = numpy.empty(m.nz)
    p[-1] = p_top
    for k in range(m.nz - 2, -1, -1):
        p[k] = p[k + 1] + rho * m.g * cb * 0.5 * (dz[k] + dz[k + 1])
    return numpy.broadcast_to(p, (m.nx, m.ny, m.nz)).copy()


def gaussian_random_field(rng, shape, corr_len):
    """Zero-mean, unit-variance field: white noise filtered by a Gaussian kernel in Fourier space."""
    w = rng.standard_normal(shape)
    ks = numpy.meshgrid(*[numpy.fft.fftfreq(n) for n in shape], indexing="ij")
    k2 = sum(k * k for k in ks)
    filt = numpy.exp(-2.0 * (math.pi ** 2) * (corr_len ** 2) * k2)
    f = numpy.real(numpy.fft.ifftn(numpy.fft.fftn(w) * filt))
    f -= f.mean()
    sd = f.std()
    return f / sd if sd > 0 else f


def geometric_spacing(n, d0, ratio=1.02):
    c = 0.5 * (n - 1)
    return d0 * ratio ** numpy.abs(numpy.arange(n) - c)


def _rock_fluid_defaults(m, phi=0.1, K=1e-12):
    m.phi[:] = phi
    m.Kx[:] = K
    m.Ky[:] = K
    m.Kz[:] = K
    m.c_f[:] = 4.5e-10
    m.c_r[:] = 1e-10
    m.cp_f[:] = 4180.0
    m.cp_r[:] = 900.0
    m.l_f[:] = 0.6
    m.l_r[:] = 2.5
    m.rho_r[:] = 2650.0
    m.rho_f[:] = 1000.0
    m.nue[:] = 1e-3


def slice_2d(nx=60, ny=1, nz=30, steps=200):
    """Vertical 2-D slice: dense plume under a Dirichlet concentration patch.

    60 x 1 x 30 nodes at 10 m x 1 m x 5 m; one species; rho = 1000 + 200 c;
    viscosity 1e-3 Pa s; K = 1e-12 m^2; porosity 0.1; diffusion 1e-9 m^2/s;
    c = 1 on the middle third of the top row; top row pressure-Dirichlet at
    hydrostatic pressure; SOR 1.8, tolerance 1e-10; CFL time-step control.
    """
    m = base_config("slice_2d", nx, ny, nz, 10.0, 1.0, 5.0, species=1)
    _rock_fluid_defaults(m, phi=0.1, K=1e-12)
    m.SPECTRANS = True
    m.FLUIDPROP = True
    m.JITFLUPRO = True
    m.fluid_properties, m.GPU_EOS = make_linear_eos(1000.0, [(0, 200.0)], 0.0, 20.0)
    m.D_fx[:] = 1e-9
    m.D_fy[:] = 1e-9
    m.D_fz[:] = 1e-9
    a, b = nx // 3, 2 * nx // 3
    m.BC[a:b, :, -1] = 1
    m.C[a:b, :, -1, 0] = 1.0
    m.BP[:, :, -1] = 1
    m.P[:] = hydrostatic(m)
    m.T[:] = 20.0
    m.dt = 86400.0
    m.dt_max = 86400.0 * 30
    m.SOR_P = 1.8
    m.CONV_P = 1e-10
    m.CONV_C = 1e-10
    m.STEPS = steps
    return m


def slice_2d_plot(nx=60, ny=1, nz=30, steps=100, t_last=2.0e7, n_plot=6):
    """slice_2d with snapshots on, as the course configs run: PLOTSAVE = True
    and PLOTTIME = linspace(0, 1, n_plot) * t_last, so the step sequence is
    shortened to land on every plot time (tse.py:312-329)."""
    m = slice_2d(nx, ny, nz, steps)
    m.__name__ = "slice_2d_plot"
    m.PLOTSAVE = True
    m.PLOTTIME = numpy.linspace(0.0, 1.0, n_plot) * t_last
    return m


CHEM_RATE = 2e-7   # 1/s, first-order decay of the slice_2d_chem species


def chem_decay_all(C, P, T, rho_f, phi, Kx, Ky, Kz, dt_chem):
    """Vectorised chemistry of slice_2d_chem (the chemical_reactions_all hook):
    first-order decay of every species, porosity growing with what decayed."""
    f = math.exp(-CHEM_RATE * dt_chem)
    return C * f, P, T, rho_f, phi * (1.0 + 1e-3 * (1.0 - f)), Kx, Ky, Kz


def chem_decay_cell(c, p, t, rho_f, phi, kx, ky, kz, dt_chem, i, j, k):
    """The same chemistry one cell at a time (the chemical_reactions hook)."""
    f = math.exp(-CHEM_RATE * dt_chem)
    return c * f, p, t, rho_f, phi * (1.0 + 1e-3 * (1.0 - f)), kx, ky, kz


def slice_2d_chem(nx=60, ny=1, nz=30, steps=40, per_cell=False):
    """slice_2d with chemistry coupling on (tse.py:1383-1417): every DTCHEM of
    accumulated step time the chemistry runs on every cell whose species
    boundary flag is not 1, through chemical_reactions_all (vectorised) or,
    with per_cell, chemical_reactions one cell at a time."""
    m = slice_2d(nx, ny, nz, steps)
    m.__name__ = "slice_2d_chemcell" if per_cell else "slice_2d_chem"
    m.CHEMREACT = True
    m.DTCHEM = 2 * 86400.0
    m.parallel_chemistry = 1
    if per_cell:
        m.chemical_reactions = chem_decay_cell
    else:
        m.chemical_reactions_all = chem_decay_all
    return m


DYNBC_T1 = 40 * 86400.0    # s: the brine patch moves and a well starts
DYNBC_T2 = 120 * 86400.0   # s: the well stops


def dynbc_patch_and_well(t, bc_inc, P, T, C, BP, BT, BC, WP, WT, WC, Kx, Ky, Kz, rho_f, nue,
                         c_f, cp_f, qx, phi, l_f, l_r):
    """dynamic_bc of slice_2d_dynbc (the hook of tse.py:1448-1458), a pure
    function of the time and bc_inc that changes its arrays in place:

    * from DYNBC_T1 (bc_inc 0 -> 1): the Dirichlet brine patch on the top row
      moves one third of the slice to the right (the old cells become free,
      the new ones hold c = 1), and a well injects fluid low in the left part;
    * from DYNBC_T2 (bc_inc 1 -> 2): the well stops and the left half of the
      top row turns pressure-free (BP = 0).

    Each change of bc_inc makes the driver re-run the equation of state."""
    nx, ny, nz = P.shape
    if bc_inc == 0 and t >= DYNBC_T1:
        a, b = nx // 3, 2 * nx // 3
        BC[a:b, :, nz - 1] = 0.0
        BC[b:, :, nz - 1] = 1.0
        C[b:, :, nz - 1, 0] = 1.0
        WP[nx // 6, :, nz // 4] = 2.0e-7
        bc_inc = 1
    elif bc_inc == 1 and t >= DYNBC_T2:
        WP[nx // 6, :, nz // 4] = 0.0
        BP[: nx // 2, :, nz - 1] = 0.0
        bc_inc = 2
    return bc_inc, P, T, C, BP, BT, BC, WP, WT, WC, Kx, Ky, Kz


def slice_2d_dynbc(nx=30, ny=1, nz=15, steps=60):
    """slice_2d at 30 x 1 x 15 nodes with dynamic boundary conditions on
    (DYNAMICBC, dynbc_patch_and_well): the brine patch moves and a well starts
    after 40 days, the well stops and part of the top turns pressure-free
    after 120 days; the linear EOS is re-run at each change."""
    m = slice_2d(nx, ny, nz, steps)
    m.__name__ = "slice_2d_dynbc"
    m.DYNAMICBC = True
    m.dynamic_bc = dynbc_patch_and_well
    m.dt_max = 86400.0 * 10
    return m


def reservoir_3d(nx=256, ny=256, nz=128, seed=2024, steps=100):
    """Bottom-heated 3-D reservoir with a dense brine patch on top.

    Node spacing grows geometrically (ratio 1.02) toward the boundaries
    (1 m in x/y, 0.5 m in z at the centre); log10 K is a Gaussian random field
    (mean -12, sd 0.5, correlation length 8 cells); porosity U(0.05, 0.25);
    two species plus heat; rho = 1000 + 200 c1 - 0.3 (T - 20); T = 80 C at
    the bottom and 20 C at the top (Dirichlet, linear initial profile);
    SIA Picard tolerance 1e-6.
    """
    rng = numpy.random.default_rng(seed)
    m = base_config("reservoir_3d", nx, ny, nz, geometric_spacing(nx, 1.0),
                    geometric_spacing(ny, 1.0), geometric_spacing(nz, 0.5),
                    species=2)
    _rock_fluid_defaults(m)
    logk = -12.0 + 0.5 * gaussian_random_field(rng, (nx, ny, nz), 8.0)
    K = 10.0 ** logk
    m.Kx[:] = K
    m.Ky[:] = K
    m.Kz[:] = K
    m.phi[:] = rng.uniform(0.05, 0.25, (nx, ny, nz))
    m.SPECTRANS = True
    m.HEATTRANS = True
    m.FLUIDPROP = True
    m.JITFLUPRO = True
    m.C_IMBLFLO = True
    m.T_IMBLFLO = True
    m.SIA = True
    m.SIA_maxit = 10
    m.SIA_conv = 1e-6
    m.fluid_properties, m.GPU_EOS = make_linear_eos(1000.0, [(0, 200.0)], 0.3, 20.0)
    for D in (m.D_fx, m.D_fy, m.D_fz):
        D[:] = 1e-9
    # temperature: Dirichlet bottom/top, linear initial profile
    m.BT[:, :, 0] = 1
    m.BT[:, :, -1] = 1
    m.T[:] = numpy.linspace(80.0, 20.0, nz)[None, None, :]
    # brine patch (species 0) on the top-centre third, Dirichlet
    a, b = nx // 3, max(nx // 3 + 1, 2 * nx // 3)
    c, d = ny // 3, max(ny // 3 + 1, 2 * ny // 3)
    m.BC[a:b, c:d, -1] = 1
    m.C[a:b, c:d, -1, 0] = 1.0
    # tracer patch (species 1): initial plume in the lower middle
    i0, i1 = nx // 4, max(nx // 4 + 1, nx // 2)
    j0, j1 = ny // 4, max(ny // 4 + 1, ny // 2)
    k0, k1 = nz // 4, max(nz // 4 + 1, nz // 2)
    m.C[i0:i1, j0:j1, k0:k1, 1] = 1.0
    m.BP[:, :, -1] = 1
    m.P[:] = hydrostatic(m)
    m.dt = 3600.0
    m.dt_max = 86400.0 * 10
    m.SOR_P = 1.9
    m.CONV_P = 1e-10
    m.CONV_C = 1e-10
    m.CONV_T = 1e-10
    m.STEPS = steps
    return m


def ensemble_member(seed, n_min=32, n_max=128, steps=50, shape=None):
    """One model of a parameter/permeability ensemble.

    Grid size per axis log-uniform in [n_min, n_max]; lognormal K (mean
    1e-12, ln-sd U(0.3, 1.0)); one source or sink cell of 1e-5 m^3/s; one
    species plus heat; top row pressure-Dirichlet.
    """
    rng = numpy.random.default_rng(seed)
    if shape is None:
        shape = tuple(int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
                      for _ in range(3))
    nx, ny, nz = shape
    m = base_config("ensemble_%d" % seed, nx, ny, nz, 1.0, 1.0, 1.0, species=1)
    _rock_fluid_defaults(m, phi=0.2)
    sd = rng.uniform(0.3, 1.0)
    K = 1e-12 * numpy.exp(sd * rng.standard_normal((nx, ny, nz)) - 0.5 * sd * sd)
    m.Kx[:] = K
    m.Ky[:] = K
    m.Kz[:] = K
    m.SPECTRANS = True
    m.HEATTRANS = True
    m.FLUIDPROP = True
    m.JITFLUPRO = True
    m.fluid_properties, m.GPU_EOS = make_linear_eos(1000.0, [(0, 200.0)], 0.3, 20.0)
    for D in (m.D_fx, m.D_fy, m.D_fz):
        D[:] = 1e-9
    m.BP[:, :, -1] = 1
    m.P[:] = hydrostatic(m)
    m.T[:] = 20.0
    m.BT[:, :, -1] = 1
    # initial tracer plume (the reference's next-dt rule reads dt_C, which
    # only exists once a species has been transported, tse.py:1490-1491)
    m.C[nx // 4:max(nx // 4 + 1, nx // 2), ny // 4:max(ny // 4 + 1, ny // 2),
        nz // 4:max(nz // 4 + 1, nz // 2), 0] = 1.0
    ci = (int(rng.integers(0, nx)), int(rng.integers(0, ny)), int(rng.integers(0, max(1, nz - 1))))
    sign = 1.0 if rng.uniform() < 0.5 else -1.0
    V = m.dx[ci[0]] * m.dy[ci[1]] * m.dz[ci[2]]
    m.WP[ci] = sign * 1e-5 * 1000.0 / V
    if sign > 0:
        m.WC[ci + (0,)] = 1e-5 * 1.0 / V
        m.WT[ci] = 1e-5 * 1000.0 * 4180.0 * 40.0 / V
    m.source_cell = ci
    m.dt = 600.0
    m.dt_max = 86400.0
    m.SOR_P = 1.9
    m.CONV_P = 1e-10
    m.CONV_C = 1e-10
    m.CONV_T = 1e-10
    m.STEPS = steps
    return m


def sloped_3d(nx=512, ny=512, nz=256, seed=7, steps=20):
    """Sloped (5 deg) anisotropic 3-D model at HBM scale.

    Lognormal K (ln-sd 0.7, mean 1e-12), Kz = 0.1 Kx; three species with
    longitudinal/transversal dispersivity 10/1 m; Smolarkiewicz correction
    on; NLTE heat (two temperature layers); OMEGA = 1; SIA on.
    """
    rng = numpy.random.default_rng(seed)
    m = base_config("sloped_3d", nx, ny, nz, 2.0, 2.0, 1.0, species=3, nlte=True)
    _rock_fluid_defaults(m, phi=0.15)
    m.beta = 5.0
    K = 1e-12 * numpy.exp(0.7 * rng.standard_normal((nx, ny, nz)) - 0.5 * 0.49)
    m.Kx[:] = K
    m.Ky[:] = K
    m.Kz[:] = 0.1 * K
    m.SPECTRANS = True
    m.HEATTRANS = True
    m.FLUIDPROP = True
    m.JITFLUPRO = True
    m.SMOLAR_C = True
    m.SIA = True
    m.SIA_maxit = 5
    m.SIA_conv = 1e-6
    m.C_IMBLFLO = True
    m.fluid_properties, m.GPU_EOS = make_linear_eos(1000.0, [(0, 200.0)], 0.3, 20.0)
    for D in (m.D_fx, m.D_fy, m.D_fz):
        D[:] = 1e-9
    m.lf_l[:] = 10.0
    m.lf_t[:] = 1.0
    m.BP[:, :, -1] = 1
    m.P[:] = hydrostatic(m)
    m.T[:] = 20.0
    m.BT[:, :, 0] = 1
    m.T[:, :, 0, :] = 60.0
    a, b = nx // 3, max(nx // 3 + 1, 2 * nx // 3)
    c, d = ny // 3, max(ny // 3 + 1, 2 * ny // 3)
    m.BC[a:b, c:d, -1] = 1
    m.C[a:b, c:d, -1, 0] = 1.0
    m.C[a:b, c:d, -1, 1] = 0.5
    m.C[a:b, c:d, -1, 2] = 0.25
    m.dt = 3600.0
    m.dt_max = 86400.0 * 10
    m.SOR_P = 1.9
    m.STEPS = steps
    return m


def serving_request(seed, n_min=16, n_max=192, steps=50, n=None):
    """One served simulation: cubic grid of log-uniform size, flow/heat/species."""
    rng = numpy.random.default_rng(seed)
    if n is None:
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
    m = base_config("request_%d" % seed, n, n, n, 1.0, 1.0, 1.0, species=1)
    _rock_fluid_defaults(m, phi=0.2)
    K = 1e-12 * numpy.exp(0.5 * rng.standard_normal((n, n, n)) - 0.125)
    m.Kx[:] = K
    m.Ky[:] = K
    m.Kz[:] = K
    m.SPECTRANS = True
    m.HEATTRANS = True
    m.FLUIDPROP = True
    m.JITFLUPRO = True
    m.fluid_properties, m.GPU_EOS = make_linear_eos(1000.0, [(0, 200.0)], 0.3, 20.0)
    for D in (m.D_fx, m.D_fy, m.D_fz):
        D[:] = 1e-9
    m.BP[:, :, -1] = 1
    m.P[:] = hydrostatic(m)
    m.T[:] = 20.0
    m.BT[:, :, 0] = 1
    m.T[:, :, 0] = 50.0
    w = max(1, n // 4)
    x0 = int(rng.integers(0, n - w + 1))
    y0 = int(rng.integers(0, n - w + 1))
    m.BC[x0:x0 + w, y0:y0 + w, -1] = 1
    m.C[x0:x0 + w, y0:y0 + w, -1, 0] = 1.0
    m.dt = 600.0
    m.dt_max = 86400.0
    m.SOR_P = 1.9
    m.STEPS = steps
    return m
