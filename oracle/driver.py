"""THE ORACLE's time loop -- test infrastructure, never the product path.

A restatement of the reference driver (tse.py:170-245 set-up, tse.py:1118-1494
step loop) over NumPy arrays, calling the oracle's C kernels.  It keeps the
reference's control flow line by line: the SIA Picard loop, the CFL clamp that
happens after the pressure solve, the species skip test, the dt hand-over
between solvers, the Smolarkiewicz second solve and the NLTE two-layer heat
solve.  Used by the tests to check the CUDA driver at sizes the committed
fixtures do not cover, and by bench.py's CPU baseline.
"""
from __future__ import annotations

import math

import numpy

from .oracle import OracleModel

FIELDS = ("phi", "Kx", "Ky", "Kz", "c_r", "cp_r", "l_r", "rho_r", "lf_l", "lf_t",
          "lt_l", "lt_t", "L", "R", "D_fx", "D_fy", "D_fz", "c_f", "cp_f", "l_f",
          "rho_f", "nue", "P", "C", "T", "BP", "BC", "BT", "WP", "WT", "WC", "qx",
          "qy", "qz", "mass")


class ConvergenceError(SystemExit):
    pass


def pymin(*a):
    m = a[0]
    for v in a[1:]:
        if v < m:
            m = v
    return m


# the snapshot tuple of tse.py:324-326, in order
SNAPSHOT_ITEMS = ("lx", "ly", "lz", "nx", "ny", "nz", "dx", "dy", "dz", "t_sim", "dt",
                  "P", "C", "T", "qx", "qy", "qz", "phi", "Kx", "Ky", "Kz", "rho_f",
                  "nue", "cp_f", "l_f", "BP", "BC", "BT", "L", "mass", "WP", "WT", "WC", "e")


def chemistry(config, S, t_sim, dt, chem):
    """The chemistry coupling of tse.py:1383-1417, once per Picard iteration:
    chem_inc accumulates dt (after the first step), and once it reaches
    DTCHEM (or in the first step) the config's chemical_reactions_all runs on
    the whole state, or chemical_reactions on each cell whose BC is not 1
    (k, j, i order, joblib with parallel_chemistry jobs)."""
    if t_sim > 0:
        chem["inc"] += dt
    else:
        chem["inc"] = 0
        chem["dt_chem"] = dt
    if chem["inc"] >= config.DTCHEM:
        chem["dt_chem"] = chem["inc"]
        chem["inc"] = 0
    BC = S["BC"]
    nx, ny, nz = BC.shape[:3]
    cells = [(i, j, k) for k in range(nz) for j in range(ny) for i in range(nx) if BC[i, j, k] != 1]
    if cells == [] or chem["inc"] != 0:
        return
    names = ("C", "P", "T", "rho_f", "phi", "Kx", "Ky", "Kz")
    if hasattr(config, "chemical_reactions_all"):
        out = config.chemical_reactions_all(*[S[n] for n in names], chem["dt_chem"])
        for n, v in zip(names, out):
            S[n] = v
    else:
        from joblib import Parallel, delayed
        res = Parallel(n_jobs=config.parallel_chemistry)(
            delayed(config.chemical_reactions)(*[S[n][i, j, k] for n in names], chem["dt_chem"],
                                               i, j, k) for i, j, k in cells)
        for (i, j, k), r in zip(cells, res):
            for n, v in zip(names, r):
                S[n][i, j, k] = v


class Plots:
    """plotresults (tse.py:312-329): with PLOTSAVE, shorten dt so the run
    lands on the next PLOTTIME (remembering the unshortened dt in dt_prev);
    on landing exactly, write the snapshot tuple with joblib (compress=3) to
    "<prefix>-<index:05d>.p" and restore dt = dt_prev.  A time that is passed
    without an exact landing is never written, and neither is any later one
    (the index stays), as in the reference."""

    def __init__(self, config, prefix):
        self.on = bool(getattr(config, "PLOTSAVE", False))
        self.times = getattr(config, "PLOTTIME", []) if self.on else []
        self.index = 0
        self.prefix = prefix
        self.written = []

    def __call__(self, t_sim, dt, dt_prev, items):
        """items(dt) -> the 34-tuple; returns the new (dt, dt_prev)."""
        if not self.on or self.index > numpy.shape(self.times)[0] - 1:
            return dt, dt_prev
        t_plot = self.times[self.index]
        if t_sim < t_plot:
            dt_prev = dt
            dt = pymin(dt, t_plot - t_sim)
        elif t_sim == t_plot:
            import joblib
            path = "{:s}-{:05d}.p".format(self.prefix, self.index)
            joblib.dump(items(dt), path, compress=3)
            self.written.append(path)
            dt = dt_prev
            self.index += 1
        return dt, dt_prev


def run_fluid_properties(config, S, T3):
    """Per-cell EOS callback over all cells (tse.py:179-199)."""
    C, P, nue, rho_f = S["C"], S["P"], S["nue"], S["rho_f"]
    c_f, cp_f, l_f, cp_r, l_r = S["c_f"], S["cp_f"], S["l_f"], S["cp_r"], S["l_r"]
    phi, Kx, Ky, Kz = S["phi"], S["Kx"], S["Ky"], S["Kz"]
    D_fx, D_fy, D_fz, rho_r = S["D_fx"], S["D_fy"], S["D_fz"], S["rho_r"]
    fp = config.fluid_properties
    nx, ny, nz = P.shape
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                c = (i, j, k)
                r = fp(C[c], T3[c], P[c], nue[c], rho_f[c], c_f[c], cp_f[c], l_f[c],
                       cp_r[c], l_r[c], phi[c], Kx[c], Ky[c], Kz[c], D_fx[c], D_fy[c],
                       D_fz[c], rho_r[c])
                (C[c], T3[c], P[c], nue[c], rho_f[c], c_f[c], cp_f[c], l_f[c], cp_r[c],
                 l_r[c], phi[c], Kx[c], Ky[c], Kz[c], D_fx[c], D_fy[c], D_fz[c],
                 rho_r[c]) = r


def update_fluid_properties(config, S):
    """tse.py:208-225: layer 0 of a 4-D (NLTE) temperature is the fluid."""
    T = S["T"]
    run_fluid_properties(config, S, T if T.ndim == 3 else T[:, :, :, 0])


def run(config, max_steps=None, on_step=None, verbose=False, plot_prefix=None):
    """Run the config; returns the final state dict (plus 'n_tsteps', 't_sim',
    'plots' = snapshot files written).  Snapshots go to
    "<plot_prefix>-<k:05d>.p" (default: the config module's name)."""
    S = {}
    for name in FIELDS:
        S[name] = numpy.array(getattr(config, name), dtype=numpy.float64, copy=True)
    nx, ny, nz = int(config.nx), int(config.ny), int(config.nz)
    S["vx"] = numpy.zeros((nx, ny, nz))
    S["vy"] = numpy.zeros((nx, ny, nz))
    S["vz"] = numpy.zeros((nx, ny, nz))
    S["e"] = numpy.zeros((nx, ny, nz))
    ZEROS = numpy.zeros((nx, ny, nz))
    ONES = numpy.ones((nx, ny, nz))
    t = config.t
    dt_max = config.dt_max
    if config.FLUIDPROP:
        update_fluid_properties(config, S)
    MAXIT_P = config.MAXIT_P if getattr(config, "MAXIT_P", 0) else 20000
    MAXIT_C = config.MAXIT_C if getattr(config, "MAXIT_C", 0) else 100
    MAXIT_T = config.MAXIT_T if getattr(config, "MAXIT_T", 0) else 100
    # numba freezes the globals at the first kernel call, i.e. after the
    # initial EOS; snapshot them from the updated state
    frozen_src = type("F", (), {})()
    for name in ("c_r", "l_r", "rho_r", "cp_r", "lf_l", "lf_t", "lt_l", "lt_t"):
        setattr(frozen_src, name, S[name])
    M = OracleModel(config)
    M.freeze_from(frozen_src)
    cmax_dt = config.dt_max          # compute_C/T default max_dt (tse.py:786, 922)
    dt = config.dt
    t_sim = getattr(config, "t_sim", 0)
    n_tsteps = 0
    numitP = numitC = numitT = num_CFL = 0
    dt_max_abs = dt_max
    dt_P = dt_C = dt_T = float("nan")
    nlte = bool(getattr(config, "NLTE_SOLV", False))
    rhof_prev = numpy.zeros_like(S["rho_f"])
    Pn = S["P"].copy()
    Cn = S["C"].copy()
    Tn = S["T"].copy()
    log = []
    plots = Plots(config, plot_prefix if plot_prefix is not None else config.__name__)

    def snapshot(dt_now):
        v = dict(lx=config.lx, ly=config.ly, lz=config.lz, nx=nx, ny=ny, nz=nz,
                 dx=config.dx, dy=config.dy, dz=config.dz, t_sim=t_sim, dt=dt_now)
        return tuple(v[k] if k in v else S[k] for k in SNAPSHOT_ITEMS)

    dt_prev = dt                     # tse.py:1121
    chem = {"inc": 0, "dt_chem": 0}  # tse.py:1132-1133
    bc_inc = 0                       # tse.py:1128-1132
    dt, dt_prev = plots(t_sim, dt, dt_prev, snapshot)   # tse.py:1177
    while t_sim < t:
        SIA_filled = False
        SIA_iter = 0
        while not SIA_filled and SIA_iter < config.SIA_maxit:
            Co_Filled = False
            CFL = 0
            if config.OMEGA_C == 0:
                dt_NeC = M.explicit_C(S["D_fx"], S["phi"])
            num_it_P = 0
            if config.FLUIDFLOW:
                while not Co_Filled:
                    dt, dt_P, S["P"], Pn, conv, num_it_P = M.compute_P(
                        S["P"], S["c_f"], S["nue"], S["rho_f"], S["phi"], S["Kx"],
                        S["Ky"], S["Kz"], S["qx"], S["qy"], S["qz"], dt, S["BP"],
                        S["WP"], max_dt=dt_max, inc_it=1.25, SOR=config.SOR_P,
                        max_it=MAXIT_P, P_conv=config.CONV_P)
                    if not conv:
                        raise ConvergenceError("* P CONVERGENCE ERROR - check dt and CONV_P in compute_P")
                    S["qx"], S["qy"], S["qz"] = M.compute_q(
                        S["P"], S["BP"], S["Kx"], S["Ky"], S["Kz"], S["qx"], S["qy"],
                        S["qz"], S["nue"], S["rho_f"])
                    if config.HEATTRANS or config.SPECTRANS:
                        S["e"] = M.flow_error(S["P"], Pn, S["qx"], S["qy"], S["qz"],
                                              S["WP"], S["phi"], S["c_f"], S["c_r"],
                                              S["rho_f"], dt)
                    if t_sim > 0:
                        dt_CFL = M.dt_cfl(S["qx"], S["qy"], S["qz"], S["phi"])
                    else:
                        dt_CFL = 1e10
                    dt_max_C = dt_max_T = dt_max_P = dt_max_abs
                    if config.OMEGA_C == 0:
                        dt_max_C = dt_NeC
                    if config.SIA:
                        dt_max = pymin(dt_max_C, dt_max_T, dt_max_P)
                    else:
                        dt_max = pymin(dt_CFL, dt_max_C, dt_max_T, dt_max_P)
                    Co_Filled = True
                    if dt > dt_max * 1.0:
                        num_CFL += num_it_P
                        CFL += 1
                        dt = dt_max
            num_it_C = 0
            if config.SPECTRANS:
                Cn = S["C"].copy()
                for n in config.SPTRANS:
                    Cv = S["C"][:, :, :, n]
                    if numpy.sum(Cv) != 0.0 or numpy.sum(S["WC"][:, :, :, n]) != 0.0:
                        Ds = [S[d][:, :, :, n] for d in ("D_fx", "D_fy", "D_fz")]
                        dt, dt_C, Cnew, conv, it = M.compute_C(
                            Cv, *Ds, S["phi"], S["rho_f"], S["qx"], S["qy"], S["qz"], dt,
                            S["BC"], S["WC"][:, :, :, n], S["R"], S["e"],
                            omega=config.OMEGA_C, SOR=config.SOR_C, max_it=MAXIT_C,
                            max_dt=cmax_dt, C_conv=config.CONV_C)
                        S["C"][:, :, :, n] = Cnew
                        num_it_C += it
                        if not conv:
                            raise ConvergenceError("* C CONVERGENCE ERROR- check dt and C_conv in compute_C")
                        if config.SMOLAR_C:
                            S["vx"], S["vy"], S["vz"] = M.smolarkiewicz(
                                S["C"][:, :, :, n], S["qx"], S["qy"], S["qz"], S["vx"],
                                S["vy"], S["vz"], dt, eps=1e-15, Sc=1.08)
                            dt, dt_C, Cnew, conv, it = M.compute_C(
                                S["C"][:, :, :, n], *Ds, S["phi"], S["rho_f"], S["vx"],
                                S["vy"], S["vz"], dt, S["BC"], S["WC"][:, :, :, n], S["R"],
                                ZEROS, omega=config.OMEGA_C, max_it=MAXIT_C,
                                SOR=config.SOR_C, max_dt=cmax_dt, C_conv=config.CONV_C)
                            S["C"][:, :, :, n] = Cnew
                            num_it_C += it
                            if not conv:
                                raise ConvergenceError("* C2 CONVERGENCE ERROR- check dt and C_conv in compute_C")
            num_it_T = 0
            if config.HEATTRANS:
                Tn = S["T"].copy()
                if nlte:
                    T4 = S["T"]
                    dt, dt_T, T0, conv, it1 = M.compute_T(
                        T4[:, :, :, 0], S["l_f"], S["cp_f"], S["rho_f"], ONES, S["qx"],
                        S["qy"], S["qz"], dt, S["BT"], ZEROS, S["e"],
                        omega=config.OMEGA_T, max_it=MAXIT_T, SOR=config.SOR_T,
                        max_dt=cmax_dt, T_conv=config.CONV_T)
                    T4[:, :, :, 0] = T0
                    dt, dt_T, T1, conv, it2 = M.compute_T(
                        T4[:, :, :, 1], ZEROS, ZEROS, ZEROS, ZEROS, S["qx"], S["qy"],
                        S["qz"], dt, S["BT"], S["WT"], S["e"], omega=config.OMEGA_T,
                        max_it=MAXIT_T, SOR=config.SOR_T, max_dt=cmax_dt,
                        T_conv=config.CONV_T)
                    T4[:, :, :, 1] = T1
                    num_itT = it1 + it2
                else:
                    dt, dt_T, S["T"], conv, num_itT = M.compute_T(
                        S["T"], S["l_f"], S["cp_f"], S["rho_f"], S["phi"], S["qx"],
                        S["qy"], S["qz"], dt, S["BT"], S["WT"], S["e"],
                        omega=config.OMEGA_T, max_it=MAXIT_T, SOR=config.SOR_T,
                        max_dt=cmax_dt, T_conv=config.CONV_T)
                num_it_T += num_itT
                if not conv:
                    raise ConvergenceError("* T CONVERGENCE ERROR - check dt and T_conv in compute_T")
                if config.SMOLAR_T:
                    S["vx"], S["vy"], S["vz"] = M.smolarkiewicz(
                        S["T"], S["qx"], S["qy"], S["qz"], S["vx"], S["vy"], S["vz"], dt,
                        eps=1e-15, Sc=1.08)
                    dt, dt_T, S["T"], conv, num_itT = M.compute_T(
                        S["T"], S["l_f"], S["cp_f"], S["rho_f"], S["phi"], S["vx"],
                        S["vy"], S["vz"], dt, S["BT"], S["WT"], ZEROS,
                        omega=config.OMEGA_T, max_it=MAXIT_T, SOR=config.SOR_T,
                        max_dt=cmax_dt, T_conv=config.CONV_T)
                    num_it_T += num_itT
                    if not conv:
                        raise ConvergenceError("* T CONVERGENCE ERROR - check dt and T_conv in compute_T")
            if config.CHEMREACT:
                chemistry(config, S, t_sim, dt, chem)
            if config.FLUIDPROP:
                update_fluid_properties(config, S)
            if config.SIA:
                SIA_diff = M.l2_norm(S["rho_f"], rhof_prev, "rhof")
                if SIA_diff < config.SIA_conv or SIA_iter == config.SIA_maxit - 1:
                    SIA_filled = True
                else:
                    rhof_prev = S["rho_f"].copy()
                    S["P"] = Pn.copy()
                    if config.HEATTRANS:
                        S["T"] = Tn.copy()
                    if config.SPECTRANS:
                        S["C"] = Cn.copy()
                    SIA_iter += 1
            else:
                SIA_filled = True
            numitP += num_it_P
            numitC += num_it_C
            numitT += num_it_T
        rec = dict(dt=dt, t_sim=t_sim, numitP=numitP, numitC=numitC, numitT=numitT,
                   num_CFL=num_CFL, dt_P=dt_P, dt_C=dt_C, dt_T=dt_T, step=n_tsteps + 1)
        log.append(rec)
        if config.DYNAMICBC:
            # tse.py:1448-1458: the hook returns the (possibly replaced) arrays;
            # a changed bc_inc re-runs the equation of state
            names = ("P", "T", "C", "BP", "BT", "BC", "WP", "WT", "WC", "Kx", "Ky", "Kz")
            bc_prev = bc_inc
            out = config.dynamic_bc(t_sim + dt, bc_inc, *[S[n] for n in names], S["rho_f"],
                                    S["nue"], S["c_f"], S["cp_f"], S["qx"], S["phi"], S["l_f"],
                                    S["l_r"])
            bc_inc = out[0]
            for n, v in zip(names, out[1:]):
                S[n] = v
            if bc_prev != bc_inc and config.FLUIDPROP:
                update_fluid_properties(config, S)
        if verbose:
            print("[t] %8.2e/%8.2e [dt] %8.2e [S] %4d [P] %3d [C] %3d [T] %3d [CFL] %d"
                  % (t_sim + dt, t, dt, n_tsteps + 1, num_it_P, num_it_C, num_it_T, CFL))
        if on_step is not None:
            on_step(rec, S)
        t_sim += dt
        n_tsteps += 1
        dt = 1e99
        if config.FLUIDFLOW:
            dt = pymin(dt_P, t - t_sim)
        if config.HEATTRANS:
            dt = pymin(dt_T, t - t_sim, dt)
        if config.SPECTRANS:
            dt = pymin(dt_C, t - t_sim, dt)
        dt, dt_prev = plots(t_sim, dt, dt_prev, snapshot)   # tse.py:1494
        if max_steps is not None and n_tsteps >= max_steps:
            break
    S["t_sim"] = t_sim
    S["n_tsteps"] = n_tsteps
    S["plots"] = list(plots.written)
    S["log"] = log
    return S
