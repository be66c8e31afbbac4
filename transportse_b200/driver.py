"""GPU time-step driver behind the TRANSPORTSE config-module API.

``Simulation(config).run()`` does what ``python tse.py config.py`` does
(tse.py:170-245 set-up, tse.py:1118-1494 step loop) with every grid field
resident on the GPU and every kernel in libtsecuda.so.  The control flow is
the reference's, line for line: the SIA Picard loop, the pressure solve with
the current dt_max (tse.py:1214-1218), the CFL clamp after the pressure solve
(tse.py:1288-1292), the species skip test (tse.py:1300-1301), the dt
hand-over from solver to solver, the Smolarkiewicz second solve
(tse.py:1318-1336), the NLTE two-layer heat solve (tse.py:1343-1354), the SIA
reset (tse.py:1433-1438) and the next-dt rule (tse.py:1486-1492).

Device layout: (nx, ny, nz) float64 fields as in the reference; species
fields are stored species-major, (S, nx, ny, nz), so each species is one
contiguous array; an NLTE temperature is (2, nx, ny, nz).

Equation of state: a config may declare ``GPU_EOS`` (see ``eos.py``); the
declaration is checked against the config's ``fluid_properties`` callback
on sample cells (exact FP64 agreement) and then evaluated by a device
kernel.  Without a declaration the callback itself runs on the host over all
cells, exactly as the reference runs it (tse.py:179-199).
"""
from __future__ import annotations

import math
import sys

import numpy
import torch

from . import eos as _eos
from .kernels import Model

FIELDS3 = ("phi", "Kx", "Ky", "Kz", "c_r", "cp_r", "l_r", "rho_r", "lf_l", "lf_t", "lt_l",
           "lt_t", "L", "R", "c_f", "cp_f", "l_f", "rho_f", "nue", "P", "BP", "BC", "BT", "WP",
           "WT", "qx", "qy", "qz")
FIELDS4 = ("D_fx", "D_fy", "D_fz", "C", "WC")

# the snapshot tuple tse2pvd.py reads (tse.py:324-326), in order
SNAPSHOT_ITEMS = ("lx", "ly", "lz", "nx", "ny", "nz", "dx", "dy", "dz", "t_sim", "dt",
                  "P", "C", "T", "qx", "qy", "qz", "phi", "Kx", "Ky", "Kz", "rho_f",
                  "nue", "cp_f", "l_f", "BP", "BC", "BT", "L", "mass", "WP", "WT", "WC", "e")


class Snapshots:
    """Result snapshots at the PLOTTIME list (plotresults, tse.py:312-329).

    With PLOTSAVE on, the step before a plot time is shortened so the run
    lands on it (the unshortened dt is remembered); at a landing the fields
    come to the host once and the tuple is written with joblib (compress=3)
    to "<prefix>-<index:05d>.p", and dt returns to the remembered value.  A
    plot time that is stepped over without an exact landing is not written,
    and then no later one is either -- the reference behaves the same way."""

    def __init__(self, config, prefix):
        self.on = bool(getattr(config, "PLOTSAVE", False))
        self.times = getattr(config, "PLOTTIME", []) if self.on else []
        self.index = 0
        self.prefix = prefix
        self.written = []

    def step(self, t_sim, dt, dt_prev, items):
        """items(dt) builds the tuple; returns the new (dt, dt_prev)."""
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


class ConvergenceError(SystemExit):
    pass


def pymin(*a):
    m = a[0]
    for v in a[1:]:
        if v < m:
            m = v
    return m


class Simulation:
    def __init__(self, config, device=None, verbose=False, precision=None, plot_prefix=None):
        """precision: 'fp64' (the reference's arithmetic) or 'fp32dc' (FP32
        sweeps with FP64 defect correction); default: config.GPU_PRECISION,
        else 'fp64'.  plot_prefix: path prefix of the PLOTSAVE snapshot files
        (default: the config module's name, in the working directory)."""
        if getattr(config, "NLTE_SOLV", False) and config.SMOLAR_T:
            raise NotImplementedError("NLTE_SOLV with SMOLAR_T is not supported by the reference")
        self.config = config
        self.verbose = verbose
        self.device = torch.device(device if device is not None else "cuda")
        self.M = Model.from_config(config, device=self.device, precision=precision)
        self.shape = (int(config.nx), int(config.ny), int(config.nz))
        self.S = {}
        self.upload_state(config)
        self.nlte = self.S["T"].dim() == 4
        self.eos = _eos.declared_eos(config) if config.FLUIDPROP else None
        if self.eos is not None:
            _eos.validate(config, self.eos)
        self.ZEROS = torch.zeros(self.shape, dtype=torch.float64, device=self.device)
        self.ONES = torch.ones(self.shape, dtype=torch.float64, device=self.device)
        for v in ("vx", "vy", "vz", "e"):
            self.S[v] = torch.zeros(self.shape, dtype=torch.float64, device=self.device)
        self.MAXIT_P = config.MAXIT_P if getattr(config, "MAXIT_P", 0) else 20000
        self.MAXIT_C = config.MAXIT_C if getattr(config, "MAXIT_C", 0) else 100
        self.MAXIT_T = config.MAXIT_T if getattr(config, "MAXIT_T", 0) else 100
        if config.FLUIDPROP:
            self.update_fluid_properties()
        # the reference's numba kernels freeze these globals at their first
        # call, i.e. after the initial EOS (tse.py:228-229)
        S = self.S
        self.M.freeze(S["c_r"], S["l_r"], S["rho_r"], S["cp_r"], S["lf_l"], S["lf_t"], S["lt_l"],
                      S["lt_t"], config.C_IMBLFLO, config.T_IMBLFLO)
        self.t_sim = getattr(config, "t_sim", 0)
        self.n_tsteps = 0
        self.log = []
        self.mass_log = []
        self.counters = dict(P=0, C=0, T=0)
        self.plots = Snapshots(config, plot_prefix if plot_prefix is not None
                               else getattr(config, "__name__", "tse"))

    # ------------------------------------------------------------ state I/O
    def upload_state(self, config):
        dev = dict(dtype=torch.float64, device=self.device)
        for name in FIELDS3:
            self.S[name] = torch.as_tensor(numpy.ascontiguousarray(getattr(config, name),
                                                                   dtype=numpy.float64), **dev)
        for name in FIELDS4:
            a = numpy.asarray(getattr(config, name), dtype=numpy.float64)
            self.S[name] = torch.as_tensor(numpy.ascontiguousarray(numpy.moveaxis(a, 3, 0)), **dev)
        T = numpy.asarray(config.T, dtype=numpy.float64)
        if T.ndim == 4:
            T = numpy.moveaxis(T, 3, 0)
        self.S["T"] = torch.as_tensor(numpy.ascontiguousarray(T), **dev)

    def swap_state(self, S):
        """Make ``S`` (a dict of device tensors with the names, shapes and
        dtypes of ``self.S``) the model's state and return the previous one.
        A caller that streams inputs from the host can then fill one set of
        buffers on a copy stream while the other set steps: later ``run``
        calls read and write ``S``."""
        if set(S) != set(self.S):
            raise ValueError("swap_state: the state names differ")
        for n, t in S.items():
            o = self.S[n]
            if t.shape != o.shape or t.dtype != o.dtype or t.device != o.device:
                raise ValueError("swap_state: %s differs in shape, dtype or device" % n)
        old, self.S = self.S, S
        return old

    def field(self, name):
        """One field as a NumPy array in the reference layout."""
        t = self.S[name].detach().cpu().numpy()
        if name in FIELDS4 or (name == "T" and t.ndim == 4):
            t = numpy.moveaxis(t, 0, 3)
        return numpy.ascontiguousarray(t)

    # ------------------------------------------------------------------ EOS
    def update_fluid_properties(self):
        """tse.py:208-225 (layer 0 of an NLTE temperature is the fluid)."""
        S = self.S
        T0 = S["T"][0] if self.nlte else S["T"]
        if self.eos is not None:
            _eos.apply(self.M, self.eos, S, T0)
        else:
            _eos.host_callback(self, T0)

    # ----------------------------------------------------------------- loop
    def snapshot(self, dt):
        """The snapshot tuple of the current state (host copies)."""
        cfg = self.config
        v = dict(lx=cfg.lx, ly=cfg.ly, lz=cfg.lz, nx=self.shape[0], ny=self.shape[1],
                 nz=self.shape[2], dx=cfg.dx, dy=cfg.dy, dz=cfg.dz, t_sim=self.t_sim, dt=dt,
                 mass=getattr(self, "mass", cfg.mass))
        return tuple(v[k] if k in v else self.field(k) for k in SNAPSHOT_ITEMS)

    def _init_loop(self):
        cfg, S = self.config, self.S
        self._L = dict(dt_max=cfg.dt_max, dt=cfg.dt, dt_P=None, dt_C=None, dt_T=None, num_CFL=0,
                       pe=(0.0,) * 6)
        # tse.py:1121 and the call before the loop, tse.py:1177
        self._L["dt"], self._L["dt_prev"] = self.plots.step(self.t_sim, cfg.dt, cfg.dt,
                                                            self.snapshot)
        self._rhof_prev = torch.zeros_like(S["rho_f"])
        self._Cn = torch.empty_like(S["C"])
        self._Tn = torch.empty_like(S["T"])

    def run(self, max_steps=None, on_step=None):
        """Advance the model (resumable: a later call continues the run)."""
        cfg, M, S = self.config, self.M, self.S
        if not hasattr(self, "_L"):
            self._init_loop()
        Ls = self._L
        t = cfg.t
        dt_max = Ls["dt_max"]
        cmax_dt = cfg.dt_max
        dt_max_abs = cfg.dt_max
        dt, dt_prev = Ls["dt"], Ls["dt_prev"]
        dt_P, dt_C, dt_T = Ls["dt_P"], Ls["dt_C"], Ls["dt_T"]
        num_CFL = Ls["num_CFL"]
        rhof_prev = self._rhof_prev
        Pn = M.Pn_buf
        Cn = self._Cn
        Tn = self._Tn
        Pex_T, Pey_T, Pez_T, Pex_C, Pey_C, Pez_C = Ls["pe"]
        steps_here = 0
        while self.t_sim < t:
            SIA_filled = False
            SIA_iter = 0
            while not SIA_filled and SIA_iter < cfg.SIA_maxit:
                Co_Filled = False
                CFL = 0
                if cfg.OMEGA_C == 0:
                    dt_NeC = M.explicit_C([S["D_fx"][s] for s in range(S["D_fx"].shape[0])],
                                          S["phi"])
                num_it_P = 0
                if cfg.FLUIDFLOW:
                    while not Co_Filled:
                        dt, dt_P, P, Pn, conv, num_it_P = M.compute_P(
                            S["P"], S["c_f"], S["nue"], S["rho_f"], S["phi"], S["Kx"], S["Ky"],
                            S["Kz"], S["qx"], S["qy"], S["qz"], dt, S["BP"], S["WP"],
                            max_dt=dt_max, inc_it=1.25, SOR=cfg.SOR_P, max_it=self.MAXIT_P,
                            P_conv=cfg.CONV_P)
                        self._halving_log("P", M.last_status)
                        if not conv:
                            raise ConvergenceError("* P CONVERGENCE ERROR - check dt and CONV_P in compute_P")
                        M.compute_q(S["P"], S["BP"], S["Kx"], S["Ky"], S["Kz"], S["qx"], S["qy"],
                                    S["qz"], S["nue"], S["rho_f"])
                        if cfg.HEATTRANS or cfg.SPECTRANS:
                            M.flow_error(S["P"], Pn, S["qx"], S["qy"], S["qz"], S["WP"], S["phi"],
                                         S["c_f"], S["c_r"], S["rho_f"], dt, out=S["e"])
                        printing = self.verbose and self.n_tsteps % cfg.PRINTOUT == 0
                        if self.t_sim > 0 and (not cfg.SIA or printing):
                            # with SIA on, dt_CFL only feeds the printout
                            dt_CFL = M.dt_cfl(S["qx"], S["qy"], S["qz"], S["phi"])
                        else:
                            dt_CFL = 1e10
                        dt_max_C = dt_max_T = dt_max_P = dt_max_abs
                        if printing and cfg.HEATTRANS:
                            Pex_T, Pey_T, Pez_T = M.peclet_T(S["qx"], S["qy"], S["qz"], S["rho_f"],
                                                             S["cp_f"], S["phi"], S["l_r"],
                                                             S["l_f"], S["BT"])
                        if printing and cfg.SPECTRANS:
                            ns = S["D_fx"].shape[0]
                            Pex_C, Pey_C, Pez_C = M.peclet_C(
                                S["qx"], S["qy"], S["qz"], [S["D_fx"][s] for s in range(ns)],
                                [S["D_fy"][s] for s in range(ns)], [S["D_fz"][s] for s in range(ns)],
                                S["BC"])
                        if cfg.OMEGA_C == 0:
                            dt_max_C = dt_NeC
                        if cfg.SIA:
                            dt_max = pymin(dt_max_C, dt_max_T, dt_max_P)
                        else:
                            dt_max = pymin(dt_CFL, dt_max_C, dt_max_T, dt_max_P)
                        if printing:
                            self._print_flow(cfg, dt, dt_CFL, dt_max_C, dt_max_T,
                                             (Pex_T, Pey_T, Pez_T, Pex_C, Pey_C, Pez_C))
                        Co_Filled = True
                        if dt > dt_max * 1.0:
                            num_CFL += num_it_P
                            CFL += 1
                            dt = dt_max
                num_it_C = 0
                if cfg.SPECTRANS:
                    Cn.copy_(S["C"])
                    # skip test of tse.py:1300-1301; a species' solve changes no
                    # other species, so all sums are taken up front (one sync)
                    sp = [int(n) for n in cfg.SPTRANS]
                    sums = M.sums([S["C"][n] for n in sp] + [S["WC"][n] for n in sp])
                    for q, n in enumerate(sp):
                        Cv = S["C"][n]
                        if sums[q] != 0.0 or sums[len(sp) + q] != 0.0:
                            Ds = (S["D_fx"][n], S["D_fy"][n], S["D_fz"][n])
                            dt, dt_C, _, conv, it = M.compute_C(
                                Cv, *Ds, S["phi"], S["rho_f"], S["qx"], S["qy"], S["qz"], dt,
                                S["BC"], S["WC"][n], S["R"], S["e"], omega=cfg.OMEGA_C,
                                SOR=cfg.SOR_C, max_it=self.MAXIT_C, max_dt=cmax_dt,
                                C_conv=cfg.CONV_C)
                            self._halving_log("C", M.last_status)
                            num_it_C += it
                            if not conv:
                                raise ConvergenceError("* C CONVERGENCE ERROR- check dt and C_conv in compute_C")
                            if cfg.SMOLAR_C:
                                M.smolarkiewicz(Cv, S["qx"], S["qy"], S["qz"], S["vx"], S["vy"],
                                                S["vz"], dt, eps=1e-15, Sc=1.08)
                                dt, dt_C, _, conv, it = M.compute_C(
                                    Cv, *Ds, S["phi"], S["rho_f"], S["vx"], S["vy"], S["vz"], dt,
                                    S["BC"], S["WC"][n], S["R"], self.ZEROS, omega=cfg.OMEGA_C,
                                    max_it=self.MAXIT_C, SOR=cfg.SOR_C, max_dt=cmax_dt,
                                    C_conv=cfg.CONV_C)
                                self._halving_log("C", M.last_status)
                                num_it_C += it
                                if not conv:
                                    raise ConvergenceError("* C2 CONVERGENCE ERROR- check dt and C_conv in compute_C")
                num_it_T = 0
                if cfg.HEATTRANS:
                    Tn.copy_(S["T"])
                    if self.nlte:
                        dt, dt_T, _, conv, it1 = M.compute_T(
                            S["T"][0], S["l_f"], S["cp_f"], S["rho_f"], self.ONES, S["qx"], S["qy"],
                            S["qz"], dt, S["BT"], self.ZEROS, S["e"], omega=cfg.OMEGA_T,
                            max_it=self.MAXIT_T, SOR=cfg.SOR_T, max_dt=cmax_dt, T_conv=cfg.CONV_T)
                        self._halving_log("T", M.last_status)
                        dt, dt_T, _, conv, it2 = M.compute_T(
                            S["T"][1], self.ZEROS, self.ZEROS, self.ZEROS, self.ZEROS, S["qx"],
                            S["qy"], S["qz"], dt, S["BT"], S["WT"], S["e"], omega=cfg.OMEGA_T,
                            max_it=self.MAXIT_T, SOR=cfg.SOR_T, max_dt=cmax_dt, T_conv=cfg.CONV_T)
                        self._halving_log("T", M.last_status)
                        num_itT = it1 + it2
                    else:
                        dt, dt_T, _, conv, num_itT = M.compute_T(
                            S["T"], S["l_f"], S["cp_f"], S["rho_f"], S["phi"], S["qx"], S["qy"],
                            S["qz"], dt, S["BT"], S["WT"], S["e"], omega=cfg.OMEGA_T,
                            max_it=self.MAXIT_T, SOR=cfg.SOR_T, max_dt=cmax_dt, T_conv=cfg.CONV_T)
                        self._halving_log("T", M.last_status)
                    num_it_T += num_itT
                    if not conv:
                        raise ConvergenceError("* T CONVERGENCE ERROR - check dt and T_conv in compute_T")
                    if cfg.SMOLAR_T:
                        M.smolarkiewicz(S["T"], S["qx"], S["qy"], S["qz"], S["vx"], S["vy"],
                                        S["vz"], dt, eps=1e-15, Sc=1.08)
                        dt, dt_T, _, conv, num_itT = M.compute_T(
                            S["T"], S["l_f"], S["cp_f"], S["rho_f"], S["phi"], S["vx"], S["vy"],
                            S["vz"], dt, S["BT"], S["WT"], self.ZEROS, omega=cfg.OMEGA_T,
                            max_it=self.MAXIT_T, SOR=cfg.SOR_T, max_dt=cmax_dt, T_conv=cfg.CONV_T)
                        self._halving_log("T", M.last_status)
                        num_it_T += num_itT
                        if not conv:
                            raise ConvergenceError("* T CONVERGENCE ERROR - check dt and T_conv in compute_T")
                if cfg.CHEMREACT:
                    self._chemistry(dt)
                if cfg.FLUIDPROP:
                    self.update_fluid_properties()
                if cfg.SIA:
                    SIA_diff = M.l2_norm(S["rho_f"], rhof_prev, "rhof")
                    if self.verbose and self.n_tsteps % cfg.PRINTOUT == 0:
                        print(" [SIA] %4d [SIA] %6.2e" % (SIA_iter, SIA_diff))
                    if SIA_diff < cfg.SIA_conv or SIA_iter == cfg.SIA_maxit - 1:
                        SIA_filled = True
                    else:
                        rhof_prev.copy_(S["rho_f"])
                        S["P"].copy_(Pn)
                        if cfg.HEATTRANS:
                            S["T"].copy_(Tn)
                        if cfg.SPECTRANS:
                            S["C"].copy_(Cn)
                        SIA_iter += 1
                else:
                    SIA_filled = True
                    if self.verbose and self.n_tsteps % cfg.PRINTOUT == 0:
                        print("")
                self.counters["P"] += num_it_P
                self.counters["C"] += num_it_C
                self.counters["T"] += num_it_T
            rec = dict(step=self.n_tsteps + 1, dt=dt, t_sim=self.t_sim,
                       numitP=self.counters["P"], numitC=self.counters["C"],
                       numitT=self.counters["T"], num_CFL=num_CFL,
                       dt_P=dt_P if dt_P is not None else float("nan"),
                       dt_C=dt_C if dt_C is not None else float("nan"),
                       dt_T=dt_T if dt_T is not None else float("nan"))
            self.log.append(rec)
            if cfg.DYNAMICBC:
                self._dynamic_bc(dt)
            if cfg.MASSBALAN or getattr(cfg, "GPU_MASSBAL", False):
                self._mass_balance(dt)
            if on_step is not None:
                on_step(rec, self)
            self.t_sim += dt
            self.n_tsteps += 1
            steps_here += 1
            if self.verbose and self.n_tsteps % cfg.PRINTOUT == 0:
                # tse.py:1481-1484, bold dt included
                print("[t] %8.2e/%8.2e [dt] \033[1m%8.2e\033[0m [S] %4d [P] %3d"
                      % (self.t_sim, t, dt, self.n_tsteps, num_it_P)
                      + " [C] %3d [T] %3d [CFL] %d" % (num_it_C, num_it_T, CFL))
            dt = 1e99
            if cfg.FLUIDFLOW:
                dt = pymin(dt_P, t - self.t_sim)
            if cfg.HEATTRANS:
                dt = pymin(dt_T, t - self.t_sim, dt)
            if cfg.SPECTRANS:
                if dt_C is None:
                    # the reference stops with NameError here (tse.py:1490-1491)
                    raise RuntimeError("name 'dt_C' is not defined: no species was transported "
                                       "in the first step (the reference stops here as well)")
                dt = pymin(dt_C, t - self.t_sim, dt)
            dt, dt_prev = self.plots.step(self.t_sim, dt, dt_prev, self.snapshot)   # tse.py:1494
            if max_steps is not None and steps_here >= max_steps:
                break
        Ls.update(dt_max=dt_max, dt=dt, dt_prev=dt_prev, dt_P=dt_P, dt_C=dt_C, dt_T=dt_T,
                  num_CFL=num_CFL, pe=(Pex_T, Pey_T, Pez_T, Pex_C, Pey_C, Pez_C))
        return self

    # -------------------------------------------------------------- hooks
    def _dynamic_bc(self, dt):
        """dynamic_bc host hook (tse.py:1448-1458): fields go to the host and back."""
        cfg = self.config
        names = ("P", "T", "C", "BP", "BT", "BC", "WP", "WT", "WC", "Kx", "Ky", "Kz", "rho_f",
                 "nue", "c_f", "cp_f", "qx", "phi", "l_f", "l_r")
        h = {n: self.field(n) for n in names}
        bc_inc = getattr(self, "_bc_inc", 0)
        out = cfg.dynamic_bc(self.t_sim + dt, bc_inc, *[h[n] for n in names])
        new_inc = out[0]
        for n, v in zip(("P", "T", "C", "BP", "BT", "BC", "WP", "WT", "WC", "Kx", "Ky", "Kz"),
                        out[1:]):
            a = numpy.asarray(v, dtype=numpy.float64)
            if n in FIELDS4 or (n == "T" and a.ndim == 4):
                a = numpy.moveaxis(a, 3, 0)
            self.S[n].copy_(torch.as_tensor(numpy.ascontiguousarray(a)))
        self._bc_inc = new_inc
        if new_inc != bc_inc and cfg.FLUIDPROP:
            self.update_fluid_properties()

    def _chemistry(self, dt):
        """Chemistry coupling (tse.py:1383-1417), a host hook once per Picard
        iteration: chem_inc accumulates dt (after the first step); when it
        reaches DTCHEM (and in the first step) the state goes to the host, the
        config's chemical_reactions_all runs on it -- or chemical_reactions on
        each cell whose BC is not 1, k-j-i order, through joblib with
        parallel_chemistry jobs -- and the results come back to the device."""
        cfg = self.config
        st = self.__dict__.setdefault("_chem", {"inc": 0, "dt_chem": 0})
        if self.t_sim > 0:
            st["inc"] += dt
        else:
            st["inc"] = 0
            st["dt_chem"] = dt
        if st["inc"] >= cfg.DTCHEM:
            st["dt_chem"] = st["inc"]
            st["inc"] = 0
        if st["inc"] != 0:
            return
        BC = self.field("BC")
        kk, jj, ii = numpy.nonzero(numpy.transpose(BC != 1, (2, 1, 0)))   # k, j, i order
        if len(ii) == 0:
            return
        names = ("C", "P", "T", "rho_f", "phi", "Kx", "Ky", "Kz")
        h = {n: self.field(n) for n in names}
        if hasattr(cfg, "chemical_reactions_all"):
            out = cfg.chemical_reactions_all(*[h[n] for n in names], st["dt_chem"])
            h = dict(zip(names, out))
        else:
            from joblib import Parallel, delayed
            cells = list(zip(ii.tolist(), jj.tolist(), kk.tolist()))
            res = Parallel(n_jobs=cfg.parallel_chemistry)(
                delayed(cfg.chemical_reactions)(*[h[n][i, j, k] for n in names], st["dt_chem"],
                                                i, j, k) for i, j, k in cells)
            for (i, j, k), r in zip(cells, res):
                for n, v in zip(names, r):
                    h[n][i, j, k] = v
        for n in names:
            a = numpy.asarray(h[n], dtype=numpy.float64)
            if n in FIELDS4 or (n == "T" and a.ndim == 4):
                a = numpy.moveaxis(a, 3, 0)
            self.S[n].copy_(torch.as_tensor(numpy.ascontiguousarray(a)))

    def _mass_balance(self, dt):
        """Mass balance at the point of tse.py:1460-1463: FP64 device totals
        (water, species, heat and their source rates) appended to
        ``mass_log``; a config's own mass_balance callback, when MASSBALAN is
        set, is called as the reference calls it, on host copies."""
        S, cfg = self.S, self.config
        T0 = S["T"][0] if self.nlte else S["T"]
        ns = S["C"].shape[0]
        tot = self.M.mass_totals(S["phi"], S["rho_f"], S["R"], [S["C"][s] for s in range(ns)],
                                 [S["WC"][s] for s in range(ns)], T0, S["cp_f"], S["rho_r"],
                                 S["cp_r"], S["WP"], S["WT"])
        self.mass_log.append({"t": self.t_sim + dt, "dt": dt, "water": tot[0],
                              "species": tot[1:1 + ns].copy(), "heat": tot[1 + ns],
                              "water_source": tot[2 + ns], "species_source": tot[3 + ns:3 + 2 * ns].copy(),
                              "heat_source": tot[3 + 2 * ns]})
        if cfg.MASSBALAN and hasattr(cfg, "mass_balance"):
            f = self.field
            self.mass = cfg.mass_balance(f("C"), f("qx"), f("qy"), f("qz"), f("WP"), f("WC"),
                                         f("WT"), f("D_fx"), f("D_fy"), f("D_fz"), dt,
                                         getattr(self, "mass", numpy.array(cfg.mass, copy=True)))

    def _halving_log(self, which, s):
        if not self.verbose or s is None or s.n_events == 0:
            return
        for q in range(s.n_events):
            if which == "P":
                print(" t:", 0, "P [", s.ev_it[q], "]: Reducing dt:", s.ev_dt[q], "=>",
                      s.ev_dt[q] / 2, "(s) L2:", s.ev_diff[q])
            else:
                print("\n  [%s] [iter %5d] [dt/s %6.2e -> %6.2e] [L2 %6.2e]"
                      % (which, s.ev_it[q], s.ev_dt[q], s.ev_dt[q] / 2, s.ev_diff[q]), end="")

    def _print_flow(self, cfg, dt, dt_CFL, dt_max_C, dt_max_T, pe):
        M, S = self.M, self.S
        if cfg.OMEGA_C + cfg.OMEGA_T < 2:
            print(" [dt_NeC] %8.2e [dt_NeT] %8.2e" % (dt_max_C, dt_max_T))
        print(" [CFL] %6.2f%% | Pe_T %.1e/%.1e/%.1e | Pe_C %.1e/%.1e/%.1e"
              % ((dt / dt_CFL * 100,) + tuple(pe)))
        _, pmax, pmin = M.field_stats(S["P"])
        _, tmax, tmin = M.field_stats(S["T"])
        _, cmax, cmin = M.field_stats(S["C"])
        print("[P+] %6.2e [P-] %6.2e [T+] %6.4f [T-] %6.4f" % (pmax, pmin, tmax, tmin)
              + " [C+] %6.4f [C-] %6.4f" % (cmax, cmin), end="")


def main(argv=None):
    """CLI: python -m transportse_b200 <config.py> [--steps N]"""
    import argparse
    import importlib.util
    import os
    ap = argparse.ArgumentParser(prog="transportse_b200")
    ap.add_argument("config")
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--quiet", action="store_true")
    a = ap.parse_args(argv)
    path = os.path.abspath(a.config)
    sys.path.append(os.path.dirname(path))
    spec = importlib.util.spec_from_file_location(os.path.basename(path)[:-3], path)
    cfg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(cfg)
    # snapshots next to the config file, named like the reference's
    sim = Simulation(cfg, verbose=not a.quiet, plot_prefix=path[:-3])
    sim.run(max_steps=a.steps)
    print("[ SIMULATION SUMMARY ]")
    print("[t/s] %8.2e/%8.2e [S] %5d [P] %5d [C] %5d [T] %5d"
          % (sim.t_sim, cfg.t, sim.n_tsteps, sim.counters["P"], sim.counters["C"],
             sim.counters["T"]))
    return sim
