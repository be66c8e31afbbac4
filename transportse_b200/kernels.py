"""Reference-named kernel front end over torch CUDA tensors.

``Model`` binds one grid (the globals a TRANSPORTSE config defines: nx, ny,
nz, dx, dy, dz, g, beta) plus the values the reference's numba kernels freeze
at their first call (c_r in compute_P; l_r, rho_r, cp_r, lt_l, lt_t and
T_IMBLFLO in compute_T; lf_l, lf_t and C_IMBLFLO in compute_C), and exposes
the reference kernels under their own names and argument lists:

    compute_P     tse.py:647     compute_q   tse.py:744
    flow_error    tse.py:409     compute_C   tse.py:783
    compute_T     tse.py:919     smolarkiewicz tse.py:1083
    l2_norm       tse.py:273     explicit_C  tse.py:385
    peclet_C/_T   tse.py:331/357 dt_cfl      tse.py:1241-1249

Arrays are float64 CUDA tensors in the reference's (nx, ny, nz) C order.
Every call goes to libtsecuda.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as ct
import math

import numpy
import torch

from . import _native as N


def _sin_cos_beta(beta_deg):
    b = float(numpy.radians(beta_deg))
    return math.sin(b), math.cos(b)


class Model:
    PRECISIONS = ("fp64", "fp32dc")

    def __init__(self, nx, ny, nz, dx, dy, dz, g, beta_deg, device=None, precision="fp64",
                 dc_cycle=256):
        """precision 'fp64': the reference's arithmetic, operation for
        operation; 'fp32dc': FP32 sweeps on a correction driven by an FP64
        residual (tse_compute_*_dc), same convergence test and dt control."""
        if precision not in self.PRECISIONS:
            raise ValueError("precision must be one of %s" % (self.PRECISIONS,))
        self.precision = precision
        self.dc_cycle = int(dc_cycle)
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.type != "cuda":
            raise RuntimeError("transportse_b200 kernels run on CUDA devices only")
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.n = self.nx * self.ny * self.nz
        f64 = dict(dtype=torch.float64, device=self.device)
        self.dx = torch.as_tensor(numpy.array(dx, dtype=numpy.float64), **f64)
        self.dy = torch.as_tensor(numpy.array(dy, dtype=numpy.float64), **f64)
        self.dz = torch.as_tensor(numpy.array(dz, dtype=numpy.float64), **f64)
        self.g = float(g)
        self.sinb, self.cosb = _sin_cos_beta(beta_deg)
        self.grid = N.TseGrid(self.nx, self.ny, self.nz, 0, self.dx.data_ptr(),
                              self.dy.data_ptr(), self.dz.data_ptr(), self.g, self.sinb,
                              self.cosb)
        L = N.lib()
        gp = ct.byref(self.grid)
        kinds = (N.TSE_WS_PRESSURE, N.TSE_WS_TRANSPORT, N.TSE_WS_REDUCE)
        if precision == "fp32dc":
            kinds += (N.TSE_WS_PRESSURE_DC, N.TSE_WS_TRANSPORT_DC)
        self.ws_bytes = max(L.tse_workspace_bytes(gp, k) for k in kinds)
        self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device=self.device)
        self.red_ws = torch.empty(L.tse_workspace_bytes(gp, N.TSE_WS_REDUCE), dtype=torch.uint8,
                                  device=self.device)
        self.status = torch.zeros(ct.sizeof(N.TseSolveStatus), dtype=torch.uint8, device=self.device)
        self.scal = torch.zeros(8, **f64)
        self.Pn_buf = torch.empty((self.nx, self.ny, self.nz), **f64)
        self.frozen = {}
        self.C_IMBLFLO = False
        self.T_IMBLFLO = False
        self.last_status = None
        self.launches = 0
        # FP64 solves' sweep kernel (args.sweep): 0 the bulk-copy staged
        # kernel where its stages fit, 1 plain loads; same cell values
        self.sweep = 0
        # mixed-precision solves: the staged FP32 sweep's variant (chunk
        # cells, ring stages, pipelines per block; 0 = the library's
        # default), chosen per grid by transportse_b200.autotune; the last
        # solve's variant as it ran
        self.sweep_variant = (0, 0, 0)
        self.last_variant = None
        # optional per-solve timing: list of (kind, start event, end event,
        # status) appended by the solver entry points when enabled
        self.timing = False
        self.timed = []
        self.sweep_timed = []
        # cell-updates = active cells relaxed once per red+black iteration
        self.cell_updates = {"P": 0, "C": 0, "T": 0}

    @classmethod
    def from_config(cls, config, device=None, precision=None):
        if precision is None:
            precision = getattr(config, "GPU_PRECISION", "fp64")
        return cls(config.nx, config.ny, config.nz, config.dx, config.dy, config.dz, config.g,
                   config.beta, device=device, precision=precision,
                   dc_cycle=getattr(config, "GPU_DC_CYCLE", 256))

    # FP32 corrections resolve a relative change of about 1e-13 of the FP64
    # iterate at best; a solve asking for a tighter tolerance runs in FP64
    DC_MIN_CONV = 1e-13

    def _solve(self, name, args_struct, conv):
        """Call tse_<name> or its mixed-precision form tse_<name>_dc."""
        L = N.lib()
        if self.precision == "fp32dc" and conv >= getattr(self, "dc_min_conv", self.DC_MIN_CONV):
            gate = getattr(self, "batch_gate", None)
            if gate is not None:
                # batched with the other models' solves (transportse_b200.batch)
                gate.submit(name, self.grid, args_struct, self.status, self.ws, self.ws_bytes,
                            self.dc_cycle)
                return
            if self.n <= self.cluster_cells:
                # small grid: the whole solve as one launch of one thread-block
                # cluster, no device-wide barriers and no host round trips,
                # leaving the rest of the GPU to other streams
                self._solve_cluster(name, args_struct)
                return
            opts = N.TseDcOptions(self.dc_cycle, getattr(self, "max_blocks", 0), int(self.timing))
            opts.chunk, opts.ring, opts.pipes = self.sweep_variant
            rc = getattr(L, "tse_%s_dc" % name)(ct.byref(self.grid), ct.byref(args_struct),
                                                ct.byref(opts), self._p(self.status),
                                                self._p(self.ws), self.ws_bytes, self._stream())
            self.last_variant = (opts.chunk, opts.ring, opts.pipes)
            if self.timing:
                # per sweep-kernel timing of this solve: (kind, launches,
                # red+black iterations, event ms)
                self.sweep_timed.append((name[-1], opts.sweep_launches, opts.sweep_iterations,
                                         opts.sweep_ms))
        else:
            rc = getattr(L, "tse_" + name)(ct.byref(self.grid), ct.byref(args_struct),
                                           self._p(self.status), self._p(self.ws), self.ws_bytes,
                                           self._stream())
        N.check(rc, "tse_" + name)

    # grids of up to this many cells solve in one cluster launch (0: never);
    # cluster_size CTAs per cluster (0: library default)
    cluster_cells = 0
    cluster_size = 16

    def _solve_cluster(self, name, args_struct):
        L = N.lib()
        bws = self.__dict__.get("_cluster_ws")
        if bws is None:
            bws = self._cluster_ws = torch.empty(int(L.tse_batch_workspace_bytes(1, self.n)),
                                                 dtype=torch.uint8, device=self.device)
        Item = N.BATCH_ITEM[name]
        items = (Item * 1)(Item(ct.pointer(self.grid), ct.pointer(args_struct),
                                self._p(self.status), self._p(self.ws), self.ws_bytes))
        opts = N.TseDcOptions(self.dc_cycle, int(self.cluster_size), 0)
        rc = getattr(L, "tse_%s_dc_batch" % name)(items, 1, ct.byref(opts), self._p(bws),
                                                  bws.numel(), self._stream())
        N.check(rc, "tse_%s_dc_batch" % name)

    # ----------------------------------------------------------- helpers
    def _t(self, a):
        """Check (or convert) an argument to a contiguous float64 device tensor."""
        if isinstance(a, torch.Tensor):
            if a.device != self.device or a.dtype != torch.float64 or not a.is_contiguous():
                a = a.to(device=self.device, dtype=torch.float64).contiguous()
            return a
        return torch.as_tensor(numpy.ascontiguousarray(a, dtype=numpy.float64),
                               device=self.device)

    @staticmethod
    def _p(t):
        return ct.c_void_p(t.data_ptr())

    def _stream(self):
        return ct.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def freeze(self, c_r, l_r, rho_r, cp_r, lf_l, lf_t, lt_l, lt_t, C_IMBLFLO, T_IMBLFLO):
        """Snapshot the globals the reference kernels freeze at first call."""
        for k, v in dict(c_r=c_r, l_r=l_r, rho_r=rho_r, cp_r=cp_r, lf_l=lf_l, lf_t=lf_t,
                         lt_l=lt_l, lt_t=lt_t).items():
            self.frozen[k] = self._t(v).clone()
        self.C_IMBLFLO = bool(C_IMBLFLO)
        self.T_IMBLFLO = bool(T_IMBLFLO)

    def _ev_start(self):
        if not self.timing:
            return None
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.current_stream(self.device))
        return e0

    def _ev_end(self, e0):
        if e0 is None:
            return None
        e1 = torch.cuda.Event(enable_timing=True)
        e1.record(torch.cuda.current_stream(self.device))
        return (e0, e1)

    def _account(self, kind, B, s, ev):
        key = (kind, B.data_ptr())
        cache = self.__dict__.setdefault("_active_cache", {})
        if key not in cache or cache[key][0] is not B:
            cache[key] = (B, int((B == 0).sum().item()))
        self.cell_updates[kind] += int(s.num_it) * cache[key][1]
        if ev is not None:
            self.timed.append((kind, ev[0], ev[1], int(s.num_it), cache[key][1]))

    def read_status(self):
        s = N.TseSolveStatus.from_buffer_copy(self.status.cpu().numpy().tobytes())
        self.last_status = s
        if s.error != 0:
            raise RuntimeError("solver kernel stopped: grid barrier wait timed out")
        return s

    # ----------------------------------------------------------- kernels
    def compute_P(self, P, c_f, nue, rho_f, phi, Kx, Ky, Kz, qx, qy, qz, dt_P, BP, WP, SOR=1.0,
                  max_it=20000, inc_it=1.05, max_dt=1e6, min_dt=1e-8, P_conv=1e-10):
        """compute_P (tse.py:647-742).  P is updated in place; the returned
        Pn is a buffer owned by the model, overwritten by the next call."""
        P = self._t(P)
        a = N.TsePressureArgs()
        a.P = P.data_ptr()
        a.Pn = self.Pn_buf.data_ptr()
        keep = [self._t(x) for x in (c_f, nue, rho_f, phi, Kx, Ky, Kz)]
        for name, t in zip(("c_f", "nue", "rho_f", "phi", "Kx", "Ky", "Kz"), keep):
            setattr(a, name, t.data_ptr())
        a.c_r = self.frozen["c_r"].data_ptr()
        BPt, WPt = self._t(BP), self._t(WP)
        a.BP, a.WP = BPt.data_ptr(), WPt.data_ptr()
        a.dt_P, a.SOR, a.inc_it, a.max_dt, a.min_dt, a.P_conv = (
            float(dt_P), float(SOR), float(inc_it), float(max_dt), float(min_dt), float(P_conv))
        a.max_it = int(max_it)
        a.sweep = int(self.sweep)
        ev = self._ev_start()
        self._solve("compute_P", a, a.P_conv)
        self.launches += 3
        ev = self._ev_end(ev)
        s = self.read_status()
        self._account("P", BPt, s, ev)
        return s.t, s.dt, P, self.Pn_buf, bool(s.converged), int(s.num_it)

    def compute_q(self, P, BP, Kx, Ky, Kz, qx, qy, qz, nue, rho_f):
        """compute_q (tse.py:744-780); qx, qy, qz are updated in place."""
        qx, qy, qz = self._t(qx), self._t(qy), self._t(qz)
        args = [self._t(x) for x in (P, BP, Kx, Ky, Kz)]
        n2 = [self._t(nue), self._t(rho_f)]
        rc = N.lib().tse_compute_q(ct.byref(self.grid), *[self._p(x) for x in args],
                                   self._p(qx), self._p(qy), self._p(qz),
                                   *[self._p(x) for x in n2], self._stream())
        N.check(rc, "tse_compute_q")
        self.launches += 1
        return qx, qy, qz

    def flow_error(self, P, Pn, qx, qy, qz, WP, phi, c_f, c_r, rho_f, dt_P, out=None):
        """flow_error (tse.py:409-446); returns e (written into ``out`` if given)."""
        args = [self._t(x) for x in (P, Pn, qx, qy, qz, WP, phi, c_f, c_r, rho_f)]
        e = out if out is not None else torch.empty_like(args[0])
        rc = N.lib().tse_flow_error(ct.byref(self.grid), *[self._p(x) for x in args],
                                    float(dt_P), self._p(e), self._stream())
        N.check(rc, "tse_flow_error")
        self.launches += 1
        return e

    def compute_C(self, C, D_fx, D_fy, D_fz, phi, rho_f, qx, qy, qz, dt_C, BC, WC, RC, e,
                  omega=1, SOR=1.0, max_it=100, inc_it=1.05, max_dt=1e6, min_dt=1e-8,
                  C_conv=1e-10):
        """compute_C (tse.py:783-916); C (one species) is updated in place."""
        C = self._t(C)
        a = N.TseSpeciesArgs()
        a.C = C.data_ptr()
        keep = [self._t(x) for x in (D_fx, D_fy, D_fz, phi, rho_f, qx, qy, qz, BC, WC, RC, e)]
        for name, t in zip(("D_fx", "D_fy", "D_fz", "phi", "rho_f", "qx", "qy", "qz", "BC", "WC",
                            "RC", "e"), keep):
            setattr(a, name, t.data_ptr())
        a.l_l = self.frozen["lf_l"].data_ptr()
        a.l_t = self.frozen["lf_t"].data_ptr()
        a.dt, a.omega, a.SOR, a.inc_it, a.max_dt, a.min_dt, a.conv = (
            float(dt_C), float(omega), float(SOR), float(inc_it), float(max_dt), float(min_dt),
            float(C_conv))
        a.max_it = int(max_it)
        a.imblflo = int(self.C_IMBLFLO)
        a.sweep = int(self.sweep)
        ev = self._ev_start()
        self._solve("compute_C", a, a.conv)
        self.launches += 3
        ev = self._ev_end(ev)
        s = self.read_status()
        self._account("C", keep[8], s, ev)
        return s.t, s.dt, C, bool(s.converged), int(s.num_it)

    def compute_T(self, T, l_f, cp_f, rho_f, phi, qx, qy, qz, dt_T, BT, WT, e, omega=1, SOR=1.0,
                  max_it=100, inc_it=1.05, max_dt=1e6, min_dt=1e-8, T_conv=1e-10):
        """compute_T (tse.py:919-1081); T (one layer) is updated in place."""
        T = self._t(T)
        a = N.TseHeatArgs()
        a.T = T.data_ptr()
        keep = [self._t(x) for x in (l_f, cp_f, rho_f, phi, qx, qy, qz, BT, WT, e)]
        for name, t in zip(("l_f", "cp_f", "rho_f", "phi", "qx", "qy", "qz", "BT", "WT", "e"), keep):
            setattr(a, name, t.data_ptr())
        a.l_r = self.frozen["l_r"].data_ptr()
        a.rho_r = self.frozen["rho_r"].data_ptr()
        a.cp_r = self.frozen["cp_r"].data_ptr()
        a.l_l = self.frozen["lt_l"].data_ptr()
        a.l_t = self.frozen["lt_t"].data_ptr()
        a.dt, a.omega, a.SOR, a.inc_it, a.max_dt, a.min_dt, a.conv = (
            float(dt_T), float(omega), float(SOR), float(inc_it), float(max_dt), float(min_dt),
            float(T_conv))
        a.max_it = int(max_it)
        a.imblflo = int(self.T_IMBLFLO)
        a.sweep = int(self.sweep)
        ev = self._ev_start()
        self._solve("compute_T", a, a.conv)
        self.launches += 3
        ev = self._ev_end(ev)
        s = self.read_status()
        self._account("T", keep[7], s, ev)
        return s.t, s.dt, T, bool(s.converged), int(s.num_it)

    def smolarkiewicz(self, C, qx, qy, qz, vx, vy, vz, dt, eps=1e-15, Sc=1.08):
        """smolarkiewicz (tse.py:1083-1116); vx, vy, vz updated in place."""
        vx, vy, vz = self._t(vx), self._t(vy), self._t(vz)
        args = [self._t(x) for x in (C, qx, qy, qz)]
        rc = N.lib().tse_smolarkiewicz(ct.byref(self.grid), *[self._p(x) for x in args],
                                       self._p(vx), self._p(vy), self._p(vz), float(dt),
                                       float(eps), float(Sc), self._stream())
        N.check(rc, "tse_smolarkiewicz")
        self.launches += 1
        return vx, vy, vz

    def _scalar(self, k=0):
        return float(self.scal[k].item())

    def l2_norm(self, New, Old, Process=""):
        """l2_norm (tse.py:273-281), evaluated on the device in FP64."""
        New, Old = self._t(New), self._t(Old)
        rc = N.lib().tse_l2_norm(self._p(New), self._p(Old), New.numel(), self._p(self.scal),
                                 self._p(self.red_ws), self.red_ws.numel(), self._stream())
        N.check(rc, "tse_l2_norm")
        self.launches += 2
        return self._scalar()

    def dt_cfl(self, qx, qy, qz, phi):
        """CFL limit of the driver (tse.py:1241-1249), reshape semantics kept."""
        args = [self._t(x) for x in (qx, qy, qz, phi)]
        rc = N.lib().tse_dt_cfl(ct.byref(self.grid), *[self._p(x) for x in args],
                                self._p(self.scal), self._p(self.red_ws), self.red_ws.numel(),
                                self._stream())
        N.check(rc, "tse_dt_cfl")
        self.launches += 2
        return self._scalar()

    def _species_list(self, D):
        if isinstance(D, (list, tuple)):
            return [self._t(x) for x in D]
        D = self._t(D) if isinstance(D, torch.Tensor) else torch.as_tensor(
            numpy.ascontiguousarray(D, dtype=numpy.float64), device=self.device)
        if D.dim() == 4:   # reference layout (nx, ny, nz, S)
            return [D[..., s].contiguous() for s in range(D.shape[3])]
        return [D]

    def explicit_C(self, D_fx, phi):
        """explicit_C (tse.py:385-396); D_fx as (nx,ny,nz,S), (S,...) list or one array."""
        Ds = self._species_list(D_fx)
        arr = (ct.c_void_p * len(Ds))(*[x.data_ptr() for x in Ds])
        ph = self._t(phi)
        rc = N.lib().tse_explicit_C(ct.byref(self.grid), arr, len(Ds), self._p(ph),
                                    self._p(self.scal), self._p(self.red_ws), self.red_ws.numel(),
                                    self._stream())
        N.check(rc, "tse_explicit_C")
        self.launches += 2
        return self._scalar()

    def field_stats(self, x):
        """(sum, max, min) of a device field in FP64."""
        x = self._t(x)
        rc = N.lib().tse_field_stats(self._p(x), x.numel(), self._p(self.scal),
                                     self._p(self.red_ws), self.red_ws.numel(), self._stream())
        N.check(rc, "tse_field_stats")
        self.launches += 2
        v = self.scal[:3].cpu().numpy()
        return float(v[0]), float(v[1]), float(v[2])

    def sums(self, fields):
        """FP64 sums of several device fields with one host round trip."""
        out = torch.empty(3 * len(fields), dtype=torch.float64, device=self.device)
        for q, x in enumerate(fields):
            x = self._t(x)
            rc = N.lib().tse_field_stats(self._p(x), x.numel(), ct.c_void_p(out.data_ptr() + 24 * q),
                                         self._p(self.red_ws), self.red_ws.numel(), self._stream())
            N.check(rc, "tse_field_stats")
            self.launches += 2
        v = out.cpu().numpy()
        return [float(v[3 * q]) for q in range(len(fields))]

    def peclet_C(self, qx, qy, qz, D_fx, D_fy, D_fz, BC):
        Dx, Dy, Dz = self._species_list(D_fx), self._species_list(D_fy), self._species_list(D_fz)
        mk = lambda L: (ct.c_void_p * len(L))(*[x.data_ptr() for x in L])
        q = [self._t(x) for x in (qx, qy, qz)]
        B = self._t(BC)
        rc = N.lib().tse_peclet_C(ct.byref(self.grid), *[self._p(x) for x in q], mk(Dx), mk(Dy),
                                  mk(Dz), len(Dx), self._p(B), self._p(self.scal),
                                  self._p(self.red_ws), self.red_ws.numel(), self._stream())
        N.check(rc, "tse_peclet_C")
        self.launches += 2
        v = self.scal[:3].cpu().numpy()
        return float(v[0]), float(v[1]), float(v[2])

    def peclet_T(self, qx, qy, qz, rho_f, cp_f, phi, l_r, l_f, BT):
        args = [self._t(x) for x in (qx, qy, qz, rho_f, cp_f, phi, l_r, l_f, BT)]
        rc = N.lib().tse_peclet_T(ct.byref(self.grid), *[self._p(x) for x in args],
                                  self._p(self.scal), self._p(self.red_ws), self.red_ws.numel(),
                                  self._stream())
        N.check(rc, "tse_peclet_T")
        self.launches += 2
        v = self.scal[:3].cpu().numpy()
        return float(v[0]), float(v[1]), float(v[2])

    def mass_totals(self, phi, rho_f, RC, C_species, WC_species, T, cp_f, rho_r, cp_r, WP, WT):
        """FP64 totals: water, species (ns), heat, then the source rates of
        water, species (ns), heat -- see tse_mass_totals."""
        ns = len(C_species)
        mk = lambda L: (ct.c_void_p * max(1, len(L)))(*[x.data_ptr() for x in L])
        args = [self._t(x) for x in (phi, rho_f, RC)]
        rest = [self._t(x) for x in (T, cp_f, rho_r, cp_r, WP, WT)]
        out = torch.zeros(2 * ns + 4, dtype=torch.float64, device=self.device)
        rc = N.lib().tse_mass_totals(ct.byref(self.grid), *[self._p(x) for x in args],
                                     mk(C_species), mk(WC_species), ns,
                                     *[self._p(x) for x in rest], self._p(out),
                                     self._p(self.red_ws), self.red_ws.numel(), self._stream())
        N.check(rc, "tse_mass_totals")
        self.launches += 2
        return out.cpu().numpy()

    def eos_linear(self, C_species, T, rho_f, rho0, species_coeffs, tcoef, T0):
        """Declared linear EOS: rho_f = rho0 + sum a_s C_s - tcoef (T - T0)."""
        m = len(species_coeffs)
        if m > 8 or any(not (0 <= int(s) < len(C_species)) for s, _ in species_coeffs):
            raise ValueError("EOS species index out of range (or more than 8 terms)")
        ptrs = (ct.c_void_p * max(1, len(C_species)))(*[x.data_ptr() for x in C_species])
        sidx = (ct.c_int32 * max(1, m))(*[int(s) for s, _ in species_coeffs])
        coef = (ct.c_double * max(1, m))(*[float(a) for _, a in species_coeffs])
        Tt = self._t(T)
        rc = N.lib().tse_eos_linear(ct.byref(self.grid), ptrs, sidx, coef, m, self._p(Tt),
                                    float(rho0), float(tcoef), float(T0), self._p(rho_f),
                                    self._stream())
        N.check(rc, "tse_eos_linear")
        self.launches += 1
        return rho_f

    def eos_form(self, kind, coef, T, out, guard=None, guard_value=0.0):
        """Declared constant or fourth-order-in-T property (tse_eos_form):
        kind 'constant' (coef = value) or 'poly4_T' (coef = 5 coefficients,
        highest power first as numpy.polyfit returns them); cells where
        ``guard`` equals ``guard_value`` keep their value."""
        f = N.TseEosForm()
        if kind == "constant":
            f.kind = N.TSE_EOS_CONSTANT
            f.coef[0] = float(coef)
        elif kind == "poly4_T":
            c = [float(v) for v in coef]
            if len(c) != 5:
                raise ValueError("poly4_T takes 5 coefficients (numpy.polyfit order)")
            f.kind = N.TSE_EOS_POLY4_T
            for q in range(5):
                f.coef[q] = c[q]
        else:
            raise ValueError("unknown EOS form %r" % (kind,))
        f.guard_value = float(guard_value)
        Tt = self._t(T) if T is not None else None
        gt = self._t(guard) if guard is not None else None
        rc = N.lib().tse_eos_form(ct.byref(self.grid), ct.byref(f),
                                  self._p(Tt) if Tt is not None else None,
                                  self._p(gt) if gt is not None else None,
                                  self._p(out), self._stream())
        N.check(rc, "tse_eos_form")
        self.launches += 1
        return out
