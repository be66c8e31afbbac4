"""THE ORACLE -- test infrastructure, never the product path.

ctypes front end of ``tse_oracle.c`` (a CPU FP64 restatement of tse.py's
numba kernels).  ``OracleModel`` exposes the reference kernels under their own
names and argument lists (tse.py:273 l2_norm, 385 explicit_C, 409 flow_error,
647 compute_P, 744 compute_q, 783 compute_C, 919 compute_T, 1083
smolarkiewicz); the grid-wide values numba freezes at first compilation (dx,
dy, dz, g, beta, c_r, l_r, rho_r, cp_r, lf_*/lt_*, C_IMBLFLO/T_IMBLFLO) are
taken from the config module at construction, like the reference's globals.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm use this module.
"""
from __future__ import annotations

import ctypes as ct
import math
import os

import numpy

from . import build as _build

_lib = None
_dp = ct.POINTER(ct.c_double)


class OGrid(ct.Structure):
    _fields_ = [("nx", ct.c_int), ("ny", ct.c_int), ("nz", ct.c_int),
                ("dx", _dp), ("dy", _dp), ("dz", _dp),
                ("g", ct.c_double), ("sinb", ct.c_double), ("cosb", ct.c_double)]


class OPFields(ct.Structure):
    _fields_ = [(n, _dp) for n in ("c_f", "nue", "rho", "phi", "Kx", "Ky", "Kz",
                                   "c_r", "BP", "WP")]


class OCFields(ct.Structure):
    _fields_ = [(n, _dp) for n in ("Dfx", "Dfy", "Dfz", "phi", "rho", "qx", "qy",
                                   "qz", "BC", "WC", "RC", "e", "l_l", "l_t")] + \
               [("imblflo", ct.c_int)]


class OTFields(ct.Structure):
    _fields_ = [(n, _dp) for n in ("l_f", "cp_f", "rho", "phi", "qx", "qy", "qz",
                                   "BT", "WT", "e", "l_r", "rho_r", "cp_r", "l_l",
                                   "l_t")] + [("imblflo", ct.c_int)]


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = ct.CDLL(path)
        L.og_l2_norm.restype = ct.c_double
        L.og_l2_norm.argtypes = [_dp, _dp, ct.c_size_t]
        L.og_explicit_C.restype = ct.c_double
        L.og_compute_P.restype = ct.c_int
        L.og_compute_C.restype = ct.c_int
        L.og_compute_T.restype = ct.c_int
        _lib = L
    return _lib


def set_threads(n):
    """Set the OpenMP thread count used by the oracle's sweeps."""
    try:
        gomp = ct.CDLL("libgomp.so.1")
        gomp.omp_set_num_threads(int(n))
    except OSError:
        os.environ["OMP_NUM_THREADS"] = str(int(n))


def _c(a):
    """Contiguous float64 copy-or-view suitable for passing to C."""
    return numpy.ascontiguousarray(a, dtype=numpy.float64)


def _p(a):
    return a.ctypes.data_as(_dp)


def sin_cos_beta(beta_deg):
    """sin/cos of the slope angle as the numba-compiled reference sees them
    (numpy.radians on the host, then libm sin/cos inside the kernel)."""
    b = float(numpy.radians(beta_deg))
    return math.sin(b), math.cos(b)


class OracleModel:
    """Reference kernels bound to one grid (one config module)."""

    def __init__(self, config):
        self.config = config
        self.nx, self.ny, self.nz = int(config.nx), int(config.ny), int(config.nz)
        self.dx = _c(config.dx)
        self.dy = _c(config.dy)
        self.dz = _c(config.dz)
        self.g = float(config.g)
        self.sinb, self.cosb = sin_cos_beta(config.beta)
        self._grid = OGrid(self.nx, self.ny, self.nz, _p(self.dx), _p(self.dy),
                           _p(self.dz), self.g, self.sinb, self.cosb)
        self.frozen = {}
        self.freeze()

    def freeze(self):
        """Snapshot the globals numba freezes at first compilation."""
        self.freeze_from(self.config)
        self.frozen["C_IMBLFLO"] = bool(self.config.C_IMBLFLO)
        self.frozen["T_IMBLFLO"] = bool(self.config.T_IMBLFLO)

    def freeze_from(self, src):
        for name in ("c_r", "l_r", "rho_r", "cp_r", "lf_l", "lf_t", "lt_l", "lt_t"):
            self.frozen[name] = _c(getattr(src, name)).copy()

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)

    # --------------------------------------------------------------- kernels
    def l2_norm(self, New, Old, Process=""):
        New, Old = _c(New), _c(Old)
        return lib().og_l2_norm(_p(New), _p(Old), New.size)

    def compute_P(self, P, c_f, nue, rho_f, phi, Kx, Ky, Kz, qx, qy, qz, dt_P,
                  BP, WP, SOR=1.0, max_it=20000, inc_it=1.05, max_dt=1e6,
                  min_dt=1e-8, P_conv=1e-10):
        P = _c(P).copy()
        Pn = numpy.empty_like(P)
        keep = [_c(a) for a in (c_f, nue, rho_f, phi, Kx, Ky, Kz)] + \
               [self.frozen["c_r"], _c(BP), _c(WP)]
        F = OPFields(*[_p(a) for a in keep])
        out = (ct.c_double * 6)()
        rc = lib().og_compute_P(ct.byref(self._grid), ct.byref(F), _p(P), _p(Pn),
                                ct.c_double(dt_P), ct.c_double(SOR), ct.c_int(int(max_it)),
                                ct.c_double(inc_it), ct.c_double(max_dt),
                                ct.c_double(min_dt), ct.c_double(P_conv), out)
        if rc != 0:
            raise MemoryError("oracle compute_P")
        self.last = list(out)
        return out[0], out[1], P, Pn, bool(out[2]), int(out[3])

    def compute_q(self, P, BP, Kx, Ky, Kz, qx, qy, qz, nue, rho_f):
        qx, qy, qz = _c(qx).copy(), _c(qy).copy(), _c(qz).copy()
        args = [_c(a) for a in (P, BP, Kx, Ky, Kz)]
        n2 = [_c(nue), _c(rho_f)]
        lib().og_compute_q(ct.byref(self._grid), *[_p(a) for a in args],
                           _p(qx), _p(qy), _p(qz), *[_p(a) for a in n2])
        return qx, qy, qz

    def flow_error(self, P, Pn, qx, qy, qz, WP, phi, c_f, c_r, rho_f, dt_P):
        args = [_c(a) for a in (P, Pn, qx, qy, qz, WP, phi, c_f, c_r, rho_f)]
        e = numpy.empty(self.shape)
        lib().og_flow_error(ct.byref(self._grid), *[_p(a) for a in args],
                            ct.c_double(dt_P), _p(e))
        return e

    def compute_C(self, C, D_fx, D_fy, D_fz, phi, rho_f, qx, qy, qz, dt_C, BC,
                  WC, RC, e, omega=1, SOR=1.0, max_it=100, inc_it=1.05,
                  max_dt=1e6, min_dt=1e-8, C_conv=1e-10):
        C = _c(C).copy()
        keep = [_c(a) for a in (D_fx, D_fy, D_fz, phi, rho_f, qx, qy, qz, BC, WC,
                                RC, e)] + [self.frozen["lf_l"], self.frozen["lf_t"]]
        F = OCFields(*[_p(a) for a in keep], int(self.frozen["C_IMBLFLO"]))
        out = (ct.c_double * 6)()
        rc = lib().og_compute_C(ct.byref(self._grid), ct.byref(F), _p(C),
                                ct.c_double(dt_C), ct.c_double(omega), ct.c_double(SOR),
                                ct.c_int(int(max_it)), ct.c_double(inc_it),
                                ct.c_double(max_dt), ct.c_double(min_dt),
                                ct.c_double(C_conv), out)
        if rc != 0:
            raise MemoryError("oracle compute_C")
        self.last = list(out)
        return out[0], out[1], C, bool(out[2]), int(out[3])

    def compute_T(self, T, l_f, cp_f, rho_f, phi, qx, qy, qz, dt_T, BT, WT, e,
                  omega=1, SOR=1.0, max_it=100, inc_it=1.05, max_dt=1e6,
                  min_dt=1e-8, T_conv=1e-10):
        T = _c(T).copy()
        keep = [_c(a) for a in (l_f, cp_f, rho_f, phi, qx, qy, qz, BT, WT, e)] + \
               [self.frozen[n] for n in ("l_r", "rho_r", "cp_r", "lt_l", "lt_t")]
        F = OTFields(*[_p(a) for a in keep], int(self.frozen["T_IMBLFLO"]))
        out = (ct.c_double * 6)()
        rc = lib().og_compute_T(ct.byref(self._grid), ct.byref(F), _p(T),
                                ct.c_double(dt_T), ct.c_double(omega), ct.c_double(SOR),
                                ct.c_int(int(max_it)), ct.c_double(inc_it),
                                ct.c_double(max_dt), ct.c_double(min_dt),
                                ct.c_double(T_conv), out)
        if rc != 0:
            raise MemoryError("oracle compute_T")
        self.last = list(out)
        return out[0], out[1], T, bool(out[2]), int(out[3])

    def smolarkiewicz(self, C, qx, qy, qz, vx, vy, vz, dt, eps=1e-15, Sc=1.08):
        vx, vy, vz = _c(vx).copy(), _c(vy).copy(), _c(vz).copy()
        args = [_c(a) for a in (C, qx, qy, qz)]
        lib().og_smolarkiewicz(ct.byref(self._grid), *[_p(a) for a in args],
                               _p(vx), _p(vy), _p(vz), ct.c_double(dt),
                               ct.c_double(eps), ct.c_double(Sc))
        return vx, vy, vz

    def explicit_C(self, D_fx, phi):
        D = numpy.asarray(D_fx)
        Dmax = _c(D.max(axis=3) if D.ndim == 4 else D)
        ph = _c(phi)
        f = lib().og_explicit_C
        f.argtypes = [ct.POINTER(OGrid), _dp, _dp]
        return f(ct.byref(self._grid), _p(Dmax), _p(ph))

    def dt_cfl(self, qx, qy, qz, phi):
        """CFL limit of tse.py:1241-1249, including its reshape (not
        transpose) of |qx|/phi and |qy|/phi before dividing by dx and dy."""
        nx, ny, nz = self.shape
        with numpy.errstate(divide="ignore", invalid="ignore"):
            a = numpy.max(numpy.reshape(numpy.abs(qx) / phi, (ny, nz, nx)) / self.dx)
            b = numpy.max(numpy.reshape(numpy.abs(qy) / phi, (nx, nz, ny)) / self.dy)
            c = numpy.max(numpy.abs(qz) / phi / self.dz)
            return 0.9 / (a + b + c)
