"""ctypes bindings of libtsecuda.so (declared in include/tse_cuda.h).

The library is built in-tree (``transportse_b200/_build/libtsecuda.so``).
There is no fallback: if the library is missing or fails to load, every
entry point raises.
"""
from __future__ import annotations

import ctypes as ct
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libtsecuda.so")

TSE_WS_PRESSURE = 1
TSE_WS_TRANSPORT = 2
TSE_WS_REDUCE = 3
TSE_WS_PRESSURE_DC = 4
TSE_WS_TRANSPORT_DC = 5

ERRORS = {-1: "invalid argument", -2: "workspace too small", -3: "kernel launch failed",
          -4: "device error"}

_dp = ct.POINTER(ct.c_double)


class TseGrid(ct.Structure):
    _fields_ = [("nx", ct.c_int32), ("ny", ct.c_int32), ("nz", ct.c_int32),
                ("reserved", ct.c_int32), ("dx", ct.c_void_p), ("dy", ct.c_void_p),
                ("dz", ct.c_void_p), ("g", ct.c_double), ("sin_beta", ct.c_double),
                ("cos_beta", ct.c_double)]


class TseSolveStatus(ct.Structure):
    _fields_ = [("t", ct.c_double), ("dt", ct.c_double), ("diff", ct.c_double),
                ("converged", ct.c_int32), ("num_it", ct.c_int32), ("num_sub_it", ct.c_int32),
                ("halvings", ct.c_int32), ("error", ct.c_int32), ("n_events", ct.c_int32),
                ("ev_it", ct.c_int32 * 8), ("ev_dt", ct.c_double * 8),
                ("ev_diff", ct.c_double * 8), ("cycles", ct.c_int32), ("reserved", ct.c_int32)]


def _ptr_fields(names):
    return [(n, ct.c_void_p) for n in names]


class TsePressureArgs(ct.Structure):
    _fields_ = _ptr_fields(["P", "Pn", "c_f", "nue", "rho_f", "phi", "Kx", "Ky", "Kz", "c_r",
                            "BP", "WP"]) + \
        [(n, ct.c_double) for n in ("dt_P", "SOR", "inc_it", "max_dt", "min_dt", "P_conv")] + \
        [("max_it", ct.c_int32), ("sweep", ct.c_int32)]


class TseSpeciesArgs(ct.Structure):
    _fields_ = _ptr_fields(["C", "D_fx", "D_fy", "D_fz", "phi", "rho_f", "qx", "qy", "qz", "BC",
                            "WC", "RC", "e", "l_l", "l_t"]) + \
        [(n, ct.c_double) for n in ("dt", "omega", "SOR", "inc_it", "max_dt", "min_dt", "conv")] + \
        [("max_it", ct.c_int32), ("imblflo", ct.c_int32), ("sweep", ct.c_int32),
         ("reserved", ct.c_int32)]


class TseHeatArgs(ct.Structure):
    _fields_ = _ptr_fields(["T", "l_f", "cp_f", "rho_f", "phi", "qx", "qy", "qz", "BT", "WT", "e",
                            "l_r", "rho_r", "cp_r", "l_l", "l_t"]) + \
        [(n, ct.c_double) for n in ("dt", "omega", "SOR", "inc_it", "max_dt", "min_dt", "conv")] + \
        [("max_it", ct.c_int32), ("imblflo", ct.c_int32), ("sweep", ct.c_int32),
         ("reserved", ct.c_int32)]


TSE_EOS_CONSTANT = 1
TSE_EOS_POLY4_T = 2


class TseEosForm(ct.Structure):
    _fields_ = [("kind", ct.c_int32), ("reserved", ct.c_int32), ("guard_value", ct.c_double),
                ("coef", ct.c_double * 5)]


class TseDcOptions(ct.Structure):
    _fields_ = [("cycle", ct.c_int32), ("max_blocks", ct.c_int32), ("timing", ct.c_int32),
                ("sweep_launches", ct.c_int32), ("sweep_iterations", ct.c_int64),
                ("sweep_ms", ct.c_double), ("host_loop", ct.c_int32), ("reserved", ct.c_int32),
                ("loop_ms", ct.c_double), ("chunk", ct.c_int32), ("ring", ct.c_int32),
                ("pipes", ct.c_int32), ("graph_runs", ct.c_int32), ("active_cells", ct.c_int64)]


def _batch_item(args_type):
    class Item(ct.Structure):
        _fields_ = [("grid", ct.POINTER(TseGrid)), ("args", ct.POINTER(args_type)),
                    ("d_status", ct.c_void_p), ("d_workspace", ct.c_void_p),
                    ("workspace_bytes", ct.c_size_t)]
    return Item


TseBatchPressure = _batch_item(TsePressureArgs)
TseBatchSpecies = _batch_item(TseSpeciesArgs)
TseBatchHeat = _batch_item(TseHeatArgs)
BATCH_ITEM = {"compute_P": TseBatchPressure, "compute_C": TseBatchSpecies,
              "compute_T": TseBatchHeat}


# name -> (restype, argtypes)
_P = ct.c_void_p
_I = ct.c_int32
_D = ct.c_double
_G = ct.POINTER(TseGrid)
_S = ct.c_size_t
_PP = ct.POINTER(ct.c_void_p)
SIGNATURES = {
    "tse_workspace_bytes": (ct.c_size_t, [_G, _I]),
    "tse_compute_P": (_I, [_G, ct.POINTER(TsePressureArgs), _P, _P, _S, _P]),
    "tse_compute_P_noalloc": (_I, [_G, ct.POINTER(TsePressureArgs), _P, _P]),
    "tse_compute_P_dc": (_I, [_G, ct.POINTER(TsePressureArgs), ct.POINTER(TseDcOptions), _P, _P,
                              _S, _P]),
    "tse_compute_C_dc": (_I, [_G, ct.POINTER(TseSpeciesArgs), ct.POINTER(TseDcOptions), _P, _P,
                              _S, _P]),
    "tse_compute_T_dc": (_I, [_G, ct.POINTER(TseHeatArgs), ct.POINTER(TseDcOptions), _P, _P, _S,
                              _P]),
    "tse_batch_workspace_bytes": (ct.c_size_t, [_I, ct.c_int64]),
    "tse_compute_P_dc_batch": (_I, [ct.POINTER(TseBatchPressure), _I, ct.POINTER(TseDcOptions), _P,
                                    _S, _P]),
    "tse_compute_C_dc_batch": (_I, [ct.POINTER(TseBatchSpecies), _I, ct.POINTER(TseDcOptions), _P,
                                    _S, _P]),
    "tse_compute_T_dc_batch": (_I, [ct.POINTER(TseBatchHeat), _I, ct.POINTER(TseDcOptions), _P, _S,
                                    _P]),
    "tse_compute_q": (_I, [_G, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "tse_flow_error": (_I, [_G, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D, _P, _P]),
    "tse_compute_C": (_I, [_G, ct.POINTER(TseSpeciesArgs), _P, _P, _S, _P]),
    "tse_compute_T": (_I, [_G, ct.POINTER(TseHeatArgs), _P, _P, _S, _P]),
    "tse_smolarkiewicz": (_I, [_G, _P, _P, _P, _P, _P, _P, _P, _D, _D, _D, _P]),
    "tse_l2_norm": (_I, [_P, _P, ct.c_int64, _P, _P, _S, _P]),
    "tse_dt_cfl": (_I, [_G, _P, _P, _P, _P, _P, _P, _S, _P]),
    "tse_explicit_C": (_I, [_G, _PP, _I, _P, _P, _P, _S, _P]),
    "tse_field_stats": (_I, [_P, ct.c_int64, _P, _P, _S, _P]),
    "tse_eos_linear": (_I, [_G, _PP, ct.POINTER(ct.c_int32), _dp, _I, _P, _D, _D, _D, _P, _P]),
    "tse_eos_form": (_I, [_G, ct.POINTER(TseEosForm), _P, _P, _P, _P]),
    "tse_peclet_C": (_I, [_G, _P, _P, _P, _PP, _PP, _PP, _I, _P, _P, _P, _S, _P]),
    "tse_peclet_T": (_I, [_G, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _S, _P]),
    "tse_mass_totals": (_I, [_G, _P, _P, _P, _PP, _PP, _I, _P, _P, _P, _P, _P, _P, _P, _P, _S,
                             _P]),
    "tse_selftest_bounded_waits": (_I, [_P, _D, _P, _S, _P]),
    "tse_batch_loop_stats": (_I, [ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int64)]),
    "tse_version": (ct.c_char_p, []),
}

_lib = None


def lib():
    """Load libtsecuda.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libtsecuda.so is not built (%s); run "
                               "`python -m transportse_b200.build`" % LIB_PATH)
        L = ct.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc, what):
    if rc != 0:
        raise RuntimeError("%s failed: %s (%d)" % (what, ERRORS.get(rc, "error"), rc))
