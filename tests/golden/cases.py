"""Seeded unit-test inputs shared by the fixture generator and the tests.

``unit_case(variant)`` builds a small config module plus random kernel
inputs; ``run_unit_calls(kernels, inputs, variant)`` calls the reference
kernel set on them.  ``kernels`` is anything exposing the reference's kernel
names with the reference's argument lists: the reference namespace itself
(when generating fixtures), the oracle's ``OracleModel``, or the CUDA
library's ``transportse_b200.kernels.Model``.
"""
from __future__ import annotations

import hashlib
import types

import numpy

from transportse_b200 import workloads


def config_checksum(cfg):
    h = hashlib.sha256()
    for name in sorted(vars(cfg)):
        if name.startswith("_"):
            continue
        v = getattr(cfg, name)
        if isinstance(v, numpy.ndarray):
            h.update(name.encode())
            h.update(numpy.ascontiguousarray(v).tobytes())
        elif isinstance(v, (int, float, bool, str)):
            h.update(("%s=%r" % (name, v)).encode())
    return h.hexdigest()


def config_attributes(cfg, skip=()):
    """The array and scalar attributes of a config module, as fixture entries
    ``cfg_<name>`` (copies: the reference changes its config's arrays in
    place while it runs)."""
    out = {}
    for name in sorted(vars(cfg)):
        if name.startswith("_") or name in skip:
            continue
        v = getattr(cfg, name)
        if isinstance(v, numpy.ndarray):
            out["cfg_" + name] = numpy.array(v, copy=True)
        elif isinstance(v, (bool, int, float, str, numpy.generic)):
            out["cfg_" + name] = numpy.array(v)
    return out


def course_eos(c_dens, c_visc):
    """(fluid_properties, GPU_EOS) of the course model with an equation of
    state, course/04-groundwater_heat_tracer_eos/config.py:197-219: unless
    species 2 holds 1, density and viscosity are fourth-order polynomials in
    T with numpy.polyfit coefficients, evaluated left to right with numba's
    products for literal integer powers (T**3 = T*(T*T), T**4 = (T*T)*(T*T))."""
    cd = [float(v) for v in c_dens]
    cv = [float(v) for v in c_visc]

    def fluid_properties(C, T, P, nue, rho_f, c_f, cp_f, l_f, cp_r, l_r, phi, Kx, Ky, Kz,
                         D_fx, D_fy, D_fz, rho_r):
        if C[2] != 1:
            t2 = T * T
            t3 = T * t2
            t4 = t2 * t2
            rho_f = cd[4] + cd[3] * T + cd[2] * t2 + cd[1] * t3 + cd[0] * t4
            nue = cv[4] + cv[3] * T + cv[2] * t2 + cv[1] * t3 + cv[0] * t4
        return (C, T, P, nue, rho_f, c_f, cp_f, l_f, cp_r, l_r, phi, Kx, Ky, Kz,
                D_fx, D_fy, D_fz, rho_r)

    decl = {"rho": {"kind": "poly4_T", "coef": cd, "unless": (2, 1.0)},
            "nue": {"kind": "poly4_T", "coef": cv, "unless": (2, 1.0)}}
    return fluid_properties, decl


def config_from_fixture(fx, name):
    """Rebuild a config module from a fixture's ``cfg_<name>`` entries, with
    the callbacks of the course models (identity EOS and chemistry unless the
    model declares its own)."""
    m = types.ModuleType(name)
    m.__file__ = name + ".py"
    keys = fx.files if hasattr(fx, "files") else list(fx)
    for k in keys:
        if k.startswith("cfg_"):
            v = numpy.array(fx[k])
            setattr(m, k[4:], v.item() if v.ndim == 0 else v)
    m.fluid_properties = workloads._identity_fluid_properties
    m.chemical_reactions = workloads._noop_chemistry
    if hasattr(m, "c_dens") and hasattr(m, "c_visc"):
        m.fluid_properties, m.GPU_EOS = course_eos(m.c_dens, m.c_visc)
    return m


def unit_case(variant):
    """variant 'a': 7x5x6, slope 5 deg, dispersion and IMBLFLO on;
    variant 'b': 6x1x9 slice, no slope, dispersion and IMBLFLO off."""
    if variant == "a":
        nx, ny, nz, seed, beta = 7, 5, 6, 101, 5.0
    else:
        nx, ny, nz, seed, beta = 6, 1, 9, 202, 0.0
    rng = numpy.random.default_rng(seed)
    dx = rng.uniform(0.5, 2.0, nx)
    dy = rng.uniform(0.5, 2.0, ny)
    dz = rng.uniform(0.5, 2.0, nz)
    cfg = workloads.base_config("unit_" + variant, nx, ny, nz, dx, dy, dz, species=2)
    cfg.beta = beta
    shp = (nx, ny, nz)
    U = lambda lo, hi: rng.uniform(lo, hi, shp)
    # frozen globals (read by the reference kernels from the config)
    cfg.c_r[:] = 1e-10 * U(0.5, 1.5)
    cfg.l_r[:] = U(1.5, 3.5)
    cfg.rho_r[:] = U(2400.0, 2800.0)
    cfg.cp_r[:] = U(800.0, 1100.0)
    if variant == "a":
        cfg.lf_l[:] = U(0.0, 2.0)
        cfg.lf_t[:] = U(0.0, 0.5)
        cfg.lt_l[:] = U(0.0, 2.0)
        cfg.lt_t[:] = U(0.0, 0.5)
        cfg.C_IMBLFLO = True
        cfg.T_IMBLFLO = True
    inp = {}
    K = 1e-12 * numpy.exp(rng.standard_normal(shp))
    inp["Kx"] = K.copy()
    inp["Ky"] = K * U(0.5, 1.5)
    inp["Kz"] = 0.3 * K
    if variant == "a":
        inp["Kx"][1, 2, 3] = 0.0   # harm() returns 0 when either side is 0
        inp["Kz"][4, 0, 2] = 0.0
    inp["nue"] = U(0.8e-3, 1.2e-3)
    inp["rho_f"] = U(995.0, 1150.0)
    inp["phi"] = U(0.05, 0.3)
    inp["c_f"] = 4.5e-10 * U(0.5, 1.5)
    cfg.beta = beta
    inp["P"] = workloads.hydrostatic(cfg) + rng.uniform(-500.0, 500.0, shp)
    BP = (rng.uniform(size=shp) < 0.1).astype(float)
    BP[:, :, -1] = 1.0
    inp["BP"] = BP
    WP = numpy.where(rng.uniform(size=shp) < 0.25, rng.uniform(-1e-4, 1e-4, shp), 0.0)
    inp["WP"] = WP
    inp["qx0"] = rng.uniform(-1e-6, 1e-6, shp)   # previous q (last planes stay)
    inp["qy0"] = rng.uniform(-1e-6, 1e-6, shp)
    inp["qz0"] = rng.uniform(-1e-6, 1e-6, shp)
    # transport inputs
    inp["tqx"] = rng.uniform(-2e-4, 2e-4, shp)
    inp["tqy"] = rng.uniform(-2e-4, 2e-4, shp)
    inp["tqz"] = rng.uniform(-2e-4, 2e-4, shp)
    Cc = rng.uniform(0.0, 1.0, shp)
    Cc[rng.uniform(size=shp) < 0.2] = 0.0
    inp["C"] = Cc
    inp["D_fx"] = 1e-5 * U(0.5, 1.5)
    inp["D_fy"] = 1e-5 * U(0.5, 1.5)
    inp["D_fz"] = 1e-5 * U(0.5, 1.5)
    inp["D_fx"][2, 0, 1] = 0.0
    BC = (rng.uniform(size=shp) < 0.15).astype(float)
    inp["BC"] = BC
    inp["WC"] = numpy.where(rng.uniform(size=shp) < 0.2, rng.uniform(0.0, 1e-4, shp), 0.0)
    inp["RC"] = U(1.0, 2.0)
    inp["e"] = rng.uniform(-1e-5, 1e-5, shp)
    inp["T"] = U(10.0, 90.0)
    inp["l_f"] = U(0.5, 0.7)
    inp["cp_f"] = U(4000.0, 4200.0)
    inp["BT"] = (rng.uniform(size=shp) < 0.15).astype(float)
    inp["WT"] = numpy.where(rng.uniform(size=shp) < 0.2, rng.uniform(-1.0, 1.0, shp), 0.0)
    Cs = rng.uniform(-0.2, 1.0, shp)
    inp["Cs"] = Cs
    inp["vx0"] = rng.uniform(-1e-6, 1e-6, shp)
    inp["vy0"] = rng.uniform(-1e-6, 1e-6, shp)
    inp["vz0"] = rng.uniform(-1e-6, 1e-6, shp)
    inp["D4"] = rng.uniform(1e-10, 1e-8, shp + (2,))
    inp["L2a"] = rng.standard_normal(shp)
    inp["L2b"] = rng.standard_normal(shp)
    return cfg, inp


class _NS:
    """Attribute view of the reference namespace dict."""

    def __init__(self, ns):
        self.__dict__.update(ns)


def run_unit_calls(kern, inp, variant):
    """Call the kernel set on the inputs; returns a dict of outputs."""
    if isinstance(kern, dict):
        kern = _NS(kern)
    c = lambda a: numpy.array(a, copy=True)
    I = inp
    out = {}
    shp = I["P"].shape
    Z = numpy.zeros(shp)
    O = numpy.ones(shp)
    pargs = lambda P: (c(P), I["c_f"], I["nue"], I["rho_f"], I["phi"], I["Kx"],
                       I["Ky"], I["Kz"], c(I["qx0"]), c(I["qy0"]), c(I["qz0"]))
    cases_p = {
        "p1": dict(dt_P=3600.0, SOR=1.0, max_it=20000, inc_it=1.25, max_dt=1e4,
                   min_dt=1e-8, P_conv=1e300),
        "p2": dict(dt_P=3600.0, SOR=1.7, max_it=20000, inc_it=1.25, max_dt=1e4,
                   min_dt=1e-8, P_conv=1e-10),
        "p3": dict(dt_P=3600.0, SOR=1.5, max_it=7, inc_it=1.05, max_dt=1e6,
                   min_dt=1e-3, P_conv=1e-14),
    }
    for name, kw in cases_p.items():
        a = pargs(I["P"])
        t_P, dt_P, P, Pn, conv, nit = kern.compute_P(
            *a, kw["dt_P"], I["BP"], I["WP"], SOR=kw["SOR"], max_it=kw["max_it"],
            inc_it=kw["inc_it"], max_dt=kw["max_dt"], min_dt=kw["min_dt"],
            P_conv=kw["P_conv"])
        out[name + "_scal"] = numpy.array([t_P, dt_P, float(conv), float(nit)])
        out[name + "_P"] = c(P)
        out[name + "_Pn"] = c(Pn)
    P2 = out["p2_P"]
    qx, qy, qz = kern.compute_q(c(P2), I["BP"], I["Kx"], I["Ky"], I["Kz"], c(I["qx0"]),
                                c(I["qy0"]), c(I["qz0"]), I["nue"], I["rho_f"])
    out["qx"], out["qy"], out["qz"] = c(qx), c(qy), c(qz)
    cfg_c_r = I["c_r_cfg"]
    e = kern.flow_error(c(P2), out["p2_Pn"], out["qx"], out["qy"], out["qz"], I["WP"],
                        I["phi"], I["c_f"], cfg_c_r, I["rho_f"], float(out["p2_scal"][0]))
    out["e"] = c(e)
    cargs = lambda: (c(I["C"]), I["D_fx"], I["D_fy"], I["D_fz"], I["phi"], I["rho_f"],
                     I["tqx"], I["tqy"], I["tqz"])
    cases_c = {
        "c1": dict(omega=1, SOR=1.0, max_it=100, conv=1e-10, min_dt=1e-8),
        "c2": dict(omega=0.5, SOR=1.3, max_it=100, conv=1e-12, min_dt=1e-8),
        "c3": dict(omega=0, SOR=1.0, max_it=100, conv=1e-10, min_dt=1e-8),
        "c4": dict(omega=1, SOR=1.0, max_it=4, conv=1e-15, min_dt=1.0),
    }
    for name, kw in cases_c.items():
        t, dt, C, conv, nit = kern.compute_C(
            *cargs(), 3600.0, I["BC"], I["WC"], I["RC"], I["e"], omega=kw["omega"],
            SOR=kw["SOR"], max_it=kw["max_it"], inc_it=1.05, max_dt=1e5,
            min_dt=kw["min_dt"], C_conv=kw["conv"])
        out[name + "_scal"] = numpy.array([t, dt, float(conv), float(nit)])
        out[name + "_C"] = c(C)
    targs = lambda T, lf, cp, rho, ph: (c(T), lf, cp, rho, ph, I["tqx"], I["tqy"], I["tqz"])
    cases_t = {
        "t1": (targs(I["T"], I["l_f"], I["cp_f"], I["rho_f"], I["phi"]), I["WT"],
               dict(omega=1, SOR=1.0, max_it=100, conv=1e-10)),
        "t2": (targs(I["T"], I["l_f"], I["cp_f"], I["rho_f"], I["phi"]), I["WT"],
               dict(omega=0.6, SOR=1.2, max_it=100, conv=1e-12)),
        # NLTE layers as driven at tse.py:1345-1353
        "t3": (targs(I["T"], I["l_f"], I["cp_f"], I["rho_f"], O), Z,
               dict(omega=1, SOR=1.0, max_it=100, conv=1e-10)),
        "t4": (targs(I["T"], Z, Z, Z, Z), I["WT"],
               dict(omega=1, SOR=1.0, max_it=100, conv=1e-10)),
    }
    for name, (a, WT, kw) in cases_t.items():
        t, dt, T, conv, nit = kern.compute_T(
            *a, 3600.0, I["BT"], WT, I["e"], omega=kw["omega"], SOR=kw["SOR"],
            max_it=kw["max_it"], inc_it=1.05, max_dt=1e5, min_dt=1e-8,
            T_conv=kw["conv"])
        out[name + "_scal"] = numpy.array([t, dt, float(conv), float(nit)])
        out[name + "_T"] = c(T)
    vx, vy, vz = kern.smolarkiewicz(c(I["Cs"]), I["tqx"], I["tqy"], I["tqz"],
                                    c(I["vx0"]), c(I["vy0"]), c(I["vz0"]), 3600.0,
                                    eps=1e-15, Sc=1.08)
    out["vx"], out["vy"], out["vz"] = c(vx), c(vy), c(vz)
    out["explicit_C"] = numpy.array(kern.explicit_C(I["D4"], I["phi"]))
    out["l2"] = numpy.array(kern.l2_norm(I["L2a"], I["L2b"], "x"))
    bad = c(I["L2a"])
    bad[0, 0, 0] = numpy.nan
    out["l2_nan"] = numpy.array(kern.l2_norm(bad, I["L2b"], "x"))
    return out


def unit_inputs_with_cfg(variant):
    cfg, inp = unit_case(variant)
    inp["c_r_cfg"] = numpy.array(cfg.c_r, copy=True)
    return cfg, inp
