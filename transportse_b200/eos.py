"""Equation of state on the GPU: declared forms of the config callback.

The reference runs ``config.fluid_properties`` per cell over the whole grid
(run_fluid_properties, tse.py:179-199; numba-compiled when JITFLUPRO is set,
tse.py:202-205).  Arbitrary Python cannot run in a CUDA kernel, so a config
that wants the EOS on the device declares its form, per property:

    GPU_EOS = {"rho": {"kind": "linear", "rho0": 1000.0,
                       "species": [(0, 200.0)], "tcoef": 0.3, "T0": 20.0},
               "nue": {"kind": "keep"}}

Kinds (``rho`` = rho_f, ``nue`` = viscosity):

* ``keep``     the callback returns the property unchanged;
* ``linear``   (rho only) rho0 + sum_s a_s * C[s] - tcoef * (T - T0), left to
               right;
* ``constant`` {"value": v};
* ``poly4_T``  {"coef": c} with five coefficients in numpy.polyfit order
               (highest power first): c[4] + c[3]*T + c[2]*T**2 + c[1]*T**3 +
               c[0]*T**4, left to right, the powers as numba computes literal
               integer powers (T**3 = T*(T*T), T**4 = (T*T)*(T*T)) -- the
               form of course/04-groundwater_heat_tracer_eos/config.py:118-124,
               197-219.

``constant`` and ``poly4_T`` take an optional guard ``"unless": (s, v)``: cells
whose species s equals v keep their value (the callback's ``if C[s] != v:``).
Every other property must be returned unchanged by the callback.  Before the
first step the declaration is checked against the callback on sample cells;
any difference (bit for bit) is an error -- so a callback in plain Python,
whose ``T**3`` goes through libm's pow, may be refused where its numba-compiled
twin is accepted.  A config without GPU_EOS runs its callback on the host over
all cells, as the reference does.
"""
from __future__ import annotations

import numpy
import torch

OUT_NAMES = ("C", "T", "P", "nue", "rho_f", "c_f", "cp_f", "l_f", "cp_r", "l_r", "phi", "Kx",
             "Ky", "Kz", "D_fx", "D_fy", "D_fz", "rho_r")


class EOSMismatch(ValueError):
    pass


KINDS = {"rho": ("keep", "linear", "constant", "poly4_T"),
         "nue": ("keep", "constant", "poly4_T")}
# property key of the declaration -> field name of the callback
FIELD = {"rho": "rho_f", "nue": "nue"}


def declared_eos(config):
    decl = getattr(config, "GPU_EOS", None)
    if decl is None:
        return None
    unknown = set(decl) - set(KINDS)
    if unknown:
        raise ValueError("GPU_EOS: unknown properties %s (declarable: rho, nue)" % sorted(unknown))
    out = {}
    for prop, kinds in KINDS.items():
        d = dict(decl.get(prop, {"kind": "keep"}))
        if d.get("kind") not in kinds:
            raise ValueError("GPU_EOS[%r]: kind %r is not one of %s" % (prop, d.get("kind"), kinds))
        if d["kind"] == "poly4_T":
            d["coef"] = [float(v) for v in d["coef"]]
            if len(d["coef"]) != 5:
                raise ValueError("GPU_EOS[%r]: poly4_T takes 5 coefficients" % prop)
        if d["kind"] == "constant":
            d["value"] = float(d["value"])
        if "unless" in d:
            if d["kind"] not in ("constant", "poly4_T"):
                raise ValueError("GPU_EOS[%r]: 'unless' applies to constant and poly4_T" % prop)
            s, v = d["unless"]
            d["unless"] = (int(s), float(v))
        out[prop] = d
    return out


def eval_linear_host(rho, C_cell, T_cell):
    """The declared linear density for one cell, with the device kernel's
    operation order (IEEE double, no contraction)."""
    r = float(rho["rho0"])
    for s, a in rho["species"]:
        r = r + float(a) * float(C_cell[s])
    return r - float(rho["tcoef"]) * (float(T_cell) - float(rho["T0"]))


def eval_form_host(d, C_cell, T_cell, old):
    """A declared property for one cell (device kernel's operation order);
    ``old`` is the value the cell keeps for 'keep' or a guarded cell."""
    kind = d["kind"]
    if kind == "keep":
        return old
    if kind == "linear":
        return eval_linear_host(d, C_cell, T_cell)
    if "unless" in d:
        s, v = d["unless"]
        if not (float(C_cell[s]) != v):
            return old
    if kind == "constant":
        return d["value"]
    c = d["coef"]
    x = float(T_cell)
    x2 = x * x
    x3 = x * x2
    x4 = x2 * x2
    r = c[4] + c[3] * x
    r = r + c[2] * x2
    r = r + c[1] * x3
    return r + c[0] * x4


def validate(config, decl, n_samples=64, seed=0):
    """Check the declaration against config.fluid_properties on sample cells."""
    rng = numpy.random.default_rng(seed)
    nx, ny, nz = int(config.nx), int(config.ny), int(config.nz)
    cells = {(0, 0, 0), (nx - 1, ny - 1, nz - 1)}
    for _ in range(n_samples):
        cells.add((int(rng.integers(nx)), int(rng.integers(ny)), int(rng.integers(nz))))
    T = numpy.asarray(config.T)
    T0 = T if T.ndim == 3 else T[:, :, :, 0]
    # probe beyond the initial state too: perturbed concentrations and
    # temperatures, and each species set to exactly 1 on its own (guards)
    nspec = numpy.asarray(config.C).shape[3]
    probes = [(0.0, None, 0.0), (0.37, None, 5.5), (1.0, None, -12.25)]
    probes += [(0.0, s, 3.25) for s in range(nspec)]
    fp = config.fluid_properties
    for c in sorted(cells):
        for dc, one, dT in probes:
            Cc = numpy.array(config.C[c], dtype=numpy.float64) + dc
            if one is not None:
                Cc[one] = 1.0
            Tc = float(T0[c]) + dT
            vals = [Cc, Tc] + [float(numpy.asarray(getattr(config, n))[c]) if numpy.asarray(
                getattr(config, n)).ndim == 3 else numpy.array(getattr(config, n)[c])
                for n in OUT_NAMES[2:]]
            out = fp(*vals)
            for k, name in enumerate(OUT_NAMES):
                if name == "C":
                    if not numpy.array_equal(numpy.asarray(out[0]), Cc):
                        raise EOSMismatch("fluid_properties changes C; GPU_EOS cannot express it")
                    continue
                got = out[k]
                if name == "rho_f":
                    want = eval_form_host(decl["rho"], Cc, Tc, vals[k])
                elif name == "nue":
                    want = eval_form_host(decl["nue"], Cc, Tc, vals[k])
                else:
                    want = vals[k]
                if not numpy.array_equal(numpy.asarray(got, dtype=numpy.float64),
                                         numpy.asarray(want, dtype=numpy.float64)):
                    raise EOSMismatch("GPU_EOS disagrees with fluid_properties for %s at cell %s"
                                      " (callback %r, declared %r)" % (name, c, got, want))
    return True


def apply(M, decl, S, T_fluid):
    """Evaluate the declared properties on the device.  Every form reads only
    C and T (which it does not change), so the order of the properties does
    not matter."""
    C = S["C"]
    for prop in ("rho", "nue"):
        d = decl[prop]
        out = S[FIELD[prop]]
        if d["kind"] == "linear":
            M.eos_linear([C[s] for s in range(C.shape[0])], T_fluid, out, d["rho0"],
                         d["species"], d["tcoef"], d["T0"])
        elif d["kind"] in ("constant", "poly4_T"):
            guard, gv = None, 0.0
            if "unless" in d:
                s, gv = d["unless"]
                if not 0 <= s < C.shape[0]:
                    raise ValueError("GPU_EOS guard species %d out of range" % s)
                guard = C[s]
            M.eos_form(d["kind"], d["value"] if d["kind"] == "constant" else d["coef"],
                       T_fluid if d["kind"] == "poly4_T" else None, out, guard, gv)


def host_callback(sim, T_fluid):
    """Run config.fluid_properties per cell on the host (tse.py:179-199)."""
    cfg = sim.config
    S = sim.S
    h = {}
    for n in OUT_NAMES:
        if n == "T":
            h[n] = T_fluid.cpu().numpy().copy()
        else:
            h[n] = sim.field(n)
    nx, ny, nz = sim.shape
    fp = cfg.fluid_properties
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                c = (i, j, k)
                r = fp(*[h[n][c] for n in OUT_NAMES])
                for q, n in enumerate(OUT_NAMES):
                    h[n][c] = r[q]
    for n in OUT_NAMES:
        a = h[n]
        if n == "T":
            T_fluid.copy_(torch.as_tensor(a))
            continue
        if a.ndim == 4:
            a = numpy.moveaxis(a, 3, 0)
        S[n].copy_(torch.as_tensor(numpy.ascontiguousarray(a)))
