"""Equation of state on the GPU: declared forms of the config callback.

The reference runs ``config.fluid_properties`` per cell over the whole grid
(run_fluid_properties, tse.py:179-199; numba-compiled when JITFLUPRO is set,
tse.py:202-205).  Arbitrary Python cannot run in a CUDA kernel, so a config
that wants the EOS on the device declares its form:

    GPU_EOS = {"rho": {"kind": "linear", "rho0": 1000.0,
                       "species": [(0, 200.0)], "tcoef": 0.3, "T0": 20.0},
               "nue": {"kind": "keep"}}

meaning rho_f = rho0 + sum_s a_s * C[s] - tcoef * (T - T0), evaluated left to
right, and every other property returned unchanged.  Before the first step
the declaration is checked against the callback on sample cells; any
difference (bit for bit) is an error.  A config without GPU_EOS runs its
callback on the host over all cells, as the reference does.
"""
from __future__ import annotations

import numpy
import torch

OUT_NAMES = ("C", "T", "P", "nue", "rho_f", "c_f", "cp_f", "l_f", "cp_r", "l_r", "phi", "Kx",
             "Ky", "Kz", "D_fx", "D_fy", "D_fz", "rho_r")


class EOSMismatch(ValueError):
    pass


def declared_eos(config):
    decl = getattr(config, "GPU_EOS", None)
    if decl is None:
        return None
    rho = decl.get("rho", {"kind": "keep"})
    nue = decl.get("nue", {"kind": "keep"})
    if rho.get("kind") not in ("linear", "keep") or nue.get("kind") != "keep":
        raise ValueError("GPU_EOS: supported forms are rho 'linear'/'keep' and nue 'keep'")
    return {"rho": rho, "nue": nue}


def eval_linear_host(rho, C_cell, T_cell):
    """The declared linear density for one cell, with the device kernel's
    operation order (IEEE double, no contraction)."""
    r = float(rho["rho0"])
    for s, a in rho["species"]:
        r = r + float(a) * float(C_cell[s])
    return r - float(rho["tcoef"]) * (float(T_cell) - float(rho["T0"]))


def validate(config, decl, n_samples=64, seed=0):
    """Check the declaration against config.fluid_properties on sample cells."""
    rng = numpy.random.default_rng(seed)
    nx, ny, nz = int(config.nx), int(config.ny), int(config.nz)
    cells = {(0, 0, 0), (nx - 1, ny - 1, nz - 1)}
    for _ in range(n_samples):
        cells.add((int(rng.integers(nx)), int(rng.integers(ny)), int(rng.integers(nz))))
    T = numpy.asarray(config.T)
    T0 = T if T.ndim == 3 else T[:, :, :, 0]
    # probe beyond the initial state too: perturbed concentrations/temperatures
    probes = [(0.0, 0.0), (0.37, 5.5), (1.0, -12.25)]
    fp = config.fluid_properties
    for c in sorted(cells):
        for dc, dT in probes:
            Cc = numpy.array(config.C[c], dtype=numpy.float64) + dc
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
                if name == "rho_f" and decl["rho"]["kind"] == "linear":
                    want = eval_linear_host(decl["rho"], Cc, Tc)
                else:
                    want = vals[k]
                if not numpy.array_equal(numpy.asarray(got, dtype=numpy.float64),
                                         numpy.asarray(want, dtype=numpy.float64)):
                    raise EOSMismatch("GPU_EOS disagrees with fluid_properties for %s at cell %s"
                                      " (callback %r, declared %r)" % (name, c, got, want))
    return True


def apply(M, decl, S, T_fluid):
    rho = decl["rho"]
    if rho["kind"] == "linear":
        C = S["C"]
        M.eos_linear([C[s] for s in range(C.shape[0])], T_fluid, S["rho_f"], rho["rho0"],
                     rho["species"], rho["tcoef"], rho["T0"])


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
