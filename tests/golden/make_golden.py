"""Generate the golden fixtures in this folder by running the reference.

The reference (thkempka/transportse) is one Python/numba script, ``tse.py``.
This script executes it UNMODIFIED, from a read-only checkout, inside a fresh
namespace (``exec``), once per synthetic config:

* unit fixtures (``unit_*.npz``): the reference's numba kernels
  (``compute_P``, ``compute_q``, ``flow_error``, ``compute_C``, ``compute_T``,
  ``smolarkiewicz``, ``explicit_C``, ``l2_norm``) are called directly on seeded
  random inputs and their outputs are stored beside the inputs.  Running the
  script with ``t = 0`` defines every kernel without stepping (its final
  summary then divides by zero steps, which is caught).
* end-to-end fixtures (``e2e_*.npz``): a step-counting ``dynamic_bc`` callback
  (tse.py:1448-1458; it returns every field unchanged) records the state after
  each time step, a ``mass_balance`` callback (tse.py:1460-1463, called after
  dynamic_bc and the equation of state it may re-run) records the fields, and
  the run stops after N steps.  A config with its own ``dynamic_bc`` keeps it:
  the recorder calls it first.
* course fixtures (``course_*.npz``): the reference's own example models
  ``course/01..04/config.py``, loaded from the checkout and run to their end
  time (PLOTSAVE as configured: the step sequence lands on every PLOTTIME; the
  snapshot files are counted, not stored).  The fixture holds the config's
  initial attributes (``cfg_<name>``) so the tests can rebuild it without the
  checkout, the per-step scalars, and fields at a few steps and at the end.

Usage:  python tests/golden/make_golden.py [--reference PATH] [--only NAME]

It needs the reference checkout and numba, so it runs on the development
machine only; the fixtures it writes are committed.
"""
from __future__ import annotations

import argparse
import contextlib
import io
import os
import sys
import uuid

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from transportse_b200 import workloads  # noqa: E402
from tests.golden import cases  # noqa: E402


class StopRun(Exception):
    pass


def _exec_reference(ref, cfg, taps=None):
    """exec tse.py with ``cfg`` as its config module; return the namespace."""
    import numba  # noqa: F401  (the reference needs it)
    name = "tsecfg_" + uuid.uuid4().hex[:10]
    cfg.__name__ = name
    if getattr(cfg, "JITFLUPRO", False):
        cfg.fluid_properties = numba.njit(cfg.fluid_properties)
    sys.modules[name] = cfg
    ns = {"__name__": "__tse_reference__"}
    cfg._ns = ns
    argv = sys.argv
    sys.argv = ["tse.py", name + ".py"]
    src = open(os.path.join(ref, "tse.py")).read()
    out = io.StringIO()
    try:
        with contextlib.redirect_stdout(out):
            try:
                exec(compile(src, os.path.join(ref, "tse.py"), "exec"), ns)
            except StopRun:
                pass
            except ZeroDivisionError:
                if ns.get("n_tsteps", 1) != 0:
                    raise
    finally:
        sys.argv = argv
        sys.modules.pop(name, None)
    ns["__stdout__"] = out.getvalue()
    return ns


def reference_namespace(ref, cfg):
    """Namespace with every kernel of tse.py defined and nothing stepped."""
    cfg.t = 0.0
    cfg.DYNAMICBC = False
    return _exec_reference(ref, cfg)


# the snapshot tuple of tse.py:324-326, in order
SNAPSHOT_ITEMS = ("lx", "ly", "lz", "nx", "ny", "nz", "dx", "dy", "dz", "t_sim", "dt",
                  "P", "C", "T", "qx", "qy", "qz", "phi", "Kx", "Ky", "Kz", "rho_f",
                  "nue", "cp_f", "l_f", "BP", "BC", "BT", "L", "mass", "WP", "WT", "WC", "e")


def run_reference(ref, cfg, steps, keep_steps, fields, keep_plots=True):
    """Run ``steps`` time steps (or to the config's end time, whichever comes
    first); record scalars every step, fields at keep_steps and at the end
    ("<field>@final").  With PLOTSAVE on, the run happens in a scratch
    directory and the snapshot files tse.py writes there are recorded item by
    item ("plot<k>_<item>"), or only counted ("n_plot_files") without
    keep_plots."""
    rec = {"dt": [], "t_sim": [], "numitP": [], "numitC": [], "numitT": [],
           "num_CFL": [], "dt_P": [], "dt_C": [], "dt_T": []}
    snaps = {}
    own_bc = cfg.dynamic_bc if getattr(cfg, "DYNAMICBC", False) else None
    own_mb = cfg.mass_balance if getattr(cfg, "MASSBALAN", False) else None
    cfg.DYNAMICBC = True
    cfg.MASSBALAN = True

    def dynamic_bc(t, bc_inc, P, T, C, BP, BT, BC, WP, WT, WC, Kx, Ky, Kz, rho_f,
                   nue, c_f, cp_f, qx, phi, l_f, l_r):
        ns = cfg._ns
        out = (bc_inc, P, T, C, BP, BT, BC, WP, WT, WC, Kx, Ky, Kz)
        if own_bc is not None:
            out = own_bc(t, bc_inc, P, T, C, BP, BT, BC, WP, WT, WC, Kx, Ky, Kz, rho_f,
                         nue, c_f, cp_f, qx, phi, l_f, l_r)
        for k in rec:
            rec[k].append(float(ns.get(k, numpy.nan)))
        return out

    def mass_balance(C, qx, qy, qz, WP, WC, WT, D_fx, D_fy, D_fz, dt, mass):
        # called after dynamic_bc and the equation of state it may re-run
        # (tse.py:1449-1463): the fields here are the step's final ones
        ns = cfg._ns
        if own_mb is not None:
            mass = own_mb(C, qx, qy, qz, WP, WC, WT, D_fx, D_fy, D_fz, dt, mass)
        step = len(rec["dt"])
        if step in keep_steps:
            for f in fields:
                snaps["%s@%d" % (f, step)] = numpy.array(ns[f], copy=True)
        if step >= steps:
            raise StopRun()
        return mass

    cfg.dynamic_bc = dynamic_bc
    cfg.mass_balance = mass_balance
    plots = {}
    if getattr(cfg, "PLOTSAVE", False):
        import glob
        import joblib
        import tempfile
        cwd = os.getcwd()
        with tempfile.TemporaryDirectory() as tmp:
            os.chdir(tmp)
            try:
                ns = _exec_reference(ref, cfg)
                files = sorted(glob.glob("*-[0-9][0-9][0-9][0-9][0-9].p"))
                for k, f in enumerate(files if keep_plots else ()):
                    for name, v in zip(SNAPSHOT_ITEMS, joblib.load(f)):
                        # later files keep only the items that differ from the
                        # first file's (a missing key means "as in plot0")
                        v = numpy.array(v)
                        p0 = plots.get("plot0_" + name)
                        if k == 0 or not (p0.shape == v.shape and numpy.array_equal(p0, v)):
                            plots["plot%d_%s" % (k, name)] = v
            finally:
                os.chdir(cwd)
        plots["n_plots" if keep_plots else "n_plot_files"] = numpy.array(len(files))
    else:
        ns = _exec_reference(ref, cfg)
    if len(rec["dt"]) < steps:
        # the run reached the config's end time
        for f in fields:
            snaps["%s@final" % f] = numpy.array(ns[f], copy=True)
    out = {("s_" + k): numpy.array(v) for k, v in rec.items()}
    out.update(plots)
    out.update(snaps)
    out["keep_steps"] = numpy.array(sorted(keep_steps))
    out["steps"] = numpy.array(steps)
    return out, ns


def gen_unit(ref, variant):
    cfg, inputs = cases.unit_inputs_with_cfg(variant)
    ns = reference_namespace(ref, cfg)
    res = cases.run_unit_calls(ns, inputs, variant)
    data = {("in_" + k): v for k, v in inputs.items()}
    data.update({("out_" + k): v for k, v in res.items()})
    # values the reference kernels see for sin/cos of the slope (numba libm)
    import numba

    @numba.njit
    def _sc(b):
        return numpy.sin(b), numpy.cos(b)
    s, c = _sc(numpy.radians(cfg.beta))
    data["sin_beta"] = numpy.array(s)
    data["cos_beta"] = numpy.array(c)
    return data


E2E = {
    # name: (builder, kwargs, steps, keep_steps, fields)
    "slice_2d": (workloads.slice_2d, {}, 200, {1, 2, 5, 10, 50, 100, 200},
                 ("P", "C", "qx", "qz")),
    "reservoir_3d": (workloads.reservoir_3d, {"nx": 12, "ny": 10, "nz": 8, "seed": 11},
                     8, {1, 2, 4, 8}, ("P", "C", "T", "qx", "qy", "qz", "rho_f")),
    "sloped_3d": (workloads.sloped_3d, {"nx": 10, "ny": 8, "nz": 6, "seed": 5},
                  5, {1, 3, 5}, ("P", "C", "T", "qx", "qy", "qz")),
    "ensemble_member": (workloads.ensemble_member, {"seed": 3, "shape": (9, 7, 8)},
                        6, {1, 3, 6}, ("P", "C", "T", "qx", "qy", "qz")),
    "serving_request": (workloads.serving_request, {"seed": 4, "n": 9},
                        5, {1, 5}, ("P", "C", "T", "qz")),
    "slice_2d_plot": (workloads.slice_2d_plot, {}, 100, {1, 50, 100}, ("P", "C", "qx", "qz")),
    "slice_2d_chem": (workloads.slice_2d_chem, {}, 24, {1, 2, 3, 12, 24}, ("P", "C", "phi", "qz")),
    "slice_2d_chemcell": (workloads.slice_2d_chem, {"per_cell": True}, 8, {1, 2, 3, 8},
                          ("P", "C", "phi", "qz")),
    "slice_2d_dynbc": (workloads.slice_2d_dynbc, {}, 60, {1, 22, 23, 24, 30, 43, 44, 45, 60},
                       ("P", "C", "qx", "qz", "rho_f", "BC", "BP", "WP")),
}


def gen_e2e(ref, name):
    builder, kw, steps, keep, fields = E2E[name]
    cfg = builder(**kw)
    data, ns = run_reference(ref, cfg, steps, keep, fields)
    data["config_checksum"] = numpy.array(cases.config_checksum(builder(**kw)))
    return data


COURSE = {
    # name: (folder under course/, fields, keep_steps) -- run to the end time
    "course_01": ("01-groundwater_flow", ("P", "qx", "qy"), {1, 10, 100}),
    "course_02": ("02-groundwater_heat_flow", ("P", "T", "qx", "qy"), {1, 10, 100}),
    "course_03": ("03-groundwater_heat_tracer_flow", ("P", "T", "C", "qx", "qy"), {1, 10, 100}),
    "course_04": ("04-groundwater_heat_tracer_eos", ("P", "T", "C", "qx", "qy", "rho_f", "nue"),
                  {1, 10, 100}),
}
# config attributes not stored: the checkout path, the raw EOS table (only
# its fitted coefficients are used), poly1d objects
COURSE_SKIP = {"CFDIR", "data"}


def load_course_config(ref, folder):
    import importlib.util
    path = os.path.join(ref, "course", folder, "config.py")
    spec = importlib.util.spec_from_file_location("course_" + folder[:2], path)
    cfg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(cfg)
    return cfg


def gen_course(ref, name):
    folder, fields, keep = COURSE[name]
    cfg = load_course_config(ref, folder)
    data = cases.config_attributes(cfg, skip=COURSE_SKIP)
    rebuilt = cases.config_from_fixture(data, name)
    data["config_checksum"] = numpy.array(cases.config_checksum(rebuilt))
    out, ns = run_reference(ref, cfg, 10 ** 9, keep, fields, keep_plots=False)
    data.update(out)
    return data


LOGS = {
    # name: (builder, kwargs, steps) -- the reference's per-step log lines
    "slice_2d": (workloads.slice_2d, {}, 30),
    "reservoir_3d": (workloads.reservoir_3d, {"nx": 12, "ny": 10, "nz": 8, "seed": 11}, 6),
}


def gen_log(ref, name):
    """The lines tse.py prints for every step (PRINTOUT = 1), from the first
    flow line on; the run stops inside the last step, after its flow lines."""
    builder, kw, steps = LOGS[name]
    cfg = builder(**kw)
    cfg.PRINTOUT = 1
    _, ns = run_reference(ref, cfg, steps, set(), ())
    lines = ns["__stdout__"].split("\n")
    first = [k for k, l in enumerate(lines) if "[CFL]" in l][0]
    return "\n".join(lines[first:]).rstrip("\n") + "\n"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("TSE_REFERENCE", "/root/reference"))
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    jobs = [("unit_a", lambda: gen_unit(a.reference, "a")),
            ("unit_b", lambda: gen_unit(a.reference, "b"))]
    jobs += [("e2e_" + n, (lambda n=n: gen_e2e(a.reference, n))) for n in E2E]
    jobs += [(n, (lambda n=n: gen_course(a.reference, n))) for n in COURSE]
    for name in LOGS:
        if a.only and a.only != "log_" + name:
            continue
        path = os.path.join(HERE, "log_%s.txt" % name)
        with open(path, "w") as f:
            f.write(gen_log(a.reference, name))
        print("wrote", path)
    for name, fn in jobs:
        if a.only and a.only != name:
            continue
        data = fn()
        path = os.path.join(HERE, name + ".npz")
        numpy.savez_compressed(path, **data)
        print("wrote", path, "%.1f KB" % (os.path.getsize(path) / 1024))


if __name__ == "__main__":
    main()
