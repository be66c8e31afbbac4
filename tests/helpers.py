"""Test helpers: NumPy adaptor over the CUDA kernels, fixture loading, errors."""
import os

import numpy

from tests.conftest import GOLDEN


def load(name):
    return numpy.load(os.path.join(GOLDEN, name + ".npz"))


def unit_inputs(fixture):
    return {k[3:]: fixture[k] for k in fixture.files if k.startswith("in_")}


def rel_err(got, ref):
    """max |got - ref| / max(|ref|max, tiny): relative to the field's scale."""
    got = numpy.asarray(got, dtype=numpy.float64)
    ref = numpy.asarray(ref, dtype=numpy.float64)
    if got.shape != ref.shape:
        raise AssertionError("shape %s != %s" % (got.shape, ref.shape))
    nan_g, nan_r = numpy.isnan(got), numpy.isnan(ref)
    if not numpy.array_equal(nan_g, nan_r):
        return numpy.inf
    g, r = got[~nan_r], ref[~nan_r]
    if g.size == 0:
        return 0.0
    scale = max(numpy.max(numpy.abs(r)), 1e-300)
    return float(numpy.max(numpy.abs(g - r)) / scale)


class NumpyKernels:
    """Reference kernel names over transportse_b200.kernels.Model, taking and
    returning NumPy arrays (so tests/golden/cases.run_unit_calls can drive it)."""

    def __init__(self, model):
        self.m = model

    def _np(self, x):
        import torch
        return x.detach().cpu().numpy().copy() if isinstance(x, torch.Tensor) else x

    def compute_P(self, *a, **k):
        r = self.m.compute_P(*a, **k)
        return r[0], r[1], self._np(r[2]), self._np(r[3]), r[4], r[5]

    def compute_q(self, *a, **k):
        return tuple(self._np(x) for x in self.m.compute_q(*a, **k))

    def flow_error(self, *a, **k):
        return self._np(self.m.flow_error(*a, **k))

    def compute_C(self, *a, **k):
        r = self.m.compute_C(*a, **k)
        return r[0], r[1], self._np(r[2]), r[3], r[4]

    def compute_T(self, *a, **k):
        r = self.m.compute_T(*a, **k)
        return r[0], r[1], self._np(r[2]), r[3], r[4]

    def smolarkiewicz(self, *a, **k):
        return tuple(self._np(x) for x in self.m.smolarkiewicz(*a, **k))

    def explicit_C(self, *a, **k):
        return self.m.explicit_C(*a, **k)

    def l2_norm(self, *a, **k):
        return self.m.l2_norm(*a, **k)


def model_for(cfg, device, precision="fp64"):
    from transportse_b200.kernels import Model
    m = Model.from_config(cfg, device=device, precision=precision)
    m.freeze(cfg.c_r, cfg.l_r, cfg.rho_r, cfg.cp_r, cfg.lf_l, cfg.lf_t, cfg.lt_l, cfg.lt_t,
             cfg.C_IMBLFLO, cfg.T_IMBLFLO)
    return m


def check_snapshots(files, fx, tol):
    """The snapshot files a run wrote against the reference's (fixture keys
    "plot<k>_<item>", a missing key meaning "as in plot0"): same count, same
    tuple layout, integers and flags equal, floating-point items within
    ``tol`` relative to each item's scale (0: bit for bit)."""
    import joblib
    from tests.golden.make_golden import SNAPSHOT_ITEMS
    n = int(fx["n_plots"])
    assert len(files) == n, (len(files), n)
    for k, f in enumerate(files):
        assert f.endswith("-%05d.p" % k), f
        got = joblib.load(f)
        assert len(got) == len(SNAPSHOT_ITEMS)
        for name, v in zip(SNAPSHOT_ITEMS, got):
            key = "plot%d_%s" % (k, name)
            ref = fx[key] if key in fx.files else fx["plot0_" + name]
            v = numpy.asarray(v)
            assert v.shape == ref.shape, (k, name, v.shape, ref.shape)
            if tol == 0 or name in ("nx", "ny", "nz", "BP", "BC", "BT", "t_sim"):
                assert numpy.array_equal(v, ref), (k, name)
            else:
                assert rel_err(v, ref) <= tol, (k, name, rel_err(v, ref))


SCALARS = ("dt", "t_sim", "numitP", "numitC", "numitT", "num_CFL")


def run_fixture_case(cfg, fx, device, precision, tmp_path, steps=None):
    """Run ``cfg`` through the GPU driver the way the fixture ``fx`` was
    recorded: per-step scalars every step, the fixture's fields at its kept
    steps (after the step's dynamic_bc and equation of state) and, when the
    fixture ran to the end time, at the end ("<field>@final").  Returns
    (scalars, fields, simulation)."""
    from transportse_b200.driver import Simulation
    keep = set(int(s) for s in fx["keep_steps"])
    fields = sorted({k.split("@")[0] for k in fx.files if "@" in k})
    got = {}
    scal = {k: [] for k in SCALARS}

    def tap(rec, sim):
        for k in scal:
            scal[k].append(rec[k])
        if rec["step"] in keep:
            for f in fields:
                got["%s@%d" % (f, rec["step"])] = sim.field(f)

    sim = Simulation(cfg, device=device, precision=precision, plot_prefix=str(tmp_path / "snap"))
    sim.run(max_steps=steps, on_step=tap)
    if any(k.endswith("@final") for k in fx.files):
        for f in fields:
            got[f + "@final"] = sim.field(f)
    return scal, got, sim


def dynamic_pressure_err(got_P, ref_P, P0):
    """The pressure change since the start (P - P0, mostly the flow-driven
    part: P itself is dominated by the hydrostatic head) compared on its own
    scale."""
    return rel_err(numpy.asarray(got_P) - P0, numpy.asarray(ref_P) - P0)
