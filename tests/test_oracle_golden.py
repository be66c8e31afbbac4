"""The oracle (C restatement of tse.py's kernels + its driver loop) against
the golden fixtures generated by running the reference itself
(tests/golden/make_golden.py).  Bit-exact agreement is required."""
import numpy
import pytest

from oracle import driver as odriver
from oracle.oracle import OracleModel
from tests.golden import cases
from tests.golden.make_golden import COURSE, E2E
from tests.helpers import check_snapshots, load


@pytest.mark.parametrize("variant", ["a", "b"])
def test_oracle_unit_kernels_bit_exact(variant):
    fx = load("unit_" + variant)
    cfg, inp = cases.unit_inputs_with_cfg(variant)
    # the committed inputs are the ones the generator used
    for k, v in inp.items():
        assert numpy.array_equal(fx["in_" + k], v), k
    m = OracleModel(cfg)
    assert m.sinb == float(fx["sin_beta"]) and m.cosb == float(fx["cos_beta"])
    out = cases.run_unit_calls(m, inp, variant)
    for k, v in out.items():
        assert numpy.array_equal(fx["out_" + k], v, equal_nan=True), k


@pytest.mark.parametrize("name", sorted(E2E))
def test_oracle_driver_bit_exact(name, tmp_path):
    builder, kw, steps, keep, fields = E2E[name]
    fx = load("e2e_" + name)
    cfg = builder(**kw)
    assert cases.config_checksum(cfg) == str(fx["config_checksum"])
    got = {}
    scal = {k: [] for k in ("dt", "t_sim", "numitP", "numitC", "numitT", "num_CFL")}

    def tap(rec, S):
        for k in scal:
            scal[k].append(rec[k])
        if rec["step"] in keep:
            for f in fields:
                got["%s@%d" % (f, rec["step"])] = S[f].copy()

    S = odriver.run(cfg, max_steps=steps, on_step=tap, plot_prefix=str(tmp_path / "snap"))
    if "n_plots" in fx.files:
        check_snapshots(S["plots"], fx, 0)
    for k, v in scal.items():
        assert numpy.array_equal(numpy.array(v), fx["s_" + k]), k
    for k in fx.files:
        if "@" in k:
            assert numpy.array_equal(fx[k], got[k]), k


@pytest.mark.parametrize("name", sorted(COURSE))
def test_oracle_course_models_bit_exact(name, tmp_path):
    """The reference's own example models (course/01..04), run to their end
    time with snapshots on: every step's dt, t and iteration counts, the fields
    at the kept steps and at the end, and the number of snapshot files."""
    fx = load(name)
    cfg = cases.config_from_fixture(fx, name)
    assert cases.config_checksum(cfg) == str(fx["config_checksum"])
    keep = set(int(s) for s in fx["keep_steps"])
    fields = sorted({k.split("@")[0] for k in fx.files if "@" in k})
    got = {}
    scal = {k: [] for k in ("dt", "t_sim", "numitP", "numitC", "numitT", "num_CFL")}

    def tap(rec, S):
        for k in scal:
            scal[k].append(rec[k])
        if rec["step"] in keep:
            for f in fields:
                got["%s@%d" % (f, rec["step"])] = S[f].copy()

    S = odriver.run(cfg, on_step=tap, plot_prefix=str(tmp_path / "snap"))
    for f in fields:
        got[f + "@final"] = S[f]
    assert len(S["plots"]) == int(fx["n_plot_files"])
    for k, v in scal.items():
        assert numpy.array_equal(numpy.array(v), fx["s_" + k]), k
    for k in fx.files:
        if "@" in k:
            assert numpy.array_equal(fx[k], got[k]), k
