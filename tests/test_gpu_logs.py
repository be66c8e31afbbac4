"""Log-line parity: with PRINTOUT = 1 the GPU driver (FP64 form) prints, for
every step, the lines the reference prints (tests/golden/log_*.txt, recorded
from tse.py): the flow line with the CFL share and the Peclet maxima, the
extrema of P, T and C, the Picard lines, and the step line -- character for
character, so logs of the two diff cleanly."""
import contextlib
import io
import os

import pytest

from tests.golden.make_golden import LOGS

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", sorted(LOGS))
def test_driver_log_lines_match_reference(name, cuda_device):
    from transportse_b200.driver import Simulation
    builder, kw, steps = LOGS[name]
    ref = open(os.path.join(HERE, "log_%s.txt" % name)).read().rstrip("\n").split("\n")
    cfg = builder(**kw)
    cfg.PRINTOUT = 1
    sim = Simulation(cfg, device=cuda_device, verbose=True)
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        sim.run(max_steps=steps)
    lines = out.getvalue().split("\n")
    first = [k for k, l in enumerate(lines) if "[CFL]" in l][0]
    got = lines[first:first + len(ref)]
    for k, (g, r) in enumerate(zip(got, ref)):
        assert g == r, (k, g, r)
    assert len(got) == len(ref)
