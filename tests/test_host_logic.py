"""Host-side logic that needs no GPU: the colour-split index arithmetic the
kernels use, the EOS declaration check, the HBM admission budget, trace and
workload determinism, and ensemble sharding across ranks."""
import threading
import time

import numpy
import pytest

from transportse_b200 import eos, workloads


def _layout(nx, ny, nz):
    nzp = nz + (nz & 1)
    H = nzp // 2
    return nzp, H, ny * H


@pytest.mark.parametrize("shape", [(3, 4, 5), (2, 1, 7), (4, 3, 6), (1, 1, 9), (5, 5, 1)])
def test_colour_split_neighbour_arithmetic(shape):
    """Compact index m = ((i*ny + j)*nzp + k) >> 1 per colour; neighbours of
    the other colour at m +- SX, m +- H, m + (k&1), m - 1 + (k&1) (the
    offsets used by the sweep kernels) -- checked against the grid."""
    nx, ny, nz = shape
    nzp, H, SX = _layout(nx, ny, nz)
    idx = {}
    for i in range(nx):
        for j in range(ny):
            for k in range(nzp):
                col = (i + j + k) & 1
                m = ((i * ny + j) * nzp + k) >> 1
                assert (col, m) not in idx
                idx[(col, m)] = (i, j, k)
    assert len(idx) == 2 * nx * ny * H
    for (col, m), (i, j, k) in idx.items():
        if k >= nz:
            continue
        other = 1 - col
        # the reference's red cells: (i + j + k) % 2 == 0 (tse.py:170-176)
        assert (col == 0) == ((i + j + k) % 2 == 0)
        if i < nx - 1:
            assert idx[(other, m + SX)] == (i + 1, j, k)
        if i > 0:
            assert idx[(other, m - SX)] == (i - 1, j, k)
        if j < ny - 1:
            assert idx[(other, m + H)] == (i, j + 1, k)
        if j > 0:
            assert idx[(other, m - H)] == (i, j - 1, k)
        if k < nz - 1:
            assert idx[(other, m + (k & 1))] == (i, j, k + 1)
        if k > 0:
            assert idx[(other, m - 1 + (k & 1))] == (i, j, k - 1)


def test_declared_eos_validates_against_callback():
    cfg = workloads.reservoir_3d(6, 5, 4, seed=1)
    decl = eos.declared_eos(cfg)
    assert eos.validate(cfg, decl)
    bad = dict(decl)
    bad["rho"] = dict(decl["rho"], tcoef=0.31)
    with pytest.raises(eos.EOSMismatch):
        eos.validate(cfg, bad)


def test_declared_polynomial_eos_of_the_course_model_validates():
    """The course model with an equation of state (course/04): density and
    viscosity polynomials in T, guarded by species 2.  The declaration matches
    the callback bit for bit (the probes include C[2] == 1, the guarded case);
    a changed coefficient, a changed guard or plain pow() powers do not."""
    from tests.golden import cases
    from tests.helpers import load
    cfg = cases.config_from_fixture(load("course_04"), "course_04")
    decl = eos.declared_eos(cfg)
    assert decl["rho"]["kind"] == "poly4_T" and decl["nue"]["unless"] == (2, 1.0)
    assert eos.validate(cfg, decl)
    bad = dict(decl, nue=dict(decl["nue"], coef=[v * (1 + 1e-12) for v in decl["nue"]["coef"]]))
    with pytest.raises(eos.EOSMismatch):
        eos.validate(cfg, bad)
    with pytest.raises(eos.EOSMismatch):
        eos.validate(cfg, dict(decl, rho=dict(decl["rho"], unless=(1, 1.0))))
    cd = [float(v) for v in cfg.c_dens]

    def pow_callback(C, T, P, nue, rho_f, *rest):
        if C[2] != 1:
            rho_f = cd[4] + cd[3] * T + cd[2] * T ** 2 + cd[1] * T ** 3 + cd[0] * T ** 4
        return (C, T, P, nue, rho_f) + rest

    # the same polynomial through libm's pow differs in the last bit somewhere
    T = numpy.random.default_rng(3).uniform(0.0, 150.0, 4000)
    rho = {"kind": "poly4_T", "coef": cd}
    assert any(eos.eval_form_host(rho, [0, 0, 0], t, 0.0) != pow_callback(
        [0, 0, 0], t, 0, 0, 0)[4] for t in T)


def test_declared_eos_forms_are_checked():
    cfg = workloads.slice_2d(6, 1, 4)
    cfg.GPU_EOS = {"rho": {"kind": "poly4_T", "coef": [1, 2, 3]}}
    with pytest.raises(ValueError):
        eos.declared_eos(cfg)
    cfg.GPU_EOS = {"nue": {"kind": "linear"}}
    with pytest.raises(ValueError):
        eos.declared_eos(cfg)
    cfg.GPU_EOS = {"rho": {"kind": "linear", "rho0": 1000.0, "species": [], "tcoef": 0.0,
                           "T0": 0.0, "unless": (0, 1.0)}}
    with pytest.raises(ValueError):
        eos.declared_eos(cfg)
    cfg.GPU_EOS = {"visc": {"kind": "keep"}}
    with pytest.raises(ValueError):
        eos.declared_eos(cfg)
    cfg.GPU_EOS = {"nue": {"kind": "constant", "value": 1e-3}}
    d = eos.declared_eos(cfg)
    assert d["rho"]["kind"] == "keep" and d["nue"]["value"] == 1e-3


def test_hbm_budget_blocks_until_release():
    from transportse_b200.ensemble import HbmBudget
    b = HbmBudget(100)
    assert b.acquire(60)
    got = []

    def late():
        got.append(b.acquire(50))

    th = threading.Thread(target=late)
    th.start()
    time.sleep(0.2)
    assert not got            # 60 + 50 > 100: waits
    b.release(60)
    th.join(timeout=5)
    assert got == [True]
    with pytest.raises(MemoryError):
        b.acquire(101)


def test_poisson_trace_is_seeded():
    from transportse_b200.serving import poisson_trace
    a = poisson_trace(5, 20.0, 3, workloads.serving_request, 2, n_min=8, n_max=12)
    b = poisson_trace(5, 20.0, 3, workloads.serving_request, 2, n_min=8, n_max=12)
    assert [x[0] for x in a] == [x[0] for x in b]
    assert a[0][0] == 0.0 and all(a[i][0] <= a[i + 1][0] for i in range(4))
    assert [x[1].nx for x in a] == [x[1].nx for x in b]


def test_workload_builders_are_deterministic():
    from tests.golden.cases import config_checksum
    for f, kw in ((workloads.reservoir_3d, dict(nx=8, ny=6, nz=5, seed=4)),
                  (workloads.sloped_3d, dict(nx=6, ny=5, nz=4, seed=2)),
                  (workloads.ensemble_member, dict(seed=7)),
                  (workloads.serving_request, dict(seed=8, n=10))):
        assert config_checksum(f(**kw)) == config_checksum(f(**kw))


def test_shard_balances_and_covers():
    from transportse_b200.ensemble import shard
    sizes = [int(x) for x in numpy.random.default_rng(0).integers(1000, 100000, 37)]
    parts = [shard(sizes, r, 4) for r in range(4)]
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(37))
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert max(loads) <= 1.25 * (sum(sizes) / 4) + max(sizes)


def test_batch_gate_launches_when_every_member_waits(monkeypatch):
    """BatchGate: no launch while a member is still between solves; one launch
    per solve kind once all wait; members that leave release the rest."""
    import threading
    import time
    from transportse_b200 import batch as B

    launched = []

    def fake_launch(self, reqs):
        launched.append(sorted(r.name for r in reqs))

    monkeypatch.setattr(B.BatchGate, "_launch", fake_launch)
    monkeypatch.setattr(B.torch.cuda, "current_stream", lambda device=None: None)
    gate = B.BatchGate("cpu")
    order = []

    def member(name, delay, solves):
        try:
            for _ in range(solves):
                time.sleep(delay)
                gate.submit(name, None, None, None, None, 0, 128)
                order.append(name)
        finally:
            gate.leave()

    for _ in range(3):
        gate.join()   # all three are members before any submits
    ths = [threading.Thread(target=member, args=a, daemon=True)
           for a in (("compute_P", 0.0, 2), ("compute_T", 0.05, 2), ("compute_P", 0.1, 1))]
    for t in ths:
        t.start()
    for t in ths:
        t.join(timeout=10)
    assert not any(t.is_alive() for t in ths)
    # first flush waits for the slowest member: all three solves together
    assert launched[0] == ["compute_P", "compute_P", "compute_T"]
    # the rest flush once the third member has left
    assert sum(len(x) for x in launched) == 5
    assert gate.members == 0 and gate.running == 0


def test_eager_batch_gate_overlaps_host_work_with_a_running_batch(monkeypatch):
    """BatchGate(eager=True): a solve goes out as soon as it waits and no batch
    runs, without waiting for the other members; the gate's lock is free while
    a batch runs, so a member submits meanwhile and its solve forms the next
    batch once the running one ends."""
    import threading
    import time
    from transportse_b200 import batch as B

    launched = []

    def fake_launch(self, reqs):
        launched.append(sorted(r.name for r in reqs))
        time.sleep(0.2)          # the batch occupies the GPU

    monkeypatch.setattr(B.BatchGate, "_launch", fake_launch)
    monkeypatch.setattr(B.torch.cuda, "current_stream", lambda device=None: None)
    gate = B.BatchGate("cpu", eager=True)
    done = {}

    def member(name, delay):
        try:
            time.sleep(delay)
            gate.submit(name, None, None, None, None, 0, 128)
            done[name] = time.perf_counter()
        finally:
            gate.leave()

    for _ in range(3):
        gate.join()
    t0 = time.perf_counter()
    ths = [threading.Thread(target=member, args=a, daemon=True)
           for a in (("compute_P", 0.0), ("compute_T", 0.05), ("compute_C", 0.1))]
    for t in ths:
        t.start()
    for t in ths:
        t.join(timeout=10)
    assert not any(t.is_alive() for t in ths)
    # the first solve went out alone; the two that arrived during it, together
    assert launched == [["compute_P"], ["compute_C", "compute_T"]]
    # the first member returned as its own batch ended, a batch before the others
    assert done["compute_T"] - t0 >= 0.4 - 0.02
    assert done["compute_T"] - done["compute_P"] >= 0.1
    assert gate.members == 0 and gate.running == 0 and not gate.launching


@pytest.mark.parametrize("eager", [False, True])
def test_batch_gate_failure_reaches_its_batch_and_the_gate_recovers(monkeypatch, eager):
    """A batched call that raises: every member of that batch gets the error,
    the gate's lock and counters are left consistent, and later solves go out
    normally."""
    import threading
    from transportse_b200 import batch as B

    calls = []

    def fake_launch(self, reqs):
        calls.append(len(reqs))
        if len(calls) == 1:
            raise RuntimeError("launch failed")

    monkeypatch.setattr(B.BatchGate, "_launch", fake_launch)
    monkeypatch.setattr(B.torch.cuda, "current_stream", lambda device=None: None)
    gate = B.BatchGate("cpu", eager=eager)
    errors, ok = [], []
    start = threading.Barrier(2)

    def member():
        try:
            start.wait()
            for k in range(2):
                try:
                    gate.submit("compute_P", None, None, None, None, 0, 128)
                    ok.append(k)
                except RuntimeError as e:
                    errors.append((k, str(e)))
        finally:
            gate.leave()

    for _ in range(2):
        gate.join()
    ths = [threading.Thread(target=member, daemon=True) for _ in range(2)]
    for t in ths:
        t.start()
    for t in ths:
        t.join(timeout=10)
    assert not any(t.is_alive() for t in ths)
    # whoever was in the first batch saw its failure; every later solve ran
    assert errors and all(k == 0 and msg == "launch failed" for k, msg in errors)
    assert len(errors) == calls[0] and len(ok) == 4 - len(errors)
    assert gate.members == 0 and gate.running == 0 and not gate.launching and not gate.pending


def _last_at_or_before(starts, q):
    """The device loop's binary search (fused_fill_kernel,
    fused_residual_kernel): the last index k with starts[k] <= q."""
    lo, hi = 0, len(starts) - 1
    while lo < hi:
        mid = (lo + hi + 1) >> 1
        if starts[mid] <= q:
            lo = mid
        else:
            hi = mid - 1
    return lo


def test_device_loop_index_maps_cover_every_chunk_and_residual_block():
    """The batched device loop maps chunk q of a launch to its model through
    the models' chunk ranges, and residual block vb to its model through the
    residual prefix sums, in which models without a residual this pass have
    no blocks: every chunk and every block lands in exactly one model, at the
    right offset, never in a model with an empty range."""
    import random
    rng = random.Random(17)
    for _ in range(300):
        n = rng.randint(1, 40)
        nchunks = [rng.randint(1, 9) for _ in range(n)]          # every model >= 1 chunk
        cfirst = [sum(nchunks[:k]) for k in range(n)]
        seen = []
        for q in range(sum(nchunks)):
            k = _last_at_or_before(cfirst, q)
            assert cfirst[k] <= q < cfirst[k] + nchunks[k]
            seen.append((k, q - cfirst[k]))
        assert seen == [(k, j) for k in range(n) for j in range(nchunks[k])]
        rb = [rng.choice([0, 0, rng.randint(1, 2048)]) for _ in range(n)]   # residual blocks
        rstart = [sum(rb[:k]) for k in range(n)]
        blocks = []
        for vb in range(sum(rb)):
            k = _last_at_or_before(rstart, vb)
            assert rb[k] > 0 and 0 <= vb - rstart[k] < rb[k]
            blocks.append((k, vb - rstart[k]))
        assert blocks == [(k, b) for k in range(n) for b in range(rb[k])]


def test_snapshot_rule_matches_the_oracle(tmp_path):
    """driver.Snapshots (product) and oracle.driver.Plots (restatement of
    tse.py:312-329) give the same dt sequence and files, including a plot time
    that a step passes without landing on it (that one and all later ones are
    never written)."""
    import types
    import numpy
    from oracle.driver import Plots
    from transportse_b200.driver import Snapshots

    for times in ([0.0, 10.0, 25.0, 40.0], [5.0, 7.3, 100.0], [3.0, 3.5]):
        cfg = types.SimpleNamespace(PLOTSAVE=True, PLOTTIME=numpy.array(times))
        outs = []
        for k, cls in enumerate((Snapshots, Plots)):
            pl = cls(cfg, str(tmp_path / ("r%d" % k)))
            step = pl.step if cls is Snapshots else pl.__call__
            t_sim, dt = 0.0, 4.0
            dt, dt_prev = step(t_sim, dt, dt, lambda d: (t_sim, d))
            seq = []
            for n in range(30):
                seq.append(dt)
                t_sim += dt
                dt = 4.0 if n % 3 else 6.5          # the solvers' next dt
                if n == 4 and times[0] == 3.0:
                    t_sim += 0.25                    # step over a plot time
                dt, dt_prev = step(t_sim, dt, dt_prev, lambda d, t=t_sim: (t, d))
            outs.append((seq, [p[-8:] for p in pl.written], pl.index))
        assert outs[0] == outs[1], times


def _staged_copies_ok(nx, ny, nz, Hstage, C=512):
    """Every bulk copy of the staged sweep for one model (the arithmetic of
    tse_dc.cuh tma_stage / tma_issue_own / tma_issue_windows and of the
    consumers' window indices) is 16-byte aligned, a multiple of 16 bytes,
    inside its array, and every shared-memory index stays inside its window."""
    nzp = nz + (nz & 1)
    H = nzp // 2
    SX = ny * H
    Nc = nx * SX
    N = (Nc + 31) & ~31
    G = ((SX + 1024 + 16 + 63) // 64) * 64            # dc_margin
    lz = lambda h: (C + 2 * h + 5 + 3) & ~3
    lx = C + 4
    assert lz(H) <= lz(Hstage)
    base = 256 * 7                                      # any 256-aligned float region
    K = [base, base + 28 * N]
    dbase = base + 56 * N
    dlen = N + 2 * G
    D = [dbase + 4 * G, dbase + 4 * (dlen + G)]
    Dlo = [dbase, dbase + 4 * dlen]
    Dhi = [dbase + 4 * dlen, dbase + 8 * dlen]
    mask = [0, ((N + 255) // 256) * 256]
    for col in (0, 1):
        for q in range((Nc + C - 1) // C):
            m0 = q * C
            cnt = min(C, N - m0)
            zs, xps, xms = (m0 - H - 1) & ~3, (m0 + SX) & ~3, (m0 - SX) & ~3
            copies = [(K[col] + 24 * m0, 24 * cnt, K[col], K[col] + 24 * N),
                      (K[col] + 24 * N + 4 * m0, 4 * cnt, K[col] + 24 * N, K[col] + 28 * N),
                      (mask[col] + m0, cnt, mask[col], mask[col] + N),
                      (D[col] + 4 * m0, 4 * cnt, Dlo[col], Dhi[col]),
                      (D[1 - col] + 4 * zs, 4 * lz(H), Dlo[1 - col], Dhi[1 - col]),
                      (D[1 - col] + 4 * xps, 4 * lx, Dlo[1 - col], Dhi[1 - col]),
                      (D[1 - col] + 4 * xms, 4 * lx, Dlo[1 - col], Dhi[1 - col])]
            for a, n, lo, hi in copies:
                if a % 16 or n % 16 or a < lo or a + n > hi:
                    return False
            oz, oxp, oxm = m0 - zs, m0 + SX - xps, m0 - SX - xms
            nval = min(C, Nc - m0)
            l = nval - 1
            if not (0 <= oz - H - 1 and l + oz + H < lz(H) and 0 <= oxp and l + oxp < lx
                    and 0 <= oxm and l + oxm < lx):
                return False
    return True


def test_staged_sweep_copies_stay_aligned_and_in_bounds():
    import random
    rng = random.Random(5)
    shapes = [(1, 1, 1), (1, 1, 2), (2, 1, 1), (3, 3, 3), (1, 1, 40), (9, 1, 31), (5, 7, 3),
              (60, 1, 30), (33, 17, 21), (2, 2, 600), (60, 40, 2), (64, 64, 32), (128, 96, 77),
              (1, 2, 1600), (1, 2, 4000)]
    shapes += [(rng.randint(1, 40), rng.randint(1, 40), rng.randint(1, 300)) for _ in range(60)]
    # single model: the stage fits its own H; fused batch: the tallest column's
    Hmax = max((nz + (nz & 1)) // 2 for _, _, nz in shapes)
    for nx, ny, nz in shapes:
        H = (nz + (nz & 1)) // 2
        # every compiled chunk size of the single-model sweep (the autotuner's
        # choices); the fused batch keeps 512
        for C in (256, 512, 1024):
            assert _staged_copies_ok(nx, ny, nz, H, C), (nx, ny, nz, C)
        assert _staged_copies_ok(nx, ny, nz, Hmax), (nx, ny, nz, "fused")


def _exact_staged_ok(nx, ny, nz, nst, count, sol, C=256):
    """Every bulk copy of the staged FP64 solve (tse_rbsolve_tma.cuh x_plan,
    the producer's copies and x_window's clamping) is 16-byte aligned in
    global and shared memory, a multiple of 16 bytes, inside its array and
    its stage slot; every shared-memory index a consumer forms stays inside
    its window; and every neighbour a set flag lets a cell read lies in the
    copied part of its window.  count: arrays per colour of the form (17
    pressure, 15 transport), sol: the solution's array index."""
    nzp = nz + (nz & 1)
    H = nzp // 2
    SX = ny * H
    Nc = nx * SX
    N = (Nc + 31) & ~31
    al = lambda b: (b + 255) & ~255
    # workspace carve of setup_pressure / setup_transport (byte offsets)
    ws = 256 * 3
    mask = [ws + al(16) + al(2 * 16384 * 8), 0]
    mask[1] = mask[0] + al(N)
    arr = [mask[1] + al(N), 0]
    arr[1] = arr[0] + 8 * count * N
    ws_end = arr[1] + 8 * count * N
    X = [arr[0] + 8 * sol * N, arr[1] + 8 * sol * N]
    # x_plan
    xo = nst * C * 8
    msk = xo + C * 8
    wz = msk + C
    lz, lx = C + 2 * H + 2, C + 2
    wxp, wxm = wz + 8 * lz, wz + 8 * lz + 8 * lx
    nbytes = (wz + 8 * lz + 16 * lx + 127) & ~127

    def clamp(s, n):
        a, e = max(s, 0), min(s + n, N)
        return (a, e) if e > a else None

    for col in (0, 1):
        for q in range((Nc + C - 1) // C):
            m0 = q * C
            cnt = min(C, N - m0)
            if cnt % 32:
                return False
            zs, xps, xms = (m0 - H) & ~1, (m0 + SX) & ~1, (m0 - SX) & ~1
            # (global address, bytes, array lo, array hi, smem offset, smem slot end)
            copies = [(arr[col] + 8 * (k * N + m0), 8 * cnt, arr[col] + 8 * k * N,
                       arr[col] + 8 * (k + 1) * N, 8 * C * k, 8 * C * (k + 1)) for k in range(nst)]
            copies.append((X[col] + 8 * m0, 8 * cnt, X[col], X[col] + 8 * N, xo, msk))
            copies.append((mask[col] + m0, cnt, mask[col], mask[col] + N, msk, wz))
            win = {}
            for name, s0, n, off in (("z", zs, lz, wz), ("xp", xps, lx, wxp), ("xm", xms, lx, wxm)):
                r = clamp(s0, n)
                win[name] = (s0, r)
                if r:
                    a, e = r
                    copies.append((X[1 - col] + 8 * a, 8 * (e - a), X[1 - col], X[1 - col] + 8 * N,
                                   off + 8 * (a - s0), off + 8 * n))
            for g, n, lo, hi, d, dend in copies:
                if g % 16 or n % 16 or d % 16 or g < lo or g + n > hi or hi > ws_end:
                    return False
                if d + n > dend or dend > nbytes:
                    return False
            oz, oxp, oxm = m0 - zs, m0 + SX - xps, m0 - SX - xms
            for l in range(min(C, Nc - m0)):
                m = m0 + l
                i, j = divmod(m // H, ny)
                k = 2 * (m % H) + ((col + i + j) & 1)
                zo = k & 1
                iz = l + oz
                idx = [("xp", l + oxp, lx), ("xm", l + oxm, lx), ("z", iz + H, lz),
                       ("z", iz - H, lz), ("z", iz + zo, lz), ("z", iz - 1 + zo, lz)]
                for _, ix, n in idx:
                    if not 0 <= ix < n:
                        return False
                if k >= nz:
                    continue
                exists = [i < nx - 1, i > 0, j < ny - 1, j > 0, k < nz - 1, k > 0]
                off = [SX, -SX, H, -H, zo, zo - 1]
                for e, (name, ix, _), o in zip(exists, idx, off):
                    if not e:
                        continue
                    s0, r = win[name]
                    if r is None or not (r[0] <= m + o < r[1]) or s0 + ix != m + o:
                        return False
    return True


def test_exact_staged_copies_stay_aligned_and_in_bounds():
    import random
    rng = random.Random(11)
    shapes = [(1, 1, 1), (1, 1, 2), (2, 1, 1), (3, 3, 3), (1, 1, 40), (9, 1, 31), (5, 7, 3),
              (60, 1, 30), (33, 17, 21), (2, 2, 600), (60, 40, 2), (24, 24, 20), (7, 3, 257),
              (3, 2, 1000), (1, 2, 3000)]
    shapes += [(rng.randint(1, 24), rng.randint(1, 24), rng.randint(1, 120)) for _ in range(40)]
    for nx, ny, nz in shapes:
        for nst, count, sol in ((9, 17, 16), (11, 17, 16), (13, 17, 16),   # pressure
                                (9, 15, 14), (11, 15, 14)):                # transport
            assert _exact_staged_ok(nx, ny, nz, nst, count, sol), (nx, ny, nz, nst)


def test_server_cancels_pending_requests():
    """A request that has not started can be withdrawn; the others stay queued."""
    from transportse_b200 import workloads
    from transportse_b200.serving import Request, Server
    s = Server(device="cpu", slots=1, hbm_budget=1 << 40, max_blocks=8)
    a = s.submit(Request(0, workloads.serving_request(1, n=8), 1, 0.0))
    b = s.submit(Request(1, workloads.serving_request(2, n=8), 1, 0.1))
    assert s.cancel(0) is True
    assert a.cancelled and a.done.is_set() and a.error is not None
    assert s.cancel(0) is False and s.cancel(7) is False
    assert [item[1] for item in s.pending] == [1] and not b.done.is_set()


def test_batch_gate_sub_batches_by_cell_budget():
    """The fused form's sub-batches: every request once, sorted by size, each
    sub-batch within the budget unless a single model alone exceeds it; no
    split under the budget, with a cluster form or with the budget off."""
    import types
    from transportse_b200 import batch as B
    gate = B.BatchGate("cpu", batch_cells=1000)
    rng = numpy.random.default_rng(4)
    reqs = []
    for i in range(40):
        n = int(rng.integers(2, 12))
        reqs.append(types.SimpleNamespace(grid=types.SimpleNamespace(nx=n, ny=n, nz=3), i=i))
    cells = lambda r: r.grid.nx * r.grid.ny * r.grid.nz
    subs = gate._subbatches(reqs)
    flat = [r for s in subs for r in s]
    assert sorted(r.i for r in flat) == list(range(40))
    assert [cells(r) for r in flat] == sorted(cells(r) for r in reqs)
    for s in subs:
        assert sum(cells(r) for r in s) <= 1000 or len(s) == 1
    assert len(subs) > 1
    assert gate._subbatches(reqs[:3]) == [reqs[:3]]
    assert B.BatchGate("cpu", batch_cells=0)._subbatches(reqs) == [reqs]
    assert B.BatchGate("cpu", cluster=8, batch_cells=1000)._subbatches(reqs) == [reqs]
    assert B.default_batch_cells("cpu") == 0


def test_server_admission_without_and_with_a_slot_limit(monkeypatch):
    """Serving host logic, with a stand-in for the model run (no GPU):
    without a slot limit every request of a burst runs at once and a later
    burst reuses the finished workers; with slots=k at most k run at once."""
    import threading
    import time

    from transportse_b200 import serving
    state = {"live": 0, "peak": 0}
    lock = threading.Lock()

    def fake_run(config, steps, device, precision, max_blocks, keep=(), gate=None):
        with lock:
            state["live"] += 1
            state["peak"] = max(state["peak"], state["live"])
        time.sleep(0.1)
        with lock:
            state["live"] -= 1
        return {"cell_updates": 1}

    monkeypatch.setattr(serving, "run_model", fake_run)
    monkeypatch.setattr(serving, "state_bytes", lambda config, precision="fp32dc": 1)
    trace = [(0.0, None, 1)] * 8 + [(0.5, None, 1)] * 8
    for slots, peak, workers in ((0, 8, 8), (3, 3, 3)):
        state.update(live=0, peak=0)
        srv = serving.Server(device="cpu", slots=slots, hbm_budget=1 << 20, precision="fp64",
                             max_blocks=8, batched=False)
        reqs, st = srv.replay(trace)
        assert st["requests"] == 16 and all(r.error is None for r in reqs)
        assert st["cell_updates"] == 16
        assert state["peak"] == peak, (slots, state["peak"])
        assert len(srv.workers) == workers, (slots, len(srv.workers))


def test_face_means_are_the_same_from_either_cell():
    """The transport assemblies form each face's means once (the face pass)
    and both cells of the face read them.  That keeps every coefficient bit for
    bit only because the two cells' expressions differ by commuted operands:
    harm2(H1, H2, d1, d2) = (d1 + d2) / (d1/H1 + d2/H2) and
    amean2(X1, X2, d1, d2) = (X1 d1 + X2 d2) / (d1 + d2) with the two cells
    swapped.  IEEE-754 addition and multiplication commute, which this checks
    on random float64 operands over many magnitudes (numpy's float64
    operations round like the GPU's FP64 without contraction)."""
    import numpy
    rng = numpy.random.default_rng(7)
    n = 200000
    H1, H2 = [10.0 ** rng.uniform(-15, 5, n) for _ in range(2)]
    X1, X2 = [rng.uniform(-1e3, 1e3, n) for _ in range(2)]
    d1, d2 = [10.0 ** rng.uniform(-3, 3, n) for _ in range(2)]

    def harm2(a, b, da, db):
        return (da + db) / (da / a + db / b)

    def amean2(a, b, da, db):
        return (a * da + b * db) / (da + db)

    assert numpy.array_equal(harm2(H1, H2, d1, d2), harm2(H2, H1, d2, d1))
    assert numpy.array_equal(amean2(X1, X2, d1, d2), amean2(X2, X1, d2, d1))
    # the heat face's conductivity mix and the species face's product
    por = amean2(X1, X2, d1, d2) * 1e-4
    lr, lf = harm2(H1, H2, d1, d2), harm2(H2 * 3, H1 * 7, d1, d2)
    lr_s, lf_s = harm2(H2, H1, d2, d1), harm2(H1 * 7, H2 * 3, d2, d1)
    por_s = amean2(X2, X1, d2, d1) * 1e-4
    assert numpy.array_equal((1 - por) * lr + por * lf, (1 - por_s) * lr_s + por_s * lf_s)
