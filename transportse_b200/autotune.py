"""Autotuner of the staged FP32 correction sweep.

The mixed-precision solves spend nearly all their time in one kernel, the
bulk-copy staged red-black sweep (``dc_sweep_tma_kernel``).  Its shape is a
compile-time choice among 18 instances:

* chunk -- cells a producer copies and a consumer group relaxes at a time
  (256, 512, 1024): larger chunks issue fewer, larger copies, smaller ones
  balance a phase's last round better on small grids;
* ring -- stages a pipeline keeps in flight (2-4), as many as shared memory
  holds for the grid's window sizes;
* pipes -- pipelines a block (2 with one block per SM, or 1 with two blocks
  per SM).

``tune_sweep`` times each variant on the model's own pressure solve (exactly
``iters`` red+black iterations, the sweep kernel's own event time, the state
restored afterwards) and sets the fastest as the model's ``sweep_variant``;
the choice is kept per grid shape, so later models of the same shape take it
without timing.  The variant changes only how the same cell updates are
scheduled: every cell update is the same; only the grouping of the
convergence check's sums follows the chunking, so the solves agree bit for bit
unless a norm falls within rounding of its tolerance.  SOR's omega is not a knob
here: it is the config's, and it sets the reference's iteration sequence.
"""
from __future__ import annotations

import statistics

import torch

CHUNKS = (256, 512, 1024)
RINGS = (2, 3, 4)
PIPES = (2, 1)
VARIANTS = tuple((c, r, p) for c in CHUNKS for p in PIPES for r in RINGS)

_chosen = {}


def _timed_solve(sim, variant, iters):
    """Sweep-kernel ms and iterations of one pressure solve of ``iters``
    iterations that never converges and stops at its first dt halving."""
    M, S = sim.M, sim.S
    M.sweep_variant = variant
    M.sweep_timed.clear()
    timing, dmin = M.timing, getattr(M, "dc_min_conv", None)
    M.timing, M.dc_min_conv = True, 0.0
    try:
        M.compute_P(S["P"], S["c_f"], S["nue"], S["rho_f"], S["phi"], S["Kx"], S["Ky"], S["Kz"],
                    S["qx"], S["qy"], S["qz"], 3600.0, S["BP"], S["WP"], SOR=1.9, max_it=iters,
                    inc_it=1.25, max_dt=1e6, min_dt=2700.0, P_conv=0.0)
    finally:
        M.timing = timing
        if dmin is None:
            del M.dc_min_conv
        else:
            M.dc_min_conv = dmin
    ms = sum(x[3] for x in M.sweep_timed)
    its = sum(x[2] for x in M.sweep_timed)
    ran = M.last_variant
    M.sweep_timed.clear()
    return ms, its, ran


def tune_sweep(sim, iters=64, repeats=3, variants=VARIANTS, cache=True):
    """Pick the fastest staged-sweep variant for ``sim``'s grid (a
    driver.Simulation in the 'fp32dc' precision); returns a record of the
    choice and every trial, and sets ``sim.M.sweep_variant``."""
    M = sim.M
    if M.precision != "fp32dc":
        raise ValueError("the sweep autotuner is for the mixed-precision form")
    key = (M.nx, M.ny, M.nz)
    if cache and key in _chosen:
        M.sweep_variant = _chosen[key]["variant"]
        return dict(_chosen[key], cached=True)
    P0 = sim.S["P"].clone()
    trials = []
    seen = set()
    failed = []
    for v in variants:
        ms_list, ran = [], None
        try:
            for _ in range(repeats):
                ms, its, ran = _timed_solve(sim, v, iters)
                ms_list.append(ms / max(1, its))
        except RuntimeError as e:
            # a trial whose solve stopped (a bounded device wait ran out)
            # is left out; the state is restored below
            failed.append({"variant": tuple(v), "error": str(e)})
            ran = None
        sim.S["P"].copy_(P0)
        if ran is None or ran[0] == 0 or ran in seen:
            continue   # the plain-load sweep ran, or a variant already timed
        seen.add(ran)
        trials.append({"chunk": ran[0], "ring": ran[1], "pipes": ran[2],
                       "us_per_iteration": 1e3 * statistics.median(ms_list)})
    torch.cuda.synchronize()
    if not trials:
        M.sweep_variant = (0, 0, 0)
        return {"variant": (0, 0, 0), "trials": [], "failed": failed,
                "note": "no staged variant fits this grid"}
    best = min(trials, key=lambda t: t["us_per_iteration"])
    rec = {"variant": (best["chunk"], best["ring"], best["pipes"]),
           "us_per_iteration": best["us_per_iteration"], "iters": iters, "trials": trials}
    if failed:
        rec["failed"] = failed
    M.sweep_variant = rec["variant"]
    if cache:
        _chosen[key] = rec
    return rec
