"""Ensembles of independent TRANSPORTSE models on one GPU.

A parameter or permeability ensemble is a list of config modules of uneven
grid sizes that share nothing.  ``Ensemble`` advances them concurrently: up
to ``concurrency`` models are resident at once, each driven by its own host
thread on its own CUDA stream through the full time-step driver
(``driver.Simulation``: SIA loop, pressure, fluxes, transport, EOS), so every
model progresses at its own pace.  Models are admitted as earlier ones finish
and their device memory is returned, under an HBM budget.

By default (``batched``, mixed-precision form) the models' threads meet at a
``BatchGate`` (transportse_b200.batch): each kind of solve of all models runs
as one fused launch -- every model's cells in one cooperative sweep sharing
its barriers, finished models dropping out -- so small models cost their
bytes rather than two device-wide barriers per iteration.  With
``batched=False`` each model solves on its own stream:
  * grids of up to ``cluster_cells`` cells: each solve is one launch of one
    thread-block cluster (tse_compute_*_dc_batch with one item);
  * larger grids: the cooperative whole-GPU sweeps, each capped to its share
    of the co-resident blocks.

More than eight concurrent streams need CUDA_DEVICE_MAX_CONNECTIONS raised
(e.g. to 32) before the process creates its CUDA context, or their launches
serialise on the default eight hardware queues.

The ctypes entry points release the GIL while they run, so the host threads
overlap; every model's result is independent of which others run beside it
(see tests/test_gpu_ensemble.py).
"""
from __future__ import annotations

import ctypes as ct
import queue
import threading
import time

import numpy
import torch

from . import _native as N
from .batch import BatchGate
from .driver import Simulation

# resident cooperative blocks per SM of the mixed-precision sweep kernel
SWEEP_BLOCKS_PER_SM = 1   # the staged sweep kernel's residency (dc_sweep_tma_kernel)


def state_bytes(config, precision="fp32dc"):
    """Device bytes a resident model needs: its fields plus solver workspace."""
    nx, ny, nz = int(config.nx), int(config.ny), int(config.nz)
    n = nx * ny * nz
    S = int(numpy.asarray(config.C).shape[-1])
    nT = 2 if numpy.asarray(config.T).ndim == 4 else 1
    # 28 3-D fields, 5 species fields, T, vx vy vz e, ZEROS ONES, Pn, rhof_prev,
    # Cn and Tn copies
    words = n * (28 + 5 * S + nT + 4 + 2 + 2 + S + nT)
    g = N.TseGrid(nx, ny, nz, 0, None, None, None, 9.81, 0.0, 1.0)
    L = N.lib()
    kinds = [N.TSE_WS_PRESSURE, N.TSE_WS_TRANSPORT]
    if precision == "fp32dc":
        kinds += [N.TSE_WS_PRESSURE_DC, N.TSE_WS_TRANSPORT_DC]
    ws = max(L.tse_workspace_bytes(ct.byref(g), k) for k in kinds)
    return 8 * words + ws + (1 << 20)


def shard(sizes, rank, world):
    """Indices of the models rank ``rank`` of ``world`` runs: models are
    independent, so ranks split them with no collective; largest first onto
    the least loaded rank (ties to the lower rank), deterministic."""
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    load = [0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += sizes[i]
        if r == rank:
            mine.append(i)
    return sorted(mine)


def cell_updates(sim):
    return sum(sim.M.cell_updates.values())


class HbmBudget:
    """Blocking byte budget for admitting models."""

    def __init__(self, total_bytes):
        self.total = int(total_bytes)
        self.free = int(total_bytes)
        self.cv = threading.Condition()

    def acquire(self, nbytes, stop=None):
        nbytes = int(nbytes)
        if nbytes > self.total:
            raise MemoryError("model needs %.2f GB, budget is %.2f GB" % (nbytes / 1e9, self.total / 1e9))
        with self.cv:
            while self.free < nbytes:
                if stop is not None and stop.is_set():
                    return False
                self.cv.wait(timeout=0.1)
            self.free -= nbytes
            return True

    def release(self, nbytes):
        with self.cv:
            self.free += int(nbytes)
            self.cv.notify_all()


def default_budget(device):
    free, total = torch.cuda.mem_get_info(device)
    return int(free * 0.85)


def block_cap(device, concurrency):
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    return max(8, (sms * SWEEP_BLOCKS_PER_SM) // max(1, concurrency))


def build_model(config, device, precision, max_blocks, dc_cycle=None, cluster_cells=0,
                cluster_size=0):
    """Set up one model (device state, workspace, initial EOS) on the calling
    thread's current stream."""
    sim = Simulation(config, device=device, precision=precision)
    sim.M.max_blocks = int(max_blocks)
    sim.M.cluster_cells = int(cluster_cells)
    if cluster_size:
        sim.M.cluster_size = int(cluster_size)
    if dc_cycle:
        sim.M.dc_cycle = int(dc_cycle)
    return sim


def step_model(sim, steps, keep=("P", "C", "T"), gate=None, joined=False):
    """Advance a built model by ``steps`` steps; returns its results.  With
    ``gate`` its mixed-precision solves are batched through it (``joined``:
    the caller has already counted this thread as a member)."""
    if gate is not None:
        if not joined:
            gate.join()
        sim.M.batch_gate = gate
        try:
            sim.run(max_steps=steps)
        finally:
            sim.M.batch_gate = None
            gate.leave()
    else:
        sim.run(max_steps=steps)
    out = {k: sim.field(k) for k in keep}
    out["cell_updates"] = cell_updates(sim)
    out["steps"] = sim.n_tsteps
    out["t_sim"] = sim.t_sim
    out["iterations"] = dict(sim.counters)
    return out


def run_model(config, steps, device, precision, max_blocks, dc_cycle=None, keep=("P", "C", "T"),
              gate=None, cluster_cells=0, cluster_size=0):
    """Run one model on the calling thread's current stream; returns results.
    With ``gate`` its mixed-precision solves are batched through it; else a
    grid of at most ``cluster_cells`` cells solves in single-cluster launches
    (``cluster_size`` CTAs) on this stream."""
    sim = build_model(config, device, precision, max_blocks, dc_cycle, cluster_cells, cluster_size)
    return step_model(sim, steps, keep, gate)


def autotune(configs, device=None, precision="fp32dc", steps=1, concurrency=(2, 4, 8),
             cycles=(128,), cluster_cells=(0,), batched=False, clusters=(8, 16)):
    """Pick the launch shape that gives the highest cell-update rate on a
    sample of the ensemble: unbatched, the concurrency (models in flight),
    the largest grid solved by single-cluster launches and the
    correction-cycle length; batched, the cluster size (CTAs per model) and
    cycle length.  Returns the best parameter set with its "rate" and all
    "trials"; the sample runs from the models' initial state each time."""
    space = []
    if batched:
        for c in clusters:
            for cyc in cycles:
                space.append({"batched": True, "cluster": c, "dc_cycle": cyc})
    else:
        for k in concurrency:
            for cc in cluster_cells:
                for cyc in cycles:
                    space.append({"batched": False, "concurrency": k, "cluster_cells": cc,
                                  "dc_cycle": cyc})
    trials = []
    best = None
    for p in space:
        _, st = Ensemble(configs, device=device, precision=precision, **p).run(steps, keep=())
        # the stepping phase's rate where set-up is apart (it dominates short samples)
        trials.append(dict(p, rate=st["stepping_cell_updates_per_s"] or st["cell_updates_per_s"]))
        if best is None or trials[-1]["rate"] > best["rate"]:
            best = dict(trials[-1])
    best["trials"] = trials
    return best


# grids up to this many cells take single-cluster solves by default
CLUSTER_CELLS = 0


class Ensemble:
    """``concurrency``: models in flight (None: 4, or every model when
    batched).  ``batched``: solve in lock step through a BatchGate (None: for
    the mixed-precision form).
    ``cluster``: CTAs per model in cluster launches (0: 16 alone, 8 batched).
    ``cluster_cells``: largest grid (cells) solved by single-cluster launches
    when not batched (None: CLUSTER_CELLS)."""

    def __init__(self, configs, device=None, precision="fp32dc", concurrency=None, hbm_budget=None,
                 max_blocks=None, dc_cycle=None, batched=None, cluster=0, cluster_cells=None):
        self.configs = list(configs)
        self.device = torch.device(device if device is not None else "cuda")
        self.precision = precision
        self.batched = (precision == "fp32dc") if batched is None else bool(batched)
        if self.batched and precision != "fp32dc":
            raise ValueError("batched solves need precision='fp32dc'")
        self.cluster_cells = CLUSTER_CELLS if cluster_cells is None else int(cluster_cells)
        if precision != "fp32dc":
            self.cluster_cells = 0
        if concurrency is None:
            concurrency = len(self.configs) if self.batched else 4
        self.concurrency = max(1, min(int(concurrency), max(1, len(self.configs))))
        self.budget = HbmBudget(hbm_budget if hbm_budget is not None else default_budget(self.device))
        self.max_blocks = max_blocks if max_blocks else block_cap(self.device, self.concurrency)
        self.dc_cycle = dc_cycle
        self.cluster = int(cluster)
        self.gate = BatchGate(self.device, cluster=self.cluster) if self.batched else None

    def run(self, steps, keep=("P", "C", "T"), prebuild=None):
        """Advance every model by ``steps`` time steps; returns (results, stats).

        prebuild (default: when every model fits the HBM budget at once): set
        every model up first, then step them, and report the two phases
        apart (``setup_s``, ``step_s``, ``stepping_cell_updates_per_s``);
        otherwise models are admitted one by one as memory frees up and only
        the whole wall time is known.  Batched runs always prebuild."""
        needs = [state_bytes(cfg, self.precision) for cfg in self.configs]
        if prebuild is None:
            prebuild = sum(needs) <= self.budget.total
        if self.batched and not prebuild:
            raise MemoryError("batched: every model must be resident at once (%.1f GB needed, "
                              "budget %.1f GB)" % (sum(needs) / 1e9, self.budget.total / 1e9))
        n = len(self.configs)
        results = [None] * n
        errors = []
        t0 = time.perf_counter()
        setup = None

        def build_all():
            sims = [None] * n
            todo = queue.Queue()
            for i in range(n):
                todo.put(i)

            def builder():
                stream = torch.cuda.Stream(device=self.device)
                with torch.cuda.device(self.device), torch.cuda.stream(stream):
                    while True:
                        try:
                            i = todo.get_nowait()
                        except queue.Empty:
                            break
                        try:
                            sims[i] = build_model(self.configs[i], self.device, self.precision,
                                                  self.max_blocks, self.dc_cycle, self.cluster_cells,
                                                  self.cluster)
                        except Exception as e:
                            errors.append((i, e))
                    stream.synchronize()
            ths = [threading.Thread(target=builder, daemon=True) for _ in range(min(8, n))]
            for th in ths:
                th.start()
            for th in ths:
                th.join()
            return sims

        if prebuild:
            sims = build_all()
            setup = time.perf_counter() - t0
            if errors:
                i, e = errors[0]
                raise RuntimeError("model %d failed: %s" % (i, e)) from e
            todo = queue.Queue()
            for i in range(n):
                todo.put(i)
            nthreads = n if self.batched else self.concurrency
            if self.batched:
                for _ in range(n):
                    self.gate.join()   # every model is a member before any solves

            def stepper():
                stream = torch.cuda.Stream(device=self.device)
                while True:
                    try:
                        i = todo.get_nowait()
                    except queue.Empty:
                        return
                    try:
                        with torch.cuda.device(self.device), torch.cuda.stream(stream):
                            results[i] = step_model(sims[i], steps, keep, self.gate, joined=True)
                            stream.synchronize()
                    except Exception as e:   # reported after all workers stop
                        errors.append((i, e))
                    sims[i] = None   # its device memory goes back to the pool

            threads = [threading.Thread(target=stepper, daemon=True) for _ in range(nthreads)]
        else:
            todo = queue.Queue()
            for i, cfg in enumerate(self.configs):
                todo.put((i, cfg))

            def admitter():
                stream = torch.cuda.Stream(device=self.device)
                while True:
                    try:
                        i, cfg = todo.get_nowait()
                    except queue.Empty:
                        return
                    self.budget.acquire(needs[i])
                    try:
                        with torch.cuda.device(self.device), torch.cuda.stream(stream):
                            results[i] = run_model(cfg, steps, self.device, self.precision,
                                                   self.max_blocks, self.dc_cycle, keep, None,
                                                   self.cluster_cells, self.cluster)
                            stream.synchronize()
                    except Exception as e:   # reported after all workers stop
                        errors.append((i, e))
                    finally:
                        self.budget.release(needs[i])

            threads = [threading.Thread(target=admitter, daemon=True) for _ in range(self.concurrency)]
        t1 = time.perf_counter()
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        t2 = time.perf_counter()
        wall = t2 - t0
        if errors:
            i, e = errors[0]
            raise RuntimeError("model %d failed: %s" % (i, e)) from e
        updates = sum(r["cell_updates"] for r in results)
        step_s = (t2 - t1) if prebuild else None
        return results, {"wall_s": wall, "cell_updates": updates,
                         "cell_updates_per_s": updates / wall if wall > 0 else 0.0,
                         "setup_s": setup, "step_s": step_s,
                         "stepping_cell_updates_per_s": (updates / step_s) if step_s else None,
                         "models": len(results), "concurrency": self.concurrency,
                         "max_blocks": self.max_blocks, "batched": self.batched,
                         "cluster_cells": self.cluster_cells,
                         "batch": self.gate.stats() if self.gate is not None else None}
