"""Batched solves across models that each run in their own host thread.

Every model of an ensemble (or every request a server is stepping) runs the
full time-step driver on its own thread and CUDA stream.  When a model
reaches a mixed-precision pressure / species / heat solve, ``Model._solve``
hands the call to the ``BatchGate`` it is attached to and waits.  Once every
live member is waiting at a solve, the gate issues the waiting calls as one
``tse_compute_*_dc_batch`` call per solve kind -- by default the fused form:
every model's cells in one cooperative sweep, the loop around the sweeps run
on the device as one CUDA graph (``cluster > 0``: one thread-block cluster
per model instead) -- and releases the members.
Members that are between solves keep the gate open (it never launches a
partial batch while one of them may still arrive), members that finish
leave, and new ones join between steps: continuous batching.

Ordering: each kind's launch goes on the gate's own stream for that kind,
which first waits on an event recorded on every member's stream; each
member's stream then waits on the launch's completion event, so a member's
later kernels (and its status read) follow its solve.  The launches of
different kinds overlap on the GPU.
"""
from __future__ import annotations

import ctypes as ct
import threading
import time
from contextlib import contextmanager

import torch

from . import _native as N

KINDS = ("compute_P", "compute_C", "compute_T")


class _Request:
    __slots__ = ("name", "grid", "args", "status", "ws", "ws_bytes", "stream", "cycle", "done",
                 "error")

    def __init__(self, name, grid, args, status, ws, ws_bytes, stream, cycle):
        self.name = name
        self.grid = grid
        self.args = args
        self.status = status
        self.ws = ws
        self.ws_bytes = ws_bytes
        self.stream = stream
        self.cycle = cycle
        self.done = False
        self.error = None


def default_batch_cells(device):
    """The fused form's default cell budget: 12M cells on a B200 (126 MB of
    L2), i.e. L2 bytes / 10.5.  Measured on the 512-model ensemble (axes
    log-uniform 32-128, 164M cells, 3 steps): models admitted into the
    running loop under 6M / 9M / 12M / 18M cells 104.4 / 107.4 / 109.3 /
    102.8 G cell-updates/s; as size-sorted sub-batches (the host loop's form)
    4M / 8M / 16M / 32M cells 90.3 / 103.4 / 104.3 / 95.2, one batch 96.0."""
    device = torch.device(device)
    if device.type != "cuda":
        return 0
    l2 = getattr(torch.cuda.get_device_properties(device), "L2_cache_size", 0)
    return int(l2 / 10.5) if l2 else 0


class BatchGate:
    """Collects the mixed-precision solves of the member models and launches
    them together.  ``cluster``: CTAs per model (0: the fused form).

    ``eager``: when to issue a batch.  False (lock step): once every live
    member waits at a solve -- the largest batches, for ensembles whose
    members step together.  True: as soon as a solve waits and no batch is
    on the GPU -- the members that arrive while a batch runs form the next
    one, so their host work between solves overlaps the GPU's work; for
    serving, whose requests differ in size and arrive over time.  Either way
    the gate's lock is free while a batch runs, and a model's results do not
    depend on which batch it was in.

    ``host_loop``: the fused form's loop around its sweep launches -- False
    (default) on the device, one CUDA graph launch per batched call; True on
    the host, a round trip per sweep launch.  Same results bit for bit.

    ``batch_cells``: the fused form streams every model's coefficient records
    once per half-sweep and keeps the FP32 corrections in L2 between
    half-sweeps -- while they fit.  A batch of more cells than this runs
    with at most this many cells solving at once: with the device-driven
    loop as one call whose models, largest first, wait and join the running
    loop as earlier ones finish (TseDcOptions.active_cells), so the GPU stays
    full until the last models; with the host loop as sub-batches of models
    of similar size, one after another.  None: default_batch_cells(device);
    0: every model at once.  A model's results do not depend on either.

    Use ``with gate.member():`` around a member thread's work, and attach the
    gate to its model (``Model.batch_gate = gate``)."""

    def __init__(self, device=None, cluster=0, eager=False, host_loop=False, batch_cells=None):
        self.device = torch.device(device if device is not None else "cuda")
        self.cluster = int(cluster)
        self.eager = bool(eager)
        self.host_loop = bool(host_loop)
        # device-driven loop: body runs per graph launch (0: the library's
        # 4096); graph launches made so far, in the statistics
        self.graph_runs = 0
        self.graph_launches = 0
        if batch_cells is None:
            batch_cells = default_batch_cells(self.device)
        self.batch_cells = int(batch_cells)
        self.cv = threading.Condition(threading.Lock())
        self.members = 0
        self.running = 0
        self.launching = False
        self.pending = []
        self.streams = {}
        self.ws = {}
        # statistics: launches per kind and models per launch
        self.launches = {k: 0 for k in KINDS}
        self.solves = {k: 0 for k in KINDS}
        # fused form: sweep launches, global iterations, sweep ms and loop ms per kind
        self.sweeps = {k: [0, 0, 0.0, 0.0] for k in KINDS}
        # host wall time inside the batched calls, and between the end of one
        # batch and the issue of the next (the members' host work while no
        # batch runs)
        self.call_s = 0.0
        self.gap_s = 0.0
        self._t_end = None

    # ------------------------------------------------------- membership
    def join(self):
        with self.cv:
            self.members += 1
            self.running += 1

    def leave(self):
        with self.cv:
            self.members -= 1
            self.running -= 1
            self._maybe_flush()

    @contextmanager
    def member(self):
        self.join()
        try:
            yield self
        finally:
            self.leave()

    # ----------------------------------------------------------- solves
    def submit(self, name, grid, args, status, ws, ws_bytes, cycle):
        """Called by a member thread in place of tse_<name>_dc; returns once
        the solve is queued behind this thread's current stream."""
        if name not in KINDS:
            raise ValueError("no batched form of %s" % name)
        req = _Request(name, grid, args, status, ws, ws_bytes,
                       torch.cuda.current_stream(self.device), int(cycle))
        with self.cv:
            if self.members < 1:
                raise RuntimeError("BatchGate.submit from a thread that has not joined the gate")
            self.pending.append(req)
            self.running -= 1
            # a waiting member issues the next batch once it may go out (its
            # own solve among the batch's), then returns to its model
            self._maybe_flush()
            while not req.done:
                self.cv.wait()
                self._maybe_flush()
        if req.error is not None:
            raise req.error

    def _maybe_flush(self):
        # caller holds self.cv; it is released while the batch runs.  The
        # requests that arrive meanwhile wait; the end of the batch wakes
        # their threads, one of which issues them
        if self.pending and not self.launching and (self.eager or self.running == 0):
            reqs, self.pending = self.pending, []
            self.launching = True
            self.cv.release()
            err = None
            t0 = time.perf_counter()
            try:
                self._launch(reqs)
            except Exception as e:   # every waiting member sees the failure
                err = e
            finally:
                t1 = time.perf_counter()
                self.cv.acquire()
                self.launching = False
                if self._t_end is not None and not self.eager:
                    self.gap_s += max(0.0, t0 - self._t_end)
                self.call_s += t1 - t0
                self._t_end = t1
            for r in reqs:
                r.error = err
                r.done = True
            self.running += len(reqs)
            self.cv.notify_all()

    def _stream(self, key):
        s = self.streams.get(key)
        if s is None:
            s = self.streams[key] = torch.cuda.Stream(device=self.device)
        return s

    def _workspace(self, key, rs, stream):
        cells = sum(r.grid.nx * r.grid.ny * r.grid.nz for r in rs)
        need = int(N.lib().tse_batch_workspace_bytes(len(rs), cells))
        t = self.ws.get(key)
        if t is None or t.numel() < need:
            with torch.cuda.stream(stream):
                t = self.ws[key] = torch.empty(need, dtype=torch.uint8, device=self.device)
        return t

    def _subbatches(self, rs):
        """The host loop's sub-batches of one kind of solve (see batch_cells)."""
        if self.cluster > 0 or self.batch_cells <= 0:
            return [rs]
        cells = lambda r: r.grid.nx * r.grid.ny * r.grid.nz
        if sum(cells(r) for r in rs) <= self.batch_cells:
            return [rs]
        out, cur, tot = [], [], 0
        for r in sorted(rs, key=cells):
            c = cells(r)
            if cur and tot + c > self.batch_cells:
                out.append(cur)
                cur, tot = [], 0
            cur.append(r)
            tot += c
        out.append(cur)
        return out

    def _launch(self, reqs):
        groups = {}
        for r in reqs:
            groups.setdefault((r.name, r.cycle), []).append(r)
        with torch.cuda.device(self.device):
            for (name, cycle), rs in groups.items():
                bs = self._stream((name, cycle))
                seen = set()
                for r in rs:
                    if r.stream.cuda_stream not in seen:
                        seen.add(r.stream.cuda_stream)
                        bs.wait_stream(r.stream)
                if self.cluster > 0 or not self.host_loop:
                    # one call; with a budget, the largest models first
                    cells = lambda r: r.grid.nx * r.grid.ny * r.grid.nz
                    self._launch_one(name, cycle, sorted(rs, key=cells, reverse=True), bs)
                else:
                    for sub in self._subbatches(rs):
                        self._launch_one(name, cycle, sub, bs)
                for r in rs:
                    r.stream.wait_stream(bs)

    def _launch_one(self, name, cycle, rs, bs):
        """One batched call of ``rs`` on the gate's stream ``bs``."""
        L = N.lib()
        ws = self._workspace((name, cycle), rs, bs)
        Item = N.BATCH_ITEM[name]
        items = (Item * len(rs))(*[Item(ct.pointer(r.grid), ct.pointer(r.args),
                                        ct.c_void_p(r.status.data_ptr()),
                                        ct.c_void_p(r.ws.data_ptr()), r.ws_bytes)
                                   for r in rs])
        opts = N.TseDcOptions(cycle, self.cluster, 1)
        opts.host_loop = int(self.host_loop)
        opts.active_cells = max(0, self.batch_cells)
        opts.graph_runs = int(self.graph_runs)
        rc = getattr(L, "tse_%s_dc_batch" % name)(items, len(rs), ct.byref(opts),
                                                  ct.c_void_p(ws.data_ptr()), ws.numel(),
                                                  ct.c_void_p(bs.cuda_stream))
        N.check(rc, "tse_%s_dc_batch" % name)
        self.launches[name] += 1
        self.solves[name] += len(rs)
        self.sweeps[name][0] += opts.sweep_launches
        self.sweeps[name][1] += opts.sweep_iterations
        self.sweeps[name][2] += opts.sweep_ms
        self.sweeps[name][3] += opts.loop_ms
        if not self.host_loop and self.cluster <= 0:
            self.graph_launches += opts.graph_runs

    def stats(self):
        # sweeps: the fused sweep kernel's launches, the global iterations
        # they ran and their own time (ms); loop_ms: the whole loop around
        # them (sweeps, events, x += d, residuals)
        return {"launches": dict(self.launches), "solves": dict(self.solves),
                "call_s": round(self.call_s, 3), "gap_s": round(self.gap_s, 3),
                "graph_launches": self.graph_launches,
                "sweeps": {k: {"launches": v[0], "iterations": v[1], "ms": round(v[2], 3),
                               "loop_ms": round(v[3], 3)}
                           for k, v in self.sweeps.items()}}
