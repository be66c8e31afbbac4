"""Serving loop: simulations arrive over time and share the GPU.

``Server`` admits requests (a config module and a number of time steps) as
slots and device memory free up, keeps each admitted model's state resident
on the GPU until its last step, and runs the admitted models concurrently,
one host thread and CUDA stream per slot.  With ``batched`` (the default for
the mixed-precision form) the slots' solves meet at a ``BatchGate``: each
kind of solve of all admitted models runs as one batched call (the fused
form: one cooperative sweep over every model's cells, its loop one CUDA
graph on the device); otherwise the cooperative sweep kernels of concurrent
solves each take a share of the SMs.  A request that arrives while others are
running starts as soon as a slot is free and its state fits the HBM budget,
and joins the next batch of solves -- continuous batching at the granularity
of solver calls.

``replay(trace)`` plays a trace of (arrival time, config, steps) in real time
and reports per-request latency (arrival to result), p50/p99 and the
aggregate cell-update rate.
"""
from __future__ import annotations

import contextlib
import heapq
import threading
import time

import numpy
import torch

from .batch import BatchGate
from .ensemble import HbmBudget, block_cap, default_budget, run_model, state_bytes


class Request:
    def __init__(self, rid, config, steps, arrival):
        self.rid = rid
        self.config = config
        self.steps = int(steps)
        self.arrival = float(arrival)
        self.bytes = None
        self.start = None
        self.finish = None
        self.result = None
        self.error = None
        self.cancelled = False
        self.done = threading.Event()

    @property
    def latency(self):
        return None if self.finish is None else self.finish - self.arrival


class Server:
    """``eager`` (batched): a batch of solves goes out only once every running
    request waits (False, lock step: the default), or as soon as one waits and
    the GPU is free (True).  Measured on 40 requests of 16-96^3, 10 steps: lock
    step 24.1 G cell-updates/s, p50 0.78 s; eager 16.8-19.5 G/s, p50 1.2-1.7 s
    -- eager batches are smaller and each batched solve has a fixed cost."""

    def __init__(self, device=None, slots=8, hbm_budget=None, precision="fp32dc", max_blocks=None,
                 keep=("P", "C", "T"), batched=None, cluster=0, eager=False):
        """``slots``: requests running at once; 0 or None: no limit, a request
        starts as soon as it has arrived and its state fits the HBM budget
        (admission by the budget alone)."""
        self.device = torch.device(device if device is not None else "cuda")
        self.slots = max(0, int(slots or 0))
        self.batched = (precision == "fp32dc") if batched is None else bool(batched)
        if self.batched and precision != "fp32dc":
            raise ValueError("batched solves need precision='fp32dc'")
        self.gate = BatchGate(self.device, cluster=cluster, eager=eager) if self.batched else None
        self.budget = HbmBudget(hbm_budget if hbm_budget is not None else default_budget(self.device))
        self.precision = precision
        self.max_blocks = max_blocks if max_blocks else block_cap(self.device, max(1, self.slots))
        self.keep = keep
        self.pending = []          # heap of (arrival, rid, request)
        self.cv = threading.Condition()
        self.stop = threading.Event()
        self.t0 = None
        self.workers = []
        self.idle = 0              # no slot limit: workers free for a request not yet claimed
        self.completed = []

    def now(self):
        return time.perf_counter() - self.t0

    def start(self):
        self.t0 = time.perf_counter()
        for _ in range(self.slots):
            self._spawn()

    def _spawn(self):
        th = threading.Thread(target=self._worker, daemon=True)
        th.start()
        self.workers.append(th)

    def submit(self, req):
        req.bytes = state_bytes(req.config, self.precision)
        if req.bytes > self.budget.total:
            raise MemoryError("request %s needs %.1f GB, more than the HBM budget"
                              % (req.rid, req.bytes / 1e9))
        with self.cv:
            heapq.heappush(self.pending, (req.arrival, req.rid, req))
            # no slot limit: the request claims an idle worker, or a new one,
            # so every request starts once it fits the budget and finished
            # workers take later requests rather than accumulating
            spawn = False
            if self.slots == 0:
                if self.idle > 0:
                    self.idle -= 1
                else:
                    spawn = True
            self.cv.notify()
        if spawn:
            self._spawn()
        return req

    def cancel(self, rid):
        """Withdraw a request that has not started; True if it was pending.
        A request already on the GPU runs to its end."""
        with self.cv:
            for k, item in enumerate(self.pending):
                if item[1] == rid:
                    req = item[2]
                    self.pending[k] = self.pending[-1]
                    self.pending.pop()
                    heapq.heapify(self.pending)
                    req.error = RuntimeError("request %s cancelled" % rid)
                    req.cancelled = True
                    req.done.set()
                    return True
        return False

    def _next(self):
        with self.cv:
            while not self.pending:
                if self.stop.is_set():
                    return None
                self.cv.wait(timeout=0.05)
            return heapq.heappop(self.pending)[2]

    def _on_stream(self, stream):
        """A request's context on its worker: the device and the worker's
        own stream current (nothing to set without a CUDA device)."""
        ctx = contextlib.ExitStack()
        if stream is not None:
            ctx.enter_context(torch.cuda.device(self.device))
            ctx.enter_context(torch.cuda.stream(stream))
        return ctx

    def _worker(self):
        stream = torch.cuda.Stream(device=self.device) if self.device.type == "cuda" else None
        while True:
            req = self._next()
            if req is None:
                return
            if not self.budget.acquire(req.bytes, stop=self.stop):
                return
            try:
                req.start = self.now()
                with self._on_stream(stream):
                    req.result = run_model(req.config, req.steps, self.device, self.precision,
                                           self.max_blocks, keep=self.keep, gate=self.gate)
                    if stream is not None:
                        stream.synchronize()
            except Exception as e:
                req.error = e
            finally:
                self.budget.release(req.bytes)
                req.finish = self.now()
                self.completed.append(req)
                if self.slots == 0:
                    with self.cv:
                        self.idle += 1
                req.done.set()

    def shutdown(self):
        self.stop.set()
        with self.cv:
            self.cv.notify_all()
        for th in self.workers:
            th.join()

    def replay(self, trace):
        """trace: list of (arrival_s, config, steps); plays it in real time."""
        self.start()
        reqs = []
        for rid, (arr, cfg, steps) in enumerate(sorted(trace, key=lambda x: x[0])):
            delay = arr - self.now()
            if delay > 0:
                time.sleep(delay)
            reqs.append(self.submit(Request(rid, cfg, steps, arr)))
        for r in reqs:
            r.done.wait()
        self.shutdown()
        errs = [r for r in reqs if r.error is not None]
        if errs:
            raise RuntimeError("request %d failed: %s" % (errs[0].rid, errs[0].error))
        lat = numpy.array([r.latency for r in reqs])
        makespan = max(r.finish for r in reqs) - min(r.arrival for r in reqs)
        updates = sum(r.result["cell_updates"] for r in reqs)
        return reqs, {"requests": len(reqs), "p50_s": float(numpy.percentile(lat, 50)),
                      "p99_s": float(numpy.percentile(lat, 99)), "mean_s": float(lat.mean()),
                      "makespan_s": makespan, "cell_updates": updates,
                      "cell_updates_per_s": updates / makespan if makespan > 0 else 0.0,
                      "slots": self.slots or "unlimited", "max_blocks": self.max_blocks,
                      "batched": self.batched,
                      "batch": self.gate.stats() if self.gate is not None else None}


def poisson_trace(n, rate, seed, builder, steps, **kw):
    """n requests with exponential inter-arrival gaps (mean 1/rate)."""
    rng = numpy.random.default_rng(seed)
    t = numpy.cumsum(rng.exponential(1.0 / rate, size=n))
    return [(float(t[i] - t[0]), builder(seed * 1000 + i, **kw), steps) for i in range(n)]
