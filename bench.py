#!/usr/bin/env python
"""Benchmark: SOR cell-updates/s of the TRANSPORTSE time-step core on B200.

Workload: the 256 x 256 x 128 bottom-heated reservoir
(transportse_b200.workloads.reservoir_3d: geometric node spacing, Gaussian
random field log10 K, porosity U(0.05, 0.25), two species plus heat, linear
EOS, SIA Picard tolerance 1e-6), synthetic seeded inputs.  One step = one
full time step of the model (SIA loop with pressure solve, fluxes, flow
error, species and heat solves, EOS).

Metric: cell-updates per second over the timed steps; a cell-update is one
active (non-Dirichlet) cell relaxed once in a red+black iteration of the
pressure, species or heat solve.  The headline ``value`` is the FP32 +
defect-correction form; the plain FP64 form (the reference's arithmetic) is
timed on the same inputs and reported beside it, with the largest relative
difference between the two forms' fields after the same steps.  ``e2e``
repeats the FP32+DC steps through the public API with the state uploaded
from pinned host memory and the solution read back every step.  The working
set (> 3 GB) exceeds L2, so no flush is needed between steps.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os

# concurrent model streams (ensemble / serving workloads) need more than the
# default eight hardware work queues; must be set before the CUDA context
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
import statistics
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

# algorithmic bytes per pressure cell-update (coefficient form, neighbour
# reuse from cache): FP64 57 B, FP32 29 B
ALG_BYTES = {"fp64": 57, "fp32dc": 29}
# what the FP64 form in the reference's operation order must stream for this
# workload (z buoyancy only): 11 coefficient words and the flag byte
EXACT_FORM_BYTES = {"fp64": 89}
# DRAM bytes per cell-update measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum of one 64-iteration launch on the 192x192x128
# reservoir, divided by its cell-updates; summaries under profiles/), scaled
# to a launch of the benchmark by its cell-updates
TRAFFIC_BYTES = {"fp32dc": 28.8, "fp64": 95.2}
DEFAULT_SHAPE = (256, 256, 128)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--shape", type=str, default=None, help="override grid, e.g. 64x64x32")
    ap.add_argument("--dc-cycle", type=int, default=0,
                    help="iterations per FP32 correction cycle (0: the model's default)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the library's default sweep variant (chunk 512, 2 pipelines)")
    ap.add_argument("--kernel-only", choices=("fp64", "fp32dc"), default=None,
                    help="time one pressure solve of exactly --iters red+black iterations "
                         "(for isolated kernel timing and profiler captures)")
    ap.add_argument("--iters", type=int, default=200)
    ap.add_argument("--variant", type=str, default=None,
                    help="kernel-only: staged sweep chunk,ring,pipes (e.g. 1024,2,2)")
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--workload", choices=("reservoir", "ensemble", "serving", "sloped"),
                    default="reservoir")
    ap.add_argument("--models", type=int, default=48, help="ensemble: models")
    ap.add_argument("--n-max", type=int, default=None, help="ensemble/serving: largest axis")
    ap.add_argument("--concurrency", type=int, default=0,
                    help="ensemble: models in flight with --streams (0 = autotune); batched, "
                         "any value > 0 skips the cycle-length autotune")
    ap.add_argument("--cluster", type=int, default=0,
                    help="ensemble/serving, batched: CTAs per model (0 = autotune / 8)")
    ap.add_argument("--streams", action="store_true",
                    help="ensemble/serving: concurrent per-model streams instead of batched "
                         "solves (one fused launch per solve kind, the default)")
    ap.add_argument("--requests", type=int, default=40, help="serving: requests")
    ap.add_argument("--rate", type=float, default=20.0, help="serving: arrivals per second")
    ap.add_argument("--slots", type=int, default=0,
                    help="serving: requests running at once (0: no limit, admission by the HBM budget)")
    ap.add_argument("--gate", choices=("eager", "lockstep"), default="lockstep",
                    help="serving, batched: issue a batch as soon as a solve waits and the GPU "
                         "is free (eager), or once every running request waits (lockstep)")
    ap.add_argument("--batch-loop", choices=("device", "host"), default="device",
                    help="ensemble/serving, batched: the fused form's loop (device: one CUDA "
                         "graph per batch solve; host: a host round trip per sweep launch)")
    ap.add_argument("--batch-cells", type=int, default=None,
                    help="ensemble/serving, batched: largest sub-batch in cells (default: a "
                         "third of L2 in FP32 corrections; 0: one batch)")
    ap.add_argument("--ensemble-models", type=int, default=512,
                    help="default run: models of the batched-ensemble key (0: leave it out)")
    ap.add_argument("--ensemble-steps", type=int, default=10,
                    help="default run: time steps of every model of the ensemble key")
    ap.add_argument("--serving-requests", type=int, default=40,
                    help="default run: requests of the serving key (0: leave it out)")
    ap.add_argument("--serving-steps", type=int, default=50,
                    help="default run: time steps of every request of the serving key")
    ap.add_argument("--serving-n-max", type=int, default=192,
                    help="default run: largest cubic edge of the serving key's requests")
    return ap.parse_args()


def with_loop(runner, a):
    """The --batch-loop choice on a runner's batch gate (per call, through
    TseDcOptions.host_loop)."""
    if getattr(runner, "gate", None) is not None:
        runner.gate.host_loop = a.batch_loop == "host"
        if a.batch_cells is not None:
            runner.gate.batch_cells = int(a.batch_cells)
    return runner


def batched_roofline(units, st, peak, peak_kind):
    """Roofline of the batched form from a batch gate's statistics: the fused
    sweep kernel's own time (global timer inside the device-driven loop's
    graph) and the loop around it, at the algorithmic 29 bytes per
    cell-update of the FP32 correction sweep."""
    sw = (st or {}).get("sweeps") or {}
    ms = sum(v["ms"] for v in sw.values())
    loop_ms = sum(v.get("loop_ms", 0.0) for v in sw.values())
    launches = sum(v["launches"] for v in sw.values())
    if ms <= 0 or launches == 0:
        return None
    b = ALG_BYTES["fp32dc"]
    achieved = units * b / (ms / 1e3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": None,
            "kernel": "fused_sweep_dev_kernel<4, 2> (all models' FP32 correction sweeps in one "
                      "cooperative launch, inside the device-driven loop)",
            "algorithmic_bytes_per_cell_update": b, "launches": launches,
            "ms_per_launch": ms / launches, "cell_updates_per_launch": units / launches,
            "loop_frac": (units * b / (loop_ms / 1e3) / 1e9 / peak) if loop_ms > 0 else None,
            "peak_source": peak_kind}


def ensemble_run(a, dev, models, steps, nmax=128, clocks=True):
    """Ensemble of independent models (log-uniform 32-nmax per axis, lognormal
    K, one source/sink, one species plus heat), FP32+DC, ``steps`` time steps
    each.  Batched (default): every model resident, each kind of solve of all
    models in one fused launch sequence (the device-driven loop), the
    correction-cycle length autotuned on a sample; unbatched (--streams):
    concurrency and cycle length autotuned on a sample."""
    from transportse_b200 import workloads
    from transportse_b200.ensemble import Ensemble, autotune
    cfgs = [workloads.ensemble_member(seed=1000 + i, n_max=nmax) for i in range(models)]
    tune = None
    batched = not a.streams
    conc = cyc = cl = None
    if batched:
        cl = max(0, a.cluster)   # 0: fused form; > 0: one cluster of that size per model
        if a.concurrency <= 0:
            # the batched form's runtime knob: the correction-cycle length
            tune = autotune(cfgs[:16], device=dev, steps=1, batched=True, clusters=(cl,),
                            cycles=(128, 256, 512))
            cyc = tune["dc_cycle"]
        kw = {"batched": True, "cluster": cl}
    else:
        if a.concurrency <= 0:
            tune = autotune(cfgs[:8], device=dev, steps=1, concurrency=(2, 4, 8), cycles=(128, 256))
            conc, cyc = tune["concurrency"], tune["dc_cycle"]
        else:
            conc = a.concurrency
        kw = {"batched": False, "concurrency": conc}
    sampler = ClockSampler(0) if clocks else None
    if sampler:
        sampler.start()
    _, st = with_loop(Ensemble(cfgs, device=dev, precision="fp32dc", dc_cycle=cyc, **kw), a).run(
        steps, keep=())
    clk = sampler.stop() if sampler else None
    cells = [c.nx * c.ny * c.nz for c in cfgs]
    value = st["stepping_cell_updates_per_s"] or st["cell_updates_per_s"]
    peak, peak_kind = measured_peak()
    roof = batched_roofline(st["cell_updates"], st["batch"], peak, peak_kind) if batched else None
    if roof is not None and st["step_s"]:
        # the whole batched form over the stepping phase: sweeps, the loop
        # around them, the transport solves and every model's host steps
        roof["form_frac"] = value * ALG_BYTES["fp32dc"] / 1e9 / peak
    return {
        "metric": "SOR cell-updates/s", "value": value, "unit": "cell-updates/s",
        "config": {"workload": "ensemble of %d models, axes log-uniform 32-%d, %d steps each, "
                               "FP32 sweeps + FP64 defect correction; value = cell-updates over "
                               "the stepping phase (one-time model set-up in setup_s)"
                               % (models, nmax, steps),
                   "models": models, "steps": steps,
                   "cells_total": int(sum(cells)), "cells_max": int(max(cells))},
        "setup_s": st["setup_s"], "step_s": st["step_s"], "cell_updates": st["cell_updates"],
        "with_setup_cell_updates_per_s": st["cell_updates_per_s"],
        "wall_s": st["wall_s"], "batched": batched, "cluster": cl, "concurrency": st["concurrency"],
        "dc_cycle": cyc, "max_blocks": st["max_blocks"], "batch_loop": a.batch_loop,
        "batch": st["batch"], "autotune": tune, "roofline": roof, "clocks": clk}


def bench_ensemble(a):
    import torch
    r = ensemble_run(a, torch.device("cuda:0"), a.models, a.steps, a.n_max or 128)
    r.update({"n_gpus": 1, "steps": a.steps, "higher_is_better": True, "dtype": "f32",
              "data": "synthetic"})
    print(json.dumps(r))


def bench_sloped(a):
    """Large sloped model (sloped_3d: beta 5 deg, anisotropic lognormal K, three
    species with dispersivity 10/1 m, Smolarkiewicz correction, NLTE heat,
    SIA), FP32+DC with FP64 mass-balance totals, against an FP64 GPU run of the
    same steps."""
    import numpy
    import torch
    from transportse_b200 import workloads
    from transportse_b200.driver import Simulation
    dev = torch.device("cuda:0")
    shape = tuple(int(x) for x in a.shape.lower().split("x")) if a.shape else (512, 512, 256)
    cfg = workloads.sloped_3d(*shape)
    cfg.GPU_MASSBAL = True
    out = {}
    fields = {}
    for prec in ("fp32dc", "fp64"):
        sim = Simulation(cfg, device=dev, precision=prec)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        cu0 = sum(sim.M.cell_updates.values())
        e0.record()
        sim.run(max_steps=a.steps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        cu = sum(sim.M.cell_updates.values()) - cu0
        out[prec] = {"ms_per_step": ms / a.steps, "cell_updates_per_s": cu / (ms / 1e3),
                     "iterations": dict(sim.counters),
                     "mass": {k: (v.tolist() if hasattr(v, "tolist") else v)
                              for k, v in sim.mass_log[-1].items()}}
        fields[prec] = {n: sim.field(n) for n in ("P", "C", "T")}
        del sim
        torch.cuda.empty_cache()
    err = {n: float(numpy.max(numpy.abs(fields["fp32dc"][n] - fields["fp64"][n]))
                    / max(numpy.max(numpy.abs(fields["fp64"][n])), 1e-300)) for n in ("P", "C", "T")}
    m32, m64 = out["fp32dc"]["mass"], out["fp64"]["mass"]
    mass_rel = {"water": abs(m32["water"] - m64["water"]) / abs(m64["water"]),
                "heat": abs(m32["heat"] - m64["heat"]) / abs(m64["heat"]),
                "species": [abs(x - y) / max(abs(y), 1e-300)
                            for x, y in zip(m32["species"], m64["species"])]}
    print(json.dumps({
        "metric": "SOR cell-updates/s", "value": out["fp32dc"]["cell_updates_per_s"],
        "unit": "cell-updates/s", "n_gpus": 1, "steps": a.steps, "higher_is_better": True,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "sloped_3d %dx%dx%d, %d SIA steps, FP32+DC vs FP64" % (shape + (a.steps,))},
        "fp32dc": out["fp32dc"], "fp64": out["fp64"], "max_rel_err_vs_fp64": err,
        "mass_rel_diff_vs_fp64": mass_rel}))


def serving_run(a, dev, requests, steps, nmax, rate=20.0, slots=0, clocks=True):
    """Poisson arrivals of cubic-grid simulations (log-uniform edge 16-nmax),
    each ``steps`` coupled flow/heat/species steps; HBM-budget admission,
    state resident on the device, continuous batching of the running
    requests' solves; p50/p99 latency (arrival to result) and the aggregate
    cell-update rate over the makespan."""
    import torch
    from transportse_b200 import workloads
    from transportse_b200.serving import Server, poisson_trace
    trace = poisson_trace(requests, rate, 5, workloads.serving_request, steps, n_min=16,
                          n_max=nmax)
    budget = min(150e9, torch.cuda.mem_get_info(dev)[0] * 0.85)
    sampler = ClockSampler(0) if clocks else None
    if sampler:
        sampler.start()
    reqs, st = with_loop(Server(device=dev, slots=slots, hbm_budget=budget, batched=not a.streams,
                                cluster=a.cluster, eager=a.gate == "eager"), a).replay(trace)
    clk = sampler.stop() if sampler else None
    peak, peak_kind = measured_peak()
    roof = batched_roofline(st["cell_updates"], st["batch"], peak, peak_kind)
    return {
        "metric": "SOR cell-updates/s", "value": st["cell_updates_per_s"], "unit": "cell-updates/s",
        "config": {"workload": "serving: %d Poisson arrivals at %.0f/s, cubic n log-uniform 16-%d, "
                               "%d steps each, %s, HBM budget %.0f GB"
                               % (requests, rate, nmax, steps,
                                  "%d slots" % slots if slots else "admission by the budget alone",
                                  budget / 1e9),
                   "requests": requests, "steps": steps},
        "latency_p50_s": st["p50_s"], "latency_p99_s": st["p99_s"], "latency_mean_s": st["mean_s"],
        "makespan_s": st["makespan_s"], "cell_updates": st["cell_updates"],
        "batched": st["batched"], "gate": a.gate, "batch_loop": a.batch_loop,
        "batch": st["batch"], "roofline": roof, "clocks": clk}


def bench_serving(a):
    import torch
    r = serving_run(a, torch.device("cuda:0"), a.requests, a.steps, a.n_max or 96, a.rate,
                    a.slots)
    r.update({"n_gpus": 1, "steps": a.steps, "higher_is_better": True, "dtype": "f32",
              "data": "synthetic"})
    print(json.dumps(r))


def shape_of(a):
    if a.shape:
        return tuple(int(x) for x in a.shape.lower().split("x"))
    return DEFAULT_SHAPE


def measured_peak():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------- CPU arm
def cpu_model():
    """The host CPU's model name (first /proc/cpuinfo entry)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_pressure_rate(shape, seconds):
    """The oracle's compute_P (C port of tse.py:647-742, OpenMP over all host
    threads) on the benchmark grid: single-iteration calls (P_conv = 1e300),
    each doing the reference's copy, red and black sweeps and L2."""
    import numpy
    from oracle import oracle as O
    from transportse_b200 import workloads
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    cfg = workloads.reservoir_3d(*shape)
    m = O.OracleModel(cfg)
    z = numpy.zeros(shape)
    args = (cfg.c_f, cfg.nue, cfg.rho_f, cfg.phi, cfg.Kx, cfg.Ky, cfg.Kz, z, z, z)
    active = int((cfg.BP == 0).sum())
    P = cfg.P.copy()
    calls, t0 = 0, time.perf_counter()
    while True:
        r = m.compute_P(P, *args, 3600.0, cfg.BP, cfg.WP, SOR=1.9, max_it=20000, inc_it=1.25,
                        max_dt=1e6, P_conv=1e300)
        P = r[2]
        calls += 1
        el = time.perf_counter() - t0
        if el >= seconds and calls >= 2:
            break
    return {"value": active * calls / el, "unit": "cell-updates/s", "cores": cores,
            "kind": "port", "cpu_model": cpu_model(),
            "sample": "%d single-iteration compute_P calls (red+black sweep, copy, L2) on the "
                      "%dx%dx%d grid, %.1f s" % ((calls,) + tuple(shape) + (el,))}


def run_reference_arm(a, rank):
    if rank != 0:
        return
    shape = shape_of(a)
    for _ in range(a.warmup):
        cpu_pressure_rate(shape, 1.0)
    vals, info = [], None
    for _ in range(a.steps):
        info = cpu_pressure_rate(shape, max(2.0, a.cpu_seconds / max(1, a.steps)))
        vals.append(info["value"])
    v = statistics.mean(vals)
    print(json.dumps({
        "impl": "reference", "metric": "SOR cell-updates/s", "value": v, "unit": "cell-updates/s",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "reservoir_3d %dx%dx%d pressure SOR sweeps" % shape,
                   "note": "single red+black iterations of compute_P on the GPU arm's grid: "
                           "pressure updates are 99.4 % of the GPU arm's cell-updates, and one "
                           "full time step of the CPU port (~8,300 pressure iterations) would "
                           "take ~20 minutes at this size"},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": info["cores"],
                         "kind": info["kind"], "cpu_model": info["cpu_model"],
                         "sample": info["sample"]},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))


# ---------------------------------------------------------------- GPU arm
class Ctx:
    def __init__(self, world, dev):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.world, self.dev = torch, dist, world, dev

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()
        self.torch.cuda.synchronize()

    def max_sum(self, ms, units):
        """(max over ranks of ms, sum over ranks of units)."""
        t = self.torch.tensor([ms, float(units)], dtype=self.torch.float64, device=self.dev)
        if self.world > 1:
            a = t[0:1].clone()
            b = t[1:2].clone()
            self.dist.all_reduce(a, op=self.dist.ReduceOp.MAX)
            self.dist.all_reduce(b, op=self.dist.ReduceOp.SUM)
            return float(a[0]), float(b[0])
        return ms, float(units)


def timed_steps(ctx, sim, steps, clocks=None):
    torch = ctx.torch
    M = sim.M
    cu0 = dict(M.cell_updates)
    it0 = dict(sim.counters)
    M.timing, M.timed, M.sweep_timed = True, [], []
    launches0 = M.launches
    if clocks:
        clocks.start()
    ctx.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        sim.run(max_steps=1)
    e1.record()
    ctx.barrier()
    clk = clocks.stop() if clocks else None
    M.timing = False
    ms = e0.elapsed_time(e1)
    updates = sum(M.cell_updates[k] - cu0[k] for k in cu0)
    p_units, p_ms, n_p, active_p = 0.0, 0.0, 0, 0
    by = {}   # per solve kind: cell-updates, event ms of the solve calls, calls
    for kind, s0, s1, nit, active in M.timed:
        ms_k = s0.elapsed_time(s1)
        b = by.setdefault(kind, [0.0, 0.0, 0])
        b[0] += float(nit) * active
        b[1] += ms_k
        b[2] += 1
        if kind == "P":
            p_units += float(nit) * active
            p_ms += ms_k
            n_p += 1
            active_p = active
    # mixed-precision form: the FP32 sweep kernel's own launches (events
    # recorded by the library around each launch on the solve's stream)
    s_units, s_ms, n_s = 0.0, 0.0, 0
    for kind, launches, iters, sms in M.sweep_timed:
        if kind == "P":
            s_units += float(iters) * active_p
            s_ms += sms
            n_s += launches
    rates = {k: {"cell_updates": u, "ms": t, "calls": n,
                 "cell_updates_per_s": u / (t / 1e3) if t > 0 else None}
             for k, (u, t, n) in sorted(by.items())}
    return {"ms": ms, "updates": updates, "launches": M.launches - launches0, "clocks": clk,
            "rates_by_solve": rates,
            "iterations": {k: sim.counters[k] - it0[k] for k in it0},
            "p_units": p_units, "p_ms": p_ms, "n_p": n_p,
            "s_units": s_units, "s_ms": s_ms, "n_s": n_s}


def e2e_steps(ctx, sim, steps):
    """Steps through the public API with host buffers: every step's inputs
    (all state fields) come from pinned host memory and its results (P, C, T
    and the Darcy fluxes) go back to pinned host memory.  The copies run on a
    copy stream into a second set of device buffers (Simulation.swap_state),
    so step s+1's upload and step s's download overlap step s+1's and step
    s's compute; the timed region starts before the first upload and ends
    after the last download."""
    torch = ctx.torch
    M = sim.M
    host = {}
    for name, tns in sim.S.items():
        h = torch.empty(tns.shape, dtype=tns.dtype, pin_memory=True)
        h.copy_(tns)
        host[name] = h
    outs = {n: torch.empty(sim.S[n].shape, dtype=torch.float64, pin_memory=True)
            for n in ("P", "C", "T", "qx", "qy", "qz")}
    h2d = sum(h.numel() * h.element_size() for h in host.values())
    d2h = sum(h.numel() * h.element_size() for h in outs.values())
    bufs = [sim.S, {n: torch.empty_like(t) for n, t in sim.S.items()}]
    comp = torch.cuda.current_stream()
    copy = torch.cuda.Stream()
    cu = dict(M.cell_updates)
    ctx.barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(comp)

    # the first upload overwrites buffers the earlier steps used
    copy.wait_stream(comp)

    def upload(dst):
        with torch.cuda.stream(copy):
            for name, h in host.items():
                dst[name].copy_(h, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(copy)
        return ev

    ready = upload(bufs[0])
    for s in range(steps):
        cur = bufs[s % 2]
        comp.wait_event(ready)
        if sim.S is not cur:
            sim.swap_state(cur)
        if s + 1 < steps:
            # the other set's last reader is step s-1's download, queued
            # earlier on the same copy stream
            ready = upload(bufs[(s + 1) % 2])
        sim.run(max_steps=1)
        done = torch.cuda.Event()
        done.record(comp)
        copy.wait_event(done)
        with torch.cuda.stream(copy):
            for n, h in outs.items():
                h.copy_(cur[n], non_blocking=True)
    comp.wait_stream(copy)
    f1.record(comp)
    ctx.barrier()
    if sim.S is not bufs[0]:
        sim.swap_state(bufs[0])
    ms, upd = ctx.max_sum(f0.elapsed_time(f1), sum(M.cell_updates[k] - cu[k] for k in cu))
    return {"value": upd / (ms / 1e3), "unit": "cell-updates/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "copies": "copy stream, double-buffered state",
            "step": "the first time step from the host inputs, every step"}


def roofline(res, precision, peak, peak_kind):
    """Roofline of the dominant kernel: algorithmic bytes / event time.
    fp32dc: the FP32 sweep kernel (dc_sweep_tma_kernel, 96 % of device time);
    fp64: the persistent FP64 solve (rb_solve_tma_kernel, one launch per
    solve, timed with its assembly and unpack kernels)."""
    if precision == "fp32dc":
        if not res["n_s"]:
            return None
        units, ms, n = res["s_units"], res["s_ms"], res["n_s"]
        name = "dc_sweep_tma_kernel<ring, pipes, chunk> (FP32 correction sweeps, bulk-copy pipelines; variant in autotune)"
    else:
        if not res["n_p"]:
            return None
        units, ms, n = res["p_units"], res["p_ms"], res["n_p"]
        name = "rb_solve_tma_kernel<PressureForm> (FP64, reference operation order, bulk-copy pipelines)"
    achieved = units * ALG_BYTES[precision] / (ms / 1e3) / 1e9
    per_launch = units / n
    out = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "traffic": TRAFFIC_BYTES[precision] * per_launch,
           "kernel": name, "algorithmic_bytes_per_cell_update": ALG_BYTES[precision],
           "traffic_bytes_per_cell_update": TRAFFIC_BYTES[precision],
           "cell_updates_per_launch": per_launch, "launches": n,
           "ms_per_launch": ms / n, "peak_source": peak_kind}
    if precision in EXACT_FORM_BYTES:
        ex = units * EXACT_FORM_BYTES[precision] / (ms / 1e3) / 1e9
        out["exact_form"] = {"bytes_per_cell_update": EXACT_FORM_BYTES[precision],
                             "achieved": ex, "frac": ex / peak}
    return out


def kernel_only(a):
    """One pressure solve of exactly a.iters iterations (P_conv = 0, so it
    never converges; max_it = a.iters and min_dt = dt, so the first dt halving
    ends it), repeated a.repeat times; prints per-launch time and bandwidth."""
    import torch
    from transportse_b200 import workloads
    from transportse_b200.driver import Simulation
    shape = shape_of(a)
    sim = Simulation(workloads.reservoir_3d(*shape), device=torch.device("cuda:0"),
                     precision=a.kernel_only)
    M, S = sim.M, sim.S
    M.dc_min_conv = 0.0   # P_conv = 0 below: keep the requested form
    if a.variant:
        M.sweep_variant = tuple(int(x) for x in a.variant.split(","))
    P0 = S["P"].clone()
    peak, kind = measured_peak()
    M.timing = a.kernel_only == "fp32dc"
    out = []
    sweep = []
    for r in range(a.repeat + 1):
        S["P"].copy_(P0)
        M.sweep_timed.clear()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = M.compute_P(S["P"], S["c_f"], S["nue"], S["rho_f"], S["phi"], S["Kx"], S["Ky"],
                          S["Kz"], S["qx"], S["qy"], S["qz"], 3600.0, S["BP"], S["WP"],
                          SOR=1.9, max_it=a.iters, inc_it=1.25, max_dt=1e6, min_dt=2700.0,
                          P_conv=0.0)
        e1.record()
        torch.cuda.synchronize()
        if r:
            out.append((e0.elapsed_time(e1), res[5]))
            if M.sweep_timed:
                sweep.append((sum(x[3] for x in M.sweep_timed), sum(x[2] for x in M.sweep_timed)))
    active = int((S["BP"] == 0).sum().item())
    ms = statistics.median(x[0] for x in out)
    its = out[0][1]
    rate = its * active / (ms / 1e3)
    st = M.last_status
    sw = None
    if sweep:
        # the sweep kernel alone (event-timed launches), without the solve's
        # FP64 setup, residual and unpack passes
        sms = statistics.median(x[0] for x in sweep)
        sw = {"ms": sms, "us_per_iteration": 1e3 * sms / sweep[0][1],
              "cell_updates_per_s": sweep[0][1] * active / (sms / 1e3),
              "frac_of_peak": sweep[0][1] * active / (sms / 1e3) * ALG_BYTES["fp32dc"] / 1e9 / peak}
    print(json.dumps({"kernel_only": a.kernel_only, "shape": list(shape), "iterations": its,
                      "variant": M.last_variant,
                      "residual_cycles": int(st.cycles), "halvings": int(st.halvings),
                      "sweep_kernel": sw,
                      "ms_per_launch": ms, "cell_updates_per_s": rate,
                      "alg_GBps": rate * ALG_BYTES[a.kernel_only] / 1e9,
                      "frac_of_peak": rate * ALG_BYTES[a.kernel_only] / 1e9 / peak,
                      "peak_GBps": peak, "peak_source": kind}))


def main():
    a = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if a.impl == "reference":
        return run_reference_arm(a, rank)
    if a.kernel_only:
        return kernel_only(a)
    if a.workload == "ensemble":
        return bench_ensemble(a)
    if a.workload == "serving":
        return bench_serving(a)
    if a.workload == "sloped":
        return bench_sloped(a)
    import numpy
    import torch
    import torch.distributed as dist
    from transportse_b200 import workloads
    from transportse_b200.driver import Simulation
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    ctx = Ctx(world, dev)
    shape = shape_of(a)
    peak, peak_kind = measured_peak()

    # ---- headline: FP32 sweeps + FP64 defect correction
    sim = Simulation(workloads.reservoir_3d(*shape), device=dev, precision="fp32dc")
    if a.dc_cycle:
        sim.M.dc_cycle = int(a.dc_cycle)
    tune = None
    if not a.no_autotune:
        # the staged sweep's chunk / ring / pipelines for this grid, timed on
        # its own pressure solve (every variant makes the same cell updates)
        from transportse_b200 import autotune
        tune = autotune.tune_sweep(sim)
    for _ in range(a.warmup):
        sim.run(max_steps=1)
    res = timed_steps(ctx, sim, a.steps, ClockSampler(local))
    ms, upd = ctx.max_sum(res["ms"], res["updates"])
    value = upd / (ms / 1e3)

    # ---- the plain FP64 form on the same inputs and steps
    fp64 = None
    if not a.no_fp64:
        sim64 = Simulation(workloads.reservoir_3d(*shape), device=dev, precision="fp64")
        for _ in range(a.warmup):
            sim64.run(max_steps=1)
        r64 = timed_steps(ctx, sim64, a.steps)
        ms64, upd64 = ctx.max_sum(r64["ms"], r64["updates"])
        err = {}
        for n in ("P", "C", "T", "qx", "qy", "qz"):
            x, y = sim.field(n), sim64.field(n)
            err[n] = float(numpy.max(numpy.abs(x - y)) / max(numpy.max(numpy.abs(y)), 1e-300))
        # the pressure change over the steps (P - P0) on its own scale: the
        # flow-driven part that the hydrostatic head would hide
        P0 = numpy.asarray(workloads.reservoir_3d(*shape).P)
        dx_, dy_ = sim.field("P") - P0, sim64.field("P") - P0
        err["P_change"] = float(numpy.max(numpy.abs(dx_ - dy_)) / max(numpy.max(numpy.abs(dy_)), 1e-300))
        fp64 = {"value": upd64 / (ms64 / 1e3), "ms_per_step": ms64 / a.steps,
                "speedup_fp32dc": value / (upd64 / (ms64 / 1e3)),
                # the plain form's relaxations for the same steps and
                # tolerances, over the FP32+DC form's time: the rate extra
                # correction sweeps cannot inflate
                "fp64_equivalent_rate_of_fp32dc": upd64 / (ms / 1e3),
                "iterations": {"fp32dc": res["iterations"], "fp64": r64["iterations"]},
                "step_time_ratio": (ms64 / a.steps) / (ms / a.steps),
                "max_rel_err_vs_fp64": err,
                "roofline": roofline(r64, "fp64", peak, peak_kind)}
        del sim64
        torch.cuda.empty_cache()
    e2e = None if a.no_e2e else e2e_steps(ctx, sim, a.steps)
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu = cpu_pressure_rate(shape, a.cpu_seconds)
    roof = roofline(res, "fp32dc", peak, peak_kind)
    ens = srv = None
    if world == 1 and (a.ensemble_models > 0 or a.serving_requests > 0):
        # the batched form and the serving loop of the same library, after
        # the single-model state is released
        del sim
        torch.cuda.empty_cache()
        if a.ensemble_models > 0:
            ens = ensemble_run(a, dev, a.ensemble_models, a.ensemble_steps)
            torch.cuda.empty_cache()
        if a.serving_requests > 0:
            srv = serving_run(a, dev, a.serving_requests, a.serving_steps, a.serving_n_max)
            torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps({
            "metric": "SOR cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "reservoir_3d %dx%dx%d, full time steps (SIA loop), "
                                   "FP32 sweeps + FP64 defect correction" % shape,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "working set > L2 (no flush)"},
            "gpu_launches": int(res["launches"]), "clocks": res["clocks"], "e2e": e2e,
            "autotune": tune,
            # pressure SOR / species / heat separately: each solve call's event
            # time (sweeps, residuals, set-up) and its cell-updates
            "rates_by_solve": res["rates_by_solve"],
            "roofline": roof, "fp64_plain": fp64, "cpu_baseline": cpu,
            # the batched form (the 512-model ensemble of log-uniform 32-128
            # axes) and the serving loop (Poisson arrivals, p50/p99), measured
            # in the same run, each with its own roofline and clocks
            "ensemble": ens, "serving": srv}))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
