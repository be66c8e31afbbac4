#!/usr/bin/env python
"""Benchmark: SOR cell-updates/s of the TRANSPORTSE time-step core on B200.

Workload (default): the 256 x 256 x 128 bottom-heated reservoir
(transportse_b200.workloads.reservoir_3d: geometric spacing, GRF log10 K,
two species plus heat, linear EOS, SIA Picard tolerance 1e-6), synthetic
seeded inputs.  One step = one full time step of the model (SIA loop with
pressure solve, fluxes, flow error, species and heat solves, EOS).

Metric: cell-updates per second over the timed steps, where a cell-update
is one active (non-Dirichlet) cell relaxed once in a red+black iteration of
the pressure, species or heat solve.  ``value`` is measured with all state
resident in HBM; ``e2e`` repeats the steps through the public API with the
state uploaded from pinned host memory and the solution read back every
step.  The working set (~2 GB) is far larger than L2, so no flush is needed.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

PRESSURE_BYTES_FP64 = 57   # algorithmic bytes per pressure cell-update, FP64 form
DEFAULT_SHAPE = (256, 256, 128)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--shape", type=str, default=None, help="override grid, e.g. 64x64x32")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def shape_of(a):
    if a.shape:
        return tuple(int(x) for x in a.shape.lower().split("x"))
    return DEFAULT_SHAPE


def measured_peak():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
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
    rho = numpy.ascontiguousarray(cfg.rho_f)
    args = (cfg.c_f, cfg.nue, rho, cfg.phi, cfg.Kx, cfg.Ky, cfg.Kz, z, z, z)
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
            "kind": "port",
            "sample": "%d single-iteration compute_P calls (red+black sweep, copy, L2) on the "
                      "%dx%dx%d grid, %.1f s" % ((calls,) + tuple(shape) + (el,))}


def run_reference_arm(a, rank):
    if rank != 0:
        return
    shape = shape_of(a)
    vals = []
    for _ in range(a.warmup):
        cpu_pressure_rate(shape, 1.0)
    info = None
    for _ in range(a.steps):
        info = cpu_pressure_rate(shape, max(2.0, a.cpu_seconds / max(1, a.steps)))
        vals.append(info["value"])
    v = statistics.mean(vals)
    line = {"impl": "reference", "metric": "SOR cell-updates/s", "value": v,
            "unit": "cell-updates/s", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "reservoir_3d %dx%dx%d pressure SOR sweeps" % shape},
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": info["cores"],
                             "kind": info["kind"], "sample": info["sample"]},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------- GPU arm
def main():
    a = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if a.impl == "reference":
        return run_reference_arm(a, rank)
    import torch
    import torch.distributed as dist
    from transportse_b200 import workloads
    from transportse_b200.driver import Simulation
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=dev)
    shape = shape_of(a)
    cfg = workloads.reservoir_3d(*shape)
    sim = Simulation(cfg, device=dev)
    M = sim.M
    for _ in range(a.warmup):
        sim.run(max_steps=1)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---------------- device-resident timed region
    cu0 = dict(M.cell_updates)
    M.timing = True
    M.timed = []
    launches0 = M.launches
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        sim.run(max_steps=1)
    e1.record()
    barrier()
    clk = clocks.stop()
    M.timing = False
    ms = e0.elapsed_time(e1)
    updates = sum(M.cell_updates[k] - cu0[k] for k in cu0)
    gpu_launches = M.launches - launches0
    # pressure-solve launches: algorithmic bytes / event duration
    p_bytes, p_ms, n_p = 0.0, 0.0, 0
    for kind, s0, s1, nit, active in M.timed:
        if kind == "P":
            p_bytes += float(nit) * active * PRESSURE_BYTES_FP64
            p_ms += s0.elapsed_time(s1)
            n_p += 1
    t = torch.tensor([ms, float(updates)], dtype=torch.float64, device=dev)
    if world > 1:
        tmax = t.clone()
        dist.all_reduce(tmax[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:2], op=dist.ReduceOp.SUM)
        ms_max, upd_all = float(tmax[0]), float(t[1])
    else:
        ms_max, upd_all = ms, float(updates)
    value = upd_all / (ms_max / 1e3)

    # ---------------- end-to-end through the public API with host buffers
    e2e = None
    if not a.no_e2e:
        host = {}
        for name, tns in sim.S.items():
            h = torch.empty(tns.shape, dtype=tns.dtype, pin_memory=True)
            h.copy_(tns)
            host[name] = h
        outs = {n: torch.empty(sim.S[n].shape, dtype=torch.float64, pin_memory=True)
                for n in ("P", "C", "T", "qx", "qy", "qz")}
        h2d = sum(h.numel() * h.element_size() for h in host.values())
        d2h = sum(h.numel() * h.element_size() for h in outs.values())
        cu1 = dict(M.cell_updates)
        barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record()
        for _ in range(a.steps):
            for name, h in host.items():
                sim.S[name].copy_(h, non_blocking=True)
            sim.run(max_steps=1)
            for n, h in outs.items():
                h.copy_(sim.S[n], non_blocking=True)
        f1.record()
        barrier()
        ms_e2e = f0.elapsed_time(f1)
        upd_e2e = sum(M.cell_updates[k] - cu1[k] for k in cu1)
        te = torch.tensor([ms_e2e, float(upd_e2e)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(te[0:1], op=dist.ReduceOp.MAX)
            tsum = torch.tensor([float(upd_e2e)], dtype=torch.float64, device=dev)
            dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
            te[1] = tsum[0]
        e2e = {"value": float(te[1]) / (float(te[0]) / 1e3), "unit": "cell-updates/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}

    peak, peak_kind = measured_peak()
    roof = None
    if n_p:
        achieved = p_bytes / (p_ms / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None,
                "kernel": "rb_solve_kernel<PressureForm> (FP64 exact, per compute_P launch)",
                "algorithmic_bytes_per_cell_update": PRESSURE_BYTES_FP64,
                "peak_source": peak_kind, "launches": n_p}
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu = cpu_pressure_rate(shape, a.cpu_seconds)
    if rank == 0:
        line = {"metric": "SOR cell-updates/s", "value": value, "unit": "cell-updates/s",
                "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
                "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "reservoir_3d %dx%dx%d, full time steps (SIA loop), "
                                       "FP64 plain form" % shape,
                           "parallelism": "replicas" if world > 1 else "single",
                           "l2": "working set > L2 (no flush)"},
                "gpu_launches": int(gpu_launches), "clocks": clk, "e2e": e2e,
                "roofline": roof, "cpu_baseline": cpu}
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
