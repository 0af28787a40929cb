#!/usr/bin/env python
"""CCZ4 SSP-RK3 point-updates/s on B200 (one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl granite|reference]
                    [--workload single_puncture_128|gauge_wave_48] [--precision fp64|mixed]

A step is one full SSP-RK3 coarse step of the workload (3 fused RHS+KO+RK
stage launches, ghost fills), inputs resident in HBM. The metric counts
interior points x RK3 steps per wall second, timed with CUDA events on the
library's stream between barriers, max over ranks. Multi-GPU runs are
independent replicas (the single-block workloads do not shard), weak scaling.

Extra objects on the JSON line:
  roofline      HBM roofline of the fused stage kernel: algorithmic bytes
                (1408 B per point-update) / its device time, measured in a
                profiling pass with CUDA events around every stage launch.
  e2e           the same metric through the C ABI with host buffers: every
                step uploads the state from pinned host memory, steps, and
                downloads the state.
  cpu_baseline  the compiled reference (oracle/_ref, Release flags, OpenMP on
                all host cores) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CCZ4 RK3 point-updates/s on 1 B200: mixed/batched vs FP64 plain, equal accuracy"
UNIT = "point-updates/s"
BYTES_PER_POINT_UPDATE = 1408  # 3 stages: (2 + 3 + 3) x 22 fields x 8 B
NV = 22

WORKLOADS = {
    # Single Brill-Lindquist puncture, M = 1 at the origin, 128^3 on [-16,16]^3,
    # r floored at dx/2, U(-1e-10, 1e-10) noise (seed 12345), CFL 0.25,
    # reference boundaries (zero-gradient level fill + 1/r falloff).
    "single_puncture_128": dict(n=128, lo=-16.0, hi=16.0, kind="bl", bc=0),
    # Gauge wave g_xx = 1 - 0.1 sin(2 pi x), 48^3 on [-0.5,0.5]^3, periodic.
    "gauge_wave_48": dict(n=48, lo=-0.5, hi=0.5, kind="gw", bc=1),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload: str, kernel: str):
    """dram bytes per stage launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def make_state(gb, w):
    n, lo, hi = w["n"], w["lo"], w["hi"]
    b = gb.GridBlock(0, 0, (n, n, n), (lo, lo, lo), (hi, hi, hi))
    if w["kind"] == "bl":
        gb.brill_lindquist(b, [1.0], [[0.0, 0.0, 0.0]], r_floor=0.5 * b.dx(0))
        gb.initial_data.add_noise(b, 1e-10, 12345)
    else:
        gb.gauge_wave(b, -0.1, 1.0)
    return b


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 100 ms in the background."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def mark(self, which):
        setattr(self, which, time.time())

    def stop(self):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except subprocess.TimeoutExpired:
                self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().splitlines() if r.strip()]
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if len(r) > 8 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 8 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) > 8:
                for k, nm in enumerate(names):
                    if r[5 + k].strip() == "Active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(w, seconds_target=15.0):
    """Compiled reference (Release flags, OpenMP on all cores) on a bounded sample:
    whole RK3 steps of the same workload until ~seconds_target of CPU work."""
    import oracle
    from oracle import Geom, Params
    n, lo, hi = w["n"], w["lo"], w["hi"]
    g = Geom((n, n, n), (lo, lo, lo), (hi, hi, hi))
    if oracle.reference_available("fast"):
        impl = oracle.Reference("fast")
        kind = "reference"
        cores = impl.max_threads()
    else:
        impl = oracle.Oracle()
        kind = "port"
        cores = os.cpu_count()
    o = oracle.Oracle()
    if w["kind"] == "bl":
        u = o.init_brill_lindquist(g, [1.0], [[0.0, 0.0, 0.0]], r_floor=0.5 * g.dx[0])
        u = oracle.add_noise(u, 1e-10, 12345)
    else:
        u = o.init_gauge_wave(g, -0.1, 1.0)
    dt = 0.25 * g.dx[0]
    bc = w["bc"]
    t = time.perf_counter()
    u = impl.rk3_steps(Params(), g, u, dt, 1, bc)
    first = time.perf_counter() - t
    steps = 1
    total = first
    extra = int(max(0, min(20, seconds_target / max(first, 1e-3) - 1)))
    if extra:
        t = time.perf_counter()
        u = impl.rk3_steps(Params(), g, u, dt, extra, bc)
        total += time.perf_counter() - t
        steps += extra
    pts = n ** 3 * steps
    return {"value": pts / total, "unit": UNIT, "cores": int(cores), "kind": kind,
            "sample": f"{steps} RK3 step(s) of the full {n}^3 workload, {total:.1f} s, "
                      f"OMP threads = {cores}"}


def run_reference(args, w, rank, world):
    if rank != 0:
        return 0
    import oracle
    if not (oracle.reference_available("fast") or os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so"))):
        print(json.dumps({"impl": "reference", "unavailable": "compiled reference library not built"}))
        return 0
    # each reference step is one RK3 step of the same workload; bound the run to ~2 minutes
    cb = cpu_baseline(w, seconds_target=min(120.0, 6.0 * max(1, args.steps)))
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": world,
            "steps": int(cb["sample"].split()[0]), "warmup": 0,
            "ms_per_step": 1000.0 * w["n"] ** 3 / cb["value"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": args.workload, "grid": f"{w['n']}^3", "precision": "fp64",
                       "parallelism": "host OpenMP"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="granite", choices=["granite", "reference"])
    ap.add_argument("--workload", default="single_puncture_128", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--variant", default="smem", choices=["global", "smem"],
                    help="stage-kernel variant: stencils from global memory or staged in shared memory")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    w = WORKLOADS[args.workload]

    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.impl == "reference":
        rc = run_reference(args, w, rank, world)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return rc

    import granite_b200 as gb
    prec = gb.PRECISION_FP64 if args.precision == "fp64" else gb.PRECISION_MIXED
    block = make_state(gb, w)
    variant = gb.VARIANT_SMEM if args.variant == "smem" else gb.VARIANT_GLOBAL
    ev = gb.Evolver(gb.CCZ4Params(device=local), variant)
    ev.add_block(block)
    ev.commit()
    ev.upload()
    dt = 0.25 * block.dx(0)
    bc = w["bc"]
    pts = w["n"] ** 3
    stream = torch.cuda.ExternalStream(ev.stream_handle(), device=local)

    for _ in range(args.warmup):
        ev.rk3_step(0, dt, prec, bc)
    ev.sync()

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    n0 = ev.launch_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ev.rk3_step(0, dt, prec, bc)
    e1.record(stream)
    ev.sync()
    torch.cuda.synchronize(local)
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    launches = ev.launch_count() - n0
    clocks = sampler.stop()
    ms_t = torch.tensor([ms], device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = pts * args.steps * world / (ms_max / 1000.0)

    # roofline pass: every stage launch bracketed by events on the library stream
    prof_steps = min(args.steps, 20)
    ev.set_profiling(True)
    ev.profile_reset()
    for _ in range(prof_steps):
        ev.rk3_step(0, dt, prec, bc)
    st_ms, st_n = ev.profile(gb.KERNEL_STAGE)
    gh_ms, gh_n = ev.profile(gb.KERNEL_GHOST)
    ev.set_profiling(False)
    peak, peak_kind = measured_peaks()
    bytes_per_launch = BYTES_PER_POINT_UPDATE * pts / 3.0
    avg_launch_ms = st_ms / max(st_n, 1)
    achieved = bytes_per_launch / (avg_launch_ms / 1000.0) / 1e9
    kname = "ccz4_stage_smem_kernel" if variant == gb.VARIANT_SMEM else "ccz4_stage_kernel"
    traffic = ncu_traffic(args.workload, kname)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "peak_source": peak_kind,
                "kernel": "ccz4_stage_smem_kernel" if variant == gb.VARIANT_SMEM else "ccz4_stage_kernel",
                "avg_launch_ms": avg_launch_ms,
                "stage_share_of_step": st_ms / max(st_ms + gh_ms, 1e-12),
                "algorithmic_bytes_per_launch": bytes_per_launch}

    # e2e through the C ABI with host buffers (pinned), copies inside the timed region
    host = torch.empty(block.array.size, dtype=torch.float64, pin_memory=True)
    hview = host.numpy().reshape(block.array.shape)
    hview[...] = block.array
    e2e_steps = max(1, min(args.steps, 20))
    ev.sync()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    x0 = torch.cuda.Event(enable_timing=True)
    x1 = torch.cuda.Event(enable_timing=True)
    x0.record(stream)
    for _ in range(e2e_steps):
        ev.upload(0, hview)
        ev.rk3_step(0, dt, prec, bc)
        ev.download(0, hview)
    x1.record(stream)
    ev.sync()
    e2e_ms = x0.elapsed_time(x1)
    wall_ms = (time.perf_counter() - t0) * 1000.0
    e2e_ms = max(e2e_ms, wall_ms)
    e_t = torch.tensor([e2e_ms], device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(e_t, op=dist.ReduceOp.MAX)
    e2e_val = pts * e2e_steps * world / (float(e_t.item()) / 1000.0)
    state_bytes = block.array.nbytes

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_baseline(w)
        except Exception as ex:  # the baseline is a reported number, not the product
            cb = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                  "sample": f"failed: {ex}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if prec == 0 else "f32+f64", "data": "synthetic",
                "config": {"workload": args.workload, "grid": f"{w['n']}^3", "ghosts": 4,
                           "fields": NV, "precision": args.precision, "kernel_variant": args.variant,
                           "points_per_step": pts, "dt": dt,
                           "l2": f"inputs larger than L2: {3 * state_bytes / 1e9:.2f} GB resident state",
                           "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
                "roofline": roofline,
                "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                        "d2h_bytes_per_step": state_bytes, "steps": e2e_steps},
                "cpu_baseline": cb,
                "clocks": clocks,
                "gpu_launches": launches}
        print(json.dumps(line))
    ev.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
