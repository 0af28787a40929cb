#!/usr/bin/env python
"""CCZ4 SSP-RK3 point-updates/s on B200 (one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl granite|reference]
                    [--workload binary_bl_4level|triple_bl_6level|single_puncture_128|gauge_wave_48]
                    [--precision mixed|fp64] [--variant global|smem]

Default workload: binary Brill-Lindquist punctures (m = 0.5 at x = +-3) on the
4-level Berger-Oliger hierarchy (coarse dx = 1 on [-64,64]^3, 80-400 uneven
blocks per level with edges from {16,24,32,48,64}, seeded), one coarse step =
the subcycled RK3 step of all levels (level L takes 2^L steps), ghost exchange
between blocks and levels, captured as one CUDA graph. value = point-updates/s
of the mixed-precision form; the FP64 plain form runs on the same hierarchy
and its throughput, the ratio and the mixed-vs-FP64 accuracy are on the line.
A point-update is one interior point advanced by one RK3 step of its level.

Timing: W warm-up steps, then K steps between barriers, timed with CUDA events
on the library's stream, max over ranks; the resident state (GBs) is far larger
than L2. Multi-GPU runs are independent replicas (weak scaling).

Extra objects on the JSON line:
  roofline      HBM roofline of the fused stage kernel: algorithmic bytes
                (1408 B per point-update) / its device time, measured in a
                profiling pass with CUDA events around every stage launch.
  e2e           the same metric through the C ABI with host buffers: every
                step uploads every block from pinned memory, steps, and
                downloads every block; three contexts take the steps in turn so
                that one's upload and another's download overlap the third's
                step ("serial": one context, copies and step in series).
  cpu_baseline  the compiled reference (oracle/_ref, Release flags, OpenMP on
                all host cores) on a bounded sample of the workload's blocks.
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
E2E_CONTEXTS = 3  # contexts of the e2e pipeline: upload, step and download in flight at once
# reference-equivalent flops per point-update: 3 RHS + KO evaluations as ccz4.cpp
# is written (10,395 each, op-counted) + the RK combine (22 fields x 3 stages x 4)
FLOPS_PER_POINT_UPDATE = 3 * 10395 + 22 * 3 * 4
NV = 22
GROUPS = [[0], [1, 2, 3, 4, 5, 6], [7, 8, 9, 10, 11, 12], [13], [14, 15, 16], [17], [18], [19, 20, 21]]

WORKLOADS = {
    "binary_bl_4level": dict(kind="hier", builder="binary"),
    # the same punctures on a small 3-level hierarchy (64^3 cells per level on
    # [-32,32]^3, blocks of 16/24/32 cells, ~0.9 GB resident): for profiling
    # under ncu, whose full captures must stay at a few GB
    "binary_bl_3level_small": dict(kind="hier", builder="binary_small"),
    "triple_bl_6level": dict(kind="hier", builder="triple"),
    # single BL puncture M = 1, 128^3 on [-16,16]^3, r >= dx/2, 1e-10 noise, reference boundaries
    "single_puncture_128": dict(kind="block", n=128, lo=-16.0, hi=16.0, data="bl", bc=0),
    # the same puncture at 256^3 (dx = 0.125)
    "single_puncture_256": dict(kind="block", n=256, lo=-16.0, hi=16.0, data="bl", bc=0),
    # gauge wave g_xx = 1 - 0.1 sin(2 pi x), 48^3 on [-0.5,0.5]^3, periodic
    "gauge_wave_48": dict(kind="block", n=48, lo=-0.5, hi=0.5, data="gw", bc=1),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload: str, kernel: str, precision: str):
    """dram bytes per stage launch from the committed ncu summary, if any: the
    line `traffic_bytes_per_launch_<precision>:`, else `traffic_bytes_per_launch:`."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    if not os.path.exists(path):
        return None
    found = {}
    for line in open(path):
        key, _, val = line.strip().partition(":")
        if key.startswith("traffic_bytes_per_launch") and val:
            try:
                found[key] = float(val.split()[0])
            except ValueError:
                pass
    return found.get(f"traffic_bytes_per_launch_{precision}", found.get("traffic_bytes_per_launch"))


class Runner:
    """One workload on one device through the library's resident-block API."""

    def __init__(self, gb, name, w, precision, variant, device, stage_config=-1, like=None):
        """like: another Runner of the same workload whose host blocks (the
        initial state) this one shares instead of building its own."""
        self.gb, self.w, self.prec = gb, w, precision
        self.ev = gb.Evolver(gb.CCZ4Params(device=device), variant)
        if stage_config >= 0:
            self.ev.force_stage_config(stage_config)
        if like is not None:
            self.h, self.blocks, self.points_per_step, self.dt = like.h, like.blocks, like.points_per_step, like.dt
        elif w["kind"] == "hier":
            self.h = hierarchy_of(gb, w)
            self.blocks = gb.block_states(self.h, noise=1e-10, seed=12345)
            self.points_per_step = self.h.point_updates_per_coarse_step()
            self.dt = 0.25 * self.h.level_dx[0]
        else:
            n, lo, hi = w["n"], w["lo"], w["hi"]
            b = gb.GridBlock(0, 0, (n, n, n), (lo, lo, lo), (hi, hi, hi))
            if w["data"] == "bl":
                gb.brill_lindquist(b, [1.0], [[0.0, 0.0, 0.0]], r_floor=0.5 * b.dx(0))
                gb.initial_data.add_noise(b, 1e-10, 12345)
            else:
                gb.gauge_wave(b, -0.1, 1.0)
            self.h = None
            self.blocks = [b]
            self.points_per_step = n ** 3
            self.dt = 0.25 * b.dx(0)
        for b in self.blocks:
            self.ev.add_block(b)
        self.ev.commit()
        self.ev.upload()
        self.state_bytes = sum(b.array.nbytes for b in self.blocks)
        # the binary hierarchy's state stays finite for 16 coarse steps (the
        # reference's equations on these punctures are not long-term stable):
        # timed runs restart from the initial state every 8 steps
        self.restore_every = 8 if self.h is not None else 0

    def restore(self):
        """Back to the initial state (the blocks' host arrays hold it)."""
        self.ev.upload()
        self.ev.sync()

    def step(self):
        if self.h is not None:
            self.ev.hierarchy_step(self.dt, self.prec, self.gb.AMR_GHOSTS)
        else:
            self.ev.rk3_step(0, self.dt, self.prec, self.w["bc"])

    def config(self):
        if self.h is None:
            n = self.w["n"]
            return {"grid": f"{n}^3", "blocks": 1}
        lv = [sum(1 for b in self.h.blocks if b.level == L) for L in range(self.h.num_levels)]
        return {"levels": self.h.num_levels, "blocks": len(self.h.blocks), "blocks_per_level": lv,
                "interior_points": self.h.interior_points(), "amr_mode": "ghosts",
                "coarse_dx": self.h.level_dx[0], "refinement_ratio": 2, "subcycling": True}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 100 ms in the background."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

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
        num = lambda s: s.strip().replace(".", "", 1).isdigit()  # noqa: E731
        sm = [float(r[1]) for r in rows if len(r) > 8 and num(r[1])]
        mx = [float(r[2]) for r in rows if len(r) > 8 and num(r[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) > 8:
                for k, nm in enumerate(names):
                    if r[5 + k].strip() == "Active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU reference (bounded samples)
# ---------------------------------------------------------------------------

def reference_impl():
    """The compiled reference (Release flags, OpenMP on all cores), else the C restatement."""
    import oracle
    if oracle.reference_available("fast"):
        impl = oracle.Reference("fast")
        return impl, "reference", impl.max_threads()
    return oracle.Oracle(), "port", os.cpu_count()


def hierarchy_of(gb, w):
    if w["builder"] == "binary":
        return gb.make_binary_hierarchy()
    if w["builder"] == "binary_small":
        return gb.make_binary_hierarchy(levels=3, coarse_n=64, extent=32.0, sizes=(16, 24, 32),
                                        blocks_per_level=(20, 100))
    return gb.make_triple_hierarchy()


def reference_jobs(w):
    """Endless sequence of (geometry, state, dt, bc) units of the workload for the
    reference: hierarchy blocks taken round-robin over the levels (so every level's
    sizes appear), each as a single block; or the workload's single block."""
    import oracle
    from oracle import Geom
    o = oracle.Oracle()
    if w["kind"] == "hier":
        import granite_b200 as gb
        h = hierarchy_of(gb, w)
        per = [[b for b in h.blocks if b.level == L] for L in range(h.num_levels)]
        order = [per[L][i] for i in range(max(len(p) for p in per)) for L in range(h.num_levels) if i < len(per[L])]
        while True:
            for b in order:
                g = Geom(b.ncells, b.lo, b.hi)
                u = o.init_brill_lindquist(g, h.masses, h.positions, r_floor=0.5 * g.dx[0])
                yield g, oracle.add_noise(u, 1e-10, 12345), 0.25 * h.level_dx[b.level], 0
    n, lo, hi = w["n"], w["lo"], w["hi"]
    g = Geom((n, n, n), (lo, lo, lo), (hi, hi, hi))
    if w["data"] == "bl":
        u = oracle.add_noise(o.init_brill_lindquist(g, [1.0], [[0.0, 0.0, 0.0]], r_floor=0.5 * g.dx[0]), 1e-10, 12345)
    else:
        u = o.init_gauge_wave(g, -0.1, 1.0)
    while True:
        yield g, u, 0.25 * g.dx[0], w["bc"]


def reference_unit(impl, job):
    """One RK3 step of one unit by the reference; returns (seconds, interior points).
    The compiled reference reports the time of its step loop alone (its
    AMRHierarchy set-up, block allocation and the copies in and out are not
    part of the step); the C restatement is timed around the whole call."""
    from oracle import Params
    g, u, dt, bc = job
    t = time.perf_counter()
    impl.rk3_steps(Params(), g, u, dt, 1, bc)
    wall = time.perf_counter() - t
    loop = impl.last_loop_seconds() if hasattr(impl, "last_loop_seconds") else wall
    return loop, int(np.prod(g.n))


def reference_sample(w, seconds_target: float):
    """The reference advancing units of the workload by whole RK3 steps until
    ~seconds_target of CPU work; returns a cpu_baseline object."""
    impl, kind, cores = reference_impl()
    total, pts, used = 0.0, 0, 0
    for job in reference_jobs(w):
        dt_s, n = reference_unit(impl, job)
        total += dt_s
        pts += n
        used += 1
        if total >= seconds_target:
            break
    what = "blocks of the hierarchy, each as a single block" if w["kind"] == "hier" else "steps of the workload block"
    sample = f"one RK3 step of each of {used} {what} ({pts} interior point-updates)"
    return {"value": pts / total, "unit": UNIT, "cores": int(cores), "kind": kind,
            "sample": f"{sample}; {total:.1f} s; OMP threads = {cores}"}


# points of one reference step sample: a few seconds of host work on a many-core host
REFERENCE_SAMPLE_POINTS = 1 << 21


def run_reference(args, w, rank, world):
    """--impl reference: W warm-up and K timed steps of the reference, each step a
    bounded sample of the workload (units until ~2.1 M interior points; the whole
    block for single-block workloads) advanced by one RK3 step on all host cores."""
    if rank != 0:
        return 0
    import oracle
    if not (oracle.reference_available("fast") or os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so"))):
        print(json.dumps({"impl": "reference", "unavailable": "compiled reference library not built"}))
        return 0
    impl, kind, cores = reference_impl()
    jobs = reference_jobs(w)

    def one_step():
        sec, pts = 0.0, 0
        while pts < REFERENCE_SAMPLE_POINTS:
            dt_s, n = reference_unit(impl, next(jobs))
            sec += dt_s
            pts += n
            if w["kind"] != "hier":
                break
        return sec, pts

    for _ in range(args.warmup):
        one_step()
    times, points = [], []
    for _ in range(args.steps):
        sec, pts = one_step()
        times.append(sec)
        points.append(pts)
    value = sum(points) / sum(times)
    what = "hierarchy blocks taken round-robin over the levels, each as a single block" if w["kind"] == "hier" \
        else "the workload block"
    cb = {"value": value, "unit": UNIT, "cores": int(cores), "kind": kind,
          "sample": f"{args.steps} steps of one RK3 step of {what}, ~{int(np.mean(points))} interior points "
                    f"per step; {sum(times):.1f} s timed; OMP threads = {cores}"}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": args.workload, "precision": "fp64", "parallelism": "host OpenMP",
                       "points_per_step": int(np.mean(points))},
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def max_over_ranks(torch, dist, world, value, device):
    """The largest of the ranks' values (the job's time is its slowest rank's):
    one all-reduce MAX over the process group; the value itself on one rank."""
    if world == 1:
        return float(value)
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(points_per_step, steps, world, ms):
    """Point-updates per second of all ranks together: every rank advances its own
    replica of the workload, the job takes the slowest rank's time."""
    return points_per_step * steps * world / (ms / 1000.0)


def timed_steps(torch, dist, world, local, run: Runner, steps: int):
    """Device time of `steps` steps (CUDA events on the library's stream, max over
    ranks). Where the workload's state leaves the finite regime within the run
    (run.restore_every > 0), the steps go in segments of that many, each from
    the initial state re-uploaded outside the timed region, so every timed step
    advances a finite state; the segments' times are summed."""
    stream = torch.cuda.ExternalStream(run.ev.stream_handle(), device=local)
    n0 = run.ev.launch_count()
    seg = run.restore_every if run.restore_every > 0 else steps
    total, done = 0.0, 0
    while done < steps:
        k = min(seg, steps - done)
        if run.restore_every > 0:
            run.restore()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(local)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            run.step()
        e1.record(stream)
        run.ev.sync()
        torch.cuda.synchronize(local)
        if world > 1:
            dist.barrier()
        total += e0.elapsed_time(e1)
        done += k
    ms = max_over_ranks(torch, dist, world, total, f"cuda:{local}")
    return ms, run.ev.launch_count() - n0


def roofline(gb, run: Runner, workload, prof_steps, kernel):
    if run.restore_every > 0:
        run.restore()
        prof_steps = min(prof_steps, run.restore_every)
    run.ev.set_profiling(True)
    run.ev.profile_reset()
    for _ in range(prof_steps):
        run.step()
    st_ms, st_n = run.ev.profile(gb.KERNEL_STAGE)
    gh_ms, _ = run.ev.profile(gb.KERNEL_GHOST)
    xf_ms, _ = run.ev.profile(gb.KERNEL_TRANSFER)
    run.ev.set_profiling(False)
    peak, peak_kind = measured_peaks()
    total_bytes = BYTES_PER_POINT_UPDATE * run.points_per_step * prof_steps
    achieved = total_bytes / (st_ms / 1000.0) / 1e9
    per_launch = total_bytes / max(st_n, 1)
    traffic = ncu_traffic(workload, kernel, "mixed" if run.prec == gb.PRECISION_MIXED else "fp64")
    # the bound that applies to this kernel: its FP64 / FP32 pipes (HBM is ~10 % busy)
    fp64_peak = gb.measure_fma_rate(run.ev.params.device, 0)
    fp32_peak = gb.measure_fma_rate(run.ev.params.device, 1)
    flops = FLOPS_PER_POINT_UPDATE * run.points_per_step * prof_steps / (st_ms / 1000.0) / 1e12
    compute = {"unit": "TFLOP/s", "achieved": flops, "flops_per_point_update": FLOPS_PER_POINT_UPDATE,
               "flops": "reference-equivalent (ccz4.cpp as written, op-counted), per point-update",
               "peak_fp64": fp64_peak, "peak_fp32": fp32_peak, "frac_of_fp64": flops / fp64_peak,
               "peak_source": "measured here: register-only FMA kernel at full occupancy"}
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_source": peak_kind, "kernel": kernel,
            "avg_launch_ms": st_ms / max(st_n, 1), "launches_per_step": st_n / prof_steps,
            "algorithmic_bytes_per_launch": per_launch,
            "stage_share_of_step": st_ms / max(st_ms + gh_ms + xf_ms, 1e-12),
            "device_ms_per_step": {"stage": st_ms / prof_steps, "ghost": gh_ms / prof_steps,
                                   "transfer": xf_ms / prof_steps},
            "compute": compute}


def accuracy(gb, a: Runner, b: Runner, steps: int):
    """Mixed (b) against FP64 (a) after the same steps, on the device: per-field
    max deviation over the interior of all blocks relative to the largest |FP64|
    of the field's tensor group, ||H||_2 and ||M||_2 ratios, and whether the
    FP64 state is still finite."""
    dev, mag, nf = a.ev.compare_states(b.ev)
    gscale = np.zeros(NV)
    for grp in GROUPS:
        gscale[grp] = mag[grp].max()
    with np.errstate(invalid="ignore"):
        rel = np.where(np.isfinite(dev), dev / np.maximum(gscale, 1e-300), np.inf)
    ha, ma = a.ev.constraint_norms(-1)
    hb, mb = b.ev.constraint_norms(-1)
    finite = nf[0] == 0 and bool(np.isfinite(ha) and np.isfinite(ma))
    return {"coarse_steps": steps, "max_rel_dev": float(rel.max()),
            "max_rel_dev_field": int(rel.argmax()), "h_l2_fp64": ha, "h_l2_mixed": hb,
            "h_l2_ratio": hb / ha if ha else None, "m_l2_ratio": mb / ma if ma else None,
            "fp64_finite": finite, "nonfinite_fp64": int(nf[0]), "nonfinite_mixed": int(nf[1])}


def accuracy_run(gb, a: Runner, b: Runner, steps: int, every: int, seconds: float):
    """FP64 (a) and mixed (b) stepped side by side from the same initial state
    (re-uploaded), compared every `every` steps up to `steps` or until the FP64
    state goes non-finite (the reference's equations on puncture data are not
    long-term stable) or `seconds` of wall time pass. Reports the comparison
    at the last step where the FP64 state was finite, the largest deviation up
    to there and while ||H||_2 of the FP64 state stayed within 10x of its
    initial value (the solution still bounded, with the field and step of that
    largest deviation), and a thinned history [step, max_rel_dev, field,
    h_l2_ratio, h_l2_fp64]."""
    for r in (a, b):
        r.ev.upload()
        r.ev.sync()
    h0 = a.ev.constraint_norms(-1)[0]
    last, worst, hist, stop = None, 0.0, [], "steps"
    worst_bounded, bounded_until, still_bounded = 0.0, 0, True
    worst_bounded_at = (None, None)  # (field, step)
    t0 = time.perf_counter()
    for s in range(1, steps + 1):
        a.step()
        b.step()
        if s % every and s != steps:
            continue
        r = accuracy(gb, a, b, s)
        if not r["fp64_finite"]:
            stop = "fp64 state non-finite"
            first_bad = s
            break
        last = r
        worst = max(worst, r["max_rel_dev"])
        if still_bounded and r["h_l2_fp64"] <= 10.0 * h0:
            if r["max_rel_dev"] >= worst_bounded:
                worst_bounded, worst_bounded_at = r["max_rel_dev"], (r["max_rel_dev_field"], s)
            bounded_until = s
        else:
            still_bounded = False
        hist.append([s, r["max_rel_dev"], r["max_rel_dev_field"], r["h_l2_ratio"], r["h_l2_fp64"]])
        if time.perf_counter() - t0 > seconds:
            stop = "time cap"
            break
    out = dict(last) if last else {"coarse_steps": 0}
    out.update({"steps_requested": steps, "check_every": every, "stopped_by": stop,
                "max_rel_dev_over_run": worst, "h_l2_fp64_initial": h0,
                "bounded_until_step": bounded_until, "max_rel_dev_while_bounded": worst_bounded,
                "max_rel_dev_while_bounded_field": worst_bounded_at[0],
                "max_rel_dev_while_bounded_step": worst_bounded_at[1],
                "wall_s": time.perf_counter() - t0,
                "history": hist[:: max(1, len(hist) // 20)] + ([hist[-1]] if hist else [])})
    if stop == "fp64 state non-finite":
        out["fp64_nonfinite_by_step"] = first_bad
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="granite", choices=["granite", "reference"])
    ap.add_argument("--workload", default="binary_bl_4level", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="headline precision (default: mixed for hierarchies, fp64 for single blocks)")
    ap.add_argument("--variant", default="tma",
                    choices=["global", "smem", "global_r168", "global_r128", "tma"],
                    help="stage-kernel variant: stencils from global memory (optionally register-capped) "
                         "or staged in shared memory")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--fp64-chi", type=float, default=0.5,
                    help="mixed precision: tiles with a point of chi below this run the FP64 algebra "
                         "(0 = FP32 algebra everywhere)")
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="mixed runs: step FP64 and mixed side by side from the initial state for up to "
                         "this many steps (coarse steps of a hierarchy), or until the FP64 state goes "
                         "non-finite, and report the deviation there (0 = only after the warm-up)")
    ap.add_argument("--accuracy-every", type=int, default=1, help="steps between accuracy checks")
    ap.add_argument("--accuracy-seconds", type=float, default=420.0,
                    help="wall-time cap of the accuracy run")
    ap.add_argument("--stage-config", type=int, default=-1,
                    help="one TMA stage-kernel configuration for every block (default: the per-class table)")
    ap.add_argument("--ghost-push", type=int, default=-1, choices=[-1, 0, 1],
                    help="GRANITE_AMR_GHOSTS: stage kernels write the same-level ghost copies (1) or the "
                         "fills copy them (0); -1 = the library default")
    ap.add_argument("--pass-overlap", type=int, default=-1, choices=[-1, 0, 1],
                    help="per-tile precision: FP64 pass beside the FP32 pass (1) or after it (0); -1 = default")
    ap.add_argument("--no-amr-reference", action="store_true",
                    help="skip the GRANITE_AMR_REFERENCE hierarchy timing")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    w = WORKLOADS[args.workload]
    hier = w["kind"] == "hier"
    precision = args.precision or ("mixed" if hier else "fp64")

    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        if args.impl == "reference":  # host cores only: the ranks just meet at the end
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=900))
        else:
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    if args.impl == "reference":
        rc = run_reference(args, w, rank, world)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return rc

    import granite_b200 as gb
    variant = gb.VARIANT_NAMES[args.variant]
    kname = {gb.VARIANT_SMEM: "ccz4_stage_smem_kernel", gb.VARIANT_TMA: "ccz4_stage_tma_kernel"}.get(
        variant, "ccz4_stage_kernel")
    prec = gb.PRECISION_MIXED if precision == "mixed" else gb.PRECISION_FP64
    def configure(r):
        if prec == gb.PRECISION_MIXED and args.fp64_chi > 0.0:
            r.ev.set_fp64_chi_threshold(args.fp64_chi)
        if args.ghost_push >= 0:
            r.ev.set_ghost_push(bool(args.ghost_push))
        if args.pass_overlap >= 0:
            r.ev.set_pass_overlap(bool(args.pass_overlap))

    run = Runner(gb, args.workload, w, prec, variant, local, args.stage_config)
    configure(run)
    compare = None
    if prec == gb.PRECISION_MIXED and not args.no_compare:
        compare = Runner(gb, args.workload, w, gb.PRECISION_FP64, variant, local, args.stage_config)

    for r in (run, compare):
        if r is None:
            continue
        for _ in range(args.warmup):
            r.step()
        r.ev.sync()
    # mixed vs FP64 on the state the timed steps start from
    acc = accuracy(gb, compare, run, args.warmup) if compare is not None else None
    if acc is not None:
        acc["fp64_chi_threshold"] = args.fp64_chi

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    ms, launches = timed_steps(torch, dist, world, local, run, args.steps)
    clocks = sampler.stop()
    value = whole_job_rate(run.points_per_step, args.steps, world, ms)
    # kernel time of the same steps (eager launches bracketed by events), clocks sampled again
    prof_steps = max(1, min(args.steps, 5 if hier else 20))
    rsampler = ClockSampler(local)
    rsampler.start()
    time.sleep(0.3)
    rl = roofline(gb, run, args.workload, prof_steps, kname)
    rl["clocks"] = rsampler.stop()

    # e2e through the C ABI with host buffers (pinned), copies inside the timed
    # region: every step uploads its input state (the workload's initial state)
    # from pinned host memory, steps, and downloads the result into a pinned
    # buffer. Up to E2E_CONTEXTS contexts hold the workload and take the steps in
    # turn, a three-stage pipeline: while one context steps (SMs), the next
    # one's upload and the previous one's download run (copy engines, one
    # direction each). Uploads, and downloads, are ordered across the contexts
    # by events on the contexts' streams, so each copy runs at the full PCIe
    # rate instead of sharing it with the other contexts' copies; before a
    # context takes its next step the host waits for its previous result. The
    # same round trip on one context, copies and step in series, is reported
    # beside it.
    def pinned_like(a):
        t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
        return t, t.numpy().reshape(a.shape)

    hosts_in = [pinned_like(b.array) for b in run.blocks]
    for (_, v), b in zip(hosts_in, run.blocks):
        v[...] = b.array
    hosts_out = [[pinned_like(b.array) for b in run.blocks]]  # one per context (more below)
    vin = [v for _, v in hosts_in]
    vouts = [[v for _, v in ho] for ho in hosts_out]

    serial_steps = max(1, min(args.steps, 3 if hier else 20))
    run.ev.sync()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(serial_steps):
        run.ev.upload(None, vin)
        run.step()
        run.ev.download(None, vouts[0])
    run.ev.sync()
    serial_ms = max_over_ranks(torch, dist, world, (time.perf_counter() - t0) * 1000.0, f"cuda:{local}")
    serial_val = whole_job_rate(run.points_per_step, serial_steps, world, serial_ms)

    # as many more contexts as the device's free memory holds (a 60 GB hierarchy
    # fits one more at most), keeping 2 GB for graphs and scratch
    free_bytes = torch.cuda.mem_get_info(local)[0]
    extra = max(0, min(E2E_CONTEXTS - 1, int((free_bytes - (2 << 30)) // max(run.ev.arena_bytes(), 1))))
    ring = [run]
    for _ in range(extra):
        r = Runner(gb, args.workload, w, prec, variant, local, args.stage_config, like=run)
        configure(r)
        r.step()  # builds its step graph
        r.ev.sync()
        ring.append(r)
    nctx = len(ring)
    hosts_out += [[pinned_like(b.array) for b in run.blocks] for _ in range(nctx - 1)]
    vouts = [[v for _, v in ho] for ho in hosts_out]
    streams = [torch.cuda.ExternalStream(r.ev.stream_handle(), device=f"cuda:{local}") for r in ring]
    e2e_steps = max(2 * nctx, min(args.steps, 16 if hier else 40))
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    last_up = last_down = None
    for s in range(e2e_steps):
        r, st = ring[s % nctx], streams[s % nctx]
        r.ev.sync()  # its previous result is on the host before the buffers are reused
        if last_up is not None:
            st.wait_event(last_up)
        r.ev.upload(None, vin)
        last_up = torch.cuda.Event()
        last_up.record(st)
        r.step()
        if last_down is not None:
            st.wait_event(last_down)
        r.ev.download(None, vouts[s % nctx], wait=False)
        last_down = torch.cuda.Event()
        last_down.record(st)
    for r in ring:
        r.ev.sync()
    e2e_ms = max_over_ranks(torch, dist, world, (time.perf_counter() - t0) * 1000.0, f"cuda:{local}")
    e2e_val = whole_job_rate(run.points_per_step, e2e_steps, world, e2e_ms)
    for r in ring[1:]:
        r.ev.close()
    del ring, streams

    # after the headline measurements: the same mixed steps with the FP32 algebra on
    # every tile, then the FP64 comparison runs (these drop and rebuild cached graphs)
    fp32_line = None
    if prec == gb.PRECISION_MIXED and args.fp64_chi > 0.0:
        # the same mixed steps with the FP32 algebra on every tile (no FP64 pass)
        run.ev.set_fp64_chi_threshold(0.0)
        for _ in range(2):
            run.step()
        fms, _ = timed_steps(torch, dist, world, local, run, args.steps)
        run.ev.set_fp64_chi_threshold(args.fp64_chi)
        fp32_line = {"value": run.points_per_step * args.steps * world / (fms / 1000.0),
                     "ms_per_step": fms / args.steps}
    cmp_line = None
    if compare is not None:
        cms, _ = timed_steps(torch, dist, world, local, compare, args.steps)
        cvalue = compare.points_per_step * args.steps * world / (cms / 1000.0)
        # the same FP64 kernel launched block by block without graphs (a per-block
        # drop-in of the reference's per-GridBlock calls)
        ksteps = max(1, min(args.steps, 5))
        compare.ev.set_batching(False)
        ums, _ = timed_steps(torch, dist, world, local, compare, ksteps)
        compare.ev.set_batching(True)
        uvalue = compare.points_per_step * ksteps * world / (ums / 1000.0)
        cmp_line = {"fp64_value": cvalue, "fp64_ms_per_step": cms / args.steps,
                    "mixed_over_fp64": value / cvalue,
                    "fp64_unbatched_value": uvalue, "fp64_unbatched_ms_per_step": ums / ksteps,
                    "fp64_unbatched_steps": ksteps, "mixed_over_fp64_unbatched": value / uvalue}

    # the reference's own hierarchy semantics (GRANITE_AMR_REFERENCE: prolongation
    # into every fine cell before and after each fine step, amr.cpp:313-329)
    amr_ref = None
    if hier and not args.no_amr_reference:
        amr_ref = {"amr_mode": "reference", "steps": max(1, min(args.steps, 5))}
        for tag, r in (("mixed", run), ("fp64", compare)):
            if r is None:
                continue
            r.ev.upload()
            for _ in range(2):
                r.ev.hierarchy_step(r.dt, r.prec, gb.AMR_REFERENCE)
            orig = r.step
            r.step = lambda r=r: r.ev.hierarchy_step(r.dt, r.prec, gb.AMR_REFERENCE)
            rms, _ = timed_steps(torch, dist, world, local, r, amr_ref["steps"])
            r.step = orig
            amr_ref[f"{tag}_value"] = r.points_per_step * amr_ref["steps"] * world / (rms / 1000.0)
            amr_ref[f"{tag}_ms_per_step"] = rms / amr_ref["steps"]
        if "fp64_value" in amr_ref:
            amr_ref["mixed_over_fp64"] = amr_ref["mixed_value"] / amr_ref["fp64_value"]

    # mixed against FP64 from the same initial state, as far as the FP64 state stays finite
    if compare is not None and args.accuracy_steps > 0:
        if prec == gb.PRECISION_MIXED and args.fp64_chi > 0.0:
            run.ev.set_fp64_chi_threshold(args.fp64_chi)
        acc = accuracy_run(gb, compare, run, args.accuracy_steps, args.accuracy_every, args.accuracy_seconds)
        acc["fp64_chi_threshold"] = args.fp64_chi
    if compare is not None:
        compare.ev.close()
        compare = None

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = reference_sample(w, seconds_target=15.0)
        except Exception as ex:  # the baseline is a reported number, not the product
            cb = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                  "sample": f"failed: {ex}"}

    if rank == 0:
        cls_cfg = {p: [run.ev.stage_config(q, c) for c in range(len(gb.STAGE_CLASS_EDGES))]
                   for p, q in (("fp64", gb.PRECISION_FP64), ("mixed", gb.PRECISION_MIXED))}
        cfg = {"workload": args.workload, "precision": precision, "kernel_variant": args.variant,
               "stage_configs": {"class_edges": list(gb.STAGE_CLASS_EDGES), **cls_cfg},
               "fp64_chi_threshold": args.fp64_chi if prec == gb.PRECISION_MIXED else None,
               "ghosts": 4, "fields": NV, "point_updates_per_step": run.points_per_step, "dt": run.dt,
               "l2": f"inputs larger than L2: {3 * run.state_bytes / 1e9:.2f} GB resident state",
               "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}
        cfg.update(run.config())
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f32+f64" if prec == gb.PRECISION_MIXED else "f64", "data": "synthetic",
                "config": cfg, "roofline": rl,
                "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": run.state_bytes,
                        "d2h_bytes_per_step": run.state_bytes, "steps": e2e_steps, "contexts": nctx,
                        "serial": {"value": serial_val, "steps": serial_steps, "contexts": 1}},
                "cpu_baseline": cb, "clocks": clocks, "gpu_launches": launches}
        if cmp_line:
            line["fp64_plain"] = cmp_line
        if fp32_line:
            line["fp32_algebra_all_tiles"] = fp32_line
        if acc:
            line["accuracy_mixed_vs_fp64"] = acc
        if amr_ref:
            line["amr_reference"] = amr_ref
        print(json.dumps(line))
    run.ev.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
