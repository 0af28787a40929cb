"""Autotuner of the TMA stage kernel per block-size class.

The reference evaluates computeRHS with one OpenMP loop per block whatever its
size (ccz4.cpp:267-270). Here the stage kernel exists in several
configurations (tile depth, ring depth, shared-memory copies of the stage input
and of the Hessian-field loop; granite_b200.stage_config_info), and the best one
depends on the block size (partial tiles along x, halo overhead per tile,
resident CTAs per SM) and on the precision. For every block-size class (edge
in STAGE_CLASS_EDGES) and precision this module times every configuration on a
level of equal cubic blocks of that edge carrying single-puncture data (about
two million interior points, so a launch takes about a millisecond), with CUDA
events around every stage launch (the library's profiler), and keeps the
fastest. The result is a table {"fp64": [cfg per class], "mixed": [...]} that
Evolver.apply_stage_table applies, and a uniform table (one configuration per
precision for every class): a level whose blocks use different configurations
runs one launch per configuration, and on hierarchies of mixed block sizes the
extra launch tails cost more than the per-class gains, so the library's
built-in default is the uniform table this module produced on a B200.

    python -m granite_b200.tuner [--out table.json] [--classes 16,24] [--configs 0,4] [--precisions mixed]
                                 [--steps 3]
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np

from . import (PRECISION_FP64, PRECISION_MIXED, STAGE_CLASS_EDGES, STAGE_CONFIGS, BC_REFERENCE, CCZ4Params,
               Evolver, GridBlock, KERNEL_STAGE, block_stage_class, stage_config_info)
from .initial_data import add_noise, brill_lindquist

PRECISIONS = {"fp64": PRECISION_FP64, "mixed": PRECISION_MIXED}


def class_level(edge: int, target_points: int = 1 << 21, dx: float = 0.25):
    """Equal cubic blocks of `edge` cells tiling a cube around one puncture at
    the origin (M = 1, r >= dx / 2, 1e-10 noise): about target_points interior
    points in all."""
    nb = max(1, round(target_points / edge ** 3))
    per = max(1, round(nb ** (1.0 / 3.0)))
    dims = [per, per, max(1, math.ceil(nb / (per * per)))]
    h = edge * dx
    lo0 = [-0.5 * d * h for d in dims]
    blocks = []
    for k in range(dims[2]):
        for j in range(dims[1]):
            for i in range(dims[0]):
                if len(blocks) == nb:
                    break
                lo = (lo0[0] + i * h, lo0[1] + j * h, lo0[2] + k * h)
                b = GridBlock(len(blocks), 0, (edge,) * 3, lo, tuple(x + h for x in lo))
                brill_lindquist(b, [1.0], [[0.0, 0.0, 0.0]], r_floor=0.5 * dx)
                add_noise(b, 1e-10, 12345 + len(blocks))
                blocks.append(b)
    return blocks, dx


def time_config(blocks, dx: float, precision: int, cfg: int, steps: int = 3, warmup: int = 1,
                fp64_chi: float = 0.5, device: int = 0) -> float:
    """Stage-kernel device time per point-stage (ns) of one configuration on a
    level of blocks (RK3 steps of level 0, every stage launch event-timed)."""
    ev = Evolver(CCZ4Params(device=device))
    try:
        ev.force_stage_config(cfg)
        for b in blocks:
            ev.add_block(b)
        ev.commit()
        ev.upload()
        if precision == PRECISION_MIXED and fp64_chi > 0.0:
            ev.set_fp64_chi_threshold(fp64_chi)
        dt = 0.25 * dx
        for _ in range(warmup):
            ev.rk3_step(0, dt, precision, BC_REFERENCE)
        ev.sync()
        ev.set_profiling(True)
        ev.profile_reset()
        for _ in range(steps):
            ev.rk3_step(0, dt, precision, BC_REFERENCE)
        ms, _n = ev.profile(KERNEL_STAGE)
        ev.set_profiling(False)
        points = sum(int(np.prod(b.ncells)) for b in blocks)
        return ms * 1e6 / (points * 3 * steps)
    finally:
        ev.close()


def tune(classes=None, configs=None, precisions=("fp64", "mixed"), steps: int = 3, fp64_chi: float = 0.5,
         device: int = 0, target_points: int = 1 << 21, margin: float = 0.01, log=None) -> dict:
    """Time every configuration for every class and precision; returns the
    table (per class the fastest configuration, or configuration 0 unless the
    fastest beats it by more than `margin`; classes not tuned keep None) and
    the timings in ns per point-stage."""
    classes = list(STAGE_CLASS_EDGES if classes is None else classes)
    configs = list(range(STAGE_CONFIGS) if configs is None else configs)
    table = {p: [None] * len(STAGE_CLASS_EDGES) for p in precisions}
    timings = {p: {} for p in precisions}
    for edge in classes:
        cls = STAGE_CLASS_EDGES.index(edge)
        assert block_stage_class((edge,) * 3) == cls
        blocks, dx = class_level(edge, target_points)
        for pname in precisions:
            row = {}
            for cfg in configs:
                t0 = time.perf_counter()
                row[cfg] = time_config(blocks, dx, PRECISIONS[pname], cfg, steps=steps, fp64_chi=fp64_chi,
                                       device=device)
                if log:
                    log(f"class {edge:3d} {pname:5s} cfg {cfg}: {row[cfg]:.4f} ns/point-stage "
                        f"({time.perf_counter() - t0:.1f} s)")
            timings[pname][str(edge)] = {str(k): v for k, v in row.items()}
            best = min(row, key=row.get)
            # configuration 0 unless another is faster by more than run-to-run noise
            if 0 in row and row[best] > (1.0 - margin) * row[0]:
                best = 0
            table[pname][cls] = best
    # one configuration per precision for every class: a level whose blocks use
    # different configurations runs one launch per configuration, and every
    # extra persistent launch adds a tail; the uniform choice minimises the sum
    # of the per-class times (configuration 0 unless beaten by the margin)
    uniform = {}
    for pname in precisions:
        rows = [timings[pname][str(e)] for e in classes]
        tot = {cfg: sum(r[str(cfg)] for r in rows) for cfg in configs}
        best = min(tot, key=tot.get)
        if 0 in tot and tot[best] > (1.0 - margin) * tot[0]:
            best = 0
        uniform[pname] = [best] * len(STAGE_CLASS_EDGES)
    return {"classes": list(STAGE_CLASS_EDGES), "table": table, "uniform_table": uniform,
            "timings_ns_per_point_stage": timings,
            "configs": {str(k): stage_config_info(k) for k in configs}, "steps": steps,
            "fp64_chi_threshold": fp64_chi, "target_points": target_points, "margin": margin}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", default=None, help="write the result (JSON) here")
    ap.add_argument("--classes", default=None, help="comma-separated class edges (default: all)")
    ap.add_argument("--configs", default=None, help="comma-separated configurations (default: all)")
    ap.add_argument("--precisions", default="fp64,mixed", help="comma-separated: fp64, mixed")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--fp64-chi", type=float, default=0.5)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    classes = [int(x) for x in args.classes.split(",")] if args.classes else None
    configs = [int(x) for x in args.configs.split(",")] if args.configs else None
    precisions = tuple(x for x in args.precisions.split(",") if x)
    res = tune(classes=classes, configs=configs, precisions=precisions, steps=args.steps, fp64_chi=args.fp64_chi,
               device=args.device, log=lambda m: print(m, file=sys.stderr, flush=True))
    try:
        import torch
        res["device_name"] = torch.cuda.get_device_name(args.device)
    except Exception:
        pass
    text = json.dumps(res, indent=1)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text + "\n")
    print(text)
    return 0


if __name__ == "__main__":
    sys.exit(main())
