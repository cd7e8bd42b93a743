"""Runs the benchmark workload for a profiler: one channel domain (by default
256 x 256 x 128 with the potential temperature, the same configuration and
seeded state as bench.py), the initial projection, W warm-up steps and S
profiled steps, then prints the device time of the steps and the per-kernel
times of one stage.

    python -m gpu_elmm_b200.profile_step [--precision mixed|fp64] [--n 256,256,128]
                                         [--warmup 1] [--steps 1] [--no-temperature]
                                         [--batched 64]

--batched D runs the batched ensemble instead: D channel domains, each axis
drawn from 32, 48, 64, 96, 128 (seed 0), one launch set for all of them.

--slabs S splits the channel (without the temperature, which split domains
do not carry) into S even z-slabs, all on GPU 0 (elmm_slabs_*).

Under `ncu -k regex:<kernel> -s <skip> -c <count>` the launches of the
profiled steps follow those of the projection and the warm-up steps; the
NVTX range "timed_steps" brackets the profiled steps.
"""
import argparse
import json

from .config import grid_of, make_config
from .workloads import log_profile_state, temperature_state
from . import lib as L


def nvtx_push(name):
    try:
        import torch
        torch.cuda.nvtx.range_push(name)
    except Exception:
        pass


def nvtx_pop():
    try:
        import torch
        torch.cuda.nvtx.range_pop()
    except Exception:
        pass


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--n", default="256,256,128")
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--stage-times", action="store_true", help="also time each kernel of stage 2 (5 repetitions)")
    ap.add_argument("--no-temperature", action="store_true", help="the channel without the temperature field")
    ap.add_argument("--batched", type=int, default=0, help="run the batched ensemble of this many domains")
    ap.add_argument("--cubes", action="store_true", help="run the array of cubes (384x384x96, stretched z)")
    ap.add_argument("--slabs", type=int, default=0, help="split the channel into this many z-slabs on GPU 0")
    a = ap.parse_args()
    if a.batched:
        return batched(a)
    if a.slabs:
        return slabs(a)
    if a.cubes:
        return cubes(a)
    n = tuple(int(x) for x in a.n.split(","))
    buoy = not a.no_temperature
    cfg = make_config(*n, precision=1 if a.precision == "mixed" else 0, buoyancy=buoy)
    g = grid_of(cfg)
    d = L.Domain(cfg)
    d.upload(*log_profile_state(g, seed=0))
    if buoy:
        d.upload_temperature(temperature_state(g, seed=0))
    d.project(1.0)
    if a.warmup:
        d.step(a.warmup)
    nvtx_push("timed_steps")  # `ncu --nvtx --nvtx-include "timed_steps/"` selects these launches
    s = d.step(a.steps)
    nvtx_pop()
    out = {"n": n, "precision": a.precision, "steps": a.steps, "ms_per_step": s.elapsed_ms / max(1, a.steps),
           "max_div": s.max_div, "kernels_per_step": s.kernels / max(1, a.steps)}
    if a.stage_times:
        out["stage2_kernel_ms"] = d.profile_stage(2, 5)
    print(json.dumps(out))
    d.close()


def slabs(a):
    n = tuple(int(x) for x in a.n.split(","))
    cfg = make_config(*n, precision=1 if a.precision == "mixed" else 0)
    b = L.Slabs(cfg, a.slabs, devices=[0] * a.slabs)
    b.upload(*log_profile_state(grid_of(cfg), seed=0))
    b.project(1.0)
    if a.warmup:
        b.step(a.warmup)
    nvtx_push("timed_steps")
    s = b.step(a.steps)
    nvtx_pop()
    print(json.dumps({"n": n, "slabs": a.slabs, "precision": a.precision, "steps": a.steps,
                      "ms_per_step": s.elapsed_ms / max(1, a.steps), "max_div": s.max_div,
                      "kernels_per_step": s.kernels / max(1, a.steps)}))
    b.close()


def cubes(a):
    from .solids import build_solids
    from .workloads import CUBES_N, cubes_boxes, cubes_config, stretched_zw
    cfg = cubes_config(precision=1 if a.precision == "mixed" else 0)
    g = grid_of(cfg)
    sol = build_solids(cfg, cubes_boxes())
    d = L.Domain(cfg)
    d.upload(*log_profile_state(g, seed=0, zW=stretched_zw(CUBES_N[2])))
    d.project(1.0)
    d.set_solids(sol)
    if a.warmup:
        d.step(a.warmup)
    nvtx_push("timed_steps")
    s = d.step(a.steps)
    nvtx_pop()
    out = {"n": CUBES_N, "precision": a.precision, "steps": a.steps, "ms_per_step": s.elapsed_ms / max(1, a.steps),
           "max_div": s.max_div, "kernels_per_step": s.kernels / max(1, a.steps), "points": sol.counts()}
    if a.stage_times:
        out["stage2_kernel_ms"] = d.profile_stage(2, 5)
    print(json.dumps(out))
    d.close()


def batched(a):
    from .workloads import uniform
    axes = (32, 48, 64, 96, 128)
    r = uniform(0, "sizes", 3 * a.batched)
    sizes = [tuple(axes[int(r[3 * q + k] * len(axes))] for k in range(3)) for q in range(a.batched)]
    ustar = 0.2 + 0.3 * uniform(0, "ustar", a.batched)
    cfgs = [make_config(*n, precision=1 if a.precision == "mixed" else 0) for n in sizes]
    b = L.Batch(cfgs)
    for q in range(a.batched):
        b.upload(q, *log_profile_state(grid_of(cfgs[q]), seed=q + 1, ustar=float(ustar[q])))
    b.project(1.0)
    if a.warmup:
        b.step(a.warmup)
    s = b.step(a.steps)
    out = {"domains": a.batched, "cells": b.cells(), "precision": a.precision, "steps": a.steps,
           "ms_per_step": s.elapsed_ms / max(1, a.steps), "kernels_per_step": s.kernels / max(1, a.steps),
           "tuning": b.tuning()}
    if a.stage_times:
        out["stage2_kernel_ms"] = b.profile_stage(2, 5)
    print(json.dumps(out))
    b.close()


if __name__ == "__main__":
    main()
