"""Benchmark of the per-timestep flow solve on B200.

Workload: one 256 x 256 x 128 channel domain per GPU (periodic x and y,
no-slip bottom with the log-law wall model, free-slip top, Smagorinsky
Cs = 0.1, RK3, dt = 0.02) with the potential temperature (0.01 K/m gradient
and +-0.05 K perturbations, adiabatic walls, buoyancy): the single large
domain on which the FP64 and the mixed path are compared.  A "step" is one RK3 time step (three stages, each
with a full pressure projection) of that domain, inputs resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun every rank steps its own independent domain (weak scaling,
no collective on the data path); the value is the total over ranks divided
by the slowest rank's time.  `--impl reference` times the CPU restatement of
the reference (the oracle, C++ FP64 with OpenMP on all host threads), since
the Fortran reference itself cannot be built here.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from gpu_elmm_b200.config import grid_of, make_config  # noqa: E402
from gpu_elmm_b200.config import FIELD_TEMPERATURE  # noqa: E402
from gpu_elmm_b200.workloads import interior, interiors, log_profile_state, temperature_state  # noqa: E402

METRIC = "cell-steps/s mixed vs FP64 plain, 1 B200, at ≤1e-5 rel err; p50/p99 latency"
N = (256, 256, 128)
WORKLOAD = ("256x256x128 channel: periodic x,y; no-slip bottom with log-law wall model (z0=0.01); "
            "free-slip top; Smagorinsky Cs=0.1; CDS2; RK3 dt=0.02; FFT(x,y)+tridiagonal(z) projection; "
            "potential temperature (KappaScalar advection, SGS diffusion Pr_sgs=0.6, adiabatic walls) with buoyancy")
DATA = ("synthetic: seeded log profile u*=0.3 + U(-0.1,0.1) perturbations on u,v,w; theta = 295 K + 0.01 K/m z "
        "+ U(-0.05,0.05) K; FP32-rounded, projected")
# words moved per cell by the momentum kernel in stages 2 and 3: reads U,V,W,nu,Pr,theta,Ustar x3;
# writes Ustar x3, U2 x3 (the per-cell figure of the momentum phase)
MOMENTUM_WORDS = 15
# timed oracle steps of the main line's cpu_baseline (a bounded sample: ~10 s on 16 cores)
CPU_STEPS = 5
# seconds of timed oracle steps in the reference arm (--impl reference)
REF_BUDGET_S = 120.0
# long run of the single domain on both paths (errors after 1, 10 and this many steps)
LONG_STEPS = 1000
# the array of cubes: steps run on both paths (device time over steps 10..CUBES_STEPS)
CUBES_STEPS = 100
# batched ensemble: domains per GPU and the axis lengths they draw from
BATCH_DOMAINS = 64
BATCH_AXES = (32, 48, 64, 96, 128)
# serving loop: requests per GPU at each arrival rate (per GPU), HBM budget
SERVE_REQUESTS = 16
SERVE_RATES = (5.0, 200.0)
SERVE_BUDGET = 40 << 30


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend=backend, timeout=timedelta(seconds=120))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def allreduce_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            os.unlink(self.path)
        except OSError:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        busy = [x for x in sm if x > 0.5 * (mx or max(sm))] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def rel(a, b):
    s = float(np.abs(b).max())
    return float(np.abs(a - b).max()) / (s if s > 0 else 1.0)


def _native_oracle():
    """The oracle built with -O3 -march=native -fopenmp on this host (the
    timed CPU baseline; the parity build of the tests keeps FMA contraction
    off), with every host thread."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    orc.build(native=True)
    threads = os.cpu_count() or 1
    orc.set_threads(threads, native=True)
    cfg = make_config(*N, buoyancy=True)
    g = grid_of(cfg)
    o = orc.Oracle(cfg, native=True)
    o.set_state(*log_profile_state(g, seed=0))
    o.set_field(FIELD_TEMPERATURE, temperature_state(g, seed=0))
    o.project(1.0)
    return o, g, threads


def cpu_baseline(steps=CPU_STEPS):
    """The FP64 oracle on all host threads, a bounded sample of the workload:
    one untimed step, then `steps` timed RK3 steps of the full domain."""
    o, g, threads = _native_oracle()
    o.step(1)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    return {"value": g.cells() * steps / dt, "unit": "cell-steps/s", "cores": threads, "kind": "port",
            "sample": f"{steps} RK3 steps of the 256x256x128 workload in FP64 after 1 untimed step "
                      f"(oracle/elmm_oracle.cpp built -O3 -march=native -fopenmp, {threads} threads)",
            "seconds": dt}


def run_reference(args, ws, rank):
    """The CPU restatement of the reference on this host's cores (the Fortran
    reference cannot be built here): W untimed RK3 steps of the full
    256x256x128 domain, then K timed ones, on rank 0 only.  A full step takes
    about 2 s on 16 cores, so the timed steps stop at REF_BUDGET_S seconds
    (estimated from the warm-up steps); the line reports the steps it timed
    ("steps") beside the ones asked for ("steps_requested")."""
    if rank != 0:
        return 0
    o, g, threads = _native_oracle()
    t0 = time.perf_counter()
    o.step(max(1, args.warmup))
    per_step = (time.perf_counter() - t0) / max(1, args.warmup)
    steps = max(1, min(args.steps, int(REF_BUDGET_S / per_step)))
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    v = g.cells() * steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell-steps/s", "n_gpus": args.gpus,
            "steps": steps, "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": dt / steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": DATA, "config": {"workload": WORKLOAD, "cells": g.cells(), "precision": "fp64"},
            "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": threads, "kind": "port",
                             "sample": f"{steps} RK3 steps of the 256x256x128 workload after {args.warmup} "
                                       f"untimed steps (the Fortran reference cannot be built here; its C++ FP64 "
                                       f"restatement in oracle/, built -O3 -march=native -fopenmp, is timed)"},
            "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, ws, rank, local):
    import torch
    from gpu_elmm_b200 import lib as L
    torch.cuda.set_device(local)
    g = grid_of(make_config(*N))
    st = log_profile_state(g, seed=rank)
    T0 = temperature_state(g, seed=rank)
    cells = g.cells()

    def domain(precision, state, temp):
        dd = L.Domain(make_config(*N, precision=precision, device=local, buoyancy=True))
        dd.upload(*state)
        dd.upload_temperature(temp)
        return dd

    # FP64 plain path on the same state
    d64 = domain(0, st, T0)
    d64.project(1.0)
    d64.step(args.warmup)
    barrier(ws)
    torch.cuda.synchronize()
    s64 = d64.step(args.steps)
    torch.cuda.synchronize()
    barrier(ws)
    ms64 = allreduce_max(s64.elapsed_ms, ws)

    # accuracy of the mixed path against FP64 after one step from the same state
    a64 = domain(0, st, T0)
    a64.project(1.0)
    ref0 = a64.download()
    a64.step(1)
    ref1 = a64.download()
    refT = a64.field(FIELD_TEMPERATURE)
    a64.close()
    d64.close()
    am = domain(1, ref0, T0)
    am.step(1)
    mix1 = am.download()
    mixT = am.field(FIELD_TEMPERATURE)
    am.close()
    errs = [rel(a, b) for a, b in zip(interiors(g, *mix1), interiors(g, *ref1))]
    nT = (g.Prnx, g.Prny, g.Prnz)
    errs.append(rel(interior(mixT, -2, nT) - 295.0, interior(refT, -2, nT) - 295.0))

    # the mixed path: headline
    dm = domain(1, st, T0)
    dm.project(1.0)
    dm.step(args.warmup)
    with Clocks(local) as clk:
        barrier(ws)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        torch.cuda.nvtx.range_push("timed_mixed")  # lets `ncu --nvtx-include timed_mixed/` select these launches
        sm = dm.step(args.steps)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
        barrier(ws)
    msm = allreduce_max(sm.elapsed_ms, ws)
    total_cells = allreduce_sum(float(cells), ws)
    value = total_cells * args.steps / (msm / 1e3)
    v64 = total_cells * args.steps / (ms64 / 1e3)
    max_div = allreduce_max(sm.max_div, ws)

    # per-step latency distribution (device time of single-step calls)
    lat = []
    for _ in range(min(args.steps, 50)):
        lat.append(dm.step(1).elapsed_ms)
    lat.sort()
    p50 = lat[len(lat) // 2]
    p99 = lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))]

    # roofline of the dominant kernel, timed live with CUDA events on the library's stream
    kt = dm.profile_stage(stage=2, reps=5)
    tiles = dm.tuning()
    mom_ms = kt["momentum"]
    alg_bytes = MOMENTUM_WORDS * 4 * cells
    peak, peak_kind = peaks()
    achieved = alg_bytes / (mom_ms / 1e3) / 1e9
    # DRAM bytes of one launch are not measurable inside a timed run; they
    # come from the committed ncu capture of this kernel on this workload
    traffic, traffic_source = None, None
    tp = os.path.join(ROOT, "profiles", "k_momentum_256x256x128_mixed.md")
    if os.path.exists(tp):
        for line in open(tp):
            if line.startswith("dram_bytes_per_launch:"):
                traffic = float(line.split(":")[1])
                traffic_source = ("stored ncu capture (dram__bytes_read.sum + dram__bytes_write.sum of one launch), "
                                  "profiles/k_momentum_256x256x128_mixed.md")

    # end to end through the C-ABI with pinned host buffers: one
    # elmm_march_host call per step (H2D of the state and temperature, one
    # step, D2H of both).  The headline takes the host arrays of the
    # reference's default build (prec=sp: real32, elmm_march_host_float);
    # e2e_fp64_host the double arrays of a prec=dp build.
    def e2e_leg(dtype, march):
        pinned = [torch.empty(a.shape, dtype=dtype, pin_memory=True).numpy() for a in st]
        for p, a in zip(pinned, dm.download()):
            p[...] = a
        pinT = torch.empty(T0.shape, dtype=dtype, pin_memory=True).numpy()
        pinT[...] = dm.field(FIELD_TEMPERATURE)
        nbytes = sum(a.nbytes for a in pinned) + pinT.nbytes
        times = []
        for _ in range(max(3, min(args.steps // 2, 40))):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            march(*pinned, pinT, n=1)  # TMarchRK3 on the host arrays
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        return total_cells / allreduce_max(statistics.median(times), ws), nbytes
    e2e64, h2d64 = e2e_leg(torch.float64, dm.march_host)
    e2e, h2d = e2e_leg(torch.float32, dm.march_host_f32)

    dm.close()
    long_run = long_run_leg(st, T0, local) if rank == 0 else None
    cubes = cubes_leg(local) if rank == 0 else None
    slabs = slabs_leg(local) if rank == 0 else None
    config0 = config0_leg(local) if rank == 0 and ws == 1 else None
    batched = batched_leg(args, ws, rank, local)
    serving = serving_leg(args, ws, rank, local)

    cpu = cpu_baseline() if (rank == 0 and ws == 1) else None
    barrier(ws)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": msm / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (FP64 reductions, zero mode, tridiagonal)", "data": DATA,
            "config": {"workload": WORKLOAD, "cells_per_gpu": cells, "precision": "mixed",
                       "l2": "inputs larger than L2 (mixed state ~0.5 GB per GPU)",
                       "parallelism": "one independent domain per GPU" if ws > 1 else "single domain"},
            "fp64_plain": {"value": v64, "unit": "cell-steps/s", "ms_per_step": ms64 / args.steps},
            "mixed_over_fp64": value / v64,
            "accuracy_vs_fp64_1step": {"u": errs[0], "v": errs[1], "w": errs[2], "p": errs[3],
                                       "theta_minus_ref": errs[4], "max_div_mixed": max_div},
            "latency_ms": {"p50": p50, "p99": p99, "what": "device time of one RK3 step"},
            "roofline": {"bound": "hbm", "kernel": "k_momentum (stage 2)", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "traffic_source": traffic_source, "algorithmic_bytes": alg_bytes,
                         "ms": mom_ms},
            "kernel_ms_stage2": kt,
            "autotuned_tiles": tiles,
            "e2e": {"value": e2e, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
                    "host_arrays": "real32 (the reference's default prec=sp build), elmm_march_host_float"},
            "e2e_fp64_host": {"value": e2e64, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d64,
                              "d2h_bytes_per_step": h2d64, "host_arrays": "real64, elmm_march_host"},
            "gpu_launches": sm.kernels,
            "clocks": clk.summary(),
            "wall_s_timed": wall,
            "long_run": long_run,
            "cubes": cubes,
            "slabs": slabs,
            "config0": config0,
            "batched": batched,
            "serving": serving,
        }
        if cpu:
            line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        print(json.dumps(line), flush=True)
    return 0


def long_run_leg(st, T0, local):
    """Config 1 on both paths from one projected state for LONG_STEPS steps:
    the relative error of the mixed path after 1, 10 and LONG_STEPS steps,
    and the vertical profiles of mean velocity, resolved TKE and theta
    averaged over the second half of the run (src/vertical_profiles.f90)."""
    from gpu_elmm_b200 import lib as L
    from gpu_elmm_b200.stats import Profiles, compare
    g = grid_of(make_config(*N))
    doms = {}
    for prec in (0, 1):
        doms[prec] = L.Domain(make_config(*N, precision=prec, device=local, buoyancy=True))
    doms[0].upload(*st)
    doms[0].upload_temperature(T0)
    doms[0].project(1.0)
    doms[1].upload(*doms[0].download())
    doms[1].upload_temperature(T0)
    prof = {0: Profiles(g), 1: Profiles(g)}
    errs = {}
    nT = (g.Prnx, g.Prny, g.Prnz)
    done = 0
    marks = sorted({1, 10, LONG_STEPS} | set(range(LONG_STEPS // 2, LONG_STEPS + 1, LONG_STEPS // 20)))
    for target in marks:
        for p in (0, 1):
            doms[p].step(target - done)
        done = target
        s = {p: doms[p].download() for p in (0, 1)}
        T = {p: doms[p].field(FIELD_TEMPERATURE) for p in (0, 1)}
        if target in (1, 10, LONG_STEPS):
            e = [rel(a, b) for a, b in zip(interiors(g, *s[1]), interiors(g, *s[0]))]
            e.append(rel(interior(T[1], -2, nT) - 295.0, interior(T[0], -2, nT) - 295.0))
            errs[str(target)] = dict(zip(("u", "v", "w", "p", "theta_minus_ref"), e))
        if target >= LONG_STEPS // 2:
            for p in (0, 1):
                prof[p].add(*s[p][:3], T[p])
    for p in (0, 1):
        doms[p].close()
    return {"steps": LONG_STEPS, "rel_err_mixed_vs_fp64": errs,
            "profiles_rel_diff": compare(prof[1].result(), prof[0].result(), keys=("u", "tke", "theta")),
            "profiles_window": f"steps {LONG_STEPS // 2}..{LONG_STEPS}, every {LONG_STEPS // 20}"}


def config0_leg(local, steps=100, cpu_steps=20):
    """Config 0, the 64x64x32 channel for its 100 steps: mixed and FP64
    device throughput from one projected state, the mixed error against FP64
    after the 100 steps, and the FP64 oracle (native build, every host
    thread) timed over cpu_steps steps from the same state, with the GPU's
    FP64 state compared with the oracle's after those steps."""
    from gpu_elmm_b200 import lib as L
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    orc.build(native=True)
    threads = orc.set_threads(os.cpu_count() or 1, native=True)
    n = (64, 64, 32)
    g = grid_of(make_config(*n))
    o = orc.Oracle(make_config(*n), native=True)
    o.set_state(*log_profile_state(g, seed=0))
    o.project(1.0)
    st = o.state()
    out = {"workload": "64x64x32 channel, config-0 physics (no temperature), 100 steps", "cells": g.cells()}
    doms = {p: L.Domain(make_config(*n, precision=p, device=local)) for p in (0, 1)}
    for p, d in doms.items():
        d.upload(*st)
    t0 = time.perf_counter()
    o.step(cpu_steps)
    cpu_s = time.perf_counter() - t0
    doms[0].step(cpu_steps)
    out["fp64_vs_oracle_after_%d" % cpu_steps] = [rel(a, b) for a, b in zip(interiors(g, *doms[0].download()),
                                                                           interiors(g, *o.state()))]
    doms[0].upload(*st)
    for p, name in ((1, "mixed"), (0, "fp64")):
        s_ = doms[p].step(steps)
        out[name] = {"cell_steps_per_s": g.cells() * steps / (s_.elapsed_ms / 1e3), "ms_per_step": s_.elapsed_ms / steps}
    out["mixed_over_fp64"] = out["mixed"]["cell_steps_per_s"] / out["fp64"]["cell_steps_per_s"]
    out["rel_err_mixed_vs_fp64_after_%d" % steps] = [rel(a, b) for a, b in zip(interiors(g, *doms[1].download()),
                                                                               interiors(g, *doms[0].download()))]
    out["cpu_oracle"] = {"cell_steps_per_s": g.cells() * cpu_steps / cpu_s, "steps": cpu_steps, "threads": threads,
                         "build": "oracle/elmm_oracle.cpp, -O3 -march=native -fopenmp (FMA contraction on)"}
    for d in doms.values():
        d.close()
    return out


def slabs_leg(local, steps=20):
    """One domain split into z-slabs (elmm_slabs_*), every slab on this GPU:
    the 256x256x128 channel with the temperature (the headline workload),
    mixed, its device time per step against the single-domain handle on the
    same state, and whether the two states (flow and temperature) agree bit
    for bit after the timed steps.  On one GPU this measures the cost of the
    split (the exchanges, the split z solve, smaller launches), not a
    speed-up."""
    from gpu_elmm_b200 import lib as L
    cfg = make_config(*N, precision=1, buoyancy=True)
    g = grid_of(cfg)
    st = log_profile_state(g, seed=0)
    T0 = temperature_state(g, seed=0)
    out = {"workload": "256x256x128 channel with temperature, mixed, every slab on one GPU", "steps": steps}
    a = L.Domain(make_config(*N, precision=1, buoyancy=True, device=local))
    a.upload(*st)
    a.upload_temperature(T0)
    a.project(1.0)
    a.step(3)
    out["single_ms_per_step"] = a.step(steps).elapsed_ms / steps
    ref = a.download() + (a.field(FIELD_TEMPERATURE),)
    a.close()
    for ns in (2, 4):
        b = L.Slabs(cfg, ns, devices=[local] * ns)
        b.upload(*st)
        b.upload_temperature(T0)
        b.project(1.0)
        b.step(3)
        s = b.step(steps)
        out[f"slabs{ns}_ms_per_step"] = s.elapsed_ms / steps
        out[f"slabs{ns}_kernels_per_step"] = s.kernels / steps
        got = b.download() + (b.field(FIELD_TEMPERATURE),)
        out[f"slabs{ns}_bit_equal_to_single"] = all(bool(np.array_equal(x, y)) for x, y in zip(got, ref))
        b.close()
    return out


def cubes_leg(local):
    """The array of cubes (384x384x96, stretched z, 8x8 cubes, mean pressure
    gradient): device time per step of both paths over CUBES_TIMED steps,
    the mixed path's error against FP64 after 1, 10 and CUBES_STEPS steps from
    one projected state, the divergence check of each, and the mean profiles
    of the second half of the run."""
    from gpu_elmm_b200 import lib as L
    from gpu_elmm_b200.solids import build_solids
    from gpu_elmm_b200.stats import Profiles, compare
    from gpu_elmm_b200.workloads import CUBES_N, cubes_boxes, cubes_config, stretched_zw
    cfgs = {p: cubes_config(precision=p, device=local) for p in (0, 1)}
    g = grid_of(cfgs[0])
    t0 = time.perf_counter()
    sol = build_solids(cfgs[0], cubes_boxes())
    t_geo = time.perf_counter() - t0
    st = log_profile_state(g, seed=0, zW=stretched_zw(CUBES_N[2]))
    doms = {p: L.Domain(cfgs[p]) for p in (0, 1)}
    doms[0].upload(*st)
    doms[0].project(1.0)
    doms[1].upload(*doms[0].download())
    for p in (0, 1):
        doms[p].set_solids(sol)
    prof = {0: Profiles(g), 1: Profiles(g)}
    errs, ms, div = {}, {0: [], 1: []}, {}
    done = 0
    marks = sorted({1, 10, CUBES_STEPS} | set(range(CUBES_STEPS // 2, CUBES_STEPS + 1, CUBES_STEPS // 10)))
    for target in marks:
        for p in (0, 1):
            s = doms[p].step(target - done)
            if done >= 10:
                ms[p].append((s.elapsed_ms, target - done))
            div[p] = s.max_div
        done = target
        sd = {p: doms[p].download() for p in (0, 1)}
        if target in (1, 10, CUBES_STEPS):
            e = [rel(a, b) for a, b in zip(interiors(g, *sd[1]), interiors(g, *sd[0]))]
            errs[str(target)] = dict(zip(("u", "v", "w", "p"), e))
        if target >= CUBES_STEPS // 2:
            for p in (0, 1):
                prof[p].add(*sd[p][:3])
    for p in (0, 1):
        doms[p].close()
    cells = g.Prnx * g.Prny * g.Prnz
    per = {p: sum(a for a, _ in ms[p]) / max(1, sum(b for _, b in ms[p])) for p in (0, 1)}
    return {"workload": f"{CUBES_N[0]}x{CUBES_N[1]}x{CUBES_N[2]} stretched z (dz_k = 0.5*1.04^(k-1)), 8x8 cubes of "
                        "16 cells at a 48-cell pitch (z0 = 0.1), mean pressure gradient in x",
            "cells": cells, "points": sol.counts(), "geometry_pass_s": t_geo,
            "mixed": {"cell_steps_per_s": cells / (per[1] / 1e3), "ms_per_step": per[1]},
            "fp64": {"cell_steps_per_s": cells / (per[0] / 1e3), "ms_per_step": per[0]},
            "mixed_over_fp64": per[0] / per[1],
            "timed_steps": sum(b for _, b in ms[1]),
            "rel_err_mixed_vs_fp64": errs, "max_div": {"mixed": div[1], "fp64": div[0]},
            "profiles_rel_diff": compare(prof[1].result(), prof[0].result(), keys=("u", "tke")),
            "profiles_window": f"steps {CUBES_STEPS // 2}..{CUBES_STEPS}, every {CUBES_STEPS // 10}"}


def gather(x, ws):
    """Every rank's x, on every rank."""
    if ws == 1:
        return [x]
    import torch.distributed as dist
    out = [None] * ws
    dist.all_gather_object(out, x)
    return out


def batched_leg(args, ws, rank, local):
    """The batched ensemble: BATCH_DOMAINS channel domains per GPU, each axis
    drawn from BATCH_AXES (seed 0), config-0 physics with each domain's own
    seed and log-profile u* in [0.2, 0.5], all stepped by one launch set and
    one CUDA graph per step; mixed and FP64, device time, max over ranks."""
    from gpu_elmm_b200 import lib as L
    from gpu_elmm_b200.workloads import uniform
    r = uniform(0, "sizes", 3 * BATCH_DOMAINS)
    sizes = [tuple(BATCH_AXES[int(r[3 * q + a] * len(BATCH_AXES))] for a in range(3)) for q in range(BATCH_DOMAINS)]
    ustar = 0.2 + 0.3 * uniform(0, "ustar", BATCH_DOMAINS)
    out = {}
    steps = max(3, min(args.steps, 20))
    for prec, name in ((1, "mixed"), (0, "fp64")):
        cfgs = [make_config(*n, precision=prec, device=local) for n in sizes]
        b = L.Batch(cfgs)
        for q, n in enumerate(sizes):
            b.upload(q, *log_profile_state(grid_of(cfgs[q]), seed=1000 * rank + q + 1, ustar=float(ustar[q])))
        b.project(1.0)
        b.step(args.warmup)
        barrier(ws)
        st = b.step(steps)
        ms = allreduce_max(st.elapsed_ms, ws)
        cells = allreduce_sum(float(b.cells()), ws)
        out[name] = {"value": cells * steps / (ms / 1e3), "unit": "cell-steps/s", "ms_per_step": ms / steps,
                     "max_div": allreduce_max(st.max_div, ws), "kernels_per_step": st.kernels / steps,
                     "autotuned_tiles": b.tuning()}
        b.close()
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["config"] = {"domains_per_gpu": BATCH_DOMAINS, "axes_from": BATCH_AXES,
                     "cells_per_gpu": int(sum(a * b * c for a, b, c in sizes)), "steps": steps,
                     "physics": "config-0 channel, u* ~ U[0.2, 0.5] per domain, seed per domain"}
    return out


def serving_shard(n, ws, rank):
    """The requests a rank serves: every ws-th of the stream, from its rank."""
    return list(range(rank, n, ws))


def serving_leg(args, ws, rank, local):
    """The serving loop under Poisson arrivals of dispersion requests (64^3 ..
    192x192x96 cells, 200..2000 steps, a passive scalar with a point source and
    a Gaussian puff).  Each rank serves every ws-th request on its own GPU;
    latency is arrival to slices on the host, p50 / p99 over all requests."""
    from gpu_elmm_b200.serve import Server, percentile, request_inputs, run_arrivals
    from gpu_elmm_b200.workloads import dispersion_request, poisson_arrivals
    reqs_all = [dispersion_request(0, q) for q in range(SERVE_REQUESTS * ws)]
    out = []
    for rate in SERVE_RATES:
        arr_all = poisson_arrivals(0, rate * ws, len(reqs_all))
        mine = serving_shard(len(reqs_all), ws, rank)
        reqs = [reqs_all[q] for q in mine]
        inputs = [request_inputs(q) for q in reqs]
        srv = Server(precision=1, budget_bytes=SERVE_BUDGET, max_active=64, chunk_steps=50, device=local)
        barrier(ws)
        done, span = run_arrivals(srv, reqs, arr_all[mine], inputs)
        st = srv.stats()
        srv.close()
        lat = [i.t_done - i.t_submit for _, i, _ in done]
        cs = float(sum(i.cells * i.steps for _, i, _ in done))
        lats = [x for part in gather(lat, ws) for x in part]
        out.append({"rate_per_s": rate * ws, "requests": len(reqs_all),
                    "p50_latency_s": percentile(lats, 50), "p99_latency_s": percentile(lats, 99),
                    "cell_steps_per_s": allreduce_sum(cs, ws) / allreduce_max(span, ws),
                    "peak_active": int(allreduce_max(float(st.peak_active), ws)),
                    "graph_builds": int(allreduce_sum(float(st.graph_builds), ws)),
                    "busy_frac": allreduce_sum(st.busy_s, ws) / (ws * allreduce_max(span, ws))})
    return {"points": out, "precision": "mixed", "budget_gb_per_gpu": SERVE_BUDGET / 2 ** 30,
            "latency": "Poisson arrival to time-averaged slices on the host (wall clock of the serving loop)",
            "workload": "dispersion requests: s x s x nz, s in {64,96,128,192}, nz in {64,96}, 200..2000 steps, "
                        "passive scalar with a continuous point source and a sigma=2 Gaussian puff"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    ws, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            rc = run_reference(args, ws, rank)
        else:
            rc = run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
