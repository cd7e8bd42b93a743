"""The serving loop (``elmm_server_*`` of include/elmm_gpu.h) and the
dispersion workload that drives it.

A request is one dispersion run: a periodic channel of s x s x nz cells with
the channel physics of the small configuration, a passive scalar released by a
continuous point source at an interior cell, an initial Gaussian puff
(sigma = 2 cells) centred there, and a number of steps; its result is the
time-averaged concentration on the horizontal and the vertical plane through
the source.  Requests arrive as a Poisson process; the library admits them as
memory and slots free up and steps all admitted requests together.

    python -m gpu_elmm_b200.serve [--rates 1,5,50,200] [--requests 24]
                                  [--precision mixed|fp64] [--budget-gb 40]

prints one JSON line per arrival rate: p50 / p99 latency (arrival to result on
the host), throughput in cell-steps/s, and the loop's own counters.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import threading
import time

import numpy as np

from .config import ElmmConfig, grid_of, make_config
from . import lib as L
from .workloads import dispersion_request, log_profile_state, poisson_arrivals, puff_state


class ServerConfig(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("precision", C.c_int32),
        ("hbm_budget_bytes", C.c_int64),
        ("max_active", C.c_int32),
        ("chunk_steps", C.c_int32),
        ("policy", C.c_int32),
        ("reserved", C.c_int32),
    ]


SERVE_FIFO, SERVE_SHORTEST_FIRST = 0, 1


class RequestInfo(C.Structure):
    _fields_ = [
        ("id", C.c_int64),
        ("status", C.c_int32),
        ("steps", C.c_int32),
        ("t_submit", C.c_double),
        ("t_admit", C.c_double),
        ("t_done", C.c_double),
        ("bytes", C.c_int64),
        ("max_div", C.c_double),
        ("cells", C.c_int64),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64), ("admitted", C.c_int64), ("finished", C.c_int64), ("failed", C.c_int64),
        ("cell_steps", C.c_int64),
        ("chunks", C.c_int64), ("graph_builds", C.c_int64),
        ("active", C.c_int32), ("queued", C.c_int32), ("peak_active", C.c_int32),
        ("reserved", C.c_int32),
        ("bytes_in_use", C.c_int64), ("bytes_peak", C.c_int64), ("budget_bytes", C.c_int64),
        ("busy_s", C.c_double),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "reserved"}


_bound = False


def _bind():
    global _bound
    lib = L.lib()
    if not _bound:
        P, dp = C.c_void_p, C.POINTER(C.c_double)
        lib.elmm_server_create.argtypes = [C.POINTER(ServerConfig), C.POINTER(P)]
        lib.elmm_server_destroy.argtypes = [P]
        lib.elmm_server_submit.argtypes = [P, C.POINTER(ElmmConfig), dp, dp, dp, dp, dp, C.c_int32,
                                           C.POINTER(C.c_int64)]
        lib.elmm_server_wait_any.argtypes = [P, C.c_int32, C.POINTER(RequestInfo)]
        lib.elmm_server_collect.argtypes = [P, C.c_int64, dp, dp]
        lib.elmm_server_stats_get.argtypes = [P, C.POINTER(ServerStats)]
        lib.elmm_server_now.argtypes = [P]
        lib.elmm_server_now.restype = C.c_double
        _bound = True
    return lib


class Server:
    """One serving loop on one device.  The input arrays of a request are
    kept referenced here until the request has been reported."""

    def __init__(self, *, precision=1, budget_bytes=8 << 30, max_active=64, chunk_steps=50, device=0,
                 policy=SERVE_FIFO):
        lib = _bind()
        c = ServerConfig(device, precision, int(budget_bytes), max_active, chunk_steps, policy, 0)
        h = C.c_void_p()
        L.check(lib.elmm_server_create(C.byref(c), C.byref(h)), "elmm_server_create")
        self.h = h
        self.precision = precision
        self.device = device
        self._inputs = {}
        self._cfgs = {}

    def close(self):
        if getattr(self, "h", None):
            _bind().elmm_server_destroy(self.h)
            self.h = None
            self._inputs.clear()

    __del__ = close

    def submit(self, cfg: ElmmConfig, U, V, W, Pr=None, S0=None, nsteps=1) -> int:
        rid = C.c_int64()
        L.check(_bind().elmm_server_submit(self.h, C.byref(cfg), L.ptr(U), L.ptr(V), L.ptr(W), L.ptr(Pr),
                                           L.ptr(S0), nsteps, C.byref(rid)), "elmm_server_submit")
        self._inputs[rid.value] = (cfg, U, V, W, Pr, S0)
        self._cfgs[rid.value] = cfg
        return rid.value

    def wait_any(self, timeout_ms=1000):
        """The next finished request (RequestInfo), or None after timeout_ms."""
        info = RequestInfo()
        r = _bind().elmm_server_wait_any(self.h, timeout_ms, C.byref(info))
        if r == 5:  # ELMM_ERR_TIMEOUT
            return None
        L.check(r, "elmm_server_wait_any")
        self._inputs.pop(info.id, None)
        return info

    def collect(self, rid: int):
        """Time-averaged slices (xy, xz) of scalar 1 of a reported request."""
        cfg = self._cfgs.pop(rid)
        g = grid_of(cfg)
        xy = np.zeros((g.Prny, g.Prnx)) if cfg.avg_slice_k > 0 else None
        xz = np.zeros((g.Prnz, g.Prnx)) if cfg.avg_slice_j > 0 else None
        L.check(_bind().elmm_server_collect(self.h, rid, L.ptr(xy), L.ptr(xz)), "elmm_server_collect")
        return xy, xz

    def stats(self) -> ServerStats:
        s = ServerStats()
        L.check(_bind().elmm_server_stats_get(self.h, C.byref(s)), "elmm_server_stats_get")
        return s

    def now(self) -> float:
        return _bind().elmm_server_now(self.h)


# ---------------------------------------------------------------- workload
def request_config(req: dict, *, precision=1, device=0, flux=1.0) -> ElmmConfig:
    """The configuration of a dispersion request: channel physics of the
    small configuration, one passive scalar with its point source at the
    centre of cell req["source"], slices through the source, and the
    averaging weight dt / (steps * dt) of a window that spans the run."""
    n, (i, j, k), steps = req["n"], req["source"], req["steps"]
    return make_config(*n, precision=precision, device=device, num_scalars=1,
                       point_sources=[(1, (i - 0.5, j - 0.5, k - 0.5), flux)],
                       avg_slice_k=k, avg_slice_j=j, avg_weight=1.0 / steps)


def request_inputs(req: dict):
    """Host arrays (U, V, W, Pr, S0) of a request: the seeded log-profile
    channel state and the Gaussian puff around the source cell."""
    g = grid_of(make_config(*req["n"]))
    U, V, W, Pr = log_profile_state(g, seed=req["seed"])
    return U, V, W, Pr, puff_state(g, req["source"])


def percentile(x, q):
    """Nearest-rank percentile: the smallest sample with at least q% of the
    samples at or below it."""
    s = np.sort(np.asarray(x, dtype=np.float64))
    if s.size == 0:
        return float("nan")
    r = int(np.ceil(q / 100.0 * s.size))
    return float(s[min(max(r, 1), s.size) - 1])


def run_arrivals(server: Server, reqs, arrivals, inputs, *, precision=1, timeout_s=600.0):
    """Submits request q at arrivals[q] seconds after the start (server
    clock) and collects every result on a second thread.  Returns a list of
    (request, RequestInfo, (xy, xz)) in completion order and the wall span
    from the first submission to the last result."""
    cfgs = [request_config(r, precision=precision, device=server.device) for r in reqs]
    done, errors = [], []
    by_id = {}
    lock = threading.Lock()

    def collector():
        t_end = time.time() + timeout_s
        while len(done) + len(errors) < len(reqs) and time.time() < t_end:
            info = server.wait_any(200)
            if info is None:
                continue
            with lock:
                q = by_id[info.id]
            if info.status != 0:
                errors.append((q, info))
                continue
            done.append((q, info, server.collect(info.id)))

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    t0 = server.now()
    for q in range(len(reqs)):
        wait = t0 + float(arrivals[q]) - server.now()
        if wait > 0:
            time.sleep(wait)
        with lock:
            rid = server.submit(cfgs[q], *inputs[q], nsteps=reqs[q]["steps"])
            by_id[rid] = q
    th.join(timeout_s)
    if errors:
        q, info = errors[0]
        raise RuntimeError(f"request {q} ended with status {info.status}")
    if len(done) != len(reqs):
        raise RuntimeError(f"{len(reqs) - len(done)} requests did not finish within {timeout_s} s")
    span = max(i.t_done for _, i, _ in done) - t0
    return done, span


def summarize(reqs, done, span, rate, server: Server):
    lat = [i.t_done - i.t_submit for _, i, _ in done]
    cell_steps = sum(i.cells * i.steps for _, i, _ in done)
    st = server.stats()
    return {
        "rate_per_s": rate,
        "requests": len(reqs),
        "p50_latency_s": percentile(lat, 50),
        "p99_latency_s": percentile(lat, 99),
        "mean_queue_s": float(np.mean([i.t_admit - i.t_submit for _, i, _ in done])),
        "cell_steps_per_s": cell_steps / span,
        "span_s": span,
        "busy_s": st.busy_s,
        "peak_active": st.peak_active,
        "graph_builds": st.graph_builds,
        "chunks": st.chunks,
        "bytes_peak": st.bytes_peak,
        "max_div": max(i.max_div for _, i, _ in done),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rates", default="1,2,5,10,20,50,100,200")
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--budget-gb", type=float, default=40.0)
    ap.add_argument("--max-active", type=int, default=64)
    ap.add_argument("--chunk-steps", type=int, default=50)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--policy", default="fifo", choices=["fifo", "shortest"])
    a = ap.parse_args()
    prec = 1 if a.precision == "mixed" else 0
    reqs = [dispersion_request(a.seed, q) for q in range(a.requests)]
    inputs = [request_inputs(r) for r in reqs]
    for rate in (float(x) for x in a.rates.split(",")):
        srv = Server(precision=prec, budget_bytes=int(a.budget_gb * (1 << 30)), max_active=a.max_active,
                     chunk_steps=a.chunk_steps, policy=SERVE_SHORTEST_FIRST if a.policy == "shortest" else SERVE_FIFO)
        arrivals = poisson_arrivals(a.seed, rate, len(reqs))
        done, span = run_arrivals(srv, reqs, arrivals, inputs, precision=prec)
        out = summarize(reqs, done, span, rate, srv)
        out["precision"] = a.precision
        out["policy"] = a.policy
        out["max_active"] = a.max_active
        print(json.dumps(out), flush=True)
        srv.close()


if __name__ == "__main__":
    main()
