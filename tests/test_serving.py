"""The serving loop: its HBM-budget allocator and workload generators on the
CPU, and on the GPU continuous batching itself: every request's result equals
the same run alone (bit for bit: each kernel choice is made per domain, so a
domain computes the same operations in any mix), admission by memory, and
requests joining while others run."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT
from gpu_elmm_b200.workloads import (REQUEST_DEPTHS, REQUEST_SIDES, dispersion_request, poisson_arrivals)

ARENA_HARNESS = r'''
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "elmm_arena.h"
using elmm::Arena;
int main() {
  static char buf[1 << 20];
  Arena a(buf, sizeof(buf));
  if (a.capacity() != sizeof(buf) || a.largest_free() != sizeof(buf)) return 1;
  struct Blk { char *p; size_t n; };
  std::vector<Blk> live;
  unsigned s = 12345;
  auto rnd = [&]() { s = s * 1103515245u + 12345u; return (s >> 8) & 0xffff; };
  for (int it = 0; it < 20000; it++) {
    if (live.empty() || rnd() % 3) {
      size_t n = 1 + rnd() % 9000;
      char *p = a.alloc(n);
      if (!p) continue;
      if (((size_t)(p - buf)) % Arena::kAlign) return 2;            // alignment
      if (p < buf || p + n > buf + sizeof(buf)) return 3;           // inside the budget
      for (auto &b : live)
        if (p < b.p + Arena::round(b.n) && b.p < p + Arena::round(n)) return 4;  // no overlap
      live.push_back({p, n});
    } else {
      size_t k = rnd() % live.size();
      if (!a.release(live[k].p)) return 5;
      live.erase(live.begin() + k);
    }
    size_t used = 0;
    for (auto &b : live) used += Arena::round(b.n);
    if (used != a.in_use()) return 6;                              // accounting
  }
  if (a.release(buf + 17)) return 7;                               // foreign pointer refused
  for (auto &b : live) a.release(b.p);
  if (!a.empty() || a.in_use() != 0 || a.free_extents() != 1 || a.largest_free() != sizeof(buf)) return 8;  // merged
  if (a.alloc(sizeof(buf) + 1)) return 9;                          // larger than the budget
  printf("ok %zu\n", a.peak());
  return 0;
}
'''


def test_arena_first_fit_merges_and_accounts():
    """The budget allocator of the serving loop (csrc/elmm_arena.h), compiled
    for the host: random allocations stay aligned, inside the budget and
    disjoint; the byte count is exact; freeing everything merges back into one
    extent."""
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "arena.cpp")
        open(src, "w").write(ARENA_HARNESS)
        exe = os.path.join(d, "arena")
        subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "gpu_elmm_b200", "csrc"), src, "-o", exe],
                       check=True)
        out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.startswith("ok"), (out.returncode, out.stdout)


def test_dispersion_requests_cover_the_sizes():
    reqs = [dispersion_request(0, q) for q in range(400)]
    assert {r["n"][0] for r in reqs} == set(REQUEST_SIDES)
    assert {r["n"][2] for r in reqs} == set(REQUEST_DEPTHS)
    for r in reqs:
        nx, ny, nz = r["n"]
        assert nx == ny and 200 <= r["steps"] <= 2000
        i, j, k = r["source"]
        assert 1 <= i <= nx and 1 <= j <= ny and 2 <= k <= nz - 1
    assert dispersion_request(0, 7) == dispersion_request(0, 7)
    assert dispersion_request(1, 7) != dispersion_request(0, 7)


def test_poisson_arrivals_have_the_rate():
    t = poisson_arrivals(3, 20.0, 20000)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert (gaps > 0).all()
    assert abs(gaps.mean() - 1 / 20.0) < 0.03 / 20.0  # 1/sqrt(20000) ~ 0.7% standard error
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.03  # exponential: coefficient of variation 1


def test_percentile_is_nearest_rank():
    from gpu_elmm_b200.serve import percentile
    x = list(range(1, 101))
    assert percentile(x, 50) == 50 and percentile(x, 99) == 99 and percentile(x, 100) == 100
    assert percentile([3.0], 99) == 3.0
    assert percentile([5, 1, 4, 2, 3], 50) == 3


# ------------------------------------------------------------------ GPU
def _small_requests():
    """Small dispersion requests of three sizes and uneven step counts."""
    return [
        {"n": (32, 32, 16), "steps": 7, "source": (5, 9, 4), "seed": 11},
        {"n": (48, 32, 16), "steps": 12, "source": (40, 2, 13), "seed": 12},
        {"n": (64, 48, 24), "steps": 5, "source": (1, 48, 2), "seed": 13},
        {"n": (32, 32, 16), "steps": 9, "source": (32, 1, 15), "seed": 14},
    ]


def _alone(req, precision):
    from gpu_elmm_b200 import lib as L
    from gpu_elmm_b200.serve import request_config, request_inputs
    d = L.Domain(request_config(req, precision=precision))
    U, V, W, Pr, S0 = request_inputs(req)
    d.upload(U, V, W, Pr)
    d.upload_scalar(1, S0)
    d.project(1.0)
    d.step(req["steps"])
    out = d.scalar_slices(1)
    d.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_server_results_equal_the_runs_alone(precision):
    """Four requests in one mix (chunks of 4 steps, so the set changes
    mid-run) give the same slices as each request run alone."""
    from gpu_elmm_b200.serve import Server, request_inputs, run_arrivals
    reqs = _small_requests()
    srv = Server(precision=precision, budget_bytes=2 << 30, max_active=8, chunk_steps=4)
    done, _ = run_arrivals(srv, reqs, np.zeros(len(reqs)), [request_inputs(r) for r in reqs], precision=precision)
    st = srv.stats()
    assert st.finished == len(reqs) and st.failed == 0 and st.peak_active >= 2
    for q, info, (xy, xz) in done:
        assert info.steps == reqs[q]["steps"]
        axy, axz = _alone(reqs[q], precision)
        assert np.array_equal(xy, axy) and np.array_equal(xz, axz), q
        assert np.abs(xy).max() > 0
    srv.close()


@pytest.mark.gpu
def test_server_admits_by_memory():
    """A budget that holds about two of the requests: never more than that on
    the device at once, and every request still finishes; one larger than the
    whole budget ends with ELMM_ERR_ADMISSION."""
    from gpu_elmm_b200.serve import Server, request_config, request_inputs, run_arrivals
    reqs = [{"n": (64, 48, 24), "steps": 6, "source": (3, 4, 5), "seed": s} for s in range(5)]
    probe = Server(precision=1, budget_bytes=2 << 30, max_active=8, chunk_steps=3)
    done, _ = run_arrivals(probe, reqs[:1], np.zeros(1), [request_inputs(reqs[0])])
    one = done[0][1].bytes
    probe.close()
    assert one > 0
    srv = Server(precision=1, budget_bytes=int(2.5 * one), max_active=8, chunk_steps=3)
    done, _ = run_arrivals(srv, reqs, np.zeros(len(reqs)), [request_inputs(r) for r in reqs])
    st = srv.stats()
    assert st.finished == len(reqs) and st.peak_active <= 2 and st.bytes_peak <= 2.5 * one
    big = {"n": (128, 128, 64), "steps": 1, "source": (3, 4, 5), "seed": 1}
    rid = srv.submit(request_config(big), *request_inputs(big), nsteps=1)
    info = srv.wait_any(60000)
    assert info is not None and info.id == rid and info.status == 7  # ELMM_ERR_ADMISSION
    srv.close()


@pytest.mark.gpu
def test_server_admits_while_others_run():
    """Continuous batching: a request that arrives while a long one runs is
    admitted and finishes before the long one does."""
    from gpu_elmm_b200.serve import Server, request_inputs, run_arrivals
    long_req = {"n": (64, 64, 32), "steps": 3000, "source": (8, 8, 8), "seed": 21}
    short = {"n": (32, 32, 16), "steps": 10, "source": (4, 4, 4), "seed": 22}
    srv = Server(precision=1, budget_bytes=2 << 30, max_active=8, chunk_steps=10)
    done, _ = run_arrivals(srv, [long_req, short], np.array([0.0, 0.05]),
                           [request_inputs(long_req), request_inputs(short)])
    info = {q: i for q, i, _ in done}
    assert info[1].t_admit < info[0].t_done and info[1].t_done < info[0].t_done
    assert srv.stats().graph_builds >= 3  # long alone, long + short, long alone again
    srv.close()


@pytest.mark.gpu
def test_server_isolates_a_failing_request():
    """A request whose flow blows up (a velocity far past the CFL limit)
    ends with ELMM_ERR_NAN; the request beside it finishes with the result it
    has alone."""
    from gpu_elmm_b200.serve import Server, request_config, request_inputs
    good = {"n": (32, 32, 16), "steps": 30, "source": (5, 9, 4), "seed": 31}
    bad = {"n": (32, 32, 16), "steps": 30, "source": (6, 6, 6), "seed": 32}
    U, V, W, Pr, S0 = request_inputs(bad)
    U = U * 1e6  # the explicit RK3 step diverges to Inf / NaN within a few steps
    srv = Server(precision=1, budget_bytes=2 << 30, max_active=8, chunk_steps=5)
    ids = {srv.submit(request_config(good), *request_inputs(good), nsteps=good["steps"]): "good",
           srv.submit(request_config(bad), U, V, W, Pr, S0, nsteps=bad["steps"]): "bad"}
    infos = {}
    while len(infos) < 2:
        info = srv.wait_any(120000)
        assert info is not None
        infos[ids[info.id]] = info
    assert infos["bad"].status == 3  # ELMM_ERR_NAN
    assert infos["good"].status == 0 and infos["good"].steps == good["steps"]
    xy, xz = srv.collect(infos["good"].id)
    axy, axz = _alone(good, 1)
    assert np.array_equal(xy, axy) and np.array_equal(xz, axz)
    srv.close()


@pytest.mark.gpu
@pytest.mark.parametrize("policy", [0, 1])
def test_server_admission_order(policy):
    """One request at a time: while a first request runs, a large and then a
    small request queue up; arrival order admits the large one next, the
    shortest-work-first policy the small one."""
    from gpu_elmm_b200.serve import Server, request_config, request_inputs
    first = {"n": (64, 64, 32), "steps": 300, "source": (3, 3, 3), "seed": 41}
    large = {"n": (64, 64, 32), "steps": 60, "source": (4, 4, 4), "seed": 42}
    small = {"n": (32, 32, 16), "steps": 10, "source": (5, 5, 5), "seed": 43}
    srv = Server(precision=1, budget_bytes=2 << 30, max_active=1, chunk_steps=10, policy=policy)
    names = {}
    for r, name in ((first, "first"), (large, "large"), (small, "small")):
        names[srv.submit(request_config(r), *request_inputs(r), nsteps=r["steps"])] = name
    order = []
    while len(order) < 3:
        info = srv.wait_any(120000)
        assert info is not None and info.status == 0
        order.append(names[info.id])
    assert order[0] == "first"
    assert order[1:] == (["large", "small"] if policy == 0 else ["small", "large"])
    srv.close()
