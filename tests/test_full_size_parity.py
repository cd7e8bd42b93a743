"""Parity with the FP64 oracle at the sizes the benchmark measures.

The other GPU tests compare the library with the oracle on small grids; this
file repeats the comparison on the configurations `bench.py` times, so that
the numbers it reports are numbers of a path checked against the oracle at
that size:

  * the 256 x 256 x 128 channel with the potential temperature (the
    headline workload): FP64 after 1 and 10 steps, mixed after 1 step;
  * the 384 x 384 x 96 stretched grid with the 8 x 8 array of cubes and a
    mean pressure gradient: FP64 after 1 step;
  * the 64 x 64 x 32 channel for the 100 steps of its configuration;
  * the same channel over 1000 steps: the vertical profiles of the mean
    velocity and of the resolved TKE of both GPU paths, averaged over steps
    500..1000, against the oracle's, within 1%;
  * one batch whose x and y lengths cover every length with a register FFT
    kernel (32, 48, 64, 96, 128, 192, 256, 384), each domain against its own
    oracle run.

Tolerances (relative = max |gpu - oracle| / max |oracle|) are those of
test_gpu_parity.py: 1e-12 for the FP64 velocities and the temperature
deviation, 1e-11 for the FP64 pressure (its conditioning floor), 1e-5 for
the mixed path (the pressure included on the headline workload); max |div u|
1e-10 (FP64), 1e-6 (mixed) and 1e-7 on the mixed headline step.  The oracle
runs on every host core.
"""
import os

import numpy as np
import pytest

from conftest import rel
from gpu_elmm_b200 import lib as L
from gpu_elmm_b200.config import FIELD_TEMPERATURE, grid_of, make_config
from gpu_elmm_b200.workloads import interior, interiors, log_profile_state, temperature_state
import oracle as orc
from oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _all_cores():
    orc.set_threads(os.cpu_count() or 1)
    yield


def _errs(g, a, b):
    return [rel(x, y) for x, y in zip(interiors(g, *a), interiors(g, *b))]


def _theta_err(g, Ta, Tb):
    n = (g.Prnx, g.Prny, g.Prnz)
    return rel(interior(Ta, -2, n) - 295.0, interior(Tb, -2, n) - 295.0)


def test_headline_channel_fp64_and_mixed():
    """256 x 256 x 128 with the potential temperature and buoyancy: the FP64
    path after 1 and 10 steps and the mixed path after 1 step, both from
    the oracle's projected state, against the oracle."""
    n = (256, 256, 128)
    cfg = make_config(*n, buoyancy=True)
    g = grid_of(cfg)
    st = log_profile_state(g, seed=0)
    T0 = temperature_state(g, seed=0)
    o = Oracle(cfg)
    o.set_state(*st)
    o.set_field(FIELD_TEMPERATURE, T0)
    o.project(1.0)
    s0, T0p = o.state(), o.get_field(FIELD_TEMPERATURE)
    doms = {}
    for prec in (0, 1):
        d = L.Domain(make_config(*n, buoyancy=True, precision=prec))
        d.upload(*s0)
        d.upload_temperature(T0p)
        doms[prec] = d
    o.step(1)
    ref1, refT1 = o.state(), o.get_field(FIELD_TEMPERATURE)
    out = {}
    for prec, d in doms.items():
        s = d.step(1)
        out[prec] = (_errs(g, d.download(), ref1), _theta_err(g, d.field(FIELD_TEMPERATURE), refT1), s.max_div)
    print("256x256x128 after 1 step vs oracle, (U, V, W, P), theta, max div:", out)
    e, et, md = out[0]
    assert max(e[:3]) < 1e-12 and e[3] < 1e-11 and et < 1e-12 and md < 1e-10, out[0]
    e, et, md = out[1]
    assert max(e) < 1e-5 and et < 1e-5 and md < 1e-7, out[1]
    doms[1].close()
    o.step(9)
    s = doms[0].step(9)
    e10 = _errs(g, doms[0].download(), o.state())
    et10 = _theta_err(g, doms[0].field(FIELD_TEMPERATURE), o.get_field(FIELD_TEMPERATURE))
    print("256x256x128 FP64 after 10 steps vs oracle:", e10, et10, s.max_div)
    assert max(e10[:3]) < 1e-12 and e10[3] < 1e-11 and et10 < 1e-12 and s.max_div < 1e-10, (e10, et10)
    doms[0].close()


def test_cube_array_fp64_one_step():
    """384 x 384 x 96, dz_k = 0.5 * 1.04^(k-1), 8 x 8 cubes of 16 cells with
    the mean pressure gradient: FP64 against the oracle after one step."""
    from gpu_elmm_b200.solids import build_solids
    from gpu_elmm_b200.workloads import CUBES_N, cubes_boxes, cubes_config, stretched_zw
    cfg = cubes_config(precision=0)
    g = grid_of(cfg)
    sol = build_solids(cfg, cubes_boxes())
    st = log_profile_state(g, seed=0, zW=stretched_zw(CUBES_N[2]))
    o = Oracle(cfg)
    o.set_state(*st)
    o.project(1.0)
    d = L.Domain(cfg)
    d.upload(*o.state())
    o.set_solids(sol)
    d.set_solids(sol)
    o.step(1)
    s = d.step(1)
    e = _errs(g, d.download(), o.state())
    print("cube array FP64 after 1 step vs oracle (U, V, W, P):", e, "max div", s.max_div)
    assert max(e[:3]) < 1e-12 and e[3] < 1e-11 and s.max_div < 1e-10, e
    d.close()


def test_channel_100_steps_fp64():
    """64 x 64 x 32 channel, the 100 steps of its configuration: FP64
    against the oracle."""
    cfg = make_config(64, 64, 32)
    g = grid_of(cfg)
    o = Oracle(cfg)
    o.set_state(*log_profile_state(g, seed=0))
    o.project(1.0)
    d = L.Domain(cfg)
    d.upload(*o.state())
    o.step(100)
    s = d.step(100)
    e = _errs(g, d.download(), o.state())
    print("64x64x32 FP64 after 100 steps vs oracle:", e, s.max_div)
    assert max(e[:3]) < 1e-12 and e[3] < 1e-11 and s.max_div < 1e-10, e
    d.close()


def test_long_run_profiles_against_the_oracle():
    """64 x 64 x 32 channel for 1000 steps from the oracle's projected state:
    the mean-velocity and resolved-TKE profiles of the FP64 and the mixed
    path, averaged over steps 500..1000 every 50 steps, within 1% of the
    oracle's."""
    from gpu_elmm_b200.stats import Profiles, compare
    cfg = make_config(64, 64, 32)
    g = grid_of(cfg)
    o = Oracle(cfg)
    o.set_state(*log_profile_state(g, seed=0))
    o.project(1.0)
    doms = {p: L.Domain(make_config(64, 64, 32, precision=p)) for p in (0, 1)}
    for d in doms.values():
        d.upload(*o.state())
    prof = {k: Profiles(g) for k in ("oracle", 0, 1)}
    done = 0
    for target in range(500, 1001, 50):
        o.step(target - done)
        for d in doms.values():
            d.step(target - done)
        done = target
        prof["oracle"].add(*o.state()[:3])
        for p, d in doms.items():
            prof[p].add(*d.download()[:3])
    ref = prof["oracle"].result()
    for p, d in doms.items():
        c = compare(prof[p].result(), ref)
        print("profiles vs oracle, precision", p, c)
        assert c["u"] < 1e-2 and c["tke"] < 1e-2, (p, c)
        d.close()


# x and y lengths of the batch: every length with its own register FFT kernel
REG_LENGTHS = (32, 48, 64, 96, 128, 192, 256, 384)


@pytest.mark.parametrize("precision", [0, 1])
def test_every_register_fft_length_in_one_batch(precision):
    """Eight channel domains in one batch whose x and y lengths cover every
    register-FFT length in both directions, two steps, each domain against
    its own oracle run."""
    sizes = [(REG_LENGTHS[q], REG_LENGTHS[(q + 3) % 8], 8) for q in range(8)]
    cfgs = [make_config(*n, precision=precision) for n in sizes]
    b = L.Batch(cfgs)
    refs = []
    for q, n in enumerate(sizes):
        c64 = make_config(*n)
        g = grid_of(c64)
        o = Oracle(c64)
        o.set_state(*log_profile_state(g, seed=q + 1))
        o.project(1.0)
        b.upload(q, *o.state())
        o.step(2)
        refs.append((g, o.state()))
    st = b.step(2)
    tol = (1e-12, 1e-11) if precision == 0 else (1e-5, None)
    for q, (g, ref) in enumerate(refs):
        e = _errs(g, b.download(q), ref)
        print(sizes[q], "precision", precision, "vs oracle:", e)
        assert max(e[:3]) < tol[0], (sizes[q], e)
        if tol[1]:
            assert e[3] < tol[1], (sizes[q], e)
    assert st.max_div < (1e-10 if precision == 0 else 1e-6)
    b.close()
