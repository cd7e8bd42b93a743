"""Smooth walls (z0 = 0): the wall model takes WMFlatStress, the u* of the
viscous-sublayer / buffer / logarithmic law iterated from the point's
previous value (src/wallmodels.f90:1190-1265, chosen at :2262-2275), on the
domain's no-slip walls.

* FP64 channel with a smooth bottom, after 1 and 10 steps against the
  oracle: U, V, W within 1e-12, P within 1e-11, max |div u| below 1e-10;
* smooth bottom and top walls on a stretched grid, FP64 against the oracle
  after 5 steps;
* the mixed path's velocity within 1e-5 of FP64 after one step;
* the autotuner's timing launches leave the wall points' u* (the start of
  the next iteration) alone: every forced tile shape gives the same state.
"""
import numpy as np
import pytest

from conftest import rel
from gpu_elmm_b200 import lib as L
from gpu_elmm_b200.config import BC_NOSLIP, BC_PERIODIC, grid_of, make_config
from gpu_elmm_b200.workloads import interiors, log_profile_state
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _errs(g, a, b):
    return [rel(x, y) for x, y in zip(interiors(g, *a), interiors(g, *b))]


def _zw(nz):
    return np.concatenate([[0.0], np.cumsum(0.5 * 1.04 ** np.arange(nz))])


def test_smooth_bottom_fp64_follows_the_oracle():
    cfg = make_config(48, 32, 24, z0=0.0)
    g = grid_of(cfg)
    o = Oracle(cfg)
    st = log_profile_state(g, seed=11)
    o.set_state(*st)
    o.project(1.0)
    d = L.Domain(cfg)
    d.upload(*st)
    d.project(1.0)  # with the wall model on the initial fields, whose u* the first stage starts from
    for n in (1, 9):
        o.step(n)
        s = d.step(n)
        e = _errs(g, d.download(), o.state())
        print("smooth bottom, FP64 vs oracle:", e, s.max_div)
        assert max(e[:3]) < 1e-12 and e[3] < 1e-11 and s.max_div < 1e-10, e
    d.close()


def test_smooth_top_and_bottom_on_a_stretched_grid():
    bt = (BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_NOSLIP, BC_NOSLIP)
    cfg = make_config(32, 24, 20, btype=bt, z0=0.0, zW=_zw(20))
    g = grid_of(cfg)
    o = Oracle(cfg)
    st = log_profile_state(g, seed=12, zW=_zw(20))
    o.set_state(*st)
    o.project(1.0)
    d = L.Domain(cfg)
    d.upload(*st)
    d.project(1.0)
    o.step(5)
    s = d.step(5)
    e = _errs(g, d.download(), o.state())
    print("smooth walls, stretched, FP64 vs oracle:", e, s.max_div)
    assert max(e[:3]) < 1e-12 and e[3] < 1e-11 and s.max_div < 1e-10, e
    d.close()


def test_smooth_bottom_mixed_follows_fp64():
    c64, c32 = make_config(48, 32, 24, z0=0.0), make_config(48, 32, 24, z0=0.0, precision=1)
    g = grid_of(c64)
    st = log_profile_state(g, seed=13)
    a, b = L.Domain(c64), L.Domain(c32)
    a.upload(*st)
    b.upload(*st)
    a.project(1.0)
    b.project(1.0)
    a.step(1)
    s = b.step(1)
    e = _errs(g, b.download(), a.download())
    print("smooth bottom, mixed vs FP64:", e, s.max_div)
    # velocity, as test_mixed_path_one_step: without buoyancy the pressure is
    # small (its largest value ~0.05) and its FP32 error relative to it is
    # the conditioning floor of the projection, reported above
    assert max(e[:3]) < 1e-5 and s.max_div < 1e-6, e
    a.close()
    b.close()


def test_every_tile_shape_leaves_a_smooth_wall_alone():
    for prec in (0, 1):
        cfg = make_config(48, 32, 24, z0=0.0, precision=prec)
        st = log_profile_state(grid_of(cfg), seed=14)
        ref = None
        for shapes in ({}, {"momentum_z_chunk": 8, "sgs_z_chunk": 8}, {"momentum_z_chunk": 32, "sgs_z_chunk": 32}):
            d = L.Domain(cfg)
            d.upload(*st)
            d.project(1.0)
            if shapes:
                d.set_tuning(**shapes)
            d.step(3)
            out = d.download()
            if ref is None:
                ref = out
            else:
                for x, y in zip(out, ref):
                    assert np.array_equal(x, y), (prec, shapes)
            d.close()
