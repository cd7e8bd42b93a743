"""The bottom and top boundary kinds of CommonBase for the temperature and
the passive scalars (src/scalarboundaries.f90:197-288): BC_DIRICHLET,
BC_NEUMANN and a BC_CONSTFLUX carried by the ghost rule (a free-slip side,
or any side of a passive scalar), whose ghost plane k_scalar_zghost writes
before each stage.

* FP64 GPU against the oracle after 1 and 5 steps: U, V, W within 1e-12,
  P within 1e-11, theta - T_ref and the scalars within 1e-11;
* mixed against FP64 after one step: velocity, theta - T_ref and the
  scalars within 1e-5;
* known answer: fluid at rest with molecular diffusion, theta linear in z
  between a Neumann bottom and a Dirichlet top stays as it is;
* the content follows the ghost-rule fluxes, (q_bottom - q_top) Lx Ly per
  unit time, on both paths;
* a batch of two domains with different scalar boundaries equals each
  domain run alone, bit for bit;
* other kinds and non-finite values are refused; a Dirichlet temperature
  at a smooth wall-model wall is accepted (tests/test_heat_flux.py).
"""
import numpy as np
import pytest

from conftest import rel
from gpu_elmm_b200 import lib as L
from gpu_elmm_b200.config import (BC_CONSTFLUX, BC_DIRICHLET, BC_NEUMANN, BC_NOSLIP, FIELD_SCALAR,
                                  FIELD_TEMPERATURE, grid_of, make_config)
from gpu_elmm_b200.workloads import interior, interiors, log_profile_state, puff_state, temperature_state
from oracle import Oracle

pytestmark = pytest.mark.gpu

N = (32, 24, 16)
CASES = {
    "neumann-dirichlet": dict(buoyancy=True, temperature_bc=((BC_NEUMANN, 0.01), (BC_DIRICHLET, 296.0))),
    "flux-top": dict(buoyancy=True, temperature_bc=((BC_CONSTFLUX, 0.15), (BC_CONSTFLUX, 0.05))),
    "scalars": dict(buoyancy=True, temperature_bc=((BC_CONSTFLUX, 0.0), (BC_NEUMANN, 0.003)), num_scalars=2,
                    scalar_bc=((BC_CONSTFLUX, 0.2), (BC_DIRICHLET, 0.5))),
}


def _fields(g, cfg, seed):
    st = log_profile_state(g, seed=seed)
    T0 = temperature_state(g, seed=seed) if cfg.enable_buoyancy else None
    S0 = [puff_state(g, (9, 7, 5)) * sc for sc in range(1, cfg.num_scalars + 1)]
    return st, T0, S0


def _load(h, st, T0, S0, oracle=False):
    if oracle:
        h.set_state(*st)
        if T0 is not None:
            h.set_field(FIELD_TEMPERATURE, T0)
        for sc, S in enumerate(S0):
            h.set_field(FIELD_SCALAR + sc, S)
    else:
        h.upload(*st)
        if T0 is not None:
            h.upload_temperature(T0)
        for sc, S in enumerate(S0):
            h.upload_scalar(sc + 1, S)


def _inner(g, F):
    return interior(F, -2, (g.Prnx, g.Prny, g.Prnz))


@pytest.mark.parametrize("nsteps", [1, 5])
@pytest.mark.parametrize("case", list(CASES))
def test_fp64_scalar_boundaries_follow_the_oracle(case, nsteps):
    cfg = make_config(*N, **CASES[case])
    g = grid_of(cfg)
    st, T0, S0 = _fields(g, cfg, 3)
    o, d = Oracle(cfg), L.Domain(cfg)
    _load(o, st, T0, S0, oracle=True)
    _load(d, st, T0, S0)
    o.project(1.0)
    d.project(1.0)
    o.step(nsteps)
    d.step(nsteps)
    for a, b, name in zip(interiors(g, *d.download()), interiors(g, *o.state()), "UVWP"):
        assert rel(a, b) < (1e-11 if name == "P" else 1e-12), (case, name, rel(a, b))
    et = rel(_inner(g, d.field(FIELD_TEMPERATURE)) - 295.0, _inner(g, o.get_field(FIELD_TEMPERATURE)) - 295.0)
    es = [rel(_inner(g, d.scalar(sc)), _inner(g, o.get_field(FIELD_SCALAR + sc - 1)))
          for sc in range(1, cfg.num_scalars + 1)]
    print(case, nsteps, "theta", et, "scalars", es)
    assert et < 1e-11 and all(e < 1e-11 for e in es), (et, es)
    d.close()


@pytest.mark.parametrize("case", list(CASES))
def test_mixed_scalar_boundaries_one_step(case):
    cfg = make_config(*N, **CASES[case])
    g = grid_of(cfg)
    st, T0, S0 = _fields(g, cfg, 4)
    d64 = L.Domain(cfg)
    _load(d64, st, T0, S0)
    d64.project(1.0)
    ref = d64.download(), d64.field(FIELD_TEMPERATURE), [d64.scalar(sc) for sc in range(1, cfg.num_scalars + 1)]
    d64.step(1)
    dm = L.Domain(make_config(*N, precision=1, **CASES[case]))
    _load(dm, *ref)
    dm.step(1)
    e = [rel(a, b) for a, b in zip(interiors(g, *dm.download())[:3], interiors(g, *d64.download())[:3])]
    e.append(rel(_inner(g, dm.field(FIELD_TEMPERATURE)) - 295.0, _inner(g, d64.field(FIELD_TEMPERATURE)) - 295.0))
    e += [rel(_inner(g, dm.scalar(sc)), _inner(g, d64.scalar(sc))) for sc in range(1, cfg.num_scalars + 1)]
    print(case, "mixed vs FP64", e)
    assert max(e) < 1e-5, e
    d64.close()
    dm.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_linear_profile_between_neumann_and_dirichlet_is_steady(precision):
    n, gam, top = N, 0.01, 300.0
    cfg = make_config(*n, sgstype=0, buoyancy=True, precision=precision,
                      temperature_bc=((BC_NEUMANN, gam), (BC_DIRICHLET, top)))
    g = grid_of(cfg)
    U, V, W, Pr = (np.zeros(s) for s in (g.shape_u(), g.shape_v(), g.shape_w(), g.shape_p()))
    T = np.zeros(g.shape_t())
    zpr = np.arange(1, n[2] + 1) - 0.5
    _inner(g, T)[...] = (top + gam * (zpr - n[2]))[:, None, None]
    d = L.Domain(cfg)
    d.upload(U, V, W, Pr)
    d.upload_temperature(T)
    d.project(1.0)
    d.step(3)
    err = np.abs(_inner(g, d.field(FIELD_TEMPERATURE)) - _inner(g, T)).max()
    print("precision", precision, "max |theta - theta0|", err)
    assert err < (1e-11 if precision == 0 else 1e-5), err
    d.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_content_follows_the_ghost_rule_fluxes(precision):
    (qb, qt), (sb, st_) = (0.15, 0.05), (0.2, -0.1)
    cfg = make_config(*N, precision=precision, buoyancy=True, num_scalars=1,
                      temperature_bc=((BC_CONSTFLUX, qb), (BC_CONSTFLUX, qt)),
                      scalar_bc=((BC_CONSTFLUX, sb), (BC_CONSTFLUX, st_)))
    g = grid_of(cfg)
    st, T0, S0 = _fields(g, cfg, 5)
    d = L.Domain(cfg)
    _load(d, st, T0, S0)
    d.project(1.0)
    h0 = _inner(g, d.field(FIELD_TEMPERATURE)).sum() - 295.0 * g.cells(), _inner(g, d.scalar(1)).sum()
    steps, dt = 5, 0.02
    d.step(steps)
    h1 = _inner(g, d.field(FIELD_TEMPERATURE)).sum() - 295.0 * g.cells(), _inner(g, d.scalar(1)).sum()
    tol = 1e-9 if precision == 0 else 2e-3
    for a, b, q0, q1 in zip(h0, h1, (qb, sb), (qt, st_)):
        expect = (q0 - q1) * g.Prnx * g.Prny * dt * steps
        assert abs((b - a) - expect) < tol * abs(expect), (b - a, expect)
    d.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_with_scalar_boundaries_equals_the_runs_alone(precision):
    cfgs = [make_config(32, 24, 16, precision=precision, num_scalars=1,
                        scalar_bc=((BC_CONSTFLUX, 0.2), (BC_DIRICHLET, 0.5))),
            make_config(48, 32, 12, precision=precision, num_scalars=1,
                        scalar_bc=((BC_NEUMANN, -0.01), (BC_CONSTFLUX, 0.0)))]
    b = L.Batch(cfgs)
    alone = []
    for di, cfg in enumerate(cfgs):
        g = grid_of(cfg)
        st, _, S0 = _fields(g, cfg, 6 + di)
        b.upload(di, *st)
        b.upload_scalar(di, 1, S0[0])
        d = L.Domain(cfg)
        _load(d, st, None, S0)
        d.project(1.0)
        d.step(3)
        alone.append((d.download(), d.scalar(1)))
        d.close()
    b.project(1.0)
    b.step(3)
    for di, (state, S) in enumerate(alone):
        for x, y in zip(b.download(di), state):
            assert np.array_equal(x, y)
        assert np.array_equal(b.scalar(di, 1), S)
    b.close()


def test_unsupported_scalar_boundaries_are_refused():
    walls = (3, 3, 3, 3, BC_NOSLIP, BC_NOSLIP)
    bad = [dict(buoyancy=True, temperature_bc=((BC_NOSLIP, 0.0), (BC_CONSTFLUX, 0.0))),
           dict(num_scalars=1, scalar_bc=((BC_CONSTFLUX, float("inf")), (BC_CONSTFLUX, 0.0)))]
    for kw in bad:
        with pytest.raises(L.ElmmError) as e:
            L.Domain(make_config(*N, **kw))
        assert e.value.code == 1, kw
    # the same kinds where they are built
    L.Domain(make_config(*N, buoyancy=True, sgstype=0, temperature_bc=((BC_DIRICHLET, 300.0), (BC_CONSTFLUX, 0.0)))).close()
    L.Domain(make_config(*N, num_scalars=1, scalar_bc=((BC_DIRICHLET, 1.0), (BC_NEUMANN, 0.1)))).close()
    L.Domain(make_config(*N, buoyancy=True, z0=0.0, temperature_bc=((BC_DIRICHLET, 300.0), (BC_CONSTFLUX, 0.0)))).close()
    L.Domain(make_config(*N, buoyancy=True, btype=walls, z0=0.0,
                         temperature_bc=((BC_CONSTFLUX, 0.0), (BC_DIRICHLET, 300.0)))).close()
