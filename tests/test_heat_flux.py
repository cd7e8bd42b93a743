"""Heat exchange at a wall-model wall.  A constant surface heat flux
(TempBtype CONSTFLUX with a non-zero sideTemp at the bottom or top): the
flux of the side's wall-model points enters the cells next to the wall
(src/scalars.f90:323-327), and a flux into the flow over a rough wall makes
the wall model's u* follow Monin-Obukhov similarity (WM_MO_FluxStress,
src/wallmodels.f90:1606-1660, 1836-1854).  A prescribed surface
temperature (TempBtype DIRICHLET): the wall model computes the points'
u* and surface flux from the temperature difference each stage
(WM_MO_Dirichlet / WM_MO_DirichletStress, src/wallmodels.f90:1664-1716,
1858-1938), starting from the state the initial projection leaves (the
wall model once on the initial fields, src/initial.f90:4331-4336).

* FP64 GPU against the oracle after 1 and 5 steps: U, V, W within 1e-12,
  P within 1e-11, theta - T_ref within 1e-11 (relative to the largest
  value), for a heated rough bottom (the Monin-Obukhov u*), a cooled bottom
  with a flux through a top wall (neutral u*, the flux terms alone), a
  heated smooth bottom (z0 = 0, WMFlatStress), a surface warmer than the
  air, between two walls a cool bottom and a warm top, and a surface
  temperature at a smooth bottom (the flat branch of ComputeViscsWM and
  ComputeUVWFluxesWM, src/wallmodels.f90:2123-2146, 2265-2275: WMFlat u*,
  and the points' temperature flux keeps its initial zero);
* mixed against FP64 after one step from the same projected state:
  velocity and theta - T_ref within 1e-5;
* the heat content grows by (q_bottom - q_top) Lx Ly per unit time on both
  paths (advection and diffusion are in flux form);
* a smooth surface temperature exchanges no heat: the heat content stays
  as it is on both paths;
* a non-finite flux is refused with ELMM_ERR_INVALID_CONFIG (a flux
  through a free-slip top, which no wall-model points carry, takes
  CommonBase's ghost rule: tests/test_scalar_bcs.py).
"""
import numpy as np
import pytest

from conftest import rel
from gpu_elmm_b200 import lib as L
from gpu_elmm_b200.config import (BC_CONSTFLUX, BC_DIRICHLET, BC_FREESLIP, BC_NOSLIP, BC_PERIODIC,
                                  FIELD_TEMPERATURE, grid_of, make_config)
from gpu_elmm_b200.workloads import interior, interiors, log_profile_state, temperature_state
from oracle import Oracle

pytestmark = pytest.mark.gpu

N = (32, 24, 16)
TWO_WALLS = (BC_PERIODIC,) * 4 + (BC_NOSLIP, BC_NOSLIP)
CASES = {
    "heated-rough": dict(heat_flux=(0.3, 0.0)),
    "cooled-top-flux": dict(heat_flux=(-0.1, 0.05), btype=TWO_WALLS),
    "heated-smooth": dict(heat_flux=(0.3, 0.0), z0=0.0),
    "warm-surface": dict(temperature_bc=((BC_DIRICHLET, 296.0), (BC_CONSTFLUX, 0.0))),
    "surfaces-two-walls": dict(temperature_bc=((BC_DIRICHLET, 294.0), (BC_DIRICHLET, 295.5)), btype=TWO_WALLS),
    "warm-smooth-surface": dict(temperature_bc=((BC_DIRICHLET, 296.0), (BC_CONSTFLUX, 0.0)), z0=0.0),
}


def _pair(case, precision=0, seed=0):
    kw = CASES[case]
    cfg = make_config(*N, buoyancy=True, precision=precision, **kw)
    g = grid_of(cfg)
    st = log_profile_state(g, seed=seed)
    T0 = temperature_state(g, seed=seed)
    o = Oracle(make_config(*N, buoyancy=True, **kw))
    o.set_state(*st)
    o.set_field(FIELD_TEMPERATURE, T0)
    d = L.Domain(cfg)
    d.upload(*st)
    d.upload_temperature(T0)
    return g, o, d


def _theta(g, F):
    return interior(F, -2, (g.Prnx, g.Prny, g.Prnz)) - 295.0


@pytest.mark.parametrize("nsteps", [1, 5])
@pytest.mark.parametrize("case", list(CASES))
def test_fp64_heat_flux_follows_the_oracle(case, nsteps):
    g, o, d = _pair(case)
    o.project(1.0)
    d.project(1.0)
    o.step(nsteps)
    d.step(nsteps)
    for a, b, name in zip(interiors(g, *d.download()), interiors(g, *o.state()), "UVWP"):
        assert rel(a, b) < (1e-11 if name == "P" else 1e-12), (case, name, rel(a, b))
    e = rel(_theta(g, d.field(FIELD_TEMPERATURE)), _theta(g, o.get_field(FIELD_TEMPERATURE)))
    print(case, nsteps, "theta", e)
    assert e < 1e-11, e
    d.close()


@pytest.mark.parametrize("case", list(CASES))
def test_mixed_heat_flux_one_step(case):
    g, _, d64 = _pair(case)
    d64.project(1.0)
    ref0 = d64.download()
    T0 = d64.field(FIELD_TEMPERATURE)
    d64.step(1)
    dm = L.Domain(make_config(*N, buoyancy=True, precision=1, **CASES[case]))
    dm.upload(*ref0)
    dm.upload_temperature(T0)
    dm.step(1)
    e = [rel(a, b) for a, b in zip(interiors(g, *dm.download())[:3], interiors(g, *d64.download())[:3])]
    et = rel(_theta(g, dm.field(FIELD_TEMPERATURE)), _theta(g, d64.field(FIELD_TEMPERATURE)))
    print(case, "mixed vs FP64", e, et)
    assert max(e) < 1e-5 and et < 1e-5, (e, et)
    d64.close()
    dm.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_heat_content_follows_the_surface_fluxes(precision):
    qb, qt = CASES["cooled-top-flux"]["heat_flux"]
    g, _, d = _pair("cooled-top-flux", precision=precision)
    d.project(1.0)
    h0 = _theta(g, d.field(FIELD_TEMPERATURE)).sum()          # cells of 1 m^3
    steps, dt = 5, 0.02
    d.step(steps)
    h1 = _theta(g, d.field(FIELD_TEMPERATURE)).sum()
    expect = (qb - qt) * g.Prnx * g.Prny * dt * steps
    tol = 1e-9 if precision == 0 else 2e-3
    assert abs((h1 - h0) - expect) < tol * abs(expect), (h1 - h0, expect)
    d.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_smooth_surface_temperature_exchanges_no_heat(precision):
    g, _, d = _pair("warm-smooth-surface", precision=precision)
    d.project(1.0)
    h0 = _theta(g, d.field(FIELD_TEMPERATURE)).sum()
    d.step(5)
    h1 = _theta(g, d.field(FIELD_TEMPERATURE)).sum()
    scale = np.abs(_theta(g, d.field(FIELD_TEMPERATURE))).sum()
    assert abs(h1 - h0) < (1e-12 if precision == 0 else 1e-5) * scale, (h1 - h0, scale)
    d.close()


def test_non_finite_flux_is_refused():
    with pytest.raises(L.ElmmError) as e:
        L.Domain(make_config(*N, buoyancy=True, heat_flux=(float("nan"), 0.0)))
    assert e.value.code == 1
    with pytest.raises(L.ElmmError) as e:
        L.Domain(make_config(*N, buoyancy=True, temperature_bc=((BC_DIRICHLET, float("inf")), (BC_CONSTFLUX, 0.0))))
    assert e.value.code == 1
    L.Domain(make_config(*N, buoyancy=True, heat_flux=(0.1, 0.0))).close()
    # a flux through the free-slip top has no wall-model points: the ghost rule carries it
    assert BC_FREESLIP == make_config(*N).Btype[5]
    L.Domain(make_config(*N, buoyancy=True, heat_flux=(0.0, 0.1))).close()
