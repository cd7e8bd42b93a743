"""A domain split into z-slabs (elmm_slabs_*), every slab on the one B200
(device copies in place of the peer copies between GPUs): the state after
the upload, the initial projection and three RK3 steps against the
single-domain handle on the same state, and the FP64 path against the
oracle.

* upload -> download returns exactly what the single-domain handle returns
  (the slabs write every element of the whole domain's host arrays, each
  plane once);
* FP64: U, V, W within 1e-12 and P within 1e-11 (relative to the largest
  value) of the single domain and of the oracle, max |div u| below 1e-10;
  the split changes only the order of the z solve's operations;
* mixed: within 1e-5 of the single-domain mixed path;
* march_host and the real32 host arrays against the double calls;
* the temperature and a passive scalar with point sources, the scalars'
  two-deep halos exchanged, against the single domain;
* even and uneven splits, 2 and 3 slabs, uniform and stretched z, slabs
  short enough for the tiled sweep kernels and taller ones.
"""
import numpy as np
import pytest

from conftest import rel
from gpu_elmm_b200 import lib as L
from gpu_elmm_b200.config import grid_of, make_config
from gpu_elmm_b200.workloads import interiors, log_profile_state
from oracle import Oracle

pytestmark = pytest.mark.gpu

N = (48, 32, 24)


def _zw(nz):
    return np.concatenate([[0.0], np.cumsum(0.5 * 1.04 ** np.arange(nz))])


def _errs(a, b):
    return [rel(x, y) for x, y in zip(a, b)]


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("split", [(2, None), (3, (6, 10, 8))], ids=["even2", "uneven3"])
def test_slabs_follow_the_single_domain(precision, split):
    ns, nz = split
    cfg = make_config(*N, precision=precision, cfl_check=1)
    st = log_profile_state(grid_of(cfg), seed=3)
    a, b = L.Domain(cfg), L.Slabs(cfg, ns, devices=[0] * ns, nz=nz)
    a.upload(*st)
    b.upload(*st)
    for x, y in zip(b.download(), a.download()):
        assert np.array_equal(x, y)
    pa, pb = a.project(1.0), b.project(1.0)
    tol = (1e-12, 1e-11) if precision == 0 else (1e-5, 1e-5)
    e = _errs(b.download(), a.download())
    print("after the projection", precision, split, e, pa.max_div, pb.max_div)
    assert max(e[:3]) < tol[0] and e[3] < tol[1], e
    sa, sb = a.step(3), b.step(3)
    e = _errs(b.download(), a.download())
    print("after 3 steps", precision, split, e, sa.max_div, sb.max_div, sa.cfl, sb.cfl)
    assert max(e[:3]) < tol[0] and e[3] < tol[1], e
    assert sb.max_div < (1e-10 if precision == 0 else 1e-6)
    assert sb.cfl == pytest.approx(sa.cfl, rel=1e-6)
    a.close()
    b.close()


def test_fp64_slabs_follow_the_oracle_on_a_stretched_grid():
    n = (32, 24, 20)
    cfg = make_config(*n, zW=_zw(n[2]))
    g = grid_of(cfg)
    o = Oracle(cfg)
    o.set_state(*log_profile_state(g, seed=7))
    b = L.Slabs(cfg, 3, devices=[0, 0, 0], nz=(5, 9, 6))
    b.upload(*o.state())
    o.project(1.0)
    b.project(1.0)
    e = _errs(interiors(g, *b.download()), interiors(g, *o.state()))
    assert max(e[:3]) < 1e-12 and e[3] < 1e-11, e
    o.step(4)
    s = b.step(4)
    e = _errs(interiors(g, *b.download()), interiors(g, *o.state()))
    print("stretched, 3 slabs, 4 steps vs oracle:", e, s.max_div)
    assert max(e[:3]) < 1e-12 and e[3] < 1e-11 and s.max_div < 1e-10, e
    b.close()


def test_tall_slabs_take_the_column_kernels():
    """A slab taller than the tiled sweeps allow (300 levels) makes every
    slab run the one-thread-per-column sweep kernels: FP64 against the
    single domain."""
    cfg = make_config(32, 32, 440, sgstype=0)
    st = log_profile_state(grid_of(cfg), seed=2)
    a, b = L.Domain(cfg), L.Slabs(cfg, 2, devices=[0, 0], nz=(300, 140))
    a.upload(*st)
    b.upload(*st)
    a.project(1.0)
    b.project(1.0)
    a.step(2)
    s = b.step(2)
    e = _errs(b.download(), a.download())
    print("300-level slabs vs single domain:", e, s.max_div)
    assert max(e[:3]) < 1e-12 and e[3] < 1e-11 and s.max_div < 1e-10, e
    a.close()
    b.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_slab_host_arrays(precision):
    """elmm_slabs_march_host equals upload, step, download on a second
    handle, bit for bit; the real32 entry points equal the double ones on
    the same values widened, their results rounded to float32."""
    cfg = make_config(*N, precision=precision)
    st = log_profile_state(grid_of(cfg), seed=5)
    a, b = L.Slabs(cfg, 2, devices=[0, 0]), L.Slabs(cfg, 2, devices=[0, 0])
    a.upload(*st)
    a.step(2)
    ref = a.download()
    arrs = [x.copy() for x in st]
    b.march_host(*arrs, n=2)
    for x, y in zip(arrs, ref):
        assert np.array_equal(x, y)
    f32 = [x.astype(np.float32) for x in st]
    wide = [x.astype(np.float64) for x in f32]
    a.upload_f32(*f32)
    b.upload(*wide)
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y)
    for x, y in zip(a.download_f32(), b.download()):
        assert x.dtype == np.float32 and np.array_equal(x, y.astype(np.float32))
    a.march_host_f32(*f32, n=2)
    b.march_host(*wide, n=2)
    for x, y in zip(f32, wide):
        assert np.array_equal(x, y.astype(np.float32))
    a.close()
    b.close()


def _theta_scalar_cfg(precision, **kw):
    return make_config(*N, precision=precision, buoyancy=True, num_scalars=1,
                       point_sources=[(1, (20.5, 14.5, 12.2), 2.0), (1, (9.5, 20.5, 3.7), 1.0)], **kw)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("split", [(2, None), (3, (6, 10, 8))], ids=["even2", "uneven3"])
def test_slabs_carry_temperature_and_scalars(precision, split):
    """Config-1 physics with the potential temperature and a passive scalar
    with two point sources (one in each half), split into slabs: the slabs
    exchange the scalars' two planes beyond each shared face and the
    diffusivity's ghost plane.  Against the single domain after the
    projection and three steps: FP64 U, V, W within 1e-12, P within 1e-11,
    theta - T_ref and the scalar within 1e-11; mixed within 1e-5."""
    from gpu_elmm_b200.config import FIELD_TEMPERATURE
    from gpu_elmm_b200.workloads import interior, puff_state, temperature_state
    ns, nz = split
    cfg = _theta_scalar_cfg(precision)
    g = grid_of(cfg)
    st = log_profile_state(g, seed=8)
    T0 = temperature_state(g, seed=8, amp=0.2)
    S0 = puff_state(g, (20, 14, 12), sigma=3.0)
    a, b = L.Domain(cfg), L.Slabs(cfg, ns, devices=[0] * ns, nz=nz)
    for h in (a, b):
        h.upload(*st)
        h.upload_temperature(T0)
        h.upload_scalar(1, S0)
    n = (g.Prnx, g.Prny, g.Prnz)
    assert np.array_equal(b.field(FIELD_TEMPERATURE), a.field(FIELD_TEMPERATURE))
    assert np.array_equal(b.scalar(1), a.scalar(1))
    a.project(1.0)
    b.project(1.0)
    a.step(3)
    sb = b.step(3)
    tol = (1e-12, 1e-11, 1e-11) if precision == 0 else (1e-5, 1e-5, 1e-5)
    e = _errs(b.download(), a.download())
    et = rel(interior(b.field(FIELD_TEMPERATURE), -2, n) - 295.0, interior(a.field(FIELD_TEMPERATURE), -2, n) - 295.0)
    es = rel(interior(b.scalar(1), -2, n), interior(a.scalar(1), -2, n))
    print("temperature and scalar, slabs vs single domain:", precision, split, e, et, es)
    assert max(e[:3]) < tol[0] and e[3] < tol[1] and et < tol[2] and es < tol[2], (e, et, es)
    assert sb.max_div < (1e-10 if precision == 0 else 1e-6)
    a.close()
    b.close()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("bc", ["warm-surface", "heated-smooth", "flux-dirichlet-top"])
def test_slabs_carry_temperature_boundaries(precision, bc):
    """The temperature's boundary kinds on split domains: a prescribed
    surface temperature at the rough bottom (the Monin-Obukhov Dirichlet
    wall model on the bottom slab), a heat flux at a smooth bottom, and a
    heat flux at the bottom under a Dirichlet top by the ghost rule (the top
    slab's ghost plane), there with a passive scalar between a Neumann
    bottom and a Dirichlet top.  Two slabs against the single domain after the
    projection and three steps: FP64 U, V, W within 1e-12, P within 1e-11,
    theta - T_ref within 1e-11; mixed within 1e-5."""
    from gpu_elmm_b200.config import BC_CONSTFLUX, BC_DIRICHLET, BC_NEUMANN, FIELD_TEMPERATURE
    from gpu_elmm_b200.workloads import interior, puff_state, temperature_state
    kw = {"warm-surface": dict(temperature_bc=((BC_DIRICHLET, 296.0), (BC_CONSTFLUX, 0.0))),
          "heated-smooth": dict(heat_flux=(0.3, 0.0), z0=0.0),
          "flux-dirichlet-top": dict(temperature_bc=((BC_CONSTFLUX, 0.2), (BC_DIRICHLET, 295.5)), num_scalars=1,
                                     scalar_bc=((BC_NEUMANN, -0.01), (BC_DIRICHLET, 0.5)))}[bc]
    cfg = make_config(*N, precision=precision, buoyancy=True, **kw)
    g = grid_of(cfg)
    st = log_profile_state(g, seed=9)
    T0 = temperature_state(g, seed=9, amp=0.2)
    a, b = L.Domain(cfg), L.Slabs(cfg, 2, devices=[0, 0])
    for h in (a, b):
        h.upload(*st)
        h.upload_temperature(T0)
        if cfg.num_scalars:
            h.upload_scalar(1, puff_state(g, (20, 14, 12), sigma=3.0))
    n = (g.Prnx, g.Prny, g.Prnz)
    a.project(1.0)
    b.project(1.0)
    a.step(3)
    b.step(3)
    tol = (1e-12, 1e-11, 1e-11) if precision == 0 else (1e-5, 1e-5, 1e-5)
    e = _errs(b.download(), a.download())
    et = rel(interior(b.field(FIELD_TEMPERATURE), -2, n) - 295.0, interior(a.field(FIELD_TEMPERATURE), -2, n) - 295.0)
    print("temperature boundaries, slabs vs single domain:", bc, precision, e, et)
    assert max(e[:3]) < tol[0] and e[3] < tol[1] and et < tol[2], (e, et)
    if cfg.num_scalars:
        es = rel(interior(b.scalar(1), -2, n), interior(a.scalar(1), -2, n))
        print("  scalar with a Neumann bottom and a Dirichlet top:", es)
        assert es < tol[2], es
    a.close()
    b.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_slabs_carry_puffs_and_slices(precision):
    """A passive scalar with a puff that restarts and clears the field, a
    second puff volume in the other slab, and both time-averaged slices (the
    xy level in the upper slab, the xz slice across both): 3 slabs against
    the single domain after 8 steps, FP64 within 1e-11, mixed within 1e-5."""
    from gpu_elmm_b200.workloads import interior, puff_state
    cfg = make_config(*N, precision=precision, num_scalars=1, avg_slice_k=17, avg_slice_j=9, avg_weight=0.1)
    g = grid_of(cfg)
    st = log_profile_state(g, seed=5)
    S0 = puff_state(g, (20, 14, 12), sigma=3.0)
    puffs = [(0.0, 1.0, 0.06, 0.03, 1)]
    vols = [(0, 1, (20, 14, 20), 3.0), (0, 1, (9, 20, 4), 1.5)]
    a, b = L.Domain(cfg), L.Slabs(cfg, 3, devices=[0] * 3, nz=(6, 10, 8))
    for h in (a, b):
        h.upload(*st)
        h.upload_scalar(1, S0)
        h.project(1.0)
        h.set_puffs(puffs, vols)
        h.step(8)
    n = (g.Prnx, g.Prny, g.Prnz)
    tol = 1e-11 if precision == 0 else 1e-5
    es = rel(interior(b.scalar(1), -2, n), interior(a.scalar(1), -2, n))
    ex = [rel(x, y) for x, y in zip(b.scalar_slices(1), a.scalar_slices(1))]
    print("puffs and slices, slabs vs single domain:", precision, es, ex)
    assert es < tol and max(ex) < tol and np.abs(a.scalar_slices(1)[0]).max() > 0, (es, ex)
    a.close()
    b.close()
