"""Immersed solid bodies (an array of cubes on a stretched grid with a mean
pressure gradient).

CPU: the geometry pass of gpu_elmm_b200/solids.py (the point lists of
GetSolidBodiesBC / SetNullifiedPoints for boxes) has the properties the
reference's construction gives them, and the oracle keeps the solid interior
at rest.  GPU: the library, given the same lists, follows the oracle
(IBMomentum, IBMassSources, NullInterior, the ScalFl viscosity and the
wall-model fluxes at the solid faces) on the FP64 path to 1e-11, and the
mixed path follows the FP64 one; so does a passive scalar among the bodies
(no advection tendency in the solid cells, the wall-model div * S of the
cells next to them)."""
import numpy as np
import pytest

from conftest import rel
from gpu_elmm_b200.config import grid_of, make_config
from gpu_elmm_b200.solids import build_solids, cube_array
from gpu_elmm_b200.workloads import interiors, log_profile_state
from oracle import Oracle

NZ = 24
ZW = np.concatenate([[0.0], np.cumsum(0.5 * 1.04 ** np.arange(NZ))])  # dz_k = 0.5 * 1.04^(k-1)


def _cfg(precision=0, n=(48, 48, NZ)):
    return make_config(*n, zW=ZW, pr_gradient_x=-0.001, precision=precision)


def _boxes():
    # 2 x 2 cubes of 8 cells at a 24-cell pitch, 8 levels tall, set 5 units into the ground
    return cube_array(2, 8.0, 24.0, float(ZW[8]), offset=8.0, depth=5.0)


def _state(cfg, seed=1):
    g = grid_of(cfg)
    return g, log_profile_state(g, seed=seed, zW=ZW)


def test_geometry_lists():
    cfg = _cfg()
    s = build_solids(cfg, _boxes())
    g = s.geometry
    c = s.counts()
    assert min(c["ib"]) > 0 and min(c["null"]) > 0 and c["scalfl"] > 0 and c["wm"] > 0
    for q in range(3):
        t = g.types[q + 1]
        for (i, j, k), pts, cf in s.ib[q]:
            assert t[k + 2, j + 2, i + 2] > 0  # forcing points are solid
            assert len(pts) == len(cf) <= 6
            for (a, b, cc) in pts:
                assert t[cc + 2, b + 2, a + 2] <= 0  # interpolation points are free
            if pts:  # the fit through zero at the wall extrapolates: weights of the other sign
                assert all(w < 0 for w in cf)
        for (i, j, k) in s.null[q]:
            assert t[k + 2, j + 2, i + 2] > 0
            for d in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
                assert t[k + d[2] + 2, j + d[1] + 2, i + d[0] + 2] > 0
    # every solid point of the interior is either an IB point or nullified
    for q in range(3):
        (nx, ny, nz) = g.grids[q + 1][0]
        solid = int((g.types[q + 1][3:nz + 3, 3:ny + 3, 3:nx + 3] > 0).sum())
        assert solid == len(s.ib[q]) + len(s.null[q])
    for comp, dr, i, j, k, dv, z0, _ in s.wm:
        assert g.typ(comp, i, j, k) < 0 and z0 == 0.1
        assert np.linalg.norm(dv) > 0
    # the ground next to and under the cubes has no wall-model point
    for q in range(3):
        for i, j in s.bottom_skip[q]:
            assert g.typ(q + 1, i, j, 1) != 0 or g.typ(q + 1, i, j, 0) > 0


def test_oracle_keeps_the_interior_at_rest():
    cfg = _cfg()
    s = build_solids(cfg, _boxes())
    g, st = _state(cfg)
    o = Oracle(cfg)
    o.set_state(*st)
    o.project(1.0)
    o.set_solids(s)
    md, _ = o.step(3)
    U, V, W, _ = o.state()
    assert md < 1e-12  # div U - Q after the projection
    for F, nl in zip((U, V, W), s.null):
        assert np.abs(F[nl[:, 2] + 2, nl[:, 1] + 2, nl[:, 0] + 2]).max() == 0
    assert np.isfinite(U).all() and np.abs(U).max() < 20


def _pair(precision, nsteps):
    from gpu_elmm_b200 import lib as L
    cfg = _cfg(precision)
    s = build_solids(cfg, _boxes())
    g, st = _state(cfg)
    o = Oracle(_cfg(0))
    o.set_state(*st)
    o.project(1.0)
    o.set_solids(s)
    d = L.Domain(cfg)
    d.upload(*st)
    d.project(1.0)
    d.set_solids(s)
    md_o, _ = o.step(nsteps)
    sd = d.step(nsteps)
    out = d.download()
    d.close()
    return g, out, o.state(), sd, md_o


@pytest.mark.gpu
@pytest.mark.parametrize("nsteps", [1, 5])
def test_fp64_cubes_match_the_oracle(nsteps):
    g, gpu, orc, sd, md_o = _pair(0, nsteps)
    e = [rel(a, b) for a, b in zip(interiors(g, *gpu), interiors(g, *orc))]
    print("FP64 errors with cubes after", nsteps, "steps (U, V, W, P):", e, "max div", sd.max_div, md_o)
    assert max(e[:3]) < 1e-11 and e[3] < 1e-10, e
    assert sd.max_div < 1e-10


@pytest.mark.gpu
def test_mixed_cubes_follow_fp64():
    g, m, _, sd, _ = _pair(1, 3)
    _, f, _, _, _ = _pair(0, 3)
    e = [rel(a, b) for a, b in zip(interiors(g, *m)[:3], interiors(g, *f)[:3])]
    print("mixed vs FP64 with cubes after 3 steps (U, V, W):", e, "max div", sd.max_div)
    assert max(e) < 1e-5, e
    assert sd.max_div < 1e-5


@pytest.mark.gpu
def test_set_solids_rejects_what_it_cannot_apply():
    """elmm_set_solids refuses (ELMM_ERR_INVALID_ARG = 6) lists it could not
    apply exactly: a forcing point next to a periodic boundary, an
    interpolation point that is itself a forcing point, a negative
    roughness length; None removes the bodies again."""
    from gpu_elmm_b200 import lib as L
    cfg = _cfg()
    s = build_solids(cfg, _boxes())
    g, st = _state(cfg)
    d = L.Domain(cfg)
    d.upload(*st)
    d.project(1.0)

    def code(sol):
        try:
            d.set_solids(sol)
            return 0
        except L.ElmmError as e:
            return e.code

    bad = build_solids(cfg, _boxes())
    (i, j, k), pts, cf = bad.ib[0][0]
    bad.ib[0][0] = ((1, j, k), pts, cf)
    assert code(bad) == 6
    bad = build_solids(cfg, _boxes())
    first = next(p for p in bad.ib[0] if p[1])
    other = bad.ib[0][1][0]
    bad.ib[0][0] = (first[0], [other] + first[1][1:], first[2])
    assert code(bad) == 6
    bad = build_solids(cfg, _boxes())
    c, dr, i, j, k, dv, z0, tf = bad.wm[0]
    bad.wm[0] = (c, dr, i, j, k, dv, -1.0, tf)
    assert code(bad) == 6
    assert code(s) == 0 and code(None) == 0 and code(s) == 0
    d.step(1)
    d.close()


@pytest.mark.gpu
def test_fp64_cubes_on_a_uniform_grid():
    """The same bodies on a uniform grid (the wall-model fluxes scale with
    1/dz instead of the stretched-grid factors; cubes of different heights,
    one of them 3 cells wide) against the oracle after 3 steps."""
    from gpu_elmm_b200 import lib as L
    from gpu_elmm_b200.solids import Box
    cfg = make_config(40, 36, 20, pr_gradient_x=-2e-3)
    boxes = [Box(6.0, 14.0, 5.0, 13.0, -3.0, 6.0), Box(22.0, 30.0, 20.0, 30.0, -3.0, 9.0),
             Box(31.0, 34.0, 6.0, 12.0, -3.0, 4.0)]
    s = build_solids(cfg, boxes)
    g = grid_of(cfg)
    st = log_profile_state(g, seed=9)
    o = Oracle(cfg)
    o.set_state(*st)
    o.project(1.0)
    o.set_solids(s)
    d = L.Domain(cfg)
    d.upload(*st)
    d.project(1.0)
    d.set_solids(s)
    o.step(3)
    sd = d.step(3)
    e = [rel(a, b) for a, b in zip(interiors(g, *d.download()), interiors(g, *o.state()))]
    print("FP64 errors with boxes on a uniform grid after 3 steps (U, V, W, P):", e)
    assert max(e[:3]) < 1e-11 and e[3] < 1e-10, e
    assert sd.max_div < 1e-10
    d.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_batch_with_cubes_and_puffs_equals_the_runs_alone(precision):
    """A batch of a cube-array domain (stretched grid) and a channel with a
    passive scalar and a puff: each domain's state after 4 steps is bit for
    bit the one it has alone (bodies and puffs are per domain)."""
    from gpu_elmm_b200 import lib as L
    cfg_c = _cfg(precision)
    sol = build_solids(cfg_c, _boxes())
    cfg_p = make_config(32, 24, 16, num_scalars=1, precision=precision)
    puffs = [(0.0, 1.0, 0.05, 0.03, 0)]
    vols = [(0, 1, (9, 7, 4), 2.0)]
    st_c = _state(cfg_c)[1]
    st_p = log_profile_state(grid_of(cfg_p), seed=6)
    b = L.Batch([cfg_c, cfg_p])
    b.upload(0, *st_c)
    b.upload(1, *st_p)
    b.project(1.0)
    b.set_solids(0, sol)
    b.set_puffs(1, puffs, vols)
    b.step(4)
    a = L.Domain(cfg_c)
    a.upload(*st_c)
    a.project(1.0)
    a.set_solids(sol)
    a.step(4)
    p = L.Domain(cfg_p)
    p.upload(*st_p)
    p.project(1.0)
    p.set_puffs(puffs, vols)
    p.step(4)
    for x, y in zip(a.download(), b.download(0)):
        assert np.array_equal(x, y)
    for x, y in zip(p.download(), b.download(1)):
        assert np.array_equal(x, y)
    assert np.array_equal(p.scalar(1), b.scalar(1, 1)) and np.abs(p.scalar(1)).max() > 0
    a.close()
    p.close()
    b.close()


def _spheres():
    # two spheres on the stretched grid: one sunk into the ground, one
    # standing free, centres off the grid lines
    from gpu_elmm_b200.solids import Sphere
    return [Sphere(14.3, 13.7, 1.1, 6.2), Sphere(33.6, 31.2, 6.4, 3.7, z0r=0.05)]


def test_sphere_geometry_lists():
    """Spheres (Sphere_Inside / Sphere_Closest): forcing points solid and
    interpolation points free, every interior solid point an IB point or
    nullified, the solid volume close to the spheres' volume, the wall-model
    points' distance vectors pointing from the free point towards the surface
    (within the surface's curvature) with each sphere's roughness."""
    cfg = _cfg()
    bodies = _spheres()
    s = build_solids(cfg, bodies)
    g = s.geometry
    c = s.counts()
    assert min(c["ib"]) > 0 and min(c["null"]) > 0 and c["scalfl"] > 0 and c["wm"] > 0
    for q in range(3):
        t = g.types[q + 1]
        for (i, j, k), pts, cf in s.ib[q]:
            assert t[k + 2, j + 2, i + 2] > 0
            for (a, b, cc) in pts:
                assert t[cc + 2, b + 2, a + 2] <= 0
        (nx, ny, nz) = g.grids[q + 1][0]
        solid = int((t[3:nz + 3, 3:ny + 3, 3:nx + 3] > 0).sum())
        assert solid == len(s.ib[q]) + len(s.null[q])
    # Pr cells inside, against the volume above the ground (cell volumes of the stretched grid)
    cz = g.c
    t0 = g.types[0]
    vol = 0.0
    for k in range(1, NZ + 1):
        dz = cz.x(cz.zW, k) - cz.x(cz.zW, k - 1)
        vol += float((t0[k + 2, 3:48 + 3, 3:48 + 3] > 0).sum()) * dz
    exact = 0.0
    import math
    for b in bodies:  # the part above z = 0 (a cap when the centre is near the ground)
        h = min(2 * b.r, b.r + b.zc)
        exact += math.pi * h * h * (3 * b.r - h) / 3
    assert abs(vol - exact) / exact < 0.15, (vol, exact)
    for comp, dr, i, j, k, dv, z0, _ in s.wm:
        assert g.typ(comp, i, j, k) < 0 and z0 in (0.1, 0.05)
        assert np.linalg.norm(dv) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ["spheres", "cylinders"])
def test_fp64_spheres_match_the_oracle(shape):
    """The same device path as the cubes, given the point lists of the
    spheres or of the cylinders: FP64 against the oracle after 3 steps, and
    the mixed path within 1e-5 of FP64."""
    from gpu_elmm_b200 import lib as L
    bodies = _spheres if shape == "spheres" else _cylinders
    out = {}
    for prec in (0, 1):
        cfg = _cfg(prec)
        s = build_solids(cfg, bodies())
        g, st = _state(cfg)
        d = L.Domain(cfg)
        d.upload(*st)
        d.project(1.0)
        d.set_solids(s)
        sd = d.step(3)
        out[prec] = (d.download(), sd.max_div)
        d.close()
    cfg = _cfg(0)
    s = build_solids(cfg, bodies())
    g, st = _state(cfg)
    o = Oracle(cfg)
    o.set_state(*st)
    o.project(1.0)
    o.set_solids(s)
    o.step(3)
    e = [rel(a, b) for a, b in zip(interiors(g, *out[0][0]), interiors(g, *o.state()))]
    em = [rel(a, b) for a, b in zip(interiors(g, *out[1][0])[:3], interiors(g, *out[0][0])[:3])]
    print(shape, ": FP64 vs oracle", e, "mixed vs FP64", em, "max div", out[0][1], out[1][1])
    assert max(e[:3]) < 1e-11 and e[3] < 1e-10 and out[0][1] < 1e-10, e
    assert max(em) < 1e-5 and out[1][1] < 1e-5, em


def _scalar_boxes_cfg(precision=0):
    return make_config(40, 36, 20, pr_gradient_x=-2e-3, num_scalars=1, precision=precision,
                       point_sources=[(1, (20.5, 16.5, 3.5), 2.0)])


def _scalar_boxes():
    from gpu_elmm_b200.solids import Box
    return [Box(6.0, 14.0, 5.0, 13.0, -3.0, 6.0), Box(22.0, 30.0, 20.0, 30.0, -3.0, 9.0),
            Box(31.0, 34.0, 6.0, 12.0, -3.0, 4.0)]


def test_scalar_lists_of_the_bodies():
    """The Pr lists for the scalars: the solid cells are the Prtype > 0
    cells, the z ghost layers included; the wall-model points are the free cells with a solid
    6-neighbour (GetSolidBodiesWM) and the bottom cells with Prtype == 0
    (GetOutsideBoundariesWM_Pr), each once, none of them solid."""
    cfg = _scalar_boxes_cfg()
    s = build_solids(cfg, _scalar_boxes())
    g = s.geometry
    nx, ny, nz = cfg.Prnx, cfg.Prny, cfg.Prnz
    t = g.types[0]
    T = lambda i, j, k: int(t[k + 2, j + 2, i + 2])
    solid = {tuple(p) for p in s.solid_pr.tolist()}
    assert len(solid) == len(s.solid_pr) == int((t[1:nz + 5, 3:ny + 3, 3:nx + 3] > 0).sum())
    assert all(T(i, j, k) > 0 and -1 <= k <= nz + 2 for (i, j, k) in solid)
    assert any(k < 1 for (_, _, k) in solid)    # the boxes reach below the ground
    wm = [tuple(p) for p in s.wm_pr.tolist()]
    assert len(wm) == len(set(wm)) and not (set(wm) & solid)
    for (i, j, k) in wm:
        near = any(T(i + a, j + b, k + c) > 0 for a, b, c in
                   ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)))
        assert T(i, j, k) <= 0 and (near or (k == 1 and T(i, j, k) == 0))
    bottom = sum(1 for j in range(1, ny + 1) for i in range(1, nx + 1) if T(i, j, 1) == 0)
    assert sum(1 for p in wm if p[2] == 1) >= bottom > 0


def _scalar_pair(precision=0):
    """The oracle and a library domain of the given precision, both from the
    same seeded state and puff, projected, then given the bodies."""
    from gpu_elmm_b200 import lib as L
    from gpu_elmm_b200.config import FIELD_SCALAR
    from gpu_elmm_b200.workloads import puff_state
    cfg = _scalar_boxes_cfg(precision)
    s = build_solids(cfg, _scalar_boxes())
    g = grid_of(cfg)
    st = log_profile_state(g, seed=9)
    S0 = puff_state(g, (18, 17, 4), sigma=3.0)
    o = Oracle(_scalar_boxes_cfg(0))
    o.set_state(*st)
    o.set_field(FIELD_SCALAR, S0)
    o.project(1.0)
    o.set_solids(s)
    d = L.Domain(cfg)
    d.upload(*st)
    d.upload_scalar(1, S0)
    d.project(1.0)  # the scalar diffusivity of the initial eddy viscosity, kept without buoyancy
    d.set_solids(s)
    return g, o, d


@pytest.mark.gpu
@pytest.mark.parametrize("nsteps", [1, 5])
def test_fp64_passive_scalar_among_boxes(nsteps):
    """A passive scalar (a puff and a continuous point source) among boxes on
    a uniform grid: no advection tendency in the solid cells
    (src/scalars.f90:259-268), and the wall-model points of the scalar, the
    free cells next to a body and the bottom cells under none, add div * S
    without the faces towards solid cells (DivergenceWM,
    src/wallmodels.f90:1150-1166).  FP64 against the oracle: U, V, W within
    1e-11, P within 1e-10, the scalar within 1e-11."""
    from gpu_elmm_b200.config import FIELD_SCALAR
    from gpu_elmm_b200.workloads import interior
    g, o, d = _scalar_pair()
    o.step(nsteps)
    d.step(nsteps)
    e = [rel(a, b) for a, b in zip(interiors(g, *d.download()), interiors(g, *o.state()))]
    n = (g.Prnx, g.Prny, g.Prnz)
    es = rel(interior(d.scalar(1), -2, n), interior(o.get_field(FIELD_SCALAR), -2, n))
    print("passive scalar among boxes, FP64 vs oracle after", nsteps, "steps:", e, es)
    assert max(e[:3]) < 1e-11 and e[3] < 1e-10 and es < 1e-11, (e, es)
    d.close()


@pytest.mark.gpu
def test_mixed_passive_scalar_among_boxes():
    from gpu_elmm_b200.workloads import interior
    g, _, d64 = _scalar_pair(0)
    _, _, dm = _scalar_pair(1)
    d64.step(3)
    dm.step(3)
    n = (g.Prnx, g.Prny, g.Prnz)
    e = [rel(a, b) for a, b in zip(interiors(g, *dm.download())[:3], interiors(g, *d64.download())[:3])]
    es = rel(interior(dm.scalar(1), -2, n), interior(d64.scalar(1), -2, n))
    print("passive scalar among boxes, mixed vs FP64 after 3 steps:", e, es)
    assert max(e) < 1e-5 and es < 1e-5, (e, es)
    d64.close()
    dm.close()


def _heated_boxes():
    from gpu_elmm_b200.solids import Box
    return [Box(6.0, 14.0, 5.0, 13.0, -3.0, 6.0, heat_flux=0.3), Box(22.0, 30.0, 20.0, 30.0, -3.0, 9.0),
            Box(31.0, 34.0, 6.0, 12.0, -3.0, 4.0, heat_flux=0.15)]


def _theta_pair(precision=0, heated=False, **ground):
    """The oracle and a library domain with the potential temperature among
    the boxes (adiabatic walls; with heated, two of them give off heat),
    from the same state, projected, then given the bodies."""
    from gpu_elmm_b200 import lib as L
    from gpu_elmm_b200.config import FIELD_TEMPERATURE
    from gpu_elmm_b200.workloads import temperature_state
    mk = lambda p: make_config(40, 36, 20, pr_gradient_x=-2e-3, buoyancy=True, precision=p, **ground)
    cfg = mk(precision)
    s = build_solids(cfg, _heated_boxes() if heated else _scalar_boxes())
    g = grid_of(cfg)
    st = log_profile_state(g, seed=4)
    T0 = temperature_state(g, seed=4, gradient=0.02, amp=0.2)
    o = Oracle(mk(0))
    o.set_state(*st)
    o.set_field(FIELD_TEMPERATURE, T0)
    o.project(1.0)
    o.set_solids(s)
    d = L.Domain(cfg)
    d.upload(*st)
    d.upload_temperature(T0)
    d.project(1.0)
    d.set_solids(s)
    return g, o, d


@pytest.mark.gpu
@pytest.mark.parametrize("nsteps", [1, 5])
def test_fp64_temperature_among_boxes(nsteps):
    """The potential temperature among boxes: no advection tendency in the
    solid cells, the wall-model div * theta of the cells next to them, and
    after each stage the fill of the solid cells with the mean of their
    fluid neighbours (src/scalars.f90:129-198; cells deep inside a body
    keep their value, as in the reference).  FP64 against the oracle: U, V,
    W within 1e-11, P within 1e-10, theta - T_ref within 1e-11."""
    from gpu_elmm_b200.config import FIELD_TEMPERATURE
    from gpu_elmm_b200.workloads import interior
    g, o, d = _theta_pair()
    o.step(nsteps)
    d.step(nsteps)
    e = [rel(a, b) for a, b in zip(interiors(g, *d.download()), interiors(g, *o.state()))]
    n = (g.Prnx, g.Prny, g.Prnz)
    et = rel(interior(d.field(FIELD_TEMPERATURE), -2, n) - 295.0, interior(o.get_field(FIELD_TEMPERATURE), -2, n) - 295.0)
    print("temperature among boxes, FP64 vs oracle after", nsteps, "steps:", e, et)
    assert max(e[:3]) < 1e-11 and e[3] < 1e-10 and et < 1e-11, (e, et)
    d.close()


@pytest.mark.gpu
def test_mixed_temperature_among_boxes():
    from gpu_elmm_b200.config import FIELD_TEMPERATURE
    from gpu_elmm_b200.workloads import interior
    g, _, d64 = _theta_pair(0)
    _, _, dm = _theta_pair(1)
    d64.step(3)
    dm.step(3)
    n = (g.Prnx, g.Prny, g.Prnz)
    e = [rel(a, b) for a, b in zip(interiors(g, *dm.download())[:3], interiors(g, *d64.download())[:3])]
    et = rel(interior(dm.field(FIELD_TEMPERATURE), -2, n) - 295.0, interior(d64.field(FIELD_TEMPERATURE), -2, n) - 295.0)
    print("temperature among boxes, mixed vs FP64 after 3 steps:", e, et)
    assert max(e) < 1e-5 and et < 1e-5, (e, et)
    d64.close()
    dm.close()


def test_heated_face_points():
    """The heated Pr wall-model points: free cells next to a heated rough
    body, q = flux x area factor (1/dz for a face below or above the cell,
    1/dx and 1/dy beside it on this grid), none next to the unheated body;
    the velocity points of a heated body carry its flux."""
    cfg = make_config(40, 36, 20, buoyancy=True)
    s = build_solids(cfg, _heated_boxes())
    g = s.geometry
    assert len(s.heat_pr) > 0
    for (i, j, k, q) in s.heat_pr:
        assert g.typ(0, i, j, k) <= 0 and q in (0.3, 0.15), (i, j, k, q)   # unit cells: area factor 1
    assert {tf for *_, tf in s.wm} == {0.0, 0.3, 0.15}


@pytest.mark.gpu
@pytest.mark.parametrize("ground", ["adiabatic", "heat-flux", "surface-temperature"])
def test_heated_boxes_on_a_heated_ground(ground):
    """Heated bodies on a ground with a surface heat flux or a surface
    temperature: the bottom cells next to a body keep the wall point or the
    solid-face point (the closer; the solid one on a tie), and the kept
    point's flux enters.  FP64 against the oracle after 3 steps: U, V, W
    within 1e-11, P within 1e-10, theta - T_ref within 1e-11."""
    from gpu_elmm_b200.config import BC_CONSTFLUX, BC_DIRICHLET, FIELD_TEMPERATURE
    from gpu_elmm_b200.workloads import interior
    kw = {"adiabatic": {}, "heat-flux": {"heat_flux": (0.2, 0.0)},
          "surface-temperature": {"temperature_bc": ((BC_DIRICHLET, 296.0), (BC_CONSTFLUX, 0.0))}}[ground]
    g, o, d = _theta_pair(heated=True, **kw)
    o.step(3)
    d.step(3)
    e = [rel(a, b) for a, b in zip(interiors(g, *d.download()), interiors(g, *o.state()))]
    n = (g.Prnx, g.Prny, g.Prnz)
    et = rel(interior(d.field(FIELD_TEMPERATURE), -2, n) - 295.0, interior(o.get_field(FIELD_TEMPERATURE), -2, n) - 295.0)
    print("heated boxes on a", ground, "ground, FP64 vs oracle:", e, et)
    assert max(e[:3]) < 1e-11 and e[3] < 1e-10 and et < 1e-11, (e, et)
    d.close()


@pytest.mark.gpu
@pytest.mark.parametrize("nsteps", [1, 5])
def test_fp64_heated_boxes(nsteps):
    """Heated bodies: the heat flux of the Pr wall-model points at their
    faces enters the temperature, and the velocity points of their faces
    take the Monin-Obukhov u* (WM_MO_FluxStress).  FP64 against the oracle:
    U, V, W within 1e-11, P within 1e-10, theta - T_ref within 1e-11; the
    mixed path within 1e-5 of FP64 after 3 steps."""
    from gpu_elmm_b200.config import FIELD_TEMPERATURE
    from gpu_elmm_b200.workloads import interior
    g, o, d = _theta_pair(heated=True)
    o.step(nsteps)
    d.step(nsteps)
    e = [rel(a, b) for a, b in zip(interiors(g, *d.download()), interiors(g, *o.state()))]
    n = (g.Prnx, g.Prny, g.Prnz)
    Td = interior(d.field(FIELD_TEMPERATURE), -2, n) - 295.0
    et = rel(Td, interior(o.get_field(FIELD_TEMPERATURE), -2, n) - 295.0)
    print("heated boxes, FP64 vs oracle after", nsteps, "steps:", e, et)
    assert max(e[:3]) < 1e-11 and e[3] < 1e-10 and et < 1e-11, (e, et)
    if nsteps == 5:
        _, _, dm = _theta_pair(1, heated=True)
        dm.step(5)
        em = [rel(a, b) for a, b in zip(interiors(g, *dm.download())[:3], interiors(g, *d.download())[:3])]
        etm = rel(interior(dm.field(FIELD_TEMPERATURE), -2, n) - 295.0, Td)
        print("heated boxes, mixed vs FP64:", em, etm)
        assert max(em) < 1e-5 and etm < 1e-5, (em, etm)
        dm.close()
    d.close()


@pytest.mark.gpu
@pytest.mark.parametrize("top", ["heat-flux", "temperature"])
def test_temperature_among_boxes_under_a_ghost_rule_top(top):
    """A free-slip top without wall-model points that carries a heat flux or
    a prescribed temperature by CommonBase's ghost rules, above boxes that
    stay clear of it: FP64 against the oracle after 3 steps (U, V, W within
    1e-11, P within 1e-10, theta - T_ref within 1e-11), the mixed path
    within 1e-5 of FP64.  A body up to the
    top face is refused with ELMM_ERR_INVALID_ARG (its velocity points
    above the body lie outside the domain; the library also refuses a fill
    that would read the ghost cell of such a side)."""
    from gpu_elmm_b200 import lib as L
    from gpu_elmm_b200.config import BC_CONSTFLUX, BC_DIRICHLET, FIELD_TEMPERATURE
    from gpu_elmm_b200.solids import Box
    from gpu_elmm_b200.workloads import interior
    kw = {"heat-flux": {"heat_flux": (0.0, 0.1)},
          "temperature": {"temperature_bc": ((BC_CONSTFLUX, 0.0), (BC_DIRICHLET, 296.0))}}[top]
    g, o, d = _theta_pair(**kw)
    o.step(3)
    d.step(3)
    e = [rel(a, b) for a, b in zip(interiors(g, *d.download()), interiors(g, *o.state()))]
    n = (g.Prnx, g.Prny, g.Prnz)
    et = rel(interior(d.field(FIELD_TEMPERATURE), -2, n) - 295.0, interior(o.get_field(FIELD_TEMPERATURE), -2, n) - 295.0)
    print("boxes under a", top, "top, FP64 vs oracle:", e, et)
    assert max(e[:3]) < 1e-11 and e[3] < 1e-10 and et < 1e-11, (e, et)
    _, _, dm = _theta_pair(1, **kw)
    dm.step(3)
    em = [rel(a, b) for a, b in zip(interiors(g, *dm.download())[:3], interiors(g, *d.download())[:3])]
    etm = rel(interior(dm.field(FIELD_TEMPERATURE), -2, n) - 295.0, interior(d.field(FIELD_TEMPERATURE), -2, n) - 295.0)
    print("boxes under a", top, "top, mixed vs FP64:", em, etm)
    assert max(em) < 1e-5 and etm < 1e-5, (em, etm)
    dm.close()
    d.close()
    cfg = make_config(40, 36, 20, buoyancy=True, **kw)
    d = L.Domain(cfg)
    with pytest.raises(L.ElmmError) as e:
        d.set_solids(build_solids(cfg, [Box(6.0, 14.0, 5.0, 13.0, -3.0, 20.0)]))   # up to the top face
    assert e.value.code == 6, e.value
    d.close()


@pytest.mark.gpu
def test_batch_with_a_scalar_among_boxes_equals_the_run_alone():
    """The scalar's cell mask is per domain: a batch of the scalar-and-boxes
    domain and a channel without bodies gives each its state alone, bit for
    bit (mixed path)."""
    from gpu_elmm_b200 import lib as L
    from gpu_elmm_b200.workloads import puff_state
    cfg_s = _scalar_boxes_cfg(1)
    sol = build_solids(cfg_s, _scalar_boxes())
    cfg_p = make_config(32, 24, 16, num_scalars=1, precision=1)
    gs, gp = grid_of(cfg_s), grid_of(cfg_p)
    st_s, st_p = log_profile_state(gs, seed=9), log_profile_state(gp, seed=6)
    S_s, S_p = puff_state(gs, (18, 17, 4), sigma=3.0), puff_state(gp, (9, 7, 4))
    b = L.Batch([cfg_s, cfg_p])
    b.upload(0, *st_s)
    b.upload(1, *st_p)
    b.upload_scalar(0, 1, S_s)
    b.upload_scalar(1, 1, S_p)
    b.project(1.0)
    b.set_solids(0, sol)
    b.step(3)
    _, _, a = _scalar_pair(1)
    a.step(3)
    p = L.Domain(cfg_p)
    p.upload(*st_p)
    p.upload_scalar(1, S_p)
    p.project(1.0)
    p.step(3)
    for x, y in zip(a.download(), b.download(0)):
        assert np.array_equal(x, y)
    assert np.array_equal(a.scalar(1), b.scalar(0, 1))
    for x, y in zip(p.download(), b.download(1)):
        assert np.array_equal(x, y)
    assert np.array_equal(p.scalar(1), b.scalar(1, 1))
    a.close()
    p.close()
    b.close()


def _cylinders():
    # a vertical cylinder sunk into the ground and a horizontal one lying
    # free in y, axes off the grid lines; unit-length caps would make the
    # cap distances exact, these are longer
    from gpu_elmm_b200.solids import Cylinder
    return [Cylinder((14.3, 13.7, -3.0), (14.3, 13.7, 6.0), 4.2),
            Cylinder((33.6, 24.0, 7.3), (33.6, 38.0, 7.3), 3.1, z0r=0.05)]


def test_cylinder_geometry_lists():
    """Cylinders (Cylinder_Inside / _Closest / _ClosestOut): forcing points
    solid and interpolation points free, every interior solid point an IB
    point or nullified, the solid volume above the ground close to the
    cylinders' volume, each cylinder's roughness on its wall-model points."""
    import math
    cfg = _cfg()
    bodies = _cylinders()
    s = build_solids(cfg, bodies)
    g = s.geometry
    c = s.counts()
    assert min(c["ib"]) > 0 and min(c["null"]) > 0 and c["scalfl"] > 0 and c["wm"] > 0
    for q in range(3):
        t = g.types[q + 1]
        for (i, j, k), pts, cf in s.ib[q]:
            assert t[k + 2, j + 2, i + 2] > 0
            for (a, b, cc) in pts:
                assert t[cc + 2, b + 2, a + 2] <= 0
        (nx, ny, nz) = g.grids[q + 1][0]
        assert int((t[3:nz + 3, 3:ny + 3, 3:nx + 3] > 0).sum()) == len(s.ib[q]) + len(s.null[q])
    cz = g.c
    t0 = g.types[0]
    vol = 0.0
    for k in range(1, NZ + 1):
        dz = cz.x(cz.zW, k) - cz.x(cz.zW, k - 1)
        vol += float((t0[k + 2, 3:48 + 3, 3:48 + 3] > 0).sum()) * dz
    exact = math.pi * 4.2 ** 2 * 6.0 + math.pi * 3.1 ** 2 * 14.0
    assert abs(vol - exact) / exact < 0.15, (vol, exact)
    for comp, dr, i, j, k, dv, z0, _ in s.wm:
        assert g.typ(comp, i, j, k) < 0 and z0 in (0.1, 0.05) and np.linalg.norm(dv) > 0


def test_cylinder_closest_points_as_written():
    """The jacket's closest point is the radial projection; a cap's closest
    point moves by the signed distance times the unnormalised cap normal
    (Plane_Closest, src/geometricshapes.f90:644-660), exact for a cylinder
    of unit length and |p2 - p1| times the distance otherwise."""
    from gpu_elmm_b200.solids import Cylinder
    c = Cylinder((10.0, 10.0, 0.0), (10.0, 10.0, 1.0), 3.0)
    assert c.closest(15.0, 10.0, 0.5) == (13.0, 10.0, 0.5)
    assert c.closest(10.2, 10.0, 5.0) == (10.2, 10.0, 1.0)
    assert c.closest_out(10.2, 10.0, 0.9) == (10.2, 10.0, 1.0)
    assert c.inside(12.9, 10.0, 0.5, 0.0) and not c.inside(10.0, 10.0, 1.2, 0.0)
    long = Cylinder((10.0, 10.0, 0.0), (10.0, 10.0, 4.0), 3.0)
    x, y, z = long.closest(10.2, 10.0, 5.0)
    assert (x, y) == (10.2, 10.0) and abs(z - (5.0 - 4.0 * 1.0)) < 1e-12   # 4 x the distance 1 below
