"""Known answers for the oracle: ghost-cell rules, the divergence after a
projection, and the viscous decay of the 2D Taylor-Green field of
task_type=2 (src/initial.f90:3900-3941)."""
import numpy as np
import pytest

from conftest import rel
from gpu_elmm_b200.config import (BC_FREESLIP, BC_NEUMANN, BC_NOSLIP, BC_PERIODIC, grid_of, make_config)
from gpu_elmm_b200.workloads import interiors, log_profile_state, taylor_green_2d
from oracle import Oracle


def fold(g, n, blo, bhi, normal):
    """Per-dimension ghost rule of BoundUVW_do_BC (src/boundaries.f90:398-1791)."""
    if 1 <= g <= n:
        return g, 1, False
    if g < 1:
        b = blo
        if b == BC_PERIODIC:
            return n + g, 1, False
        if b in (BC_NOSLIP, BC_FREESLIP) and normal:
            return (1, 1, True) if g == 0 else (-g, -1, False)
        if b == BC_NOSLIP:
            return 1 - g, -1, False
        return 1, 1, False
    b = bhi
    if b == BC_PERIODIC:
        return g - n, 1, False
    if b in (BC_NOSLIP, BC_FREESLIP) and normal:
        return (n, 1, True) if g == n + 1 else (2 * n + 2 - g, -1, False)
    if b == BC_NOSLIP:
        return 2 * n + 1 - g, -1, False
    return n, 1, False


@pytest.mark.parametrize("bt", [(3, 3, 3, 3, 1, 2), (3, 3, 3, 3, 1, 1), (3, 3, 3, 3, 3, 3), (3, 3, 3, 3, 5, 2)])
def test_ghost_cells_fold_per_dimension(bt):
    """The sequential x, y, z passes of BoundUVW equal a per-dimension fold;
    the CUDA kernels rely on this."""
    cfg = make_config(8, 6, 5, btype=bt)
    g = grid_of(cfg)
    o = Oracle(cfg)
    rng = np.random.default_rng(2)
    st = [rng.standard_normal(s) for s in (g.shape_u(), g.shape_v(), g.shape_w(), g.shape_p())]
    o.set_state(*st)
    o.bound()
    U, V, W, _ = o.state()
    for comp, (F, ext) in enumerate(((U, (g.Unx, g.Uny, g.Unz)), (V, (g.Vnx, g.Vny, g.Vnz)), (W, (g.Wnx, g.Wny, g.Wnz)))):
        for k in range(-2, ext[2] + 4):
            for j in range(-2, ext[1] + 4):
                for i in range(-2, ext[0] + 4):
                    fx = fold(i, ext[0], bt[0], bt[1], comp == 0)
                    fy = fold(j, ext[1], bt[2], bt[3], comp == 1)
                    fz = fold(k, ext[2], bt[4], bt[5], comp == 2)
                    want = 0.0 if (fx[2] or fy[2] or fz[2]) else fx[1] * fy[1] * fz[1] * F[fz[0] + 2, fy[0] + 2, fx[0] + 2]
                    assert F[k + 2, j + 2, i + 2] == want, (comp, i, j, k)


def test_projection_is_divergence_free():
    cfg = make_config(32, 24, 16)
    g = grid_of(cfg)
    o = Oracle(cfg)
    o.set_state(*log_profile_state(g, seed=0))
    assert o.project(1.0) < 1e-13
    md, _ = o.step(2)
    assert md < 1e-13


def test_taylor_green_decay():
    """Small-amplitude 2D Taylor-Green vortex on a periodic box of side 2:
    with Smagorinsky off, each mode decays at the rate of the discrete
    Laplacian, exp(-nu * 2 * (4/dx^2) sin^2(pi dx / 2) * t)."""
    n, L = 32, 2.0
    dx = L / n
    nu, dt, steps = 0.05, 0.002, 50
    cfg = make_config(n, n, 4, btype=(3, 3, 3, 3, 3, 3), dx=dx, dy=dx, dz=dx, dt=dt, nu=nu, sgstype=0)
    g = grid_of(cfg)
    amp = 1e-4
    U, V, W, P = taylor_green_2d(g, dx=dx, dy=dx, amp=amp)
    o = Oracle(cfg)
    o.set_state(U, V, W, P)
    o.step(steps)
    Ui, Vi, _, _ = interiors(g, *o.state())
    U0, V0, _, _ = interiors(g, U, V, W, P)
    lam = 2 * (4 / dx ** 2) * np.sin(np.pi * dx / 2) ** 2
    decay = np.exp(-nu * lam * dt * steps)
    assert rel(Ui, U0 * decay) < 1e-6
    assert rel(Vi, V0 * decay) < 1e-6


def _buoyant_channel(seed=0, n=(16, 12, 10), **kw):
    from gpu_elmm_b200.config import FIELD_TEMPERATURE, grid_of, make_config
    from gpu_elmm_b200.workloads import log_profile_state, temperature_state
    cfg = make_config(*n, buoyancy=True, **kw)
    g = grid_of(cfg)
    o = Oracle(cfg)
    o.set_state(*log_profile_state(g, seed=seed))
    o.set_field(FIELD_TEMPERATURE, temperature_state(g, seed=seed))
    o.project(1.0)
    return g, o


def test_temperature_heat_is_conserved():
    """Adiabatic (zero-flux) walls and periodic x, y: KappaScalar and the
    diffusion are in flux form, so the heat content only changes by the
    wall-model divergence term, which is of the size of the discrete
    divergence (~1e-15) times theta."""
    from gpu_elmm_b200.config import FIELD_TEMPERATURE
    from gpu_elmm_b200.workloads import interior
    g, o = _buoyant_channel()
    n = (g.Prnx, g.Prny, g.Prnz)
    h0 = interior(o.get_field(FIELD_TEMPERATURE), -2, n).sum()
    o.step(5)
    T = interior(o.get_field(FIELD_TEMPERATURE), -2, n)
    assert np.isfinite(T).all()
    assert abs(T.sum() - h0) / abs(h0) < 1e-12
    # the run did transport heat: the field changed
    assert np.abs(T - T.mean()).max() > 0


def test_buoyancy_vanishes_for_the_reference_temperature():
    """theta = temperature_ref everywhere: the FD2 buoyancy term
    A/2 (T(k+1) + T(k)) - A T_ref vanishes, so the flow equals the run without
    the temperature field up to the rounding of (W + g) - g in the reference's
    order of operations."""
    from gpu_elmm_b200.config import FIELD_TEMPERATURE, grid_of, make_config
    from gpu_elmm_b200.workloads import log_profile_state
    cfg0 = make_config(16, 12, 10)
    cfg1 = make_config(16, 12, 10, buoyancy=True)
    g = grid_of(cfg0)
    st = log_profile_state(g, seed=3)
    a, b = Oracle(cfg0), Oracle(cfg1)
    a.set_state(*st)
    b.set_state(*st)
    b.set_field(FIELD_TEMPERATURE, np.full(g.shape_t(), 295.0))
    a.project(1.0)
    b.project(1.0)
    a.step(2)
    b.step(2)
    for x, y, tol in zip(a.state(), b.state(), (1e-12, 1e-12, 1e-12, 1e-11)):  # P: conditioning floor
        assert rel(x, y) < tol


def _dispersion_channel(n=(16, 12, 10), source=(5, 7, 4), flux=2.5, steps=0, seed=0, avg=True):
    """A channel with one passive scalar: a Gaussian puff around the source
    cell and a continuous point source at its centre."""
    from gpu_elmm_b200.config import FIELD_SCALAR, grid_of, make_config
    from gpu_elmm_b200.workloads import log_profile_state, puff_state
    i, j, k = source
    pos = (i - 0.5, j - 0.5, k - 0.5)  # the cell centre (dx = dy = dz = 1, origin 0)
    cfg = make_config(*n, num_scalars=1, point_sources=[(1, pos, flux)],
                      avg_slice_k=k if avg else 0, avg_slice_j=j if avg else 0,
                      avg_weight=1.0 / steps if steps else 0.0)
    g = grid_of(cfg)
    o = Oracle(cfg)
    o.set_state(*log_profile_state(g, seed=seed))
    o.set_field(FIELD_SCALAR, puff_state(g, source))
    o.project(1.0)
    return cfg, g, o


def test_point_source_adds_its_flux():
    """Zero-flux walls and periodic x, y: the scalar content changes only by
    the point source, flux * dt per step (the RK3 weights of a stage sum to
    one over a step), and by the wall-model divergence term (~1e-15)."""
    from gpu_elmm_b200.config import FIELD_SCALAR
    from gpu_elmm_b200.workloads import interior
    flux, nsteps = 2.5, 4
    cfg, g, o = _dispersion_channel(flux=flux)
    n = (g.Prnx, g.Prny, g.Prnz)
    m0 = interior(o.get_field(FIELD_SCALAR), -2, n).sum()  # cell volume 1
    o.step(nsteps)
    S = interior(o.get_field(FIELD_SCALAR), -2, n)
    assert np.isfinite(S).all()
    assert abs((S.sum() - m0) - flux * cfg.dt * nsteps) < 1e-11 * max(1.0, abs(m0))


def test_scalar_averages_are_the_mean_of_the_steps():
    """The time-averaged slices equal the mean, over the steps, of the
    scalar's slice planes after each step (avg_weight = 1 / steps)."""
    from gpu_elmm_b200.config import FIELD_SCALAR
    from gpu_elmm_b200.workloads import interior
    nsteps, src = 3, (5, 7, 4)
    cfg, g, o = _dispersion_channel(steps=nsteps, source=src)
    n = (g.Prnx, g.Prny, g.Prnz)
    xy, xz = np.zeros((g.Prny, g.Prnx)), np.zeros((g.Prnz, g.Prnx))
    for _ in range(nsteps):
        o.step(1)
        S = interior(o.get_field(FIELD_SCALAR), -2, n)
        xy += S[src[2] - 1] / nsteps
        xz += S[:, src[1] - 1, :] / nsteps
    axy, axz = o.scalar_slices(1)
    assert rel(axy, xy) < 1e-14 and rel(axz, xz) < 1e-14
    assert np.abs(axy).max() > 0


def test_scalar_diffusivity_is_set_once_without_buoyancy():
    """Without buoyancy TDiff is computed once, after the initial projection
    (src/initial.f90:4296-4313), and then kept: ComputeTDiff runs per stage
    only with buoyancy (src/dynamics.f90:904)."""
    from gpu_elmm_b200.config import FIELD_TDIFF, FIELD_VISCOSITY
    from gpu_elmm_b200.workloads import interior
    cfg, g, o = _dispersion_channel()
    n = (g.Prnx, g.Prny, g.Prnz)
    nu = interior(o.get_field(FIELD_VISCOSITY), -1, n)
    td0 = interior(o.get_field(FIELD_TDIFF), -1, n).copy()
    want = (nu - cfg.molecular_viscosity) / 0.6 + cfg.molecular_diffusivity
    assert rel(td0, want) < 1e-15
    o.step(2)
    assert np.array_equal(interior(o.get_field(FIELD_TDIFF), -1, n), td0)
    assert not np.array_equal(interior(o.get_field(FIELD_VISCOSITY), -1, n), nu)


def test_point_source_cell_follows_gridcoords():
    """GridCoords on a uniform grid: nint((x - xU(0)) / dx + 0.5), clamped; a
    point outside the domain adds no source."""
    from gpu_elmm_b200.config import FIELD_SCALAR, grid_of, make_config
    from gpu_elmm_b200.workloads import interior
    n = (8, 8, 6)
    for pos, cell in (((2.2, 3.9, 1.0), (3, 4, 1)), ((7.99, 0.0, 5.5), (8, 1, 6))):
        cfg = make_config(*n, num_scalars=1, point_sources=[(1, pos, 1.0)], sgstype=0, wallmodeltype=0)
        g = grid_of(cfg)
        o = Oracle(cfg)
        o.set_state(np.zeros(g.shape_u()), np.zeros(g.shape_v()), np.zeros(g.shape_w()))
        o.step(1)
        S = interior(o.get_field(FIELD_SCALAR), -2, n)
        i, j, k = cell
        assert S[k - 1, j - 1, i - 1] > 0 and np.count_nonzero(S) > 0
    cfg = make_config(*n, num_scalars=1, point_sources=[(1, (9.5, 1.0, 1.0), 1.0)], sgstype=0, wallmodeltype=0)
    o = Oracle(cfg)
    o.set_state(np.zeros(g.shape_u()), np.zeros(g.shape_v()), np.zeros(g.shape_w()))
    o.step(1)
    assert np.count_nonzero(o.get_field(FIELD_SCALAR)) == 0


def test_puff_windows_follow_prepare_puffs():
    """The oracle's PreparePuffs / DoPuffs (src/puffs.f90:30-126) on one
    scalar: the amount a puff adds per step is dt_fraction * flux * dt (the
    RK3 weights sum to one), with dt_fraction as the reference computes it,
    including the restart branch's `time + dt - max(...) / dt` (negative, so
    nothing is added, on a restart after t = 0), and `clear` empties the
    scalar at each release."""
    import numpy as np
    from gpu_elmm_b200.config import grid_of, make_config
    from gpu_elmm_b200.workloads import interior
    from oracle import Oracle
    cfg = make_config(16, 12, 8, num_scalars=2, sgstype=0, wallmodeltype=0)
    g = grid_of(cfg)
    o = Oracle(cfg)
    z = [np.zeros(s) for s in (g.shape_u(), g.shape_v(), g.shape_w(), g.shape_p())]
    o.set_state(*z)
    o.set_puffs([(0.03, 0.5, 0.1, 0.05, 1), (0.0, 1.0, 10.0, 0.07, 0)],
                [(0, 1, (5, 6, 3), 2.0), (0, 1, (6, 6, 3), 1.0), (1, 2, (10, 7, 4), 3.0)])
    n = (g.Prnx, g.Prny, g.Prnz)
    sums = []
    for _ in range(9):
        o.step(1)
        sums.append((interior(o.get_field(16), -2, n).sum(), interior(o.get_field(17), -2, n).sum()))
    s1 = [round(a, 10) for a, _ in sums]
    s2 = [round(b, 10) for _, b in sums]
    # puff 1 (once, 0.07 long from t = 0): fraction 0.02 (restart at t = 0), 1, 1, 0.5, then 0
    assert s2 == [0.0012, 0.0612, 0.1212, 0.1512, 0.1512, 0.1512, 0.1512, 0.1512, 0.1512]
    # puff 0: release at t = 0.02 (negative fraction), full steps at 0.04, 0.06, then closed;
    # cleared at the next release (t = 0.12, the 7th step)
    assert s1 == [0.0, 0.0, 0.06, 0.12, 0.12, 0.12, 0.0, 0.06, 0.12]


def test_smooth_wall_ustar_follows_the_log_law():
    """A smooth bottom wall (z0 = 0, WMFlatStress): for a uniform flow U = 5
    every diffusive and advective flux vanishes except the wall flux, so the
    U tendency of the first level is -u*^2 / dz.  Its u* satisfies the law of
    WMFlatUstar (src/wallmodels.f90:1190-1240) in the logarithmic layer,
    u = u* (ln(z+)/0.4 + 5.5), to the iteration's tolerance (1e-4); a rough
    wall gives u* = 0.41 u / ln(z/z0) instead (WMRoughUstar)."""
    import math
    nu, dz, vel = 1.0 / 70000, 0.5, 5.0
    cfg = make_config(16, 12, 8, dz=dz, z0=0.0, nu=nu)
    g = grid_of(cfg)
    U, V, W, Pr = (np.zeros(s) for s in (g.shape_u(), g.shape_v(), g.shape_w(), g.shape_p()))
    U[...] = vel
    o = Oracle(cfg)
    o.set_state(U, V, W, Pr)
    o.run_stage(1, 2)                       # SGS with the wall fluxes, then the momentum tendency
    tend = o.get_field(8)[2 + 1, 2 + 1:2 + 1 + g.Uny, 2 + 1:2 + 1 + g.Unx]   # Ustar(:, :, 1)
    assert np.ptp(tend) == 0 and tend.max() < 0
    us = math.sqrt(-tend.max() * dz)
    zpl = (dz / 2) * us / nu
    assert zpl > 30                         # the logarithmic branch
    assert abs(vel / us - (math.log(zpl) / 0.4 + 5.5)) / (vel / us) < 1e-3
    o2 = Oracle(make_config(16, 12, 8, dz=dz, z0=1e-4, nu=nu))
    o2.set_state(U, V, W, Pr)
    o2.run_stage(1, 2)
    us2 = math.sqrt(-o2.get_field(8)[3, 3, 3] * dz)
    assert abs(us2 - vel * 0.41 / math.log((dz / 2) / 1e-4)) < 1e-12


@pytest.mark.parametrize("heat_flux", [(0.2, 0.0), (-0.1, 0.05)], ids=["heated", "cooled-with-top-flux"])
def test_surface_heat_flux_enters_through_the_wall_points(heat_flux):
    """A constant surface heat flux at a wall-model wall (TempBtype
    CONSTFLUX, which becomes the flux of the side's wall-model points,
    src/wallmodels.f90:590-627): the heat content grows by
    (q_bottom - q_top) Lx Ly per unit time (RK3's weights add to one per
    step), up to the wall-model divergence term.  The top here is a second
    wall-model wall."""
    from gpu_elmm_b200.config import FIELD_TEMPERATURE
    from gpu_elmm_b200.workloads import interior
    qb, qt = heat_flux
    g, o = _buoyant_channel(btype=(BC_PERIODIC,) * 4 + (BC_NOSLIP, BC_NOSLIP), heat_flux=heat_flux)
    n = (g.Prnx, g.Prny, g.Prnz)
    h0 = interior(o.get_field(FIELD_TEMPERATURE), -2, n).sum()      # cells of 1 m^3
    steps, dt = 4, 0.02
    o.step(steps)
    h1 = interior(o.get_field(FIELD_TEMPERATURE), -2, n).sum()
    expect = (qb - qt) * g.Prnx * g.Prny * dt * steps
    assert abs((h1 - h0) - expect) < 1e-9 * abs(expect) + 1e-12 * abs(h0)


def test_unstable_surface_flux_follows_monin_obukhov():
    """Uniform flow U over a rough bottom with a heat flux q > 0 into the
    flow (WM_MO_FluxStress, src/wallmodels.f90:1606-1660, 1836-1854): the U
    tendency of the first level is -u*^2 / dz.  u* is the reference's
    iteration from the initial u* = 1 (u* and z/L relaxed by halves until u*
    changes by less than 1e-3), restated here step by step; it stops within
    2% of the fixed point U = u*/0.4 (ln(z/z0) - PsiM(z/L)) with the
    Businger-Dyer PsiM and L = -u*^3 T_ref / (0.4 g q), found by bisection,
    and gives more drag than the neutral law with the same von Karman
    constant (0.4; the neutral WMRoughUstar uses 0.41).  A flux out of the
    flow keeps WMRoughUstar."""
    import math
    from gpu_elmm_b200.config import FIELD_TEMPERATURE
    from gpu_elmm_b200.workloads import temperature_state
    dz, vel, z0, tref, grav = 1.0, 5.0, 0.01, 295.0, 9.81

    def tendency_ustar(q):
        cfg = make_config(16, 12, 8, dz=dz, z0=z0, buoyancy=True, heat_flux=(q, 0.0))
        g = grid_of(cfg)
        U, V, W, Pr = (np.zeros(s) for s in (g.shape_u(), g.shape_v(), g.shape_w(), g.shape_p()))
        U[...] = vel
        o = Oracle(cfg)
        o.set_state(U, V, W, Pr)
        o.set_field(FIELD_TEMPERATURE, temperature_state(g, gradient=0.0, amp=0.0, t0=tref))
        o.run_stage(1, 2)
        tend = o.get_field(8)[2 + 1, 2 + 1:2 + 1 + g.Uny, 2 + 1:2 + 1 + g.Unx]
        assert np.ptp(tend) == 0 and tend.max() < 0
        return math.sqrt(-tend.max() * dz)

    def psim(zeta):
        if zeta < 0:
            x = (1 - 15 * zeta) ** 0.25
            return math.log((1 + x * x) / 2 * ((1 + x) / 2) ** 2) - 2 * math.atan(x) + math.pi / 2
        return -4.8 * zeta

    z = dz / 2
    neutral = vel * 0.41 / math.log(z / z0)
    assert abs(tendency_ustar(-0.3) - neutral) < 1e-12
    q = 0.3
    us = tendency_ustar(q)
    f32 = lambda v: float(np.float32(v))            # default-real literals of the reference
    u, zl, psi = 1.0, 0.0, 0.0
    for it in range(1, 51):
        u2 = u
        u = u + (max(vel * 0.4 / math.log(max(z / z0 - psi, f32(1e-5))), 0.0) - u) / 2
        zl = -10000.0 if u < f32(1e-4) else zl + (z * (0.4 * (grav / tref) * q) / -(u * u * u) - zl) / 2
        psi = psim(zl)
        if abs(u - u2) / max(abs(u), 1e-3) < f32(1e-3):
            break
    assert it > 3 and abs(us - u) < 1e-13, (us, u)
    # the fixed point of the similarity law, by bisection
    fp = lambda v: v - 0.4 * vel / (math.log(z / z0) - psim(z * 0.4 * (grav / tref) * q / -v ** 3))
    lo, hi = 0.05, 2.0
    for _ in range(200):
        mid = (lo + hi) / 2
        lo, hi = (mid, hi) if fp(lo) * fp(mid) > 0 else (lo, mid)
    assert abs(us - lo) / lo < 2e-2, (us, lo)
    assert us > 0.4 * vel / math.log(z / z0)      # more drag than the neutral law with its 0.4


def test_linear_temperature_profile_is_steady():
    """Fluid at rest with molecular diffusion only (no SGS model, so no
    wall model), theta linear in z with the gradient of a Neumann bottom and
    the value of a Dirichlet top at the top face (CommonBase BC_NEUMANN and
    BC_DIRICHLET, src/scalarboundaries.f90:203-288): the ghost rules continue
    the line, so the discrete Laplacian vanishes, and the buoyancy of a
    z-only field is a gradient the projection removes; theta stays as it
    is."""
    from gpu_elmm_b200.config import BC_DIRICHLET, FIELD_TEMPERATURE
    from gpu_elmm_b200.workloads import interior
    n, gam, top = (16, 12, 10), 0.01, 300.0
    cfg = make_config(*n, sgstype=0, buoyancy=True, temperature_bc=((BC_NEUMANN, gam), (BC_DIRICHLET, top)))
    g = grid_of(cfg)
    U, V, W, Pr = (np.zeros(s) for s in (g.shape_u(), g.shape_v(), g.shape_w(), g.shape_p()))
    T = np.zeros(g.shape_t())
    zpr = np.arange(1, n[2] + 1) - 0.5
    interior(T, -2, n)[...] = (top + gam * (zpr - n[2]))[:, None, None]
    o = Oracle(cfg)
    o.set_state(U, V, W, Pr)
    o.set_field(FIELD_TEMPERATURE, T)
    o.project(1.0)
    o.step(3)
    T1 = interior(o.get_field(FIELD_TEMPERATURE), -2, n)
    assert np.abs(T1 - interior(T, -2, n)).max() < 1e-11
    assert np.abs(interiors(g, *o.state())[2]).max() < 1e-14


@pytest.mark.parametrize("field", ["temperature", "scalar"])
def test_ghost_rule_fluxes_change_the_content(field):
    """CommonBase's BC_CONSTFLUX ghost rule, arr(nz+1) = arr(nz) -
    q dzW(nz) / TDiff: a flux through the free-slip top of the temperature
    (a flux at a free-slip side has no wall-model points), or through both z
    sides of a passive scalar (the scalars keep the ghost rule at a
    wall-model wall too), changes the content by (q_bottom - q_top) Lx Ly
    per unit time."""
    from gpu_elmm_b200.config import BC_CONSTFLUX, FIELD_SCALAR, FIELD_TEMPERATURE
    from gpu_elmm_b200.workloads import interior, puff_state
    n = (16, 12, 10)
    if field == "temperature":
        (qb, qt), fid = (0.15, 0.05), FIELD_TEMPERATURE
        g, o = _buoyant_channel(n=n, temperature_bc=((BC_CONSTFLUX, qb), (BC_CONSTFLUX, qt)))
    else:
        (qb, qt), fid = (0.2, -0.1), FIELD_SCALAR
        cfg = make_config(*n, num_scalars=1, scalar_bc=((BC_CONSTFLUX, qb), (BC_CONSTFLUX, qt)))
        g = grid_of(cfg)
        o = Oracle(cfg)
        o.set_state(*log_profile_state(g, seed=2))
        o.set_field(FIELD_SCALAR, puff_state(g, (8, 6, 4)))
        o.project(1.0)
    h0 = interior(o.get_field(fid), -2, n).sum()
    steps, dt = 4, 0.02
    o.step(steps)
    h1 = interior(o.get_field(fid), -2, n).sum()
    expect = (qb - qt) * n[0] * n[1] * dt * steps
    assert abs((h1 - h0) - expect) < 1e-9 * abs(expect) + 1e-12 * abs(h0), (h1 - h0, expect)


@pytest.mark.parametrize("dtheta", [2.0, -2.0], ids=["warm-surface", "cool-surface"])
def test_surface_temperature_flux_follows_monin_obukhov(dtheta):
    """A prescribed surface temperature at a rough wall-model bottom
    (WM_MO_Dirichlet, src/wallmodels.f90:1664-1716, 1858-1884): for a
    uniform flow U over air at a uniform theta every other temperature flux
    vanishes, so the first level's temperature tendency is the wall-model
    flux q over dz (TemperatureExtra's temperature_flux * area_factor).
    q and u* solve the similarity laws of Zilitinkevich and Esau,
    u* = 0.4 U / (ln(z/z0) - PsiM(z/L)), q = -(theta - theta_s) 0.47 u* /
    (ln(z/z0) - PsiH(z/L)), z/L = -z g q / (0.4 T_ref u*^3), to the
    iteration's tolerance on z/L (1e-3); a warm surface heats the air and a
    cool one cools it."""
    import math
    from gpu_elmm_b200.config import BC_CONSTFLUX, BC_DIRICHLET, FIELD_TEMPERATURE, FIELD_TEMPERATURE_ADV
    from gpu_elmm_b200.workloads import temperature_state
    dz, vel, z0, tref, grav, ta = 1.0, 5.0, 0.01, 295.0, 9.81, 295.0
    cfg = make_config(16, 12, 8, dz=dz, z0=z0, buoyancy=True,
                      temperature_bc=((BC_DIRICHLET, ta + dtheta), (BC_CONSTFLUX, 0.0)))
    g = grid_of(cfg)
    U, V, W, Pr = (np.zeros(s) for s in (g.shape_u(), g.shape_v(), g.shape_w(), g.shape_p()))
    U[...] = vel
    o = Oracle(cfg)
    o.set_state(U, V, W, Pr)
    o.set_field(FIELD_TEMPERATURE, temperature_state(g, gradient=0.0, amp=0.0, t0=ta))
    o.run_stage(1, 2)
    tend = o.get_field(FIELD_TEMPERATURE_ADV)[2 + 1, 2 + 1:2 + 1 + g.Prny, 2 + 1:2 + 1 + g.Prnx]
    assert np.ptp(tend) == 0
    q = tend.max() * dz
    assert (q > 0) == (dtheta > 0)

    def psi(zeta):
        if zeta < 0:
            x = (1 - 6 * zeta * 0.4) ** 0.25
            return (math.log((1 + x * x) / 2 * ((1 + x) / 2) ** 2) - 2 * math.atan(x) + math.pi / 2,
                    2 * math.log((1 + x * x) / 2))
        return -3 * (zeta * 0.4) ** (5 / 6), -2.5 * (zeta * 0.4) ** 0.8

    z = dz / 2
    qq, us = 0.0, 0.4 * vel / math.log(z / z0)
    for _ in range(500):                      # the fixed point, by damped substitution
        zl = -z * grav * qq / (0.4 * tref * us ** 3)
        pm, ph = psi(zl)
        us = 0.5 * us + 0.5 * 0.4 * vel / (math.log(z / z0) - pm)
        qq = 0.5 * qq + 0.5 * (dtheta * us * 0.47 / (math.log(z / z0) - ph))
    assert abs(q - qq) / abs(qq) < 1e-2, (q, qq)
