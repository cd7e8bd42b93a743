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


def _buoyant_channel(seed=0, n=(16, 12, 10)):
    from gpu_elmm_b200.config import FIELD_TEMPERATURE, grid_of, make_config
    from gpu_elmm_b200.workloads import log_profile_state, temperature_state
    cfg = make_config(*n, buoyancy=True)
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
