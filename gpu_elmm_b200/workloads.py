"""Seeded synthetic inputs of the benchmark configurations.

The reference has no generator for these fields (its only random numbers live
in the turbulent-inlet code, src/turbinlet.f90), so the project defines one:

* counter-based: value = splitmix64(key(seed, field) XOR linear index), the
  linear index being the Fortran linear index of the interior cell
  (i-1) + n1*((j-1) + n2*(k-1)) of that velocity component;
* uniform in [0, 1) from the top 53 bits, scaled to +-amplitude;
* every value is rounded to FP32, because the reference reads initial fields
  from float32 VTK files (src/initial.f90:3674-3710).

Arrays are numpy arrays in the reference's Fortran layout, stored as
(k, j, i) C-order so that x is contiguous: U(-2:Unx+3, -2:Uny+3, -2:Unz+3) is
``U[k+2, j+2, i+2]``; Pr(-1:Prnx+2, ...) is ``Pr[k+1, j+1, i+1]``.
"""
from __future__ import annotations

import numpy as np

from .config import Grid

_MASK = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64, copy=True)
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        z = x
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


FIELD_KEYS = {"u": 1, "v": 2, "w": 3, "theta": 4, "ustar": 5, "sizes": 6, "requests": 7, "arrivals": 8}


def uniform(seed: int, field: str, n: int) -> np.ndarray:
    """n uniform numbers in [0, 1) of stream (seed, field)."""
    key = (np.uint64(seed & 0xFFFFFFFF) << np.uint64(24)) ^ (np.uint64(FIELD_KEYS[field]) << np.uint64(56))
    idx = np.arange(n, dtype=np.uint64)
    r = splitmix64(idx ^ key)
    return (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def zpr_of(grid: Grid, dz: float, zmin: float = 0.0, zW=None) -> np.ndarray:
    """zPr(1:Prnz), src/initial.f90:4452-4455."""
    if zW is not None:
        zW = np.asarray(zW, dtype=np.float64)
        return (zW[:-1] + zW[1:]) / 2.0
    k = np.arange(1, grid.Prnz + 1, dtype=np.float64)
    zw = k * dz + zmin
    zwm = (k - 1) * dz + zmin
    return (zwm + zw) / 2.0


def log_profile_state(grid: Grid, *, seed=0, ustar=0.3, z0=0.01, amp=0.1, dz=1.0,
                      zmin=0.0, zW=None):
    """u = (u*/0.41) ln(zPr/z0) + U(-amp, amp), v, w = U(-amp, amp), each
    rounded to FP32; returns host arrays (U, V, W, Pr) with zero ghosts."""
    g = grid
    U = np.zeros(g.shape_u())
    V = np.zeros(g.shape_v())
    W = np.zeros(g.shape_w())
    Pr = np.zeros(g.shape_p())
    zpr = zpr_of(g, dz, zmin, zW)
    nu_ = g.Unx * g.Uny * g.Unz
    ru = uniform(seed, "u", nu_).reshape(g.Unz, g.Uny, g.Unx)
    prof = (ustar / 0.41) * np.log(zpr[: g.Unz] / z0)
    interior(U, -2, (g.Unx, g.Uny, g.Unz))[...] = prof[:, None, None] + amp * (2.0 * ru - 1.0)
    rv = uniform(seed, "v", g.Vnx * g.Vny * g.Vnz).reshape(g.Vnz, g.Vny, g.Vnx)
    interior(V, -2, (g.Vnx, g.Vny, g.Vnz))[...] = amp * (2.0 * rv - 1.0)
    rw = uniform(seed, "w", g.Wnx * g.Wny * g.Wnz).reshape(g.Wnz, g.Wny, g.Wnx)
    interior(W, -2, (g.Wnx, g.Wny, g.Wnz))[...] = amp * (2.0 * rw - 1.0)
    for a in (U, V, W):
        a[...] = a.astype(np.float32).astype(np.float64)
    return U, V, W, Pr


def temperature_state(grid: Grid, *, seed=0, t0=295.0, gradient=0.01, amp=0.05, dz=1.0, zmin=0.0, zW=None):
    """Potential temperature theta = t0 + gradient * zPr + U(-amp, amp), rounded
    to FP32; returns the host array Temperature(-2:nx+3,-2:ny+3,-2:nz+3) with
    zero ghosts (the library fills them)."""
    g = grid
    T = np.zeros(g.shape_t())
    zpr = zpr_of(g, dz, zmin, zW)
    r = uniform(seed, "theta", g.cells()).reshape(g.Prnz, g.Prny, g.Prnx)
    interior(T, -2, (g.Prnx, g.Prny, g.Prnz))[...] = (t0 + gradient * zpr[: g.Prnz])[:, None, None] + \
        amp * (2.0 * r - 1.0)
    T[...] = T.astype(np.float32).astype(np.float64)
    return T


def puff_state(grid: Grid, center, *, sigma=2.0, amp=1.0):
    """A Gaussian puff of passive scalar, amp exp(-r^2 / (2 sigma^2)) with r
    the distance in cells from the centre cell (i, j, k), the shortest
    periodic distance along x and y; rounded to FP32.  Returns the host array
    Scalar(-2:nx+3,-2:ny+3,-2:nz+3) with zero ghosts."""
    g = grid
    S = np.zeros(g.shape_t())
    ci, cj, ck = center

    def dist(idx, c, n, periodic):
        d = np.abs(idx - c).astype(np.float64)
        return np.minimum(d, n - d) if periodic else d

    di = dist(np.arange(1, g.Prnx + 1), ci, g.Prnx, True)
    dj = dist(np.arange(1, g.Prny + 1), cj, g.Prny, True)
    dk = dist(np.arange(1, g.Prnz + 1), ck, g.Prnz, False)
    r2 = dk[:, None, None] ** 2 + dj[None, :, None] ** 2 + di[None, None, :] ** 2
    interior(S, -2, (g.Prnx, g.Prny, g.Prnz))[...] = amp * np.exp(-r2 / (2.0 * sigma * sigma))
    S[...] = S.astype(np.float32).astype(np.float64)
    return S


# dispersion requests of the serving workload: horizontal sides and depths
REQUEST_SIDES = (64, 96, 128, 192)
REQUEST_DEPTHS = (64, 96)


def dispersion_request(seed: int, index: int, *, min_steps=200, max_steps=2000):
    """Request `index` of stream `seed`: a channel of s x s x nz cells
    (s from REQUEST_SIDES, nz from REQUEST_DEPTHS, so 64^3 .. 192x192x96),
    min_steps..max_steps steps, and the interior cell (i, j, k) of its
    continuous point source, which is also the centre of the initial puff
    (k in 2..nz-1, away from the walls).  Returns a dict."""
    r = uniform(seed, "requests", 8 * (index + 1))[8 * index:8 * index + 8]
    s = REQUEST_SIDES[int(r[0] * len(REQUEST_SIDES))]
    nz = REQUEST_DEPTHS[int(r[1] * len(REQUEST_DEPTHS))]
    steps = min_steps + int(r[2] * (max_steps - min_steps + 1))
    i = 1 + int(r[3] * s)
    j = 1 + int(r[4] * s)
    k = 2 + int(r[5] * (nz - 2))
    return {"n": (s, s, nz), "steps": steps, "source": (i, j, k), "seed": seed * 1000003 + index}


def poisson_arrivals(seed: int, rate: float, count: int) -> np.ndarray:
    """Arrival times (s) of a Poisson process of the given rate: cumulative
    exponential gaps -ln(1 - U) / rate."""
    u = uniform(seed, "arrivals", count)
    return np.cumsum(-np.log1p(-u) / rate)


def interior(a: np.ndarray, lo: int, n: tuple) -> np.ndarray:
    """Interior view a(1:nx,1:ny,1:nz) of a Fortran-layout array with lower bound lo."""
    nx, ny, nz = n
    o = 1 - lo
    return a[o:o + nz, o:o + ny, o:o + nx]


def interiors(grid: Grid, U, V, W, Pr):
    g = grid
    return (interior(U, -2, (g.Unx, g.Uny, g.Unz)), interior(V, -2, (g.Vnx, g.Vny, g.Vnz)),
            interior(W, -2, (g.Wnx, g.Wny, g.Wnz)), interior(Pr, -1, (g.Prnx, g.Prny, g.Prnz)))


def taylor_green_2d(grid: Grid, *, dx: float, dy: float, amp=1.0):
    """2D Taylor-Green field of task_type=2 (src/initial.f90:3900-3941):
    U = -cos(pi x) sin(pi y), V = sin(pi x) cos(pi y) on the staggered points,
    P = -(cos(2 pi x) + cos(2 pi y))/4; a domain of side 2 in x and y."""
    g = grid
    U = np.zeros(g.shape_u())
    V = np.zeros(g.shape_v())
    W = np.zeros(g.shape_w())
    Pr = np.zeros(g.shape_p())
    xu = np.arange(1, g.Unx + 1) * dx
    yu = (np.arange(1, g.Uny + 1) - 0.5) * dy
    xv = (np.arange(1, g.Vnx + 1) - 0.5) * dx
    yv = np.arange(1, g.Vny + 1) * dy
    xp = (np.arange(1, g.Prnx + 1) - 0.5) * dx
    yp = (np.arange(1, g.Prny + 1) - 0.5) * dy
    uu = -amp * np.cos(np.pi * xu)[None, :] * np.sin(np.pi * yu)[:, None]
    vv = amp * np.sin(np.pi * xv)[None, :] * np.cos(np.pi * yv)[:, None]
    pp = -(amp ** 2) * (np.cos(2 * np.pi * xp)[None, :] + np.cos(2 * np.pi * yp)[:, None]) / 4
    interior(U, -2, (g.Unx, g.Uny, g.Unz))[...] = uu[None]
    interior(V, -2, (g.Vnx, g.Vny, g.Vnz))[...] = vv[None]
    interior(Pr, -1, (g.Prnx, g.Prny, g.Prnz))[...] = pp[None]
    return U, V, W, Pr


# ------------------------------------------------ the array of cubes
# 384 x 384 x 96 cells, dx = dy = 1, dz_k = 0.5 * 1.04^(k-1) (z extent ~527),
# 8 x 8 cubes of 16 cells (16 levels tall) at a 48-cell pitch, rough (z0 =
# 0.1), driven by a uniform mean pressure gradient in x
CUBES_N = (384, 384, 96)
CUBES_PR_GRADIENT_X = -2e-4


def stretched_zw(nz: int, first: float = 0.5, ratio: float = 1.04) -> np.ndarray:
    """zW(0:nz) of the geometrically stretched grid, dz_k = first * ratio^(k-1)."""
    return np.concatenate([[0.0], np.cumsum(first * ratio ** np.arange(nz))])


def cubes_config(precision=0, device=0, n=CUBES_N, **kw):
    from .config import make_config
    return make_config(*n, zW=stretched_zw(n[2]), pr_gradient_x=CUBES_PR_GRADIENT_X, precision=precision,
                       device=device, **kw)


def cubes_boxes(n=CUBES_N, per_side=8, edge=16.0, pitch=48.0, levels=16):
    """The solid bodies: cubes from x, y = 16 + 48 a to 32 + 48 a and from
    below the ground up to zW(levels)."""
    from .solids import cube_array
    zw = stretched_zw(n[2])
    return cube_array(per_side, edge, pitch, float(zw[levels]), offset=(pitch - edge) / 2, depth=5.0)
