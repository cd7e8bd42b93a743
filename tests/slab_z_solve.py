"""The z solve of a domain split into z-slabs, restated with numpy: the
algorithm of k_slab_tri_pivots / k_slab_tri_fmap / k_slab_tri_fwd /
k_slab_tri_bwd (gpu_elmm_b200/csrc/elmm_slabs.cuh), written for ranks that
each hold one slab and exchange through a gather callback.  Test code: the
world-size-2 gloo test runs it on two CPU ranks against the oracle's Poisson
solve (the tridiagonal z system of src/poisson.f90:23-60 behind FFTs in x
and y).

Per (kx, ky) column the Thomas sweeps are affine recurrences,
    y(k) = r(k) iv(k) - Ab(k) iv(k) y(k-1),   x(k) = y(k) - At(k) iv(k) x(k+1),
so a slab maps its entry value to its exit value with two numbers per
column (A, B), and the slabs exchange only those maps.  The (0,0) column is
gathered whole and solved by every slab with the zero-mean prefix sums.
"""
import numpy as np


def z_coefficients(zW):
    """Ab, At, dzc, dzf (index 1..nz) of a z grid with faces zW[0..nz], the
    centre ghosts mirrored at the walls."""
    zW = np.asarray(zW, float)
    nz = len(zW) - 1
    zP = np.empty(nz + 2)
    zP[1:nz + 1] = (zW[:-1] + zW[1:]) / 2
    zP[0] = zW[0] - (zP[1] - zW[0])
    zP[nz + 1] = zW[nz] + (zW[nz] - zP[nz])
    Ab, At, dzc, dzf = (np.zeros(nz + 2) for _ in range(4))
    for k in range(1, nz + 1):
        Ab[k] = 1 / ((zP[k] - zP[k - 1]) * (zW[k] - zW[k - 1]))
        At[k] = 1 / ((zP[k + 1] - zP[k]) * (zW[k] - zW[k - 1]))
        dzc[k] = zW[k] - zW[k - 1]
        dzf[k] = zP[k + 1] - zP[k]
    Ab[1] = 0
    At[nz] = 0
    return Ab, At, dzc, dzf


def eigenvalues(nx, ny, dx, dy):
    """lam[ky, kx] of the half spectrum; the (0,0) entry is the zero mode."""
    lx = -4 * np.sin(np.pi * np.arange(nx // 2 + 1) / nx) ** 2 / dx ** 2
    ly = -4 * np.sin(np.pi * np.arange(ny) / ny) ** 2 / dy ** 2
    return ly[:, None] + lx[None, :]


def slab_pivots(lam, Ab, At, k0, nzl):
    """Reciprocal pivots of levels k0+1..k0+nzl, from the whole column's
    recurrence (zero for the zero mode)."""
    mode = np.ones(lam.shape, bool)
    mode[0, 0] = False
    lamm = np.where(mode, lam, 0.0)
    c = np.zeros(lam.shape)
    iv = np.zeros((nzl,) + lam.shape)
    for k in range(1, k0 + nzl + 1):
        den = (-(Ab[k] + At[k]) + lamm) - (Ab[k] * c if k > 1 else 0.0)
        v = np.where(mode, 1.0 / np.where(mode, den, 1.0), 0.0)
        c = At[k] * v
        if k > k0:
            iv[k - k0 - 1] = v
    return iv


def run_rank(r_hat, lam, Ab, At, dzc, dzf, k0, nzg, rank, gather):
    """x_hat of this rank's levels.  r_hat: (nzl, ny, nx/2+1) complex, the
    transformed right-hand side of levels k0+1..k0+nzl; rank: the slab index;
    gather(obj) returns every rank's obj in slab order."""
    nzl = r_hat.shape[0]
    ab, at = Ab[k0 + 1:k0 + nzl + 1], At[k0 + 1:k0 + nzl + 1]
    iv = slab_pivots(lam, Ab, At, k0, nzl)
    A = np.zeros(lam.shape, complex)
    B = np.ones(lam.shape)
    for k in range(nzl):
        b = -ab[k] * iv[k]
        A = r_hat[k] * iv[k] + b * A
        B = b * B
    fmaps = gather((A, B, r_hat[:, 0, 0].copy()))
    # the exact entry from the slabs below, forward replay, backward map
    y = np.zeros(lam.shape, complex)
    for q in range(rank):
        y = fmaps[q][0] + fmaps[q][1] * y
    Y = np.empty_like(r_hat)
    A2 = np.zeros(lam.shape, complex)
    G = np.ones(lam.shape)
    for k in range(nzl):
        y = r_hat[k] * iv[k] - ab[k] * iv[k] * y
        Y[k] = y
        A2 = A2 + G * y
        G = G * (-at[k] * iv[k])
    bmaps = gather((A2, G))
    x = np.zeros(lam.shape, complex)
    for q in range(len(bmaps) - 1, rank, -1):
        x = bmaps[q][0] + bmaps[q][1] * x
    X = np.empty_like(r_hat)
    for k in range(nzl - 1, -1, -1):
        x = Y[k] - at[k] * iv[k] * x
        X[k] = x
    # the zero mode from the whole gathered column
    r0 = np.concatenate([m[2] for m in fmaps])
    F, xx, sx = 0.0, 0.0, 0.0
    x0 = np.zeros(nzg, complex)
    for k in range(1, nzg):
        F = F + r0[k - 1] * dzc[k]
        x0[k - 1] = xx
        sx += xx
        xx = xx + F * dzf[k]
    sx += xx
    sx = sx / nzg
    x0[:nzg - 1] -= sx
    x0[nzg - 1] = xx - sx
    X[:, 0, 0] = x0[k0:k0 + nzl]
    return X
