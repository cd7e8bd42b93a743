"""The oracle's Poisson solve against a dense solve of the discrete operator
of Residue_variable_z (src/poisson.f90:23-60) with the ghost rules of
Bound_Phi (src/boundaries.f90:1817-1948)."""
import numpy as np
import pytest

from conftest import rel
from gpu_elmm_b200.config import BC_NOSLIP, BC_FREESLIP, BC_PERIODIC, make_config, grid_of
from oracle import Oracle


def dense_operator(nx, ny, nz, dx, dy, zW, zper):
    """Matrix of Lap(Phi) on the interior cells, x fastest."""
    zW = np.asarray(zW, float)
    zP = np.empty(nz + 2)
    zP[1:nz + 1] = (zW[:-1] + zW[1:]) / 2
    # ghost centres as the grid extension of src/initial.f90:4405-4432 gives them
    zP[0] = zW[0] - (zP[1] - zW[0])
    zP[nz + 1] = zW[nz] + (zW[nz] - zP[nz])
    N = nx * ny * nz
    A = np.zeros((N, N))
    idx = lambda i, j, k: (i % nx) + nx * ((j % ny) + ny * k)
    for k in range(nz):
        kk = k + 1
        Ab = 1 / ((zP[kk] - zP[kk - 1]) * (zW[kk] - zW[kk - 1]))
        At = 1 / ((zP[kk + 1] - zP[kk]) * (zW[kk] - zW[kk - 1]))
        for j in range(ny):
            for i in range(nx):
                r = idx(i, j, k)
                for (a, b) in ((1, 0), (-1, 0)):
                    A[r, idx(i + a, j, k)] += 1 / dx ** 2
                    A[r, r] -= 1 / dx ** 2
                for (a, b) in ((1, 0), (-1, 0)):
                    A[r, idx(i, j + a, k)] += 1 / dy ** 2
                    A[r, r] -= 1 / dy ** 2
                # z neighbours: Neumann ghost Phi(0)=Phi(1) makes the face term vanish
                if k > 0 or zper:
                    A[r, idx(i, j, (k - 1) % nz)] += Ab
                    A[r, r] -= Ab
                if k < nz - 1 or zper:
                    A[r, idx(i, j, (k + 1) % nz)] += At
                    A[r, r] -= At
    return A


@pytest.mark.parametrize("case", ["uniform", "stretched", "zperiodic"])
def test_poisson_matches_dense_solve(case):
    nx, ny, nz = 6, 4, 5
    btype = [BC_PERIODIC] * 4 + ([BC_PERIODIC] * 2 if case == "zperiodic" else [BC_NOSLIP, BC_FREESLIP])
    zW = None
    if case == "stretched":
        dz = 0.5 * 1.04 ** np.arange(nz)
        zW = np.concatenate([[0.0], np.cumsum(dz)])
    cfg = make_config(nx, ny, nz, btype=tuple(btype), dx=0.7, dy=1.3, dz=0.9, zW=zW, sgstype=0)
    g = grid_of(cfg)
    o = Oracle(cfg)
    rng = np.random.default_rng(0)
    r = rng.standard_normal((nz, ny, nx))
    # compatibility: zero flux-weighted mean
    zw = zW if zW is not None else np.arange(nz + 1) * 0.9
    w = np.diff(zw)
    r -= (r * w[:, None, None]).sum() / (w.sum() * nx * ny)
    RHS = np.zeros(g.shape_rhs())
    RHS[1:-1, 1:-1, 1:-1] = r
    Phi = o.poisson(RHS)[2:-2, 2:-2, 2:-2]
    A = dense_operator(nx, ny, nz, 0.7, 1.3, zw, case == "zperiodic")
    # residual of the oracle solution and agreement with the minimum-norm dense solve
    res = A @ Phi.ravel() - r.ravel()
    assert np.abs(res).max() < 1e-12 * np.abs(r).max() * 10
    x = np.linalg.lstsq(A, r.ravel(), rcond=None)[0]
    x -= x.mean()
    assert rel(Phi.ravel() - Phi.mean(), x) < 1e-12
    assert abs(Phi.mean()) < 1e-14


def test_poisson_residual_large():
    cfg = make_config(48, 32, 24, sgstype=0)
    g = grid_of(cfg)
    o = Oracle(cfg)
    rng = np.random.default_rng(1)
    r = rng.standard_normal((24, 32, 48))
    r -= r.mean()
    RHS = np.zeros(g.shape_rhs())
    RHS[1:-1, 1:-1, 1:-1] = r
    P = o.poisson(RHS)[2:-2, 2:-2, 2:-2]
    Pe = np.pad(P, 1)
    Pe[:, :, 0], Pe[:, :, -1] = Pe[:, :, -2], Pe[:, :, 1]
    Pe[:, 0, :], Pe[:, -1, :] = Pe[:, -2, :], Pe[:, 1, :]
    Pe[0], Pe[-1] = Pe[1], Pe[-2]
    c = Pe[1:-1, 1:-1, 1:-1]
    lap = (Pe[1:-1, 1:-1, 2:] - 2 * c + Pe[1:-1, 1:-1, :-2]) + (Pe[1:-1, 2:, 1:-1] - 2 * c + Pe[1:-1, :-2, 1:-1]) + \
          (Pe[2:, 1:-1, 1:-1] - 2 * c + Pe[:-2, 1:-1, 1:-1])
    assert np.abs(lap - r).max() < 1e-12
