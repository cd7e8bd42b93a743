"""elmm_poisson_solve_noalloc: the Poisson solve for callers that cannot
allocate device memory (a host whose memory pool already owns the GPU, or a
caller that must not let cudaMalloc/cudaFree synchronise the device).  It
solves the same problem as elmm_poisson_solver_execute, on device arrays
that the caller owns, with its working memory in one fixed array inside the
library.

The GPU test calls it through the C-ABI twice in a row and compares each
result with the handle-based solver on the same right-hand side, at the
tolerance of the other Poisson tests.  The second call of a pair gets a new
right-hand side (and, in one case, a new grid), so a result that leaned on
what the previous call left in the shared array would show up here.  The
grid spacings are exact binary fractions, which the handle-based solver
needs in order to accept the grid as uniform.

This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel

NEUMANN_Z = (3, 3, 3, 3, 5, 5)
PERIODIC = (3, 3, 3, 3, 3, 3)
ERR_INVALID_ARG = 6


def _rhs(n, seed):
    """Host RHS(0:nx+1, 0:ny+1, 0:nz+1) with a zero-mean random interior."""
    rng = np.random.default_rng(seed)
    r = rng.standard_normal((n[2], n[1], n[0]))
    r -= r.mean()
    RHS = np.zeros((n[2] + 2, n[1] + 2, n[0] + 2))
    RHS[1:-1, 1:-1, 1:-1] = r
    return RHS


def _args(n, L, bcs):
    return (C.c_int32 * 3)(*n), (C.c_double * 3)(*L), (C.c_int32 * 6)(*bcs)


def _solve_noalloc(n, L, bcs, RHS):
    """One call with caller-owned device buffers; Phi starts at 7 so that
    untouched ghosts can be checked."""
    import torch

    from gpu_elmm_b200 import lib as Lb

    rhs_d = torch.from_numpy(RHS).to("cuda:0")
    phi_d = torch.full((n[2] + 4, n[1] + 4, n[0] + 4), 7.0, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    nn, LL, bb = _args(n, L, bcs)
    st = Lb.lib().elmm_poisson_solve_noalloc(nn, LL, bb, 0, C.c_void_p(phi_d.data_ptr()),
                                             C.c_void_p(rhs_d.data_ptr()), None)
    assert st == 0, Lb.lib().elmm_last_error()
    torch.cuda.synchronize()
    return phi_d.cpu().numpy()


def _solve_handle(n, L, bcs, RHS):
    from gpu_elmm_b200 import lib as Lb

    ps = Lb.PoissonSolver(n, L=L, bcs=bcs, precision=0)
    Phi = np.full((n[2] + 4, n[1] + 4, n[0] + 4), 7.0)
    ps.execute(Phi, RHS)
    ps.close()
    return Phi


@pytest.mark.gpu
@pytest.mark.parametrize("grids", [
    [((48, 32, 20), (48.0, 32.0, 20.0), NEUMANN_Z)] * 2,
    [((40, 24, 16), (10.0, 12.0, 2.0), PERIODIC), ((64, 60, 30), (32.0, 15.0, 15.0), NEUMANN_Z)],
], ids=["same-grid", "new-grid"])
def test_noalloc_matches_handle_solver_twice(grids):
    for call, (n, L, bcs) in enumerate(grids):
        RHS = _rhs(n, seed=10 + call)
        got = _solve_noalloc(n, L, bcs, RHS)
        want = _solve_handle(n, L, bcs, RHS)
        assert rel(got[2:-2, 2:-2, 2:-2], want[2:-2, 2:-2, 2:-2]) < 1e-12, call
        ghosts = np.ones(got.shape, bool)
        ghosts[2:-2, 2:-2, 2:-2] = False
        assert (got[ghosts] == 7.0).all(), call


def test_noalloc_rejects_grids_beyond_its_scratch():
    """A grid whose working set exceeds the fixed array is refused before any
    GPU work, with a message that names the bytes it would need."""
    from gpu_elmm_b200 import lib as Lb

    nn, LL, bb = _args((256, 256, 128), (1.0, 1.0, 1.0), NEUMANN_Z)
    st = Lb.lib().elmm_poisson_solve_noalloc(nn, LL, bb, 0, C.c_void_p(16), C.c_void_p(16), None)
    assert st == ERR_INVALID_ARG
    msg = Lb.lib().elmm_last_error()
    msg = msg.decode() if isinstance(msg, bytes) else str(msg)
    assert "bytes of scratch" in msg and str(16 * 1024 * 1024) in msg


@pytest.mark.gpu
def test_noalloc_on_a_side_stream_matches_the_oracle():
    """The work is enqueued on the caller's stream: a non-default stream,
    synchronised alone before Phi is read, twice in a row with new
    right-hand sides, each result against the oracle's Poisson solve of the
    same discrete problem at 1e-12."""
    import torch

    from gpu_elmm_b200 import lib as Lb
    from gpu_elmm_b200.config import make_config
    from oracle import Oracle

    n, L, bcs = (48, 40, 24), (24.0, 10.0, 12.0), NEUMANN_Z
    cfg = make_config(*n, btype=bcs, dx=L[0] / n[0], dy=L[1] / n[1], dz=L[2] / n[2], sgstype=0)
    orc = Oracle(cfg)
    side = torch.cuda.Stream()
    nn, LL, bb = _args(n, L, bcs)
    for call in range(2):
        RHS = _rhs(n, seed=30 + call)
        with torch.cuda.stream(side):
            rhs_d = torch.from_numpy(RHS).to("cuda:0", non_blocking=False)
            phi_d = torch.full((n[2] + 4, n[1] + 4, n[0] + 4), 7.0, dtype=torch.float64, device="cuda:0")
        side.synchronize()
        st = Lb.lib().elmm_poisson_solve_noalloc(nn, LL, bb, 0, C.c_void_p(phi_d.data_ptr()),
                                                 C.c_void_p(rhs_d.data_ptr()), C.c_void_p(side.cuda_stream))
        assert st == 0, Lb.lib().elmm_last_error()
        side.synchronize()
        got = phi_d.cpu().numpy()
        want = orc.poisson(RHS)
        assert rel(got[2:-2, 2:-2, 2:-2], want[2:-2, 2:-2, 2:-2]) < 1e-12, call
        assert (got[0] == 7.0).all() and (got[:, :, 1] == 7.0).all(), call
