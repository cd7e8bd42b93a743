"""The split-domain path without a GPU.

* Two gloo ranks (world size 2) each hold one z-slab of a domain, run the
  z solve of the slab kernels (restated with numpy in slab_z_solve.py)
  behind FFTs in x and y, exchange only the sweep maps and the (0,0)
  column through torch.distributed, and together reproduce the oracle's
  Poisson solve of the whole domain (uniform and stretched z) to 1e-12.
* The C-ABI of elmm_slabs_* checks its arguments before it looks for a GPU.
"""
import ctypes as C
import json
import os
import socket
import subprocess
import sys
import tempfile

import numpy as np

from conftest import ROOT

RANK_SCRIPT = r'''
import json, os, sys
sys.path.insert(0, {root!r})
sys.path.insert(0, os.path.join({root!r}, "tests"))
sys.path.insert(0, os.path.join({root!r}, "oracle"))
import numpy as np
import torch.distributed as dist
from slab_z_solve import eigenvalues, run_rank, z_coefficients

dist.init_process_group("gloo")
ws, rank = dist.get_world_size(), dist.get_rank()

def gather(obj):
    out = [None] * ws
    dist.all_gather_object(out, obj)
    return out

nx, ny, nz, dx, dy = 24, 16, 20, 0.7, 1.3
split = [8, 12]
k0 = sum(split[:rank])
res = {{}}
for case in ("uniform", "stretched"):
    zW = np.arange(nz + 1) * 0.9 if case == "uniform" else \
        np.concatenate([[0.0], np.cumsum(0.5 * 1.04 ** np.arange(nz))])
    rng = np.random.default_rng(5)
    r = rng.standard_normal((nz, ny, nx))
    w = np.diff(zW)
    r -= (r * w[:, None, None]).sum() / (w.sum() * nx * ny)   # compatible right-hand side
    Ab, At, dzc, dzf = z_coefficients(zW)
    lam = eigenvalues(nx, ny, dx, dy)
    r_hat = np.fft.fft(np.fft.rfft(r[k0:k0 + split[rank]], axis=2), axis=1)
    X = run_rank(r_hat, lam, Ab, At, dzc, dzf, k0, nz, rank, gather)
    phi = np.fft.irfft(np.fft.ifft(X, axis=1), n=nx, axis=2)
    parts = gather(phi)
    if rank == 0:
        from gpu_elmm_b200.config import make_config, grid_of
        from oracle import Oracle
        cfg = make_config(nx, ny, nz, dx=dx, dy=dy, dz=0.9, zW=None if case == "uniform" else zW, sgstype=0)
        RHS = np.zeros(grid_of(cfg).shape_rhs())
        RHS[1:-1, 1:-1, 1:-1] = r
        ref = Oracle(cfg).poisson(RHS)[2:-2, 2:-2, 2:-2]
        got = np.concatenate(parts, axis=0)
        res[case] = float(np.abs(got - ref).max() / np.abs(ref).max())
dist.barrier()
if rank == 0:
    json.dump(res, open(os.path.join({tmp!r}, "result.json"), "w"))
dist.destroy_process_group()
'''


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_split_the_z_solve_and_reproduce_the_oracle():
    with tempfile.TemporaryDirectory() as tmp:
        script = os.path.join(tmp, "rank.py")
        open(script, "w").write(RANK_SCRIPT.format(root=ROOT, tmp=tmp))
        env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
               "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), script]
        r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-3000:]
        res = json.load(open(os.path.join(tmp, "result.json")))
    print("split z solve vs oracle:", res)
    assert res["uniform"] < 1e-12 and res["stretched"] < 1e-12, res


def test_slab_entry_points_check_their_arguments_first():
    from gpu_elmm_b200 import lib as L
    from gpu_elmm_b200.config import make_config
    lib = L.lib()
    h = C.c_void_p()
    assert lib.elmm_slabs_create(None, 2, None, None, C.byref(h)) == 6
    cfg = make_config(32, 32, 16)
    assert lib.elmm_slabs_create(C.byref(cfg), 0, None, None, C.byref(h)) == 6          # no slab
    assert lib.elmm_slabs_create(C.byref(cfg), 17, None, None, C.byref(h)) == 6         # over ELMM_MAX_SLABS
    nz = (C.c_int32 * 2)(8, 6)
    assert lib.elmm_slabs_create(C.byref(cfg), 2, None, nz, C.byref(h)) == 6            # 14 != 16 levels
    nz = (C.c_int32 * 2)(13, 3)
    assert lib.elmm_slabs_create(C.byref(cfg), 2, None, nz, C.byref(h)) == 6            # a slab under 4 levels
    refine = make_config(32, 32, 16, precision=1, max_refine_sweeps=2)
    assert lib.elmm_slabs_create(C.byref(refine), 2, None, None, C.byref(h)) == 1       # defect correction: not built
    per = make_config(32, 32, 16, btype=(3, 3, 3, 3, 3, 3))
    assert lib.elmm_slabs_create(C.byref(per), 2, None, None, C.byref(h)) == 1          # periodic z: not built
    for f in (lib.elmm_slabs_destroy(None), lib.elmm_slabs_upload_state(None, None, None, None, None),
              lib.elmm_slabs_download_state(None, None, None, None, None),
              lib.elmm_slabs_project(None, 1.0, None), lib.elmm_slabs_step(None, 1, None),
              lib.elmm_slabs_upload_temperature(None, None), lib.elmm_slabs_upload_scalar(None, 1, None),
              lib.elmm_slabs_download_field(None, 12, None)):
        assert f == 6
