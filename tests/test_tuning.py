"""The autotuner's tile shapes change no result.

Before the first step of a batch the autotuner times the candidate tile
shapes of the z solve (16 / 32 spectral columns), the FP32 scalar stage
(8 / 4 rows) and the z chunk of the momentum and SGS kernels (8 / 16 / 32
planes) and keeps the fastest.  Each shape only changes how the work is
partitioned, so forcing any candidate (elmm_batch_set_tuning) must give the
autotuned run's state bit for bit, on the FP64 and the mixed path, for a
batch with a temperature, a passive scalar and uneven domain sizes."""
import numpy as np
import pytest

from gpu_elmm_b200.config import grid_of, make_config
from gpu_elmm_b200.workloads import log_profile_state, puff_state, temperature_state

SIZES = [(48, 32, 40), (64, 48, 24), (32, 32, 16)]
CANDIDATES = [dict(scalar_tile_rows=4), dict(tri_tile_cols=32), dict(momentum_z_chunk=8), dict(momentum_z_chunk=32),
              dict(sgs_z_chunk=8), dict(sgs_z_chunk=32),
              dict(scalar_tile_rows=4, tri_tile_cols=32, momentum_z_chunk=32, sgs_z_chunk=8)]


def _run(precision, shapes=None, steps=2):
    from gpu_elmm_b200 import lib as L
    cfgs = [make_config(*n, precision=precision, buoyancy=True, num_scalars=1, avg_slice_k=3, avg_weight=0.5)
            for n in SIZES]
    b = L.Batch(cfgs)
    for q, n in enumerate(SIZES):
        g = grid_of(cfgs[q])
        b.upload(q, *log_profile_state(g, seed=20 + q))
        b.upload_scalar(q, 1, puff_state(g, (5, 6, 4)))
    b.project(1.0)
    if shapes is not None:
        b.set_tuning(**shapes)
    b.step(steps)
    out = [(b.download(q), b.scalar(q, 1)) for q in range(len(SIZES))]
    tun = b.tuning()
    b.close()
    return out, tun


def _equal(a, b):
    for (sa, ca), (sb, cb) in zip(a, b):
        for x, y in zip(sa, sb):
            if not np.array_equal(x, y):
                return False
        if not np.array_equal(ca, cb):
            return False
    return True


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_every_tile_shape_gives_the_same_state(precision):
    ref, tun = _run(precision)
    assert tun["momentum_z_chunk"] in (8, 16, 32) and tun["sgs_z_chunk"] in (8, 16, 32)
    for shapes in CANDIDATES:
        got, t2 = _run(precision, shapes)
        for k, v in shapes.items():
            assert t2[k] == v
        assert _equal(got, ref), shapes


@pytest.mark.gpu
def test_out_of_set_shapes_are_refused():
    from gpu_elmm_b200 import lib as L
    b = L.Batch([make_config(32, 32, 16)])
    for bad in (dict(scalar_tile_rows=3), dict(tri_tile_cols=8), dict(momentum_z_chunk=12), dict(sgs_z_chunk=64)):
        with pytest.raises(L.ElmmError) as e:
            b.set_tuning(**bad)
        assert e.value.code == 6
    b.close()
