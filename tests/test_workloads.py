"""Seeded synthetic inputs (gpu_elmm_b200.workloads)."""
import numpy as np

from gpu_elmm_b200.config import grid_of, make_config
from gpu_elmm_b200.workloads import interiors, log_profile_state, splitmix64, uniform


def test_splitmix64_known_values():
    # first outputs of splitmix64 seeded with 0 (the published generator)
    z = splitmix64(np.array([0, 0x9E3779B97F4A7C15], dtype=np.uint64))
    assert int(z[0]) == 0xE220A8397B1DCDAF
    assert int(z[1]) == 0x6E789E6AA1B965F4


def test_streams_are_deterministic_and_distinct():
    a = uniform(0, "u", 1000)
    assert np.array_equal(a, uniform(0, "u", 1000))
    assert not np.array_equal(a, uniform(1, "u", 1000))
    assert not np.array_equal(a, uniform(0, "v", 1000))
    assert a.min() >= 0 and a.max() < 1 and abs(a.mean() - 0.5) < 0.05


def test_log_profile_state():
    g = grid_of(make_config(16, 12, 8))
    U, V, W, P = log_profile_state(g, seed=0)
    Ui, Vi, Wi, Pi = interiors(g, U, V, W, P)
    assert np.array_equal(U.astype(np.float32).astype(np.float64), U)
    prof = (0.3 / 0.41) * np.log((np.arange(1, 9) - 0.5) / 0.01)
    assert np.abs(Ui.mean(axis=(1, 2)) - prof).max() < 0.05
    assert np.abs(Vi).max() <= 0.1 and np.abs(Wi).max() <= 0.1
    assert (P == 0).all()
    # ghosts are left zero for the library / oracle to fill
    assert (U[:2] == 0).all() and (U[:, :, -3:] == 0).all()


def test_profiles_of_a_known_field():
    """Vertical profiles (src/vertical_profiles.f90): mean, resolved variance
    and resolved TKE of a field with a known answer."""
    import numpy as np
    from gpu_elmm_b200.config import grid_of, make_config
    from gpu_elmm_b200.stats import Profiles
    from gpu_elmm_b200.workloads import interior
    g = grid_of(make_config(8, 6, 5))
    U, V, W = np.zeros(g.shape_u()), np.zeros(g.shape_v()), np.zeros(g.shape_w())
    k = np.arange(1, g.Unz + 1)[:, None, None]
    i = np.arange(1, g.Unx + 1)[None, None, :]
    j = np.arange(1, g.Wny + 1)[None, :, None]
    interior(U, -2, (g.Unx, g.Uny, g.Unz))[...] = k + 0.5 * (-1.0) ** i
    interior(W, -2, (g.Wnx, g.Wny, g.Wnz))[...] = 0.3 * (-1.0) ** j
    p = Profiles(g)
    p.add(U, V, W)
    p.add(U, V, W)
    r = p.result()
    assert np.allclose(r["u"], np.arange(1, g.Unz + 1)) and np.allclose(r["uu"], 0.25)
    assert np.allclose(r["ww"][1:g.Wnz + 1], 0.09) and r["ww"][0] == 0 and r["ww"][g.Prnz] == 0
    want = (0.25 + 0.0 + (r["ww"][:-1] + r["ww"][1:]) / 2) / 2
    assert np.allclose(r["tke"], want)


def test_vtk_frames_round_trip(tmp_path):
    """Frames and slices in the reference's legacy-VTK layout (float32
    big-endian rectilinear grids, src/outputs.f90:2260-2300) read back to the
    FP32-rounded fields on the right staggered coordinates."""
    import numpy as np
    from gpu_elmm_b200.config import grid_of, make_config
    from gpu_elmm_b200.vtk import read_rectilinear, write_scalar_slices, write_uvw
    from gpu_elmm_b200.workloads import interior, log_profile_state
    g = grid_of(make_config(8, 6, 5))
    U, V, W, Pr = log_profile_state(g, seed=4)
    write_uvw(g, U, V, W, str(tmp_path / "frame_"))
    (x, y, z), f = read_rectilinear(str(tmp_path / "frame_W.vtk"))
    assert np.allclose(z, np.arange(1, g.Wnz + 1)) and np.allclose(x, np.arange(1, 9) - 0.5)
    assert np.array_equal(f["W"], interior(W, -2, (g.Wnx, g.Wny, g.Wnz)).astype(np.float32))
    raw = open(tmp_path / "frame_U.vtk", "rb").read()
    assert raw.startswith(b"# vtk DataFile Version 2.0\n") and b"DATASET RECTILINEAR_GRID\n" in raw
    first = interior(U, -2, (g.Unx, g.Uny, g.Unz))[0, 0, 0]
    assert np.array([first], dtype=">f4").tobytes() in raw  # big-endian float32
    xy = np.arange(48.0).reshape(6, 8)
    xz = np.arange(40.0).reshape(5, 8)
    write_scalar_slices(g, xy, xz, 3, 2, str(tmp_path / "c"))
    (_, _, zz), f = read_rectilinear(str(tmp_path / "c_xy.vtk"))
    assert np.allclose(zz, [2.5]) and np.array_equal(f["scalar01_avg"][0], xy.astype(np.float32))
    (_, yy, _), f = read_rectilinear(str(tmp_path / "c_xz.vtk"))
    assert np.allclose(yy, [1.5]) and np.array_equal(f["scalar01_avg"][:, 0, :], xz.astype(np.float32))
