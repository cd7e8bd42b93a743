"""The single-precision host boundary: the reference's default release build
is prec=sp (src/make_release:2, knd = real32 in src/parameters.f90:17-21), so
its arrays are real32 and it binds the PoisSolver *_float variants
(src/poisson.f90:82-84, :152-154).

GPU: the *_float entry points, given float32 host arrays, leave the device in
the state the double entry points leave it in for the same values (float32
widens exactly), so every float32 result is the double result rounded to
float32, bit for bit: state upload / download, the temperature, two calls of
march_host, and the uniform and stretched Poisson solvers.

CPU: the Fortran interface module include/elmm_gpu.f90 binds only entry
points the header declares, covers every *_float one, and lays out
elmm_config in the order of the C struct."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from gpu_elmm_b200.config import ElmmConfig, FIELD_TEMPERATURE, grid_of, make_config
from gpu_elmm_b200.workloads import log_profile_state, temperature_state

F90 = os.path.join(ROOT, "include", "elmm_gpu.f90")
HEADER = os.path.join(ROOT, "include", "elmm_gpu.h")


def _f32(arrays):
    return [np.ascontiguousarray(a, dtype=np.float32) for a in arrays]


def _rounded(arrays):
    return [np.asarray(a, dtype=np.float64).astype(np.float32) for a in arrays]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_float_state_round_trip_and_march_host(precision):
    from gpu_elmm_b200 import lib as L
    n = (48, 32, 24)
    cfg = make_config(*n, buoyancy=True, precision=precision)
    g = grid_of(cfg)
    st = log_profile_state(g, seed=6)          # FP32-representable values
    T0 = temperature_state(g, seed=6)
    a, b = L.Domain(cfg), L.Domain(cfg)
    a.upload(*st)
    a.upload_temperature(T0)
    b.upload_f32(*_f32(st))
    b.upload_temperature_f32(np.ascontiguousarray(T0, dtype=np.float32))
    for x, y in zip(b.download_f32(), _rounded(a.download())):
        assert np.array_equal(x, y)
    a.project(1.0)
    b.project(1.0)
    # march_host: the double host arrays of `a` and float32 ones of `b`; after
    # each call the float32 arrays equal the double ones rounded
    ha = [x.copy() for x in a.download()] + [a.field(FIELD_TEMPERATURE)]
    hb = _rounded(ha)
    for it in range(2):
        ha = [x.astype(np.float32).astype(np.float64) for x in ha]  # the same values on both sides
        a.march_host(*ha, n=1 + it)
        b.march_host_f32(*hb, n=1 + it)
        for x, y, name in zip(hb, _rounded(ha), ("U", "V", "W", "Pr", "T")):
            assert np.array_equal(x, y), (it, name)
    assert np.array_equal(b.field_f32(FIELD_TEMPERATURE), a.field(FIELD_TEMPERATURE).astype(np.float32))
    a.close()
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("zstretch", [False, True])
def test_float_poisson_solver_equals_the_double_one(zstretch):
    from gpu_elmm_b200 import lib as L
    n = (48, 32, 20)
    zW = np.concatenate([[0.0], np.cumsum(0.5 * 1.04 ** np.arange(n[2]))]).astype(np.float32).astype(np.float64) \
        if zstretch else None
    Ls = (48.0, 32.0, 20.0)
    rng = np.random.default_rng(2)
    r = rng.standard_normal((n[2], n[1], n[0]))
    w = np.diff(zW) if zstretch else np.ones(n[2])
    r -= (r * w[:, None, None]).sum() / (w.sum() * n[0] * n[1])
    RHS = np.zeros((n[2] + 2, n[1] + 2, n[0] + 2))
    RHS[1:-1, 1:-1, 1:-1] = r
    RHS = RHS.astype(np.float32).astype(np.float64)
    for prec in (0, 1):
        pd = L.PoissonSolver(n, L=Ls, precision=prec, zW=zW)
        pf = L.PoissonSolver(n, L=Ls, precision=prec, zW=zW, host_f32=True)
        Phi = np.full((n[2] + 4, n[1] + 4, n[0] + 4), 7.0)
        Phif = np.full(Phi.shape, 7.0, dtype=np.float32)
        pd.execute(Phi, RHS)
        pf.execute(Phif, RHS.astype(np.float32))
        assert np.array_equal(Phif, Phi.astype(np.float32)), prec
        pd.close()
        pf.close()


def _f90_source():
    src = open(F90).read()
    return "\n".join(line.split("!")[0] for line in src.splitlines())


def test_fortran_module_binds_declared_entry_points():
    from test_abi import declared_functions
    f90 = set(re.findall(r"function\s+(elmm_\w+)\s*\(", _f90_source(), flags=re.I))
    declared = set(declared_functions())
    assert f90 and f90 <= declared, sorted(f90 - declared)
    floats = {n for n in declared if n.endswith("_float")}
    assert len(floats) >= 10 and floats <= f90, sorted(floats - f90)


def test_fortran_config_follows_the_c_struct():
    src = _f90_source()
    body = re.search(r"type, bind\(C\) :: elmm_config(.*?)end type", src, flags=re.S | re.I).group(1)
    names = []
    for line in body.splitlines():
        if "::" in line:
            for part in line.split("::")[1].split(","):
                nm = re.sub(r"\(.*", "", part).strip()
                if nm:
                    names.append(nm)
    assert names == [f[0] for f in ElmmConfig._fields_], names


def test_float_entry_points_refuse_null_handles():
    """Without a GPU: argument checks come first."""
    from gpu_elmm_b200 import lib as L
    lib = L.lib()
    assert lib.elmm_upload_state_float(None, None, None, None, None) == 6
    assert lib.elmm_download_field_float(None, 0, None) == 6
    assert lib.elmm_march_host_float(None, None, None, None, None, None, 1, None) == 6
    assert lib.elmm_poisson_solver_execute_float(None, None, None) == 6
