"""C-ABI surface of libelmm_gpu.so: every entry point declared in
include/elmm_gpu.h is exported, the ctypes mirrors have the C layout, and
argument / configuration errors come back as status codes without a GPU."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from conftest import ROOT
from gpu_elmm_b200 import config as cfgmod
from gpu_elmm_b200 import lib as L

HEADER = os.path.join(ROOT, "include", "elmm_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(elmm_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 24 and "elmm_step" in names and "elmm_poisson_solver_execute" in names
    lib = L.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (elmm_\w+)", out))
    assert set(names) <= exported


def _c_layout():
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "elmm_gpu.h"
#define O(s, f) printf(#s "." #f " %zu\n", offsetof(s, f));
int main(void) {
  printf("elmm_config.size %zu\n", sizeof(elmm_config));
  printf("elmm_stats.size %zu\n", sizeof(elmm_stats));
  O(elmm_config, Btype) O(elmm_config, xmin) O(elmm_config, zW) O(elmm_config, dt)
  O(elmm_config, sgstype) O(elmm_config, z0) O(elmm_config, pr_gradient_x) O(elmm_config, precision)
  O(elmm_config, refine_tol) O(elmm_config, device) O(elmm_config, TempBtype) O(elmm_config, molecular_diffusivity)
  O(elmm_config, num_scalars) O(elmm_config, ScalBtype) O(elmm_config, sideScal) O(elmm_config, num_point_sources)
  O(elmm_config, point_sources) O(elmm_config, avg_slice_k) O(elmm_config, avg_slice_j) O(elmm_config, avg_weight)
  O(elmm_point_source, position) O(elmm_point_source, flux)
  printf("elmm_point_source.size %zu\n", sizeof(elmm_point_source));
  O(elmm_stats, time) O(elmm_stats, max_div) O(elmm_stats, refine_sweeps) O(elmm_stats, elapsed_ms)
  printf("elmm_ib_point.size %zu\n", sizeof(elmm_ib_point));
  printf("elmm_wm_point.size %zu\n", sizeof(elmm_wm_point));
  printf("elmm_solids.size %zu\n", sizeof(elmm_solids));
  printf("elmm_puff.size %zu\n", sizeof(elmm_puff));
  printf("elmm_puff_volume.size %zu\n", sizeof(elmm_puff_volume));
  O(elmm_puff, clear) O(elmm_puff_volume, zk) O(elmm_puff_volume, flux)
  O(elmm_ib_point, interp) O(elmm_ib_point, kk) O(elmm_ib_point, coef)
  O(elmm_wm_point, dist) O(elmm_wm_point, z0)
  O(elmm_solids, ib) O(elmm_solids, n_null) O(elmm_solids, null_ijk) O(elmm_solids, n_scalfl) O(elmm_solids, scalfl)
  O(elmm_solids, n_wm) O(elmm_solids, wm) O(elmm_solids, n_bottom_skip) O(elmm_solids, bottom_skip_ij)
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        open(c, "w").write(prog)
        exe = os.path.join(d, "l")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    return dict((l.split()[0], int(l.split()[1])) for l in out.splitlines())


def test_ctypes_layout_matches_c():
    lay = _c_layout()
    assert lay["elmm_config.size"] == C.sizeof(cfgmod.ElmmConfig)
    assert lay["elmm_stats.size"] == C.sizeof(cfgmod.ElmmStats)
    assert lay["elmm_point_source.size"] == C.sizeof(cfgmod.ElmmPointSource)
    for key, off in lay.items():
        s, f = key.split(".")
        if f == "size":
            continue
        cls = {"elmm_config": cfgmod.ElmmConfig, "elmm_stats": cfgmod.ElmmStats,
               "elmm_point_source": cfgmod.ElmmPointSource, "elmm_ib_point": cfgmod.ElmmIBPoint,
               "elmm_wm_point": cfgmod.ElmmWMPoint, "elmm_solids": cfgmod.ElmmSolids,
               "elmm_puff": cfgmod.ElmmPuff, "elmm_puff_volume": cfgmod.ElmmPuffVolume}[s]
        assert getattr(cls, f).offset == off, key
    for s, cls in (("elmm_ib_point", cfgmod.ElmmIBPoint), ("elmm_wm_point", cfgmod.ElmmWMPoint),
                   ("elmm_solids", cfgmod.ElmmSolids), ("elmm_puff", cfgmod.ElmmPuff),
                   ("elmm_puff_volume", cfgmod.ElmmPuffVolume)):
        assert lay[s + ".size"] == C.sizeof(cls), s


def test_config_defaults_and_errors_without_gpu():
    lib = L.lib()
    c = cfgmod.ElmmConfig()
    assert lib.elmm_config_defaults(C.byref(c), 64, 64, 32) == 0
    assert c.Btype[4] == cfgmod.BC_NOSLIP and c.Btype[5] == cfgmod.BC_FREESLIP
    assert abs(c.molecular_viscosity - 1 / 70000) < 1e-20 and c.wallmodeltype == 1
    h = C.c_void_p()
    bad = cfgmod.make_config(64, 64, 32)
    bad.Btype[0] = 1  # no-slip x needs the FFT in x: refused
    assert lib.elmm_create(C.byref(bad), C.byref(h)) == 1
    assert b"periodic" in lib.elmm_last_error()
    bad = cfgmod.make_config(64, 64, 32)
    bad.Prnx = 7 * 11
    assert lib.elmm_create(C.byref(bad), C.byref(h)) == 1
    bad = cfgmod.make_config(64, 64, 32)
    bad.abi_version = 99
    assert lib.elmm_create(C.byref(bad), C.byref(h)) == 1
    bad = cfgmod.make_config(64, 64, 32, num_scalars=1, point_sources=[(2, (1.0, 1.0, 1.0), 1.0)])
    assert lib.elmm_create(C.byref(bad), C.byref(h)) == 1
    assert b"scalar_number" in lib.elmm_last_error()
    bad = cfgmod.make_config(64, 64, 32, num_scalars=5)
    assert lib.elmm_create(C.byref(bad), C.byref(h)) == 1
    bad = cfgmod.make_config(64, 64, 32, num_scalars=1, avg_slice_k=33)
    assert lib.elmm_create(C.byref(bad), C.byref(h)) == 1
    bad = cfgmod.make_config(64, 64, 32, num_scalars=1)
    bad.ScalBtype[4] = 1  # no-slip is not a kind of scalar side
    assert lib.elmm_create(C.byref(bad), C.byref(h)) == 1
    assert lib.elmm_create(None, C.byref(h)) == 6
    assert lib.elmm_step(None, 1, None) == 6


def test_no_cpu_fallback_without_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(L.ElmmError) as e:
        L.Domain(cfgmod.make_config(32, 24, 16))
    assert e.value.code == 4  # ELMM_ERR_CUDA


def test_new_entry_points_refuse_null_handles_without_gpu():
    """The solid-body, puff and host-array entry points check their handle
    before touching a device: NULL comes back as ELMM_ERR_INVALID_ARG (6)."""
    lib = L.lib()
    assert lib.elmm_set_solids(None, None) == 6
    assert lib.elmm_set_puffs(None, None, 0, None, 0) == 6
    assert lib.elmm_march_host(None, None, None, None, None, None, 1, None) == 6
    assert lib.elmm_batch_set_solids(None, 0, None) == 6
    assert lib.elmm_batch_set_puffs(None, 0, None, 0, None, 0) == 6
    assert b"NULL" in lib.elmm_last_error()
