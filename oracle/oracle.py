"""ctypes front end of the FP64 CPU oracle (oracle/elmm_oracle.cpp).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, always as the checker or the timed
CPU baseline, never as a code path of the library.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libelmm_oracle.so")
# the timed CPU baseline: the same source built with -O3 -march=native for
# the host that runs it (oracle/Makefile, target `native`)
NATIVE_PATH = os.path.join(HERE, "_build", "libelmm_oracle_native.so")

_libs = {}


def build(force: bool = False, native: bool = False) -> str:
    """Builds the parity library, or with native=True the timed baseline
    (make rebuilds it whenever the host CPU differs from the one it was
    built for)."""
    if native:
        subprocess.run(["make", "-s", "-C", HERE, "native"], check=True)
        return NATIVE_PATH
    if force or not os.path.exists(LIB_PATH) or (
            os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "elmm_oracle.cpp"))):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib(native: bool = False):
    if native not in _libs:
        path = NATIVE_PATH if native else LIB_PATH
        if not os.path.exists(path):
            build(native=native)
        L = C.CDLL(path)
        P = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.orc_create.restype = P
        L.orc_create.argtypes = [P]
        L.orc_destroy.argtypes = [P]
        L.orc_sizes.argtypes = [P, C.POINTER(C.c_int32)]
        L.orc_set_field.argtypes = [P, C.c_int, dp]
        L.orc_get_field.argtypes = [P, C.c_int, dp]
        L.orc_project.argtypes = [P, C.c_double, dp]
        L.orc_step.argtypes = [P, C.c_int, dp, dp]
        L.orc_run_stage.argtypes = [P, C.c_int, C.c_int]
        L.orc_clock.argtypes = [P, dp]
        L.orc_poisson.argtypes = [P, dp, dp]
        L.orc_bound_uvw.argtypes = [P]
        L.orc_num_threads.argtypes = [C.c_int]
        L.orc_num_threads.restype = C.c_int
        L.orc_scalar_slices.argtypes = [P, C.c_int, dp, dp]
        L.orc_set_solids.argtypes = [P, P]
        L.orc_set_puffs.argtypes = [P, P, C.c_int, P, C.c_int]
        _libs[native] = L
    return _libs[native]


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_threads(n: int, native: bool = False) -> int:
    return lib(native).orc_num_threads(n)


class Oracle:
    """One domain of the CPU restatement; field arrays use the host layout of
    gpu_elmm_b200.workloads (Fortran bounds, x contiguous)."""

    def __init__(self, cfg, native: bool = False):
        """native=True: an instance of the timed -march=native build."""
        self.cfg = cfg
        self.L = lib(native)
        self.h = self.L.orc_create(C.byref(cfg))
        if not self.h:
            raise ValueError("oracle rejected the configuration")
        s = (C.c_int32 * 12)()
        self.L.orc_sizes(self.h, s)
        self.sizes = tuple(s)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def _shape(self, field):
        Prnx, Prny, Prnz, Unx, Uny, Unz, Vnx, Vny, Vnz, Wnx, Wny, Wnz = self.sizes
        if field in (0, 5, 8):
            return (Unz + 6, Uny + 6, Unx + 6)
        if field in (1, 6, 9):
            return (Vnz + 6, Vny + 6, Vnx + 6)
        if field in (2, 7, 10):
            return (Wnz + 6, Wny + 6, Wnx + 6)
        if field in (12, 14) or 16 <= field < 24:  # Temperature, Scalar, their _adv: (-2:n+3)
            return (Prnz + 6, Prny + 6, Prnx + 6)
        return (Prnz + 4, Prny + 4, Prnx + 4)

    def set_field(self, field, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == self._shape(field), (a.shape, self._shape(field))
        self.L.orc_set_field(self.h, field, _ptr(a))

    def get_field(self, field):
        a = np.empty(self._shape(field))
        self.L.orc_get_field(self.h, field, _ptr(a))
        return a

    def set_state(self, U, V, W, Pr=None):
        self.set_field(0, U)
        self.set_field(1, V)
        self.set_field(2, W)
        if Pr is not None:
            self.set_field(3, Pr)

    def state(self):
        return tuple(self.get_field(f) for f in (0, 1, 2, 3))

    def project(self, coef=1.0) -> float:
        md = C.c_double(0)
        self.L.orc_project(self.h, coef, C.byref(md))
        return md.value

    def step(self, n=1):
        md = C.c_double(0)
        cfl = C.c_double(0)
        self.L.orc_step(self.h, n, C.byref(md), C.byref(cfl))
        return md.value, cfl.value

    def clock(self):
        """(time, length of the last step)."""
        out = (C.c_double * 2)()
        self.L.orc_clock(self.h, out)
        return out[0], out[1]

    def run_stage(self, stage, stop):
        r = self.L.orc_run_stage(self.h, stage, stop)
        assert r == 0

    def poisson(self, RHS):
        Prnx, Prny, Prnz = self.sizes[:3]
        RHS = np.ascontiguousarray(RHS, dtype=np.float64)
        assert RHS.shape == (Prnz + 2, Prny + 2, Prnx + 2)
        Phi = np.zeros((Prnz + 4, Prny + 4, Prnx + 4))
        self.L.orc_poisson(self.h, _ptr(RHS), _ptr(Phi))
        return Phi

    def scalar_slices(self, sc):
        """Time-averaged slices of scalar sc: xy (Prny, Prnx), xz (Prnz, Prnx)."""
        Prnx, Prny, Prnz = self.sizes[:3]
        xy, xz = np.zeros((Prny, Prnx)), np.zeros((Prnz, Prnx))
        assert self.L.orc_scalar_slices(self.h, sc, _ptr(xy), _ptr(xz)) == 0
        return xy, xz

    def set_puffs(self, puffs, volumes):
        """puffs as (start, end, period, duration, clear), volumes as
        (puff, scalar_number, (i, j, k), flux)."""
        from gpu_elmm_b200.config import make_puffs
        P, n_p, V, n_v = make_puffs(puffs, volumes)
        assert self.L.orc_set_puffs(self.h, C.cast(P, C.c_void_p), n_p, C.cast(V, C.c_void_p), n_v) == 0
        self._puffs = (P, V)

    def set_solids(self, solids):
        """Installs solid bodies: a gpu_elmm_b200.solids.Solids (or None)."""
        st = None if solids is None else solids.struct()
        assert self.L.orc_set_solids(self.h, None if st is None else C.cast(C.byref(st), C.c_void_p)) == 0
        self._solids = solids

    def bound(self):
        self.L.orc_bound_uvw(self.h)
