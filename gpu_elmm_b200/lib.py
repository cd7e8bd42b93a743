"""ctypes front end of libelmm_gpu.so (include/elmm_gpu.h).

Host arrays use the reference's Fortran layout (see workloads.py).  Every
call goes to the CUDA library; there is no CPU fallback: if the shared
library is missing or no CUDA device is usable, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .config import (FIELD_SCALAR, FIELD_SCALAR_ADV, MAX_SCALARS, ElmmConfig, ElmmStats, Grid, STATUS_NAMES,
                     grid_of)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libelmm_gpu.so")

_lib = None

_dp = C.POINTER(C.c_double)

KERNEL_NAMES = ("sgs", "momentum", "fftx_fwd", "ffty_fwd", "tri", "ffty_inv", "fftx_inv", "project", "prref", "ghosts",
                "temperature")
KERNEL_COUNT = len(KERNEL_NAMES)


class ElmmError(RuntimeError):
    def __init__(self, code: int, what: str, msg: str):
        super().__init__(f"{what}: {STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Loads the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} not built: run `make -C gpu_elmm_b200` (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.elmm_version.restype = C.c_char_p
        L.elmm_last_error.restype = C.c_char_p
        L.elmm_config_defaults.argtypes = [C.POINTER(ElmmConfig), C.c_int32, C.c_int32, C.c_int32]
        L.elmm_create.argtypes = [C.POINTER(ElmmConfig), C.POINTER(P)]
        L.elmm_destroy.argtypes = [P]
        L.elmm_upload_state.argtypes = [P, _dp, _dp, _dp, _dp]
        L.elmm_download_state.argtypes = [P, _dp, _dp, _dp, _dp]
        L.elmm_upload_temperature.argtypes = [P, _dp]
        L.elmm_upload_scalar.argtypes = [P, C.c_int32, _dp]
        L.elmm_set_solids.argtypes = [P, P]
        L.elmm_set_puffs.argtypes = [P, P, C.c_int32, P, C.c_int32]
        L.elmm_batch_set_solids.argtypes = [P, C.c_int32, P]
        L.elmm_batch_set_puffs.argtypes = [P, C.c_int32, P, C.c_int32, P, C.c_int32]
        L.elmm_march_host.argtypes = [P, _dp, _dp, _dp, _dp, _dp, C.c_int32, C.POINTER(ElmmStats)]
        L.elmm_download_scalar_slices.argtypes = [P, C.c_int32, _dp, _dp]
        L.elmm_reset_scalar_averages.argtypes = [P]
        L.elmm_download_field.argtypes = [P, C.c_int32, _dp]
        L.elmm_frame_begin.argtypes = [P]
        L.elmm_frame_wait.argtypes = [P, _dp, _dp, _dp, _dp]
        L.elmm_project.argtypes = [P, C.c_double, C.POINTER(ElmmStats)]
        L.elmm_step.argtypes = [P, C.c_int32, C.POINTER(ElmmStats)]
        L.elmm_run_stage.argtypes = [P, C.c_int32, C.c_int32]
        L.elmm_profile_stage.argtypes = [P, C.c_int32, C.c_int32, _dp]
        L.elmm_poisson_solver_new.argtypes = [C.POINTER(P), C.POINTER(C.c_int32), _dp, C.POINTER(C.c_int32),
                                              C.c_int32, C.c_int32]
        L.elmm_poisson_solver_nonuniform_z_new.argtypes = [C.POINTER(P), C.POINTER(C.c_int32), _dp, _dp, _dp,
                                                           C.POINTER(C.c_int32), C.c_int32, C.c_int32]
        L.elmm_poisson_solver_execute.argtypes = [P, _dp, _dp]
        L.elmm_poisson_solver_finalize.argtypes = [P]
        L.elmm_batch_create.argtypes = [C.POINTER(ElmmConfig), C.c_int32, C.POINTER(P)]
        L.elmm_batch_destroy.argtypes = [P]
        L.elmm_batch_upload_state.argtypes = [P, C.c_int32, _dp, _dp, _dp, _dp]
        L.elmm_batch_download_state.argtypes = [P, C.c_int32, _dp, _dp, _dp, _dp]
        L.elmm_batch_upload_scalar.argtypes = [P, C.c_int32, C.c_int32, _dp]
        L.elmm_batch_download_field.argtypes = [P, C.c_int32, C.c_int32, _dp]
        L.elmm_batch_download_scalar_slices.argtypes = [P, C.c_int32, C.c_int32, _dp, _dp]
        L.elmm_batch_project.argtypes = [P, C.c_double]
        L.elmm_batch_profile_stage.argtypes = [P, C.c_int32, C.c_int32, _dp]
        L.elmm_batch_tuning.argtypes = [P, C.POINTER(C.c_int32)]
        L.elmm_batch_step.argtypes = [P, C.c_int32, C.POINTER(ElmmStats)]
        L.elmm_batch_cells.argtypes = [P]
        L.elmm_batch_cells.restype = C.c_int64
        L.elmm_set_fault_injection.argtypes = [P, C.c_int32, C.c_int32]
        L.elmm_batch_get_tuning.argtypes = [P, C.POINTER(C.c_int32), C.c_int32]
        L.elmm_get_tuning.argtypes = [P, C.POINTER(C.c_int32), C.c_int32]
        L.elmm_set_tuning.argtypes = [P, C.POINTER(C.c_int32), C.c_int32]
        L.elmm_batch_set_tuning.argtypes = [P, C.POINTER(C.c_int32), C.c_int32]
        fp = C.POINTER(C.c_float)
        L.elmm_upload_state_float.argtypes = [P, fp, fp, fp, fp]
        L.elmm_download_state_float.argtypes = [P, fp, fp, fp, fp]
        L.elmm_download_field_float.argtypes = [P, C.c_int32, fp]
        L.elmm_upload_temperature_float.argtypes = [P, fp]
        L.elmm_upload_scalar_float.argtypes = [P, C.c_int32, fp]
        L.elmm_march_host_float.argtypes = [P, fp, fp, fp, fp, fp, C.c_int32, C.POINTER(ElmmStats)]
        L.elmm_poisson_solver_new_float.argtypes = [C.POINTER(P), C.POINTER(C.c_int32), fp, C.POINTER(C.c_int32),
                                                    C.c_int32, C.c_int32]
        L.elmm_poisson_solver_nonuniform_z_new_float.argtypes = [C.POINTER(P), C.POINTER(C.c_int32), fp, fp, fp,
                                                                 C.POINTER(C.c_int32), C.c_int32, C.c_int32]
        L.elmm_poisson_solver_execute_float.argtypes = [P, fp, fp]
        L.elmm_poisson_solver_finalize_float.argtypes = [P]
        ip = C.POINTER(C.c_int32)
        L.elmm_slabs_create.argtypes = [C.POINTER(ElmmConfig), C.c_int32, ip, ip, C.POINTER(P)]
        L.elmm_slabs_destroy.argtypes = [P]
        L.elmm_slabs_upload_state.argtypes = [P, _dp, _dp, _dp, _dp]
        L.elmm_slabs_download_state.argtypes = [P, _dp, _dp, _dp, _dp]
        L.elmm_slabs_project.argtypes = [P, C.c_double, C.POINTER(ElmmStats)]
        L.elmm_slabs_step.argtypes = [P, C.c_int32, C.POINTER(ElmmStats)]
        L.elmm_slabs_march_host.argtypes = [P, _dp, _dp, _dp, _dp, C.c_int32, C.POINTER(ElmmStats)]
        L.elmm_slabs_upload_temperature.argtypes = [P, _dp]
        L.elmm_slabs_upload_scalar.argtypes = [P, C.c_int32, _dp]
        L.elmm_slabs_download_field.argtypes = [P, C.c_int32, _dp]
        L.elmm_slabs_set_puffs.argtypes = [P, P, C.c_int32, P, C.c_int32]
        L.elmm_slabs_download_scalar_slices.argtypes = [P, C.c_int32, _dp, _dp]
        L.elmm_slabs_upload_state_float.argtypes = [P, fp, fp, fp, fp]
        L.elmm_slabs_download_state_float.argtypes = [P, fp, fp, fp, fp]
        L.elmm_slabs_march_host_float.argtypes = [P, fp, fp, fp, fp, C.c_int32, C.POINTER(ElmmStats)]
        _lib = L
    return _lib


def check(code: int, what: str):
    if code != 0:
        raise ElmmError(code, what, lib().elmm_last_error().decode())


def ptr(a):
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous, "host arrays: C-contiguous float64"
    return a.ctypes.data_as(_dp)


def fptr(a):
    """A float32 host array (the *_float entry points of a single-precision host)."""
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous, "host arrays: C-contiguous float32"
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Domain:
    """One domain whose state stays resident on the GPU (an elmm_handle)."""

    def __init__(self, cfg: ElmmConfig):
        self.cfg = cfg
        self.grid: Grid = grid_of(cfg)
        h = C.c_void_p()
        check(lib().elmm_create(C.byref(cfg), C.byref(h)), "elmm_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().elmm_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, U, V, W, Pr=None):
        check(lib().elmm_upload_state(self.h, ptr(U), ptr(V), ptr(W), ptr(Pr)), "elmm_upload_state")

    def download(self):
        g = self.grid
        U, V, W, Pr = np.zeros(g.shape_u()), np.zeros(g.shape_v()), np.zeros(g.shape_w()), np.zeros(g.shape_p())
        check(lib().elmm_download_state(self.h, ptr(U), ptr(V), ptr(W), ptr(Pr)), "elmm_download_state")
        return U, V, W, Pr

    def field_shape(self, fid: int):
        """Host shape of field fid (ELMM_FIELD_*)."""
        g = self.grid
        shape = {0: g.shape_u(), 5: g.shape_u(), 8: g.shape_u(), 1: g.shape_v(), 6: g.shape_v(), 9: g.shape_v(),
                 2: g.shape_w(), 7: g.shape_w(), 10: g.shape_w(), 12: g.shape_t(), 14: g.shape_t()}.get(fid, g.shape_p())
        if FIELD_SCALAR <= fid < FIELD_SCALAR_ADV + MAX_SCALARS:
            shape = g.shape_t()
        return shape

    def field(self, fid: int, out=None):
        a = np.zeros(self.field_shape(fid)) if out is None else out
        check(lib().elmm_download_field(self.h, fid, ptr(a)), "elmm_download_field")
        return a

    def upload_temperature(self, T):
        """Temperature(-2:nx+3,-2:ny+3,-2:nz+3), host array (enable_buoyancy)."""
        check(lib().elmm_upload_temperature(self.h, ptr(T)), "elmm_upload_temperature")

    def temperature(self):
        return self.field(12)

    def march_host(self, U, V, W, Pr, T=None, n=1) -> ElmmStats:
        """TMarchRK3 on host arrays: upload, n steps, write the state back into
        the same arrays (elmm_march_host)."""
        st = ElmmStats()
        check(lib().elmm_march_host(self.h, ptr(U), ptr(V), ptr(W), ptr(Pr), ptr(T), n, C.byref(st)),
              "elmm_march_host")
        return st

    def tuning(self):
        """Tile shapes chosen by the autotuner at the first step (or set); the keys of Batch.TUNING_KEYS."""
        out = (C.c_int32 * 4)()
        check(lib().elmm_get_tuning(self.h, out, 4), "elmm_get_tuning")
        return dict(zip(("scalar_tile_rows", "tri_tile_cols", "momentum_z_chunk", "sgs_z_chunk"), list(out)))

    def set_tuning(self, **shapes):
        cur = self.tuning()
        cur.update(shapes)
        keys = ("scalar_tile_rows", "tri_tile_cols", "momentum_z_chunk", "sgs_z_chunk")
        vals = (C.c_int32 * 4)(*[cur[k] for k in keys])
        check(lib().elmm_set_tuning(self.h, vals, 4), "elmm_set_tuning")

    def set_fault_injection(self, wait_limit=1 << 20, skip_plane=-1):
        """Fault injection for tests of the timeout path (elmm_set_fault_injection)."""
        check(lib().elmm_set_fault_injection(self.h, wait_limit, skip_plane), "elmm_set_fault_injection")

    # single-precision host arrays (a host built with prec=sp): float32 arrays
    # in the same layouts
    def upload_f32(self, U, V, W, Pr=None):
        check(lib().elmm_upload_state_float(self.h, fptr(U), fptr(V), fptr(W), fptr(Pr)), "elmm_upload_state_float")

    def download_f32(self):
        g = self.grid
        out = [np.zeros(s, dtype=np.float32) for s in (g.shape_u(), g.shape_v(), g.shape_w(), g.shape_p())]
        check(lib().elmm_download_state_float(self.h, *[fptr(a) for a in out]), "elmm_download_state_float")
        return tuple(out)

    def field_f32(self, fid):
        a = np.zeros(self.field_shape(fid), dtype=np.float32)
        check(lib().elmm_download_field_float(self.h, fid, fptr(a)), "elmm_download_field_float")
        return a

    def upload_temperature_f32(self, T):
        check(lib().elmm_upload_temperature_float(self.h, fptr(T)), "elmm_upload_temperature_float")

    def march_host_f32(self, U, V, W, Pr, T=None, n=1) -> ElmmStats:
        st = ElmmStats()
        check(lib().elmm_march_host_float(self.h, fptr(U), fptr(V), fptr(W), fptr(Pr), fptr(T), n, C.byref(st)),
              "elmm_march_host_float")
        return st

    def set_puffs(self, puffs, volumes):
        """Puff sources: puffs as (start, end, period, duration, clear),
        volumes as (puff, scalar_number, (i, j, k), flux); [] removes them."""
        from .config import make_puffs
        P, n_p, V, n_v = make_puffs(puffs, volumes)
        check(lib().elmm_set_puffs(self.h, C.cast(P, C.c_void_p), n_p, C.cast(V, C.c_void_p), n_v), "elmm_set_puffs")
        self._puffs = (P, V)

    def set_solids(self, solids):
        """Installs solid bodies (gpu_elmm_b200.solids.Solids, or None to remove them)."""
        st = None if solids is None else solids.struct()
        check(lib().elmm_set_solids(self.h, None if st is None else C.cast(C.byref(st), C.c_void_p)),
              "elmm_set_solids")

    def upload_scalar(self, sc, S):
        """Scalar(-2:nx+3,-2:ny+3,-2:nz+3,sc), host array, sc in 1..num_scalars."""
        check(lib().elmm_upload_scalar(self.h, sc, ptr(S)), "elmm_upload_scalar")

    def scalar(self, sc):
        return self.field(FIELD_SCALAR + sc - 1)

    def scalar_slices(self, sc):
        """Time-averaged slices of scalar sc: xy (Prny, Prnx) at avg_slice_k and
        xz (Prnz, Prnx) at avg_slice_j (None where the slice is off)."""
        g = self.grid
        xy = np.zeros((g.Prny, g.Prnx)) if self.cfg.avg_slice_k > 0 else None
        xz = np.zeros((g.Prnz, g.Prnx)) if self.cfg.avg_slice_j > 0 else None
        check(lib().elmm_download_scalar_slices(self.h, sc, ptr(xy), ptr(xz)), "elmm_download_scalar_slices")
        return xy, xz

    def reset_scalar_averages(self):
        check(lib().elmm_reset_scalar_averages(self.h), "elmm_reset_scalar_averages")

    def project(self, coef=1.0) -> ElmmStats:
        st = ElmmStats()
        check(lib().elmm_project(self.h, coef, C.byref(st)), "elmm_project")
        return st

    def step(self, n=1) -> ElmmStats:
        st = ElmmStats()
        check(lib().elmm_step(self.h, n, C.byref(st)), "elmm_step")
        return st

    def run_stage(self, stage, stop):
        check(lib().elmm_run_stage(self.h, stage, stop), "elmm_run_stage")

    def profile_stage(self, stage=2, reps=5):
        """Mean device time (ms) of each kernel of one RK3 stage, CUDA events on the library's stream."""
        ms = (C.c_double * KERNEL_COUNT)()
        check(lib().elmm_profile_stage(self.h, stage, reps, ms), "elmm_profile_stage")
        return dict(zip(KERNEL_NAMES, list(ms)))

    def frame_begin(self):
        check(lib().elmm_frame_begin(self.h), "elmm_frame_begin")

    def frame_wait(self):
        g = self.grid
        U, V, W, Pr = np.zeros(g.shape_u()), np.zeros(g.shape_v()), np.zeros(g.shape_w()), np.zeros(g.shape_p())
        check(lib().elmm_frame_wait(self.h, ptr(U), ptr(V), ptr(W), ptr(Pr)), "elmm_frame_wait")
        return U, V, W, Pr


class Batch:
    """n independent domains of uneven sizes stepped together (elmm_batch)."""

    def __init__(self, cfgs):
        self.cfgs = list(cfgs)
        arr = (ElmmConfig * len(self.cfgs))(*self.cfgs)
        self._arr = arr
        h = C.c_void_p()
        check(lib().elmm_batch_create(arr, len(self.cfgs), C.byref(h)), "elmm_batch_create")
        self.h = h
        self.grids = [grid_of(c) for c in self.cfgs]

    def close(self):
        if getattr(self, "h", None):
            lib().elmm_batch_destroy(self.h)
            self.h = None

    __del__ = close

    def cells(self) -> int:
        return lib().elmm_batch_cells(self.h)

    def upload(self, d, U, V, W, Pr=None):
        check(lib().elmm_batch_upload_state(self.h, d, ptr(U), ptr(V), ptr(W), ptr(Pr)), "elmm_batch_upload_state")

    def download(self, d):
        g = self.grids[d]
        U, V, W, Pr = np.zeros(g.shape_u()), np.zeros(g.shape_v()), np.zeros(g.shape_w()), np.zeros(g.shape_p())
        check(lib().elmm_batch_download_state(self.h, d, ptr(U), ptr(V), ptr(W), ptr(Pr)),
              "elmm_batch_download_state")
        return U, V, W, Pr

    def upload_scalar(self, d, sc, S):
        check(lib().elmm_batch_upload_scalar(self.h, d, sc, ptr(S)), "elmm_batch_upload_scalar")

    def scalar(self, d, sc):
        a = np.zeros(self.grids[d].shape_t())
        check(lib().elmm_batch_download_field(self.h, d, FIELD_SCALAR + sc - 1, ptr(a)), "elmm_batch_download_field")
        return a

    def scalar_slices(self, d, sc):
        g, c = self.grids[d], self.cfgs[d]
        xy = np.zeros((g.Prny, g.Prnx)) if c.avg_slice_k > 0 else None
        xz = np.zeros((g.Prnz, g.Prnx)) if c.avg_slice_j > 0 else None
        check(lib().elmm_batch_download_scalar_slices(self.h, d, sc, ptr(xy), ptr(xz)),
              "elmm_batch_download_scalar_slices")
        return xy, xz

    def project(self, coef=1.0):
        check(lib().elmm_batch_project(self.h, coef), "elmm_batch_project")

    def step(self, n=1) -> ElmmStats:
        st = ElmmStats()
        check(lib().elmm_batch_step(self.h, n, C.byref(st)), "elmm_batch_step")
        return st

    def set_solids(self, d, solids):
        """Solid bodies of domain d (gpu_elmm_b200.solids.Solids, or None)."""
        st = None if solids is None else solids.struct()
        check(lib().elmm_batch_set_solids(self.h, d, None if st is None else C.cast(C.byref(st), C.c_void_p)),
              "elmm_batch_set_solids")

    def set_puffs(self, d, puffs, volumes):
        """Puff sources of domain d, as for Domain.set_puffs."""
        from .config import make_puffs
        P, n_p, V, n_v = make_puffs(puffs, volumes)
        check(lib().elmm_batch_set_puffs(self.h, d, C.cast(P, C.c_void_p), n_p, C.cast(V, C.c_void_p), n_v),
              "elmm_batch_set_puffs")
        self.__dict__.setdefault("_puffs", {})[d] = (P, V)

    TUNING_KEYS = ("scalar_tile_rows", "tri_tile_cols", "momentum_z_chunk", "sgs_z_chunk")

    def tuning(self):
        """Tile shapes chosen by the autotuner at the first step (or set)."""
        out = (C.c_int32 * len(self.TUNING_KEYS))()
        check(lib().elmm_batch_get_tuning(self.h, out, len(out)), "elmm_batch_get_tuning")
        return dict(zip(self.TUNING_KEYS, list(out)))

    def set_tuning(self, **shapes):
        """Sets tile shapes instead of the autotuner (keys of TUNING_KEYS;
        the ones not given keep their values)."""
        cur = self.tuning()
        cur.update(shapes)
        vals = (C.c_int32 * len(self.TUNING_KEYS))(*[cur[k] for k in self.TUNING_KEYS])
        check(lib().elmm_batch_set_tuning(self.h, vals, len(vals)), "elmm_batch_set_tuning")

    def profile_stage(self, stage=2, reps=5):
        """Mean device time (ms) of each kernel kind of one RK3 stage over the whole batch."""
        ms = (C.c_double * KERNEL_COUNT)()
        check(lib().elmm_batch_profile_stage(self.h, stage, reps, ms), "elmm_batch_profile_stage")
        return dict(zip(KERNEL_NAMES, list(ms)))


class Slabs:
    """One domain split into z-slabs (an elmm_slabs handle): slab s holds
    levels k0+1..k0+nz[s] on GPU devices[s]; the host arrays are the whole
    domain's, as for Domain."""

    def __init__(self, cfg: ElmmConfig, nslabs: int, devices=None, nz=None):
        self.cfg = cfg
        self.grid: Grid = grid_of(cfg)
        dv = (C.c_int32 * nslabs)(*devices) if devices is not None else None
        nzs = (C.c_int32 * nslabs)(*nz) if nz is not None else None
        h = C.c_void_p()
        check(lib().elmm_slabs_create(C.byref(cfg), nslabs, dv, nzs, C.byref(h)), "elmm_slabs_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().elmm_slabs_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, U, V, W, Pr=None):
        check(lib().elmm_slabs_upload_state(self.h, ptr(U), ptr(V), ptr(W), ptr(Pr)), "elmm_slabs_upload_state")

    def download(self):
        g = self.grid
        U, V, W, Pr = np.zeros(g.shape_u()), np.zeros(g.shape_v()), np.zeros(g.shape_w()), np.zeros(g.shape_p())
        check(lib().elmm_slabs_download_state(self.h, ptr(U), ptr(V), ptr(W), ptr(Pr)), "elmm_slabs_download_state")
        return U, V, W, Pr

    def project(self, coef=1.0) -> ElmmStats:
        st = ElmmStats()
        check(lib().elmm_slabs_project(self.h, coef, C.byref(st)), "elmm_slabs_project")
        return st

    def step(self, n=1) -> ElmmStats:
        st = ElmmStats()
        check(lib().elmm_slabs_step(self.h, n, C.byref(st)), "elmm_slabs_step")
        return st

    def upload_temperature(self, T):
        check(lib().elmm_slabs_upload_temperature(self.h, ptr(T)), "elmm_slabs_upload_temperature")

    def upload_scalar(self, sc, S):
        check(lib().elmm_slabs_upload_scalar(self.h, sc, ptr(S)), "elmm_slabs_upload_scalar")

    def field(self, fid):
        """ELMM_FIELD_TEMPERATURE or ELMM_FIELD_SCALAR + sc - 1 of the whole domain."""
        a = np.zeros(self.grid.shape_t())
        check(lib().elmm_slabs_download_field(self.h, fid, ptr(a)), "elmm_slabs_download_field")
        return a

    def scalar(self, sc):
        return self.field(FIELD_SCALAR + sc - 1)

    def set_puffs(self, puffs, volumes):
        """Puff sources as Domain.set_puffs (cells of the whole domain)."""
        from .config import make_puffs
        P, n_p, V, n_v = make_puffs(puffs, volumes)
        check(lib().elmm_slabs_set_puffs(self.h, C.cast(P, C.c_void_p), n_p, C.cast(V, C.c_void_p), n_v),
              "elmm_slabs_set_puffs")
        self._puffs = (P, V)

    def scalar_slices(self, sc):
        g = self.grid
        xy = np.zeros((g.Prny, g.Prnx)) if self.cfg.avg_slice_k > 0 else None
        xz = np.zeros((g.Prnz, g.Prnx)) if self.cfg.avg_slice_j > 0 else None
        check(lib().elmm_slabs_download_scalar_slices(self.h, sc, ptr(xy), ptr(xz)), "elmm_slabs_download_scalar_slices")
        return xy, xz

    def march_host(self, U, V, W, Pr, n=1) -> ElmmStats:
        """elmm_slabs_march_host: the arrays are updated in place."""
        st = ElmmStats()
        check(lib().elmm_slabs_march_host(self.h, ptr(U), ptr(V), ptr(W), ptr(Pr), n, C.byref(st)),
              "elmm_slabs_march_host")
        return st

    # real32 host arrays of a prec=sp host
    def upload_f32(self, U, V, W, Pr=None):
        check(lib().elmm_slabs_upload_state_float(self.h, fptr(U), fptr(V), fptr(W), fptr(Pr)),
              "elmm_slabs_upload_state_float")

    def download_f32(self):
        g = self.grid
        out = [np.zeros(s, dtype=np.float32) for s in (g.shape_u(), g.shape_v(), g.shape_w(), g.shape_p())]
        check(lib().elmm_slabs_download_state_float(self.h, *[fptr(a) for a in out]), "elmm_slabs_download_state_float")
        return tuple(out)

    def march_host_f32(self, U, V, W, Pr, n=1) -> ElmmStats:
        st = ElmmStats()
        check(lib().elmm_slabs_march_host_float(self.h, fptr(U), fptr(V), fptr(W), fptr(Pr), n, C.byref(st)),
              "elmm_slabs_march_host_float")
        return st


class PoissonSolver:
    """The PoisSolver-compatible solver (poisson_solver_new/_execute/_finalize);
    host_f32=True: the *_float variants of a single-precision host (float32
    lengths, grid and arrays)."""

    def __init__(self, n, L=None, bcs=(3, 3, 3, 3, 5, 5), precision=0, device=0, zW=None, host_f32=False):
        self.n = tuple(int(x) for x in n)
        self.f32 = host_f32
        nn = (C.c_int32 * 3)(*self.n)
        bb = (C.c_int32 * 6)(*bcs)
        h = C.c_void_p()
        if host_f32:
            if zW is None:
                LL = (C.c_float * 3)(*L)
                check(lib().elmm_poisson_solver_new_float(C.byref(h), nn, LL, bb, precision, device),
                      "poisson_solver_new_float")
            else:
                zW = np.ascontiguousarray(zW, dtype=np.float32)
                zPr = ((zW[:-1] + zW[1:]) / 2).astype(np.float32)
                self._keep = (zW, zPr)
                Lxy = (C.c_float * 2)(L[0], L[1])
                check(lib().elmm_poisson_solver_nonuniform_z_new_float(C.byref(h), nn, Lxy, fptr(zPr), fptr(zW), bb,
                                                                       precision, device),
                      "poisson_solver_nonuniform_z_new_float")
        elif zW is None:
            LL = (C.c_double * 3)(*L)
            check(lib().elmm_poisson_solver_new(C.byref(h), nn, LL, bb, precision, device), "poisson_solver_new")
        else:
            zW = np.ascontiguousarray(zW, dtype=np.float64)
            zPr = (zW[:-1] + zW[1:]) / 2
            self._keep = (zW, zPr)
            Lxy = (C.c_double * 2)(L[0], L[1])
            check(lib().elmm_poisson_solver_nonuniform_z_new(C.byref(h), nn, Lxy, ptr(zPr), ptr(zW), bb, precision,
                                                             device), "poisson_solver_nonuniform_z_new")
        self.h = h

    def execute(self, Phi, RHS):
        if self.f32:
            check(lib().elmm_poisson_solver_execute_float(self.h, fptr(Phi), fptr(RHS)), "poisson_solver_execute_float")
        else:
            check(lib().elmm_poisson_solver_execute(self.h, ptr(Phi), ptr(RHS)), "poisson_solver_execute")
        return Phi

    def close(self):
        if getattr(self, "h", None):
            lib().elmm_poisson_solver_finalize(self.h)
            self.h = None

    __del__ = close
