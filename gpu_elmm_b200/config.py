"""ctypes mirror of ``elmm_config`` / ``elmm_stats`` (include/elmm_gpu.h).

The fields are the module globals of the reference that the hot path reads
(src/parameters.f90, src/subgrid.f90:18, src/filters.f90:14), so a host that
already parsed an ELMM configuration can fill the struct one to one.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

ABI_VERSION = 5

# Boundary-condition codes of src/parameters.f90:249-250.
BC_NOSLIP, BC_FREESLIP, BC_PERIODIC, BC_DIRICHLET, BC_NEUMANN, BC_CONSTFLUX = 1, 2, 3, 4, 5, 6
# Sides We, Ea, So, No, Bo, To (src/parameters.f90:193, zero-based here).
WE, EA, SO, NO, BO, TO = range(6)

PREC_FP64, PREC_MIXED = 0, 1

FIELD_U, FIELD_V, FIELD_W, FIELD_PR, FIELD_VISCOSITY = 0, 1, 2, 3, 4
FIELD_U2, FIELD_V2, FIELD_W2 = 5, 6, 7
FIELD_USTAR, FIELD_VSTAR, FIELD_WSTAR, FIELD_PHI = 8, 9, 10, 11
FIELD_TEMPERATURE, FIELD_TDIFF, FIELD_TEMPERATURE_ADV = 12, 13, 14
FIELD_SCALAR, FIELD_SCALAR_ADV = 16, 20  # + (sc - 1)

MAX_SCALARS, MAX_POINT_SOURCES = 4, 8

STATUS_NAMES = {
    0: "ELMM_OK", 1: "ELMM_ERR_INVALID_CONFIG", 2: "ELMM_ERR_OOM", 3: "ELMM_ERR_NAN",
    4: "ELMM_ERR_CUDA", 5: "ELMM_ERR_TIMEOUT", 6: "ELMM_ERR_INVALID_ARG", 7: "ELMM_ERR_ADMISSION",
}


class ElmmPointSource(C.Structure):
    """ScalarPointSource (src/pointsources.f90:8-13)."""
    _fields_ = [
        ("scalar_number", C.c_int32),
        ("reserved", C.c_int32),
        ("position", C.c_double * 3),
        ("flux", C.c_double),
    ]


class ElmmConfig(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("Prnx", C.c_int32), ("Prny", C.c_int32), ("Prnz", C.c_int32),
        ("Btype", C.c_int32 * 6),
        ("xmin", C.c_double), ("ymin", C.c_double), ("zmin", C.c_double),
        ("dxmin", C.c_double), ("dymin", C.c_double), ("dzmin", C.c_double),
        ("zW", C.POINTER(C.c_double)),
        ("dt", C.c_double),
        ("molecular_viscosity", C.c_double),
        ("C_Smagorinsky", C.c_double),
        ("filter_ratio", C.c_double),
        ("sgstype", C.c_int32),
        ("wallmodeltype", C.c_int32),
        ("z0", C.c_double * 6),
        ("enable_pr_gradient_x_uniform", C.c_int32),
        ("enable_pr_gradient_y_uniform", C.c_int32),
        ("pr_gradient_x", C.c_double), ("pr_gradient_y", C.c_double),
        ("precision", C.c_int32),
        ("max_refine_sweeps", C.c_int32),
        ("refine_tol", C.c_double),
        ("enable_CFL_check", C.c_int32),
        ("device", C.c_int32),
        ("enable_buoyancy", C.c_int32),
        ("TempBtype", C.c_int32 * 6),
        ("sideTemp", C.c_double * 6),
        ("temperature_ref", C.c_double),
        ("grav_acc", C.c_double),
        ("molecular_diffusivity", C.c_double),
        ("num_scalars", C.c_int32),
        ("ScalBtype", C.c_int32 * 6),
        ("sideScal", C.c_double * 6),
        ("num_point_sources", C.c_int32),
        ("reserved0", C.c_int32),
        ("point_sources", ElmmPointSource * MAX_POINT_SOURCES),
        ("avg_slice_k", C.c_int32),
        ("avg_slice_j", C.c_int32),
        ("avg_weight", C.c_double),
        ("variable_time_steps", C.c_int32),
        ("reserved1", C.c_int32),
        ("CFL", C.c_double),
        ("dt_max", C.c_double),
        ("end_time", C.c_double),
    ]


MAX_PUFFS, MAX_PUFF_VOLUMES = 4, 16


class ElmmPuff(C.Structure):
    """PuffSource (src/puffs.f90:15-21)."""
    _fields_ = [("start_time", C.c_double), ("end_time", C.c_double), ("period", C.c_double),
                ("duration", C.c_double), ("clear", C.c_int32), ("reserved", C.c_int32)]


class ElmmPuffVolume(C.Structure):
    """A ScalarFlVolume of a puff."""
    _fields_ = [("puff", C.c_int32), ("scalar_number", C.c_int32), ("xi", C.c_int32), ("yj", C.c_int32),
                ("zk", C.c_int32), ("reserved", C.c_int32), ("flux", C.c_double)]


def make_puffs(puffs, volumes):
    """ctypes arrays and counts for elmm_set_puffs: puffs as (start, end,
    period, duration, clear), volumes as (puff, scalar_number, (i, j, k), flux)."""
    P = (ElmmPuff * max(1, len(puffs)))()
    for n, (a, b, per, dur, clr) in enumerate(puffs):
        P[n] = ElmmPuff(a, b, per, dur, int(clr), 0)
    V = (ElmmPuffVolume * max(1, len(volumes)))()
    for n, (p, sc, (i, j, k), fl) in enumerate(volumes):
        V[n] = ElmmPuffVolume(p, sc, i, j, k, 0, fl)
    return P, len(puffs), V, len(volumes)


IB_MAX_INTERP = 6


class ElmmIBPoint(C.Structure):
    """TIBPoint (src/immersedboundary.f90:552-564)."""
    _fields_ = [
        ("xi", C.c_int32), ("yj", C.c_int32), ("zk", C.c_int32), ("interp", C.c_int32),
        ("ii", C.c_int32 * IB_MAX_INTERP), ("jj", C.c_int32 * IB_MAX_INTERP), ("kk", C.c_int32 * IB_MAX_INTERP),
        ("coef", C.c_double * IB_MAX_INTERP),
    ]


class ElmmWMPoint(C.Structure):
    """WMPointUVW at a solid face (src/wallmodels.f90:68-98)."""
    _fields_ = [
        ("component", C.c_int32), ("direction", C.c_int32),
        ("xi", C.c_int32), ("yj", C.c_int32), ("zk", C.c_int32), ("reserved", C.c_int32),
        ("dist", C.c_double * 3), ("z0", C.c_double), ("temperature_flux", C.c_double),
    ]


class ElmmSolids(C.Structure):
    _fields_ = [
        ("n_ib", C.c_int64 * 3), ("ib", C.POINTER(ElmmIBPoint) * 3),
        ("n_null", C.c_int64 * 3), ("null_ijk", C.POINTER(C.c_int32) * 3),
        ("n_scalfl", C.c_int64), ("scalfl", C.POINTER(ElmmIBPoint)),
        ("n_wm", C.c_int64), ("wm", C.POINTER(ElmmWMPoint)),
        ("n_bottom_skip", C.c_int64 * 3), ("bottom_skip_ij", C.POINTER(C.c_int32) * 3),
        ("n_solid_pr", C.c_int64), ("solid_pr_ijk", C.POINTER(C.c_int32)),
        ("n_wm_pr", C.c_int64), ("wm_pr_ijk", C.POINTER(C.c_int32)),
        ("n_heat_pr", C.c_int64), ("heat_pr_ijk", C.POINTER(C.c_int32)), ("heat_pr_q", C.POINTER(C.c_double)),
        ("n_wall_pr", C.c_int64), ("wall_pr_ijk", C.POINTER(C.c_int32)),
    ]


class ElmmStats(C.Structure):
    _fields_ = [
        ("steps_done", C.c_int32),
        ("nan_detected", C.c_int32),
        ("time", C.c_double),
        ("dt", C.c_double),
        ("cfl", C.c_double),
        ("max_div", C.c_double),
        ("refine_sweeps", C.c_int32),
        ("kernels", C.c_int32),
        ("elapsed_ms", C.c_double),
    ]


@dataclass
class Grid:
    """Sizes of the staggered grid, src/initial.f90:871-896."""

    Prnx: int
    Prny: int
    Prnz: int
    btype: tuple

    @property
    def Unx(self):
        return self.Prnx if self.btype[EA] == BC_PERIODIC else self.Prnx - 1

    @property
    def Uny(self):
        return self.Prny

    @property
    def Unz(self):
        return self.Prnz

    @property
    def Vnx(self):
        return self.Prnx

    @property
    def Vny(self):
        return self.Prny if self.btype[NO] == BC_PERIODIC else self.Prny - 1

    @property
    def Vnz(self):
        return self.Prnz

    @property
    def Wnx(self):
        return self.Prnx

    @property
    def Wny(self):
        return self.Prny

    @property
    def Wnz(self):
        return self.Prnz if self.btype[TO] == BC_PERIODIC else self.Prnz - 1

    # host (Fortran-layout) shapes as numpy (k, j, i) arrays
    def shape_u(self):
        return (self.Unz + 6, self.Uny + 6, self.Unx + 6)

    def shape_v(self):
        return (self.Vnz + 6, self.Vny + 6, self.Vnx + 6)

    def shape_w(self):
        return (self.Wnz + 6, self.Wny + 6, self.Wnx + 6)

    def shape_p(self):
        return (self.Prnz + 4, self.Prny + 4, self.Prnx + 4)

    def shape_rhs(self):
        return (self.Prnz + 2, self.Prny + 2, self.Prnx + 2)

    def shape_t(self):
        """Temperature(-2:Prnx+3,-2:Prny+3,-2:Prnz+3)."""
        return (self.Prnz + 6, self.Prny + 6, self.Prnx + 6)

    def cells(self):
        return self.Prnx * self.Prny * self.Prnz


def make_config(Prnx, Prny, Prnz, *, btype=(BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC,
                                           BC_NOSLIP, BC_FREESLIP),
                dx=1.0, dy=1.0, dz=1.0, dt=0.02, nu=1.0 / 70000, cs=0.1, sgstype=1,
                wallmodeltype=None, z0=0.01, precision=PREC_FP64, zW=None,
                pr_gradient_x=None, pr_gradient_y=None, max_refine_sweeps=0,
                refine_tol=1e-6, cfl_check=0, device=0, origin=(0.0, 0.0, 0.0), buoyancy=False,
                temperature_ref=295.0, grav_acc=9.81, prandtl=0.7, num_scalars=0, point_sources=(),
                avg_slice_k=0, avg_slice_j=0, avg_weight=0.0, variable_dt=False, cfl=0.5, dt_max=None,
                end_time=0.0, heat_flux=(0.0, 0.0), temperature_bc=None, scalar_bc=None):
    """Builds an ElmmConfig.  The wall model defaults to on when an SGS model
    is on (src/initial.f90:2782-2787).  ``zW`` (Prnz+1 values) selects the
    stretched-z grid; the array is kept alive on the returned struct.
    ``buoyancy`` adds the potential-temperature field with adiabatic
    (zero-flux) bottom and top and periodic x and y, or with the constant
    surface heat fluxes ``heat_flux`` = (sideTemp at the bottom, at the top),
    K m/s positive upward, at wall-model walls; ``num_scalars`` passive
    scalars get zero-flux walls.  ``temperature_bc`` / ``scalar_bc`` set the
    bottom and top kinds of CommonBase instead: ((kind, value) at the
    bottom, (kind, value) at the top), kind BC_CONSTFLUX, BC_DIRICHLET or
    BC_NEUMANN.  ``point_sources``: (scalar_number,
    (x, y, z), flux) triples.  ``avg_slice_k`` / ``avg_slice_j`` select the
    time-averaged slices, ``avg_weight`` the weight of one step.
    ``variable_dt`` switches on the variable time steps of TimeStepLength
    with target ``cfl``, longest step ``dt_max`` (default ``dt``) and, if
    positive, ``end_time``."""
    c = ElmmConfig()
    c.abi_version = ABI_VERSION
    c.Prnx, c.Prny, c.Prnz = Prnx, Prny, Prnz
    for s in range(6):
        c.Btype[s] = btype[s]
    c.xmin, c.ymin, c.zmin = origin
    c.dxmin, c.dymin, c.dzmin = dx, dy, dz
    if zW is not None:
        zw = np.ascontiguousarray(zW, dtype=np.float64)
        assert zw.shape == (Prnz + 1,)
        c._zw_keepalive = zw
        c.zW = zw.ctypes.data_as(C.POINTER(C.c_double))
        c.zmin = float(zw[0])
    c.dt = dt
    c.molecular_viscosity = nu
    c.C_Smagorinsky = cs
    c.filter_ratio = 1.0
    c.sgstype = sgstype
    if wallmodeltype is None:
        wallmodeltype = 1 if sgstype > 0 else 0
    c.wallmodeltype = wallmodeltype
    for s in range(6):
        c.z0[s] = z0
    if pr_gradient_x is not None:
        c.enable_pr_gradient_x_uniform = 1
        c.pr_gradient_x = pr_gradient_x
    if pr_gradient_y is not None:
        c.enable_pr_gradient_y_uniform = 1
        c.pr_gradient_y = pr_gradient_y
    c.precision = precision
    c.max_refine_sweeps = max_refine_sweeps
    c.refine_tol = refine_tol
    c.enable_CFL_check = cfl_check
    c.device = device
    c.enable_buoyancy = 1 if buoyancy else 0
    for s in range(6):
        c.TempBtype[s] = BC_PERIODIC if btype[s] == BC_PERIODIC else BC_CONSTFLUX
        c.sideTemp[s] = 0.0
    c.sideTemp[BO], c.sideTemp[TO] = heat_flux
    if temperature_bc is not None:
        (c.TempBtype[BO], c.sideTemp[BO]), (c.TempBtype[TO], c.sideTemp[TO]) = temperature_bc
    c.temperature_ref = temperature_ref
    c.grav_acc = grav_acc
    c.molecular_diffusivity = nu / prandtl
    c.num_scalars = num_scalars
    for s in range(6):
        c.ScalBtype[s] = BC_PERIODIC if btype[s] == BC_PERIODIC else BC_CONSTFLUX
        c.sideScal[s] = 0.0
    if scalar_bc is not None:
        (c.ScalBtype[BO], c.sideScal[BO]), (c.ScalBtype[TO], c.sideScal[TO]) = scalar_bc
    assert len(point_sources) <= MAX_POINT_SOURCES
    c.num_point_sources = len(point_sources)
    for q, (sc, pos, flux) in enumerate(point_sources):
        c.point_sources[q].scalar_number = sc
        for a in range(3):
            c.point_sources[q].position[a] = pos[a]
        c.point_sources[q].flux = flux
    c.avg_slice_k, c.avg_slice_j, c.avg_weight = avg_slice_k, avg_slice_j, avg_weight
    c.variable_time_steps = 1 if variable_dt else 0
    c.CFL = cfl
    c.dt_max = dt if dt_max is None else dt_max
    c.end_time = end_time
    return c


def grid_of(cfg: ElmmConfig) -> Grid:
    return Grid(cfg.Prnx, cfg.Prny, cfg.Prnz, tuple(cfg.Btype[s] for s in range(6)))
