/*
 * elmm_gpu.h -- C-ABI of the B200 (sm_100a) per-timestep flow solve of ELMM.
 *
 * This library replaces, behind plain C entry points, the RK3 stage loop of
 * the ELMM LES model and the external Poisson solver it calls:
 *
 *   TMarchRK3(U,V,W,Pr,Temperature,Moisture,Scalar,delta)   src/tsteps.f90:24-243
 *       called from the time loop in src/main.f90:112
 *   PressureCorrection(U,V,W,Pr,Q,coef)                      src/pressure.f90:169-266
 *       called for the initial projection in src/initial.f90:4290
 *   poisson_solver_new / _execute / _finalize (PoisSolver)   src/poisson.f90:76-210
 *       (module of the un-vendored PoisFFT / poisson-solver library)
 *
 * Conventions
 *   - Every entry point returns an int status: ELMM_OK (0) or an ELMM_ERR_* code.
 *     The Fortran host maps a nonzero status to error_stop (src/stop.f90).
 *   - Host arrays are Fortran-ordered (x fastest) with the reference's bounds:
 *       U(-2:Unx+3,-2:Uny+3,-2:Unz+3), V(-2:Vnx+3,..), W(-2:Wnx+3,..)  (src/main.f90:231-233)
 *       Pr(-1:Prnx+2,-1:Prny+2,-1:Prnz+2), Viscosity likewise            (src/main.f90:234, :272)
 *       Phi(-1:Prnx+2,..), RHS(0:Prnx+1,..)                               (src/pressure.f90:189-190)
 *     where Unx = Prnx if x is periodic else Prnx-1, and likewise Vny, Wnz
 *     (src/initial.f90:871-896).
 *   - A handle owns all of its device memory; the state U, V, W, Pr stays
 *     resident in HBM between calls.  Calls on one handle are serialised by the
 *     caller; different handles may be used from different host threads.
 *   - No entry point falls back to the CPU: without a usable CUDA device every
 *     call that needs one returns ELMM_ERR_CUDA.
 */
#ifndef ELMM_GPU_H
#define ELMM_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ELMM_ABI_VERSION 5

/* Status codes. */
enum {
  ELMM_OK = 0,
  ELMM_ERR_INVALID_CONFIG = 1, /* a config field is out of range or unsupported */
  ELMM_ERR_OOM = 2,            /* device allocation failed */
  ELMM_ERR_NAN = 3,            /* NaN/Inf in the input state or produced by a step */
  ELMM_ERR_CUDA = 4,           /* a CUDA call failed, or no device */
  ELMM_ERR_TIMEOUT = 5,        /* a bounded device-side wait gave up */
  ELMM_ERR_INVALID_ARG = 6,    /* NULL pointer, bad size, bad field id */
  ELMM_ERR_ADMISSION = 7       /* request refused by the HBM budget of a serving loop */
};

/* Boundary-condition codes: the values of BC_NOSLIP.. in src/parameters.f90:249-250. */
enum {
  ELMM_BC_NOSLIP = 1,
  ELMM_BC_FREESLIP = 2,
  ELMM_BC_PERIODIC = 3,
  ELMM_BC_DIRICHLET = 4,
  ELMM_BC_NEUMANN = 5,
  ELMM_BC_CONSTFLUX = 6
};

/* Side indices (src/parameters.f90:193 numbers them We=1..To=6; here 0..5). */
enum { ELMM_WE = 0, ELMM_EA = 1, ELMM_SO = 2, ELMM_NO = 3, ELMM_BO = 4, ELMM_TO = 5 };

/* Arithmetic of the state and of the stencil / FFT kernels. */
enum {
  ELMM_PREC_FP64 = 0,  /* plain FP64 everywhere */
  ELMM_PREC_MIXED = 1  /* FP32 state, stencils and FFT; FP64 reductions, FP64
                          zero-wavenumber mode and FP64 divergence residual for
                          the defect correction of the pressure solve */
};

/* Fields that elmm_download_field can return (host layout as above). */
enum {
  ELMM_FIELD_U = 0, ELMM_FIELD_V = 1, ELMM_FIELD_W = 2, ELMM_FIELD_PR = 3,
  ELMM_FIELD_VISCOSITY = 4,
  ELMM_FIELD_U2 = 5, ELMM_FIELD_V2 = 6, ELMM_FIELD_W2 = 7,
  ELMM_FIELD_USTAR = 8, ELMM_FIELD_VSTAR = 9, ELMM_FIELD_WSTAR = 10,
  ELMM_FIELD_PHI = 11,
  ELMM_FIELD_TEMPERATURE = 12,   /* Temperature(-2:Prnx+3,-2:Prny+3,-2:Prnz+3) */
  ELMM_FIELD_TDIFF = 13,         /* TDiff(-1:Prnx+2,...), turbulent + molecular diffusivity */
  ELMM_FIELD_TEMPERATURE_ADV = 14, /* Temperature_adv(-2:...), the stage tendency */
  ELMM_FIELD_SCALAR = 16,        /* + (sc - 1): Scalar(-2:Prnx+3,-2:Prny+3,-2:Prnz+3,sc) */
  ELMM_FIELD_SCALAR_ADV = 20     /* + (sc - 1): Scalar_adv(-2:...,sc), the stage tendency */
};

/* Passive scalars and their point sources (src/scalars.f90:88-381,
 * src/pointsources.f90:1-68). */
#define ELMM_MAX_SCALARS 4
#define ELMM_MAX_POINT_SOURCES 8

/* ScalarPointSource (src/pointsources.f90:8-13): a continuous source of
 * `flux` units per time unit at `position`, released into the single grid
 * cell that contains it (GridCoords, src/boundaries.f90:54-97) as a volume
 * source flux / volumePr of that cell. */
typedef struct elmm_point_source {
  int32_t scalar_number;        /* 1..num_scalars */
  int32_t reserved;             /* 0 */
  double position[3];           /* x, y, z */
  double flux;                  /* total flux, units per time unit */
} elmm_point_source;

/*
 * Configuration of one domain.  It carries the module globals of
 * src/parameters.f90 that the hot path reads, filled by the host from its own
 * parsed configuration (src/initial.f90 ReadConfiguration).
 */
typedef struct elmm_config {
  int32_t abi_version;          /* must be ELMM_ABI_VERSION */
  int32_t Prnx, Prny, Prnz;     /* pressure-grid cells (src/parameters.f90:55) */
  int32_t Btype[6];             /* velocity BC per side, ELMM_BC_* */
  double xmin, ymin, zmin;      /* im_xmin.. : xU(0), yV(0), zW(0) */
  double dxmin, dymin, dzmin;   /* uniform spacings */
  const double *zW;             /* NULL: uniform z.  Else zW(0:Prnz), Prnz+1 values,
                                   the stretched grid of zgrid.txt (src/initial.f90:254-283) */
  double dt;                    /* dt_constant (src/parameters.f90:89) */
  double molecular_viscosity;   /* src/parameters.f90:133 (1/70000 by default) */
  double C_Smagorinsky;         /* src/subgrid.f90:18 (0.122 by default) */
  double filter_ratio;          /* filter_ratios(filtertype), 1.0 (src/filters.f90:14) */
  int32_t sgstype;              /* 0: molecular only, 1: Smagorinsky (src/subgrid.f90:15) */
  int32_t wallmodeltype;        /* 0: off, 1: log-law wall model at no-slip sides */
  double z0[6];                 /* roughness per side z0W..z0T (src/parameters.f90:145); 0: smooth wall (WMFlatStress) */
  int32_t enable_pr_gradient_x_uniform, enable_pr_gradient_y_uniform;
  double pr_gradient_x, pr_gradient_y; /* mean pressure-gradient forcing (src/dynamics.f90:83-117) */
  int32_t precision;            /* ELMM_PREC_* */
  int32_t max_refine_sweeps;    /* mixed path: defect-correction sweeps, 0..3 */
  double refine_tol;            /* mixed path: max|div u| that triggers a sweep */
  int32_t enable_CFL_check;     /* compute the CFL number each step (src/dynamics.f90:541) */
  int32_t device;               /* CUDA device ordinal */
  /* Potential temperature: transport by ScalarRK3 (src/scalars.f90:88-381) and
   * buoyancy in the W tendency (BuoyancyForce, src/dynamics.f90:608-690).
   * Supported: TempBtype periodic on the periodic x and y sides, and at the
   * bottom and top the kinds of CommonBase (src/scalarboundaries.f90:197-288):
   * ELMM_BC_DIRICHLET (sideTemp the value at the face), ELMM_BC_NEUMANN
   * (the gradient) or ELMM_BC_CONSTFLUX (the flux, K m/s positive upward;
   * 0 is adiabatic).  At a wall-model wall a flux is a surface heat flux:
   * it enters the cells next to the wall through the wall-model points
   * (src/scalars.f90:323-327), and a flux into the flow over a rough wall
   * makes the wall model's u* follow Monin-Obukhov similarity
   * (WM_MO_FluxStress, src/wallmodels.f90:1836-1854, 2255-2259).  A
   * Dirichlet value there is a surface temperature: the Monin-Obukhov wall
   * model computes the points' u* and surface flux from the temperature
   * difference each stage (WM_MO_Dirichlet / WM_MO_DirichletStress,
   * src/wallmodels.f90:1664-1716, 1858-1938) at a rough wall (z0 > 0);
   * at a smooth wall (z0 = 0) the flat branch runs (WMFlat u*, and the
   * points' flux keeps its initial zero, src/wallmodels.f90:2123-2146,
   * 2265-2275).
   * Elsewhere the ghost rules of CommonBase carry the kind. */
  int32_t enable_buoyancy;      /* 0: no temperature field */
  int32_t TempBtype[6];         /* temperature BC per side (src/initial.f90:347-352) */
  double sideTemp[6];           /* BC values: value, gradient or flux of the kind */
  double temperature_ref;       /* src/parameters.f90:220 (295 K) */
  double grav_acc;              /* src/parameters.f90:146 (9.81) */
  double molecular_diffusivity; /* molecular_viscosity / Prandtl (src/initial.f90:791; Prandtl 0.7) */
  /* Passive scalars (ScalarRK3's loop over num_of_scalars, src/scalars.f90:217-223):
   * the same KappaScalar advection, scalar diffusion with TDiff and wall-model
   * term as the temperature, plus point sources.  Without buoyancy TDiff is
   * set once by the initial projection and then kept, as in the reference
   * (src/initial.f90:4296-4313; src/dynamics.f90:904 updates it only with
   * buoyancy).  Supported ScalBtype: as TempBtype, every kind by the ghost
   * rules of CommonBase (the wall-model points carry no scalar flux). */
  int32_t num_scalars;          /* 0..ELMM_MAX_SCALARS */
  int32_t ScalBtype[6];         /* scalar BC per side (src/initial.f90:508-519) */
  double sideScal[6];           /* BC values: value, gradient or flux of the kind */
  int32_t num_point_sources;    /* 0..ELMM_MAX_POINT_SOURCES */
  int32_t reserved0;            /* 0 */
  elmm_point_source point_sources[ELMM_MAX_POINT_SOURCES];
  /* Time-averaged scalar slices (Scalar_avg of src/outputs.f90:1043-1045,
   * restricted to two planes): after every step avg += Scalar * avg_weight,
   * with avg_weight = dt / (timeavg2 - timeavg1) for an averaging window
   * that spans the run.  In FP64 on both precision paths. */
  int32_t avg_slice_k;          /* horizontal plane k = 1..Prnz, 0: none */
  int32_t avg_slice_j;          /* vertical x-z plane j = 1..Prny, 0: none */
  double avg_weight;            /* the weight of a step of length dt (variable steps: scaled by their length / dt) */
  /* Variable time steps: the variable_time_steps branch of TimeStepLength
   * (src/dynamics.f90:517-529, :547-548).  Each step takes, from the state
   * at its start, dt = min(CFL / U_dx_max, dt_max) with U_dx_max the largest
   * sum over the three directions of the larger face speed / spacing of a
   * cell; dt_max when the flow is at rest; the smallest positive normal
   * double when U_dx_max is NaN (the step then reports ELMM_ERR_NAN); and,
   * with end_time > 0, the step that would pass end_time ends there.  A step
   * that starts at end_time takes its CFL length and the call returns
   * ELMM_ERR_INVALID_ARG (the run was over).  The length of the last step
   * and the time come back in elmm_stats.  Off: the constant dt above. */
  int32_t variable_time_steps;
  int32_t reserved1;            /* 0 */
  double CFL;                   /* target CFL number of the variable steps */
  double dt_max;                /* the longest variable step */
  double end_time;              /* > 0: no variable step passes this time */
} elmm_config;

/* Diagnostics of elmm_step / elmm_project. */
typedef struct elmm_stats {
  int32_t steps_done;           /* steps completed by this call */
  int32_t nan_detected;         /* 1 if a NaN was seen in the CFL / divergence check */
  double time;                  /* simulated time after the call */
  double dt;                    /* time step used */
  double cfl;                   /* CFL number of the last step (enable_CFL_check) */
  double max_div;               /* max |div u| after the last projection, FP64 */
  int32_t refine_sweeps;        /* defect-correction sweeps run in the last stage */
  int32_t kernels;              /* kernel launches of the library in this call */
  double elapsed_ms;            /* device time of the call (CUDA events) */
} elmm_stats;

typedef struct elmm_handle elmm_handle;

/* Library identification: returns a static string. */
const char *elmm_version(void);

/* Fills *cfg with the reference defaults for a Prnx x Prny x Prnz box
 * (periodic x,y, no-slip bottom, free-slip top, Smagorinsky + wall model). */
int elmm_config_defaults(elmm_config *cfg, int32_t Prnx, int32_t Prny, int32_t Prnz);

/* Allocates the device state of one domain (the module arrays of src/dynamics.f90:13-17,
 * src/main.f90:229-285) and prepares the wall-model points
 * (src/wallmodels.f90:690-909) and the Poisson solver. */
int elmm_create(const elmm_config *cfg, elmm_handle **out);
int elmm_destroy(elmm_handle *h);

/* Host -> device copy of the state.  U, V, W, Pr are host arrays in the
 * Fortran layout above; Pr may be NULL (zero).  Returns ELMM_ERR_NAN if an
 * interior value is not finite. */
int elmm_upload_state(elmm_handle *h, const double *U, const double *V,
                      const double *W, const double *Pr);

/* Device -> host copy of the state, ghost cells filled as BoundUVW / Bound_Pr
 * leave them (src/boundaries.f90:398-1812, :1951-2091).  NULL pointers are skipped. */
int elmm_download_state(elmm_handle *h, double *U, double *V, double *W, double *Pr);

/* Device -> host copy of one field (ELMM_FIELD_*). */
int elmm_download_field(elmm_handle *h, int32_t field, double *host);

/* Host -> device copy of Temperature(-2:Prnx+3,-2:Prny+3,-2:Prnz+3) (interior
 * read; enable_buoyancy must be set).  Returns ELMM_ERR_NAN for non-finite
 * interior values.  The state is read back with elmm_download_field
 * (ELMM_FIELD_TEMPERATURE). */
int elmm_upload_temperature(elmm_handle *h, const double *T);

/* Host -> device copy of passive scalar sc (1..num_scalars) from
 * Scalar(-2:Prnx+3,-2:Prny+3,-2:Prnz+3,sc) (only the interior is read).
 * Returns ELMM_ERR_NAN for non-finite values. */
int elmm_upload_scalar(elmm_handle *h, int32_t sc, const double *S);

/* ---- puffs ----------------------------------------------------------------
 * PuffSource of src/puffs.f90:15-21: volume sources of passive scalars that
 * are switched on in windows of `duration` every `period` between
 * `start_time` and `end_time`; `clear` zeroes the puff's scalars at each
 * release.  The reference builds them in custom code (CustomPuffSources,
 * src/puffs.f90:129-139); here the host passes them.  Every elmm_step
 * applies PreparePuffs at the start of the step (the fraction of the step
 * that a window covers, :30-84) and DoPuffs in each scalar stage after the
 * point sources (:86-126, src/scalars.f90:366-372). */
#define ELMM_MAX_PUFFS 4
#define ELMM_MAX_PUFF_VOLUMES 16
typedef struct elmm_puff {
  double start_time, end_time, period, duration;
  int32_t clear, reserved;
} elmm_puff;

/* ScalarFlVolume of a puff: cell (xi, yj, zk) of the pressure grid, the
 * scalar it feeds (1..num_scalars) and its flux per unit volume. */
typedef struct elmm_puff_volume {
  int32_t puff;           /* 0..npuffs-1 */
  int32_t scalar_number;
  int32_t xi, yj, zk, reserved;
  double flux;
} elmm_puff_volume;

/* Installs the puffs of a single-domain handle (npuffs = 0 removes them);
 * their clock starts at the handle's current time.  Up to ELMM_MAX_PUFFS
 * puffs and ELMM_MAX_PUFF_VOLUMES volumes; ELMM_ERR_INVALID_ARG otherwise or
 * for a cell, scalar or puff index out of range.  elmm_run_stage does not
 * advance the puffs. */
int elmm_set_puffs(elmm_handle *h, const elmm_puff *puffs, int32_t npuffs, const elmm_puff_volume *volumes,
                   int32_t nvolumes);

/* ---- immersed solid bodies ----------------------------------------------
 * The host describes its solid bodies by the point lists its own geometry
 * pass builds once at start-up: GetSolidBodiesBC (FindInsideCells,
 * FindNeighbouringCells, InitImBoundaries, GetSolidBodiesWM_UVW;
 * src/immersedboundary.f90:1750-1771, src/solidbodies.f90:75-206) and
 * SetNullifiedPoints (src/initial.f90:4861-4962).  The library then applies,
 * every RK3 stage as TMarchRK3 does (src/tsteps.f90:146-206):
 *   - the viscosity of the ScalFl points from their interpolation points
 *     (SubgridStresses, src/dynamics.f90:899-902);
 *   - the wall-model fluxes at the solid faces (ComputeUVWFluxesWM and the
 *     wmfluxes-*-inc.f90 corrections, src/wallmodels.f90:2159-2338);
 *   - IBMomentum, IBMassSources and NullInterior (src/tsteps.f90:360-567).
 * Indices are the reference's: 1..n of the point's own field; interpolation
 * points may lie one cell into the ghost layer. */
#define ELMM_IB_MAX_INTERP 6

/* TIBPoint (src/immersedboundary.f90:552-564): the value at (xi,yj,zk) is
 * replaced by sum_n coef[n] * F(ii[n],jj[n],kk[n]) (TIBPoint_Interpolate,
 * :637-651); interp = 0 sets it to zero. */
typedef struct elmm_ib_point {
  int32_t xi, yj, zk;
  int32_t interp;
  int32_t ii[ELMM_IB_MAX_INTERP], jj[ELMM_IB_MAX_INTERP], kk[ELMM_IB_MAX_INTERP];
  double coef[ELMM_IB_MAX_INTERP];
} elmm_ib_point;

/* WMPointUVW at a solid face (src/wallmodels.f90:68-98, built by
 * GetSolidBodiesWM_UVW, src/immersedboundary.f90:139-306): a free velocity
 * point of `component` (1 U, 2 V, 3 W) whose neighbour in `direction`
 * (1..6 = -x, +x, -y, +y, -z, +z) is solid; dist is the vector to the
 * nearest point of the body, z0 its roughness length (> 0; 0 for a smooth
 * face, which needs a positive molecular viscosity), temperature_flux the
 * body's heat flux (SolidBody%temperature_flux of a rough body; with a
 * temperature, a flux into the flow makes the point's u* follow
 * WM_MO_FluxStress). */
typedef struct elmm_wm_point {
  int32_t component, direction;
  int32_t xi, yj, zk, reserved;
  double dist[3];
  double z0;
  double temperature_flux;
} elmm_wm_point;

typedef struct elmm_solids {
  int64_t n_ib[3];                   /* UIBPoints, VIBPoints, WIBPoints */
  const elmm_ib_point *ib[3];
  int64_t n_null[3];                 /* Unull, Vnull, Wnull: (i, j, k) triples */
  const int32_t *null_ijk[3];
  int64_t n_scalfl;                  /* ScalFlIBPoints (viscosity interpolation) */
  const elmm_ib_point *scalfl;
  int64_t n_wm;                      /* wall-model points at solid faces */
  const elmm_wm_point *wm;
  /* (i, j) pairs of the bottom-wall plane k = 1 that carry no wall-model
   * point, per component: GetOutsideBoundariesWM_UVW adds a bottom point only
   * where Xtype(i,j,1) == 0 and Xtype(i,j,0) <= 0 (src/wallmodels.f90:700-820) */
  int64_t n_bottom_skip[3];
  const int32_t *bottom_skip_ij[3];
  /* With a temperature or passive scalars, (i, j, k) triples: the solid Pr
   * cells (Prtype > 0, FindInsideCells, src/solidbodies.f90:75-206; i, j in
   * 1..n, k in -1..nz+2, the z ghost layers included), where the advection
   * tendency of a scalar is zeroed (src/scalars.f90:259-268), and
   * the Pr wall-model points of the scalar equations, whose div * S term
   * skips the faces towards solid cells (DivergenceWM,
   * src/wallmodels.f90:1117-1168): the fluid cells with a solid neighbour
   * (GetSolidBodiesWM, src/immersedboundary.f90:14-138) and the cells of a
   * wall-model wall with Prtype = 0 (src/wallmodels.f90:467-687), each
   * once (1..n).  Without a temperature or passive scalars both may be
   * empty. */
  int64_t n_solid_pr;
  const int32_t *solid_pr_ijk;
  int64_t n_wm_pr;
  const int32_t *wm_pr_ijk;
  /* With a temperature: the Pr wall-model points at solid faces that carry
   * a heat flux, (i, j, k) 1..n and temperature_flux x area_factor
   * (K / s; ComputeAreaFactor, src/wallmodels.f90:173-203), which each
   * temperature stage adds to the cell (TemperatureExtra,
   * src/scalars.f90:323-327). */
  int64_t n_heat_pr;
  const int32_t *heat_pr_ijk;
  const double *heat_pr_q;
  /* With a temperature: the Pr wall-model points of the no-slip z walls
   * that RemoveDuplicateWMPoints keeps (src/wallmodels.f90:373-410: the
   * point closer to its wall, a cell next to a body keeping the solid-face
   * point on a tie), (i, j, k) 1..n; they carry the wall's surface flux or
   * surface temperature. */
  int64_t n_wall_pr;
  const int32_t *wall_pr_ijk;
} elmm_solids;

/* Installs the solid bodies of a single-domain handle (copied; the host
 * arrays may be freed afterwards).  Requirements, checked here
 * (ELMM_ERR_INVALID_ARG otherwise): indices in range; no interpolation point
 * of a list is a forcing point of the same list; no forcing or nullified
 * point within one cell of a periodic boundary; a no-slip bottom wall with
 * the wall model; with a temperature no body whose solid cells border the
 * ghost cells of a side that has a heat flux or a prescribed temperature
 * and no wall-model points, the Pr lists above as for passive scalars, the heated
 * faces' points (each body's heat flux, src/immersedboundary.f90:118, 267)
 * and the kept wall points.  After each
 * temperature stage the solid cells with fluid neighbours take the mean of
 * those (src/scalars.f90:129-198).  The next elmm_step
 * applies IBMomentum once first, as the first call of TMarchRK3 does
 * (src/tsteps.f90:44-48).  Passing NULL removes the bodies. */
int elmm_set_solids(elmm_handle *h, const elmm_solids *s);

/* The time-averaged slices of scalar sc: xy(1:Prnx,1:Prny) at avg_slice_k and
 * xz(1:Prnx,1:Prnz) at avg_slice_j, column-major; either pointer may be NULL.
 * elmm_reset_scalar_averages zeroes both accumulators of every scalar. */
int elmm_download_scalar_slices(elmm_handle *h, int32_t sc, double *xy, double *xz);
int elmm_reset_scalar_averages(elmm_handle *h);

/* Asynchronous frame: copies U, V, W, Pr on a side stream into pinned staging
 * buffers owned by the handle and returns at once.  elmm_frame_wait blocks
 * until the copy has finished and copies the frame into the host arrays.
 * Replaces the pthread frame writer of src/frames_common.f90:120-164. */
int elmm_frame_begin(elmm_handle *h);
int elmm_frame_wait(elmm_handle *h, double *U, double *V, double *W, double *Pr);

/* PressureCorrection(U,V,W,Pr,Q,coef) on the resident state
 * (src/pressure.f90:169-266, Q = 0): the initial projection uses coef = 1
 * (src/initial.f90:4290).  Then, as the end of InitialConditions
 * (src/initial.f90:4291-4336): the initial eddy viscosity and scalar
 * diffusivity, and the wall model once on the projected fields (the u* and
 * surface fluxes its points carry into the first stage). */
int elmm_project(elmm_handle *h, double coef, elmm_stats *stats);

/* nsteps calls of TMarchRK3 (src/tsteps.f90:24-243) on the resident state. */
int elmm_step(elmm_handle *h, int32_t nsteps, elmm_stats *stats);

/* TMarchRK3(U,V,W,Pr,Temperature,...) on host arrays (src/tsteps.f90:24-243,
 * called from src/main.f90:112), for a host that keeps the state in its own
 * arrays between steps: uploads U, V, W, Pr (and Temperature when
 * enable_buoyancy is set; NULL otherwise), runs nsteps steps and writes the
 * state back, ghosts filled as BoundUVW / Bound_Pr leave them.  The host
 * copies of the fields overlap the device-side unpacking and packing of the
 * neighbouring fields; page-locked host arrays give the full copy bandwidth.
 * Equivalent to elmm_upload_state + elmm_upload_temperature + elmm_step +
 * elmm_download_state + elmm_download_field(ELMM_FIELD_TEMPERATURE). */
int elmm_march_host(elmm_handle *h, double *U, double *V, double *W, double *Pr, double *Temperature,
                    int32_t nsteps, elmm_stats *stats);

/* ---- single-precision host arrays ------------------------------------------
 * The reference's default release build is single precision: make_release
 * passes prec=sp (src/make_release:2), so knd = real32 (src/parameters.f90:
 * 17-21) and the host's U, V, W, Pr, Temperature, Scalar, Phi and RHS are
 * real32.  These entry points take float host arrays in the same layouts as
 * their double counterparts above; the library widens them on the way in
 * and rounds to nearest on the way out.  The device keeps the handle's own
 * precision (ELMM_PREC_*).  Same checks and status codes as the double
 * versions; elmm_march_host_float copies field by field (no overlap of the
 * copies). */
int elmm_upload_state_float(elmm_handle *h, const float *U, const float *V, const float *W, const float *Pr);
int elmm_download_state_float(elmm_handle *h, float *U, float *V, float *W, float *Pr);
int elmm_download_field_float(elmm_handle *h, int32_t field, float *host);
int elmm_upload_temperature_float(elmm_handle *h, const float *T);
int elmm_upload_scalar_float(elmm_handle *h, int32_t sc, const float *S);
int elmm_march_host_float(elmm_handle *h, float *U, float *V, float *W, float *Pr, float *Temperature,
                          int32_t nsteps, elmm_stats *stats);

/* One RK3 stage up to a stop point, for operator-level checks:
 *   stop = 1: after SubgridStresses (Viscosity, wall-model fluxes)
 *   stop = 2: after Convection + OtherTerms + BoundUVW (U2, Ustar)
 *   stop = 3: the full stage (projection and swap)
 * stage is 1..3.  Fields are read back with elmm_download_field. */
int elmm_run_stage(elmm_handle *h, int32_t stage, int32_t stop);

/* Fault injection for tests of the failure path (no counterpart in the
 * reference).  The momentum and SGS kernels wait for each plane's copies on
 * an mbarrier with a bounded number of tries; after wait_limit tries
 * (1048576 by default) a block gives up, waits (bounded) for its own copies
 * still in flight, leaves the tile undone and makes elmm_step return
 * ELMM_ERR_TIMEOUT; the handle stays usable.  skip_plane >= 0 makes the
 * kernels issue no copy for that plane index (0..Prnz+1), so its wait runs
 * out; -1 restores normal operation.  Set a small wait_limit with it (a few
 * hundred tries) so that the test is quick; the state after such a step is
 * incomplete and should be uploaded again. */
int elmm_set_fault_injection(elmm_handle *h, int32_t wait_limit, int32_t skip_plane);

/* Kernel timing of one stage (no counterpart in the reference; the
 * reference's per-part timers are src/tsteps.f90:113, :234-238): runs the
 * kernels of RK3 stage `stage` `reps` times on the handle's stream, each
 * bracketed by CUDA events, and writes the mean duration in ms of each
 * kernel kind to ms[ELMM_NKERNELS] in the order of ELMM_KERNEL_NAMES; "ghosts"
 * is the sum of the stage's ghost-shell launches, "temperature" the
 * temperature stage (0 without a temperature field).  The state advances as by
 * `reps` stages. */
#define ELMM_NKERNELS 11
#define ELMM_KERNEL_NAMES "sgs,momentum,fftx_fwd,ffty_fwd,tri,ffty_inv,fftx_inv,project,prref,ghosts,temperature"
int elmm_profile_stage(elmm_handle *h, int32_t stage, int32_t reps, double *ms);

/*
 * PoisSolver-compatible solver (the interface of src/poisson.f90:108-121,
 * :132, :178-189, :201).  Solves the discrete problem of Residue_variable_z
 * (src/poisson.f90:23-60): periodic x and y, periodic or staggered Neumann z,
 * by FFT in x and y and a tridiagonal solve in z.  bcs[6] are
 * ELMM_BC_PERIODIC or ELMM_BC_NEUMANN per side.
 */
typedef struct elmm_poisson elmm_poisson;
int elmm_poisson_solver_new(elmm_poisson **out, const int32_t n[3], const double L[3],
                            const int32_t bcs[6], int32_t precision, int32_t device);
int elmm_poisson_solver_nonuniform_z_new(elmm_poisson **out, const int32_t n[3],
                                         const double Lxy[2], const double *zPr,
                                         const double *zW, const int32_t bcs[6],
                                         int32_t precision, int32_t device);
/* Phi(-1:nx+2,-1:ny+2,-1:nz+2) out (interior written, ghosts untouched),
 * RHS(0:nx+1,0:ny+1,0:nz+1) in; host arrays.  Returns ELMM_ERR_NAN if an
 * interior RHS value is not finite (Phi then holds no solution). */
int elmm_poisson_solver_execute(elmm_poisson *s, double *Phi, const double *RHS);
int elmm_poisson_solver_finalize(elmm_poisson *s);
/* The float variants that a prec=sp host binds (poisson_solver_new_float,
 * poisson_solver_nonuniform_z_new_float, ..._execute_float,
 * ..._finalize_float: src/poisson.f90:82-84, :152-154): lengths, zPr(1:nz),
 * zW(0:nz), Phi and RHS are float host arrays with the bounds above.  The
 * arithmetic is the solver's `precision`.  One solver handle serves both the
 * uniform and the nonuniform-z execute and finalize calls. */
int elmm_poisson_solver_new_float(elmm_poisson **out, const int32_t n[3], const float L[3], const int32_t bcs[6],
                                  int32_t precision, int32_t device);
int elmm_poisson_solver_nonuniform_z_new_float(elmm_poisson **out, const int32_t n[3], const float Lxy[2],
                                               const float *zPr, const float *zW, const int32_t bcs[6],
                                               int32_t precision, int32_t device);
int elmm_poisson_solver_execute_float(elmm_poisson *s, float *Phi, const float *RHS);
int elmm_poisson_solver_finalize_float(elmm_poisson *s);

/*
 * No counterpart in the reference.  The solve of elmm_poisson_solver_execute
 * (FP64, uniform z grid) on arrays that are already in device memory,
 * without allocating anything.  It is meant for callers that cannot call
 * cudaMalloc: a host whose memory pool already owns the GPU's memory (a
 * CUDA Fortran or OpenACC program, or a framework's caching allocator, that
 * reserved it up front), and a caller on a path where cudaMalloc/cudaFree
 * would synchronise the whole device.
 *
 * Its working memory (spectral buffer, box copy of Phi, FFT tables and
 * descriptors) is one fixed array of ELMM_NOALLOC_SCRATCH_BYTES in the
 * library's device image: every GPU that loads the library holds those
 * 16 MiB until the process exits.  That covers grids up to about 64x64x64
 * or 128x128x48; a grid needing more is rejected with ELMM_ERR_INVALID_ARG
 * and a message giving the bytes it needs.  The caller still owns the input
 * and the output:
 *   RHS  device pointer, RHS(0:nx+1,0:ny+1,0:nz+1), interior read
 *   Phi  device pointer, Phi(-1:nx+2,-1:ny+2,-1:nz+2), interior written,
 *        ghosts untouched
 * n, L and bcs mean what they mean for elmm_poisson_solver_new.  The call
 * enqueues its work on `stream` (a cudaStream_t of `device`; NULL is the
 * legacy default stream) and returns with the caller's current device as it
 * found it: Phi is ready once the stream gets there.  Non-finite RHS values are not reported.
 *
 * The first call on a device does a one-time set-up (it looks up the
 * array's device address and raises the kernels' shared-memory limit), so
 * make that first call before any stream capture.  The device image that
 * holds the array may itself be loaded only then (lazy module loading), so
 * also make that first call before the host's memory pool reserves the
 * GPU's memory; if the image cannot be loaded the call returns ELMM_ERR_OOM
 * with a message naming the fixed array.  The set-up is tied to the CUDA
 * context: after the context is destroyed and created again (for example
 * by cudaDeviceReset) the next call repeats it.  Every call shares the
 * one array: calls whose work overlaps on the GPU (two streams, or two host
 * threads on one device) race and give wrong results, so order them on one
 * stream or with events.
 */
#define ELMM_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
int elmm_poisson_solve_noalloc(const int32_t n[3], const double L[3], const int32_t bcs[6],
                               int32_t device, double *Phi, const double *RHS, void *stream);

/*
 * Batched ensemble: n independent domains of uneven sizes stepped together.
 * Every kernel of a stage runs once for the whole batch over a device table of
 * domains; each RK3 step is one captured CUDA graph.
 */
typedef struct elmm_batch elmm_batch;
int elmm_batch_create(const elmm_config *cfgs, int32_t n, elmm_batch **out);
int elmm_batch_destroy(elmm_batch *b);
int elmm_batch_upload_state(elmm_batch *b, int32_t d, const double *U, const double *V,
                            const double *W, const double *Pr);
int elmm_batch_download_state(elmm_batch *b, int32_t d, double *U, double *V, double *W,
                              double *Pr);
int elmm_batch_upload_scalar(elmm_batch *b, int32_t d, int32_t sc, const double *S);
int elmm_batch_download_field(elmm_batch *b, int32_t d, int32_t field, double *host);
int elmm_batch_download_scalar_slices(elmm_batch *b, int32_t d, int32_t sc, double *xy, double *xz);
int elmm_batch_project(elmm_batch *b, double coef);
/* The tile shapes the autotuner chose at the first step (out[0]: rows of a
 * tile of the FP32 scalar stage, out[1]: spectral columns of a tile of the z
 * solve); the defaults before it. */
int elmm_batch_tuning(const elmm_batch *b, int32_t out[2]);
/* All the tile shapes (no counterpart in the reference, whose CPU loops take
 * their L1-sized tiles from src/tiling.f90): out[0] rows of a scalar-stage
 * tile (8, 4), out[1] spectral columns of a z-solve tile (16, 32), out[2]
 * and out[3] the z chunk of the momentum and of the SGS kernel (8, 16, 32
 * planes); the first n of ELMM_TUNE_KNOBS.  elmm_batch_set_tuning sets the
 * first n shapes instead of the autotuner (the others keep their values;
 * ELMM_ERR_INVALID_ARG for a value outside its set).  No shape changes a
 * result. */
#define ELMM_TUNE_KNOBS 4
int elmm_batch_get_tuning(const elmm_batch *b, int32_t *out, int32_t n);
int elmm_batch_set_tuning(elmm_batch *b, const int32_t *vals, int32_t n);
/* The same for a single-domain handle (tuned at its first step too). */
int elmm_get_tuning(const elmm_handle *h, int32_t *out, int32_t n);
int elmm_set_tuning(elmm_handle *h, const int32_t *vals, int32_t n);

/* elmm_set_solids and elmm_set_puffs for domain d of a batch: each domain
 * keeps its own bodies and puffs, and computes the same values as alone. */
int elmm_batch_set_solids(elmm_batch *b, int32_t d, const elmm_solids *s);
int elmm_batch_set_puffs(elmm_batch *b, int32_t d, const elmm_puff *puffs, int32_t npuffs,
                         const elmm_puff_volume *volumes, int32_t nvolumes);
/* elmm_profile_stage for a whole batch */
int elmm_batch_profile_stage(elmm_batch *b, int32_t stage, int32_t reps, double *ms);
int elmm_batch_step(elmm_batch *b, int32_t nsteps, elmm_stats *stats);
/* total interior cells of the batch (for cell-steps/s) */
int64_t elmm_batch_cells(const elmm_batch *b);

/*
 * Serving loop with continuous batching (dispersion runs of different grid
 * sizes).  A worker thread owns the device: every admitted request is a
 * domain whose state stays in HBM, and all admitted requests advance together
 * through one batched launch set per RK3 step (one CUDA graph, rebuilt when
 * the set changes).  Between chunks of at most chunk_steps steps, and while a
 * chunk runs, queued requests are admitted in arrival order as long as their
 * memory fits the server's HBM budget (one device allocation made at
 * creation; a request's fields are carved from it) and fewer than max_active
 * requests are on the device.  A request that has run its steps leaves the
 * set; the time-averaged slices of its scalar 1 are copied to the host and
 * its memory returns to the budget.  Each request computes exactly what it
 * computes alone (every kernel choice is made per domain).
 */
typedef struct elmm_server elmm_server;

#define ELMM_SERVER_MAX_ACTIVE 256

typedef struct elmm_server_config {
  int32_t device;
  int32_t precision;            /* ELMM_PREC_*, shared by every request */
  int64_t hbm_budget_bytes;     /* device memory the server holds for requests */
  int32_t max_active;           /* requests on the device at once, 1..ELMM_SERVER_MAX_ACTIVE */
  int32_t chunk_steps;          /* steps between admission points, >= 1 */
  int32_t policy;               /* ELMM_SERVE_FIFO or ELMM_SERVE_SHORTEST_FIRST */
  int32_t reserved;             /* 0 */
} elmm_server_config;

/* Admission order of queued requests: arrival order, or the least work
 * (cells x steps) first, which lowers the median latency under load. */
enum { ELMM_SERVE_FIFO = 0, ELMM_SERVE_SHORTEST_FIRST = 1 };

typedef struct elmm_request_info {
  int64_t id;
  int32_t status;               /* ELMM_OK, or the ELMM_ERR_* that ended the request */
  int32_t steps;                /* steps run */
  double t_submit, t_admit, t_done; /* seconds on the server clock (elmm_server_now) */
  int64_t bytes;                /* device memory the request held */
  double max_div;               /* max |div u| after its last step */
  int64_t cells;                /* Prnx * Prny * Prnz */
} elmm_request_info;

typedef struct elmm_server_stats {
  int64_t submitted, admitted, finished, failed;
  int64_t cell_steps;           /* interior cells x steps of all finished chunks */
  int64_t chunks, graph_builds;
  int32_t active, queued, peak_active;
  int32_t reserved;
  int64_t bytes_in_use, bytes_peak, budget_bytes;
  double busy_s;                /* device time of the chunks (CUDA events) */
} elmm_server_stats;

int elmm_server_create(const elmm_server_config *cfg, elmm_server **out);
/* Stops the worker after its current chunk; unfinished requests are dropped. */
int elmm_server_destroy(elmm_server *s);
/* Queues a request of nsteps steps.  cfg->precision and cfg->device must be
 * the server's.  U, V, W, Pr (may be NULL) and S0 (scalar 1, may be NULL for
 * zero) are host arrays in the layouts of elmm_upload_state and
 * elmm_upload_scalar; they must stay valid until the request is reported by
 * elmm_server_wait_any.  A request that does not fit the whole budget, even
 * with no other request on the device, ends with status ELMM_ERR_ADMISSION. */
int elmm_server_submit(elmm_server *s, const elmm_config *cfg, const double *U, const double *V,
                       const double *W, const double *Pr, const double *S0, int32_t nsteps,
                       int64_t *id);
/* Waits up to timeout_ms for a finished request that has not been reported
 * yet and fills *info; ELMM_ERR_TIMEOUT when none finished in time. */
int elmm_server_wait_any(elmm_server *s, int32_t timeout_ms, elmm_request_info *info);
/* Copies the time-averaged slices of scalar 1 of a reported request (layouts
 * of elmm_download_scalar_slices; NULL skips one) and forgets the request. */
int elmm_server_collect(elmm_server *s, int64_t id, double *xy, double *xz);
int elmm_server_stats_get(elmm_server *s, elmm_server_stats *st);
/* Seconds since the server was created, on the clock of elmm_request_info. */
double elmm_server_now(const elmm_server *s);

/* ------------------------------------------------------------------------
 * One domain split into z-slabs over several GPUs (the reference's domain
 * decomposition over MPI ranks, src/custom_mpi.f90:331-344, with its ghost
 * exchanges, src/exchange_mpi.f90:84-503, and the PFFT solve,
 * src/poisson.f90:107-114).  One process drives every slab: slab s holds
 * levels k0+1 .. k0+nz_slab[s] on devices[s] (several slabs may share a
 * device).  The slabs exchange one ghost plane per field with their
 * neighbours (peer copies over NVLink between GPUs) and solve the z
 * tridiagonal systems by exchanging three numbers per column and slab, so
 * the spectral buffer never crosses between GPUs.  The result equals the
 * single-domain handle's to rounding.
 *
 * Built for the flow, the temperature and passive scalars (point and puff
 * sources, time-averaged slices): walls in z (no periodic z), constant dt,
 * no solid bodies or defect-correction sweeps (ELMM_ERR_INVALID_CONFIG
 * otherwise).  The slabs also exchange the
 * scalars' two planes beyond each shared face (KappaScalar's stencil) and
 * the diffusivity's ghost plane.  nz_slab may be NULL for an even
 * split; every slab needs at least 4 levels, and the levels must add up to
 * Prnz.  devices may be NULL for cfg->device.
 *
 * Host arrays are the whole domain's, in the layouts of elmm_upload_state;
 * the download writes every element the single-domain download writes. */
#define ELMM_MAX_SLABS 16
typedef struct elmm_slabs elmm_slabs;
int elmm_slabs_create(const elmm_config *cfg, int32_t nslabs, const int32_t *devices, const int32_t *nz_slab,
                      elmm_slabs **out);
int elmm_slabs_destroy(elmm_slabs *h);
int elmm_slabs_upload_state(elmm_slabs *h, const double *U, const double *V, const double *W, const double *Pr);
int elmm_slabs_download_state(elmm_slabs *h, double *U, double *V, double *W, double *Pr);
/* The temperature and passive scalar sc (1..num_scalars) from the whole
 * domain's arrays in the layout of elmm_upload_temperature, after the
 * state and before elmm_slabs_project; elmm_slabs_download_field reads
 * ELMM_FIELD_TEMPERATURE or ELMM_FIELD_SCALAR + sc - 1 back. */
int elmm_slabs_upload_temperature(elmm_slabs *h, const double *T);
int elmm_slabs_upload_scalar(elmm_slabs *h, int32_t sc, const double *S);
int elmm_slabs_download_field(elmm_slabs *h, int32_t field, double *host);
/* Puff sources (as elmm_set_puffs; the volumes' cells are the whole
 * domain's) and the time-averaged slices of scalar sc (as
 * elmm_download_scalar_slices: the xz slice assembled from every slab). */
int elmm_slabs_set_puffs(elmm_slabs *h, const elmm_puff *puffs, int32_t npuffs, const elmm_puff_volume *volumes,
                         int32_t nvolumes);
int elmm_slabs_download_scalar_slices(elmm_slabs *h, int32_t sc, double *xy, double *xz);
/* PressureCorrection on the uploaded state, as elmm_project. */
int elmm_slabs_project(elmm_slabs *h, double coef, elmm_stats *stats);
/* nsteps RK3 steps, as elmm_step: with every slab on one device each step
 * is one CUDA graph over the slabs' streams (captured at the first call);
 * slabs on several devices launch eagerly.  stats->elapsed_ms is the device
 * time from the first slab's start to the last slab's end. */
int elmm_slabs_step(elmm_slabs *h, int32_t nsteps, elmm_stats *stats);
/* TMarchRK3 on the host arrays, as elmm_march_host: upload, nsteps steps,
 * download into the same arrays. */
int elmm_slabs_march_host(elmm_slabs *h, double *U, double *V, double *W, double *Pr, int32_t nsteps,
                          elmm_stats *stats);
/* The real32 host arrays of a prec=sp host (as elmm_upload_state_float):
 * widened to double on the device after the copy, narrowed before it. */
int elmm_slabs_upload_state_float(elmm_slabs *h, const float *U, const float *V, const float *W, const float *Pr);
int elmm_slabs_download_state_float(elmm_slabs *h, float *U, float *V, float *W, float *Pr);
int elmm_slabs_march_host_float(elmm_slabs *h, float *U, float *V, float *W, float *Pr, int32_t nsteps,
                                elmm_stats *stats);

/* Last error message of this thread (static storage). */
const char *elmm_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* ELMM_GPU_H */
