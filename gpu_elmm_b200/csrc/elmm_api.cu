// elmm_api.cu -- host side of libelmm_gpu.so: the C-ABI of include/elmm_gpu.h.
//
// A single-domain handle is a batch of one; every stage kernel runs once per
// batch over the domain table (see elmm_kernels.cuh).  One RK3 step of a
// batch is captured once into a CUDA graph and replayed.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <array>
#include <functional>
#include <limits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <initializer_list>
#include <mutex>
#include <string>
#include <deque>
#include <vector>
#include <type_traits>

#include "../../include/elmm_gpu.h"
#include "elmm_kernels2.cuh"
#include "elmm_poisson_reg.cuh"
#include "elmm_temperature.cuh"
#include "elmm_solids.cuh"
#include "elmm_slabs.cuh"
#include "elmm_arena.h"

using namespace elmm;

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;

static int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

#define CU(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) {                                                                  \
      return fail(e_ == cudaErrorMemoryAllocation ? ELMM_ERR_OOM : ELMM_ERR_CUDA,             \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                        \
    }                                                                                         \
  } while (0)

// RK3 coefficients, src/parameters.f90:317-320
static const double kAlpha[3] = {4.0 / 15.0, 1.0 / 15.0, 1.0 / 6.0};
static const double kBeta[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
static const double kRho[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};

static bool factorize(int n, FFTFactors &f) {
  f.n = n;
  f.nfac = 0;
  int r = n;
  for (int p : {4, 2, 3, 5}) {
    while (r % p == 0) {
      if (f.nfac >= kMaxFac) return false;
      f.fac[f.nfac++] = p;
      r /= p;
    }
  }
  return r == 1;
}

static int round_up(int a, int b) { return (a + b - 1) / b * b; }

// cuTensorMapEncodeTiled from the driver the runtime already loaded, so the
// library does not link against libcuda itself.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// A 3-D tile map over one box field: x the padded row (pitch elements), y
// the ny+2 rows, z the nz+2 planes.  Boxes are one plane deep; out-of-range
// elements read as zero.
template <typename T>
static int encode_box_map(CUtensorMap *m, T *base, long long pitch, int ny, int nz, unsigned bx, unsigned by) {
  auto enc = tensor_map_encoder();
  if (!enc) return fail(ELMM_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  cuuint64_t dims[3] = {(cuuint64_t)pitch, (cuuint64_t)(ny + 2), (cuuint64_t)(nz + 2)};
  cuuint64_t strides[2] = {(cuuint64_t)pitch * sizeof(T), (cuuint64_t)pitch * (ny + 2) * sizeof(T)};
  cuuint32_t box[3] = {bx, by, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)base,
                   dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(ELMM_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return ELMM_OK;
}

// ------------------------------------------------------- host grid tables
// The same formulas as src/initial.f90:4395-4480 (and the oracle).
struct HostGrid {
  int nx, ny, nz;
  std::vector<double> zW, zPr, dzPr, dzW;  // index k + 2, k in [-2, nz+3] (dzW to nz+2)
  std::vector<double> dxPr, dyPr;          // index i (1..n)
  bool uniform_xy;
  std::vector<double> width;               // index k (1..nz)
  double dzmin;
};

static void make_grid(const elmm_config &c, HostGrid &g) {
  int nx = c.Prnx, ny = c.Prny, nz = c.Prnz;
  g.nx = nx; g.ny = ny; g.nz = nz;
  std::vector<double> zW2(nz + 7);  // k in [-3, nz+3] -> k + 3
  auto Z = [&](int k) -> double & { return zW2[k + 3]; };
  if (c.zW) {
    for (int k = 0; k <= nz; k++) Z(k) = c.zW[k];
    if (c.Btype[ELMM_BO] == ELMM_BC_PERIODIC)
      for (int j = -1; j >= -3; j--) Z(j) = Z(0) - (Z(nz - 1) - Z(nz - 1 + j));
    else
      for (int j = -1; j >= -3; j--) Z(j) = Z(0) - (Z(-j) - Z(0));
    if (c.Btype[ELMM_TO] == ELMM_BC_PERIODIC)
      for (int j = nz + 1; j <= nz + 3; j++) Z(j) = Z(nz - 1) + (Z(j - nz + 1) - Z(0));
    else
      for (int j = nz + 1; j <= nz + 3; j++) Z(j) = Z(nz - 1) + (Z(nz - 1) - Z(nz - 1 - (j - nz + 1)));
  } else {
    for (int k = -3; k <= nz + 3; k++) Z(k) = k * c.dzmin + c.zmin;
  }
  g.zW.assign(nz + 6, 0.0); g.zPr.assign(nz + 6, 0.0); g.dzPr.assign(nz + 6, 0.0); g.dzW.assign(nz + 6, 0.0);
  for (int k = -2; k <= nz + 3; k++) {
    g.zW[k + 2] = Z(k);
    g.zPr[k + 2] = (Z(k - 1) + Z(k)) / 2.0;
    g.dzPr[k + 2] = Z(k) - Z(k - 1);
  }
  for (int k = -2; k <= nz + 2; k++) g.dzW[k + 2] = g.zPr[k + 1 + 2] - g.zPr[k + 2];
  g.dzmin = c.dzmin;
  if (c.zW) {
    double m = g.dzPr[0];
    for (int k = -2; k <= nz + 3; k++) m = std::min(m, g.dzPr[k + 2]);
    g.dzmin = m;
  }
  g.dxPr.assign(nx + 1, 0.0); g.dyPr.assign(ny + 1, 0.0);
  for (int i = 1; i <= nx; i++) g.dxPr[i] = (i * c.dxmin + c.xmin) - ((i - 1) * c.dxmin + c.xmin);
  for (int j = 1; j <= ny; j++) g.dyPr[j] = (j * c.dymin + c.ymin) - ((j - 1) * c.dymin + c.ymin);
  g.uniform_xy = true;
  for (int i = 2; i <= nx; i++) g.uniform_xy &= g.dxPr[i] == g.dxPr[1];
  for (int j = 2; j <= ny; j++) g.uniform_xy &= g.dyPr[j] == g.dyPr[1];
  g.width.assign(nz + 1, 0.0);
  for (int k = 1; k <= nz; k++)
    g.width[k] = c.filter_ratio * std::pow(g.dxPr[1] * g.dyPr[1] * g.dzPr[k + 2], 1.0 / 3.0);
}

// the BC kinds of CommonBase a non-periodic scalar side takes
// (src/scalarboundaries.f90:197-288)
static bool scalar_bc_kind(int k) {
  return k == ELMM_BC_CONSTFLUX || k == ELMM_BC_DIRICHLET || k == ELMM_BC_NEUMANN;
}

// the z sides of a scalar slot whose ghost plane k_scalar_zghost writes:
// the rules of CommonBase a fold of the interior does not give (a zero
// flux or gradient is the fold); a temperature flux or surface temperature
// at a wall with wall-model points (wm_points[side]) enters through the
// points instead
template <typename T>
static void set_zghosts(ScalSlot<T> &sl, const int32_t *bt, const double *side, const int *wm_points) {
  for (int h = 0; h < 2; h++) {
    const int s = h ? ELMM_TO : ELMM_BO;
    const bool points = wm_points && wm_points[s];
    sl.zg[h] = (bt[s] == ELMM_BC_DIRICHLET && !points) || (bt[s] == ELMM_BC_NEUMANN && side[s] != 0) ||
               (bt[s] == ELMM_BC_CONSTFLUX && side[s] != 0 && !points);
    sl.zside[h] = side[s];
  }
}

static int check_config(const elmm_config &c) {
  if (c.abi_version != ELMM_ABI_VERSION) return fail(ELMM_ERR_INVALID_CONFIG, "abi_version mismatch");
  if (c.Prnx < 4 || c.Prny < 4 || c.Prnz < 4) return fail(ELMM_ERR_INVALID_CONFIG, "grid must be at least 4 cells per axis");
  if ((long long)c.Prnx * c.Prny * c.Prnz > (1LL << 31)) return fail(ELMM_ERR_INVALID_CONFIG, "grid too large");
  for (int s = 0; s < 6; s++) {
    int b = c.Btype[s];
    if (b != ELMM_BC_NOSLIP && b != ELMM_BC_FREESLIP && b != ELMM_BC_PERIODIC && b != ELMM_BC_NEUMANN)
      return fail(ELMM_ERR_INVALID_CONFIG, "unsupported boundary condition code " + std::to_string(b));
  }
  for (int a = 0; a < 3; a++)
    if ((c.Btype[2 * a] == ELMM_BC_PERIODIC) != (c.Btype[2 * a + 1] == ELMM_BC_PERIODIC))
      return fail(ELMM_ERR_INVALID_CONFIG, "periodic boundary conditions must be set on both sides of an axis");
  if (c.Btype[ELMM_WE] != ELMM_BC_PERIODIC || c.Btype[ELMM_SO] != ELMM_BC_PERIODIC)
    return fail(ELMM_ERR_INVALID_CONFIG, "the FFT Poisson solver needs periodic x and y");
  if (c.zW && c.Btype[ELMM_BO] == ELMM_BC_PERIODIC)
    return fail(ELMM_ERR_INVALID_CONFIG, "periodic z needs a uniform z grid");
  FFTFactors f;
  if (!factorize(c.Prnx, f) || !factorize(c.Prny, f))
    return fail(ELMM_ERR_INVALID_CONFIG, "Prnx and Prny must factor into 2, 3 and 5");
  if (c.Prnx > 4096 || c.Prny > 4096 || c.Prnz > 2048) return fail(ELMM_ERR_INVALID_CONFIG, "axis too long");
  if (!(c.dxmin > 0 && c.dymin > 0 && c.dzmin > 0 && c.dt > 0))
    return fail(ELMM_ERR_INVALID_CONFIG, "spacings and dt must be positive");
  if (c.precision != ELMM_PREC_FP64 && c.precision != ELMM_PREC_MIXED)
    return fail(ELMM_ERR_INVALID_CONFIG, "unknown precision");
  if (c.variable_time_steps &&
      !(c.CFL > 0 && std::isfinite(c.CFL) && c.dt_max > 0 && std::isfinite(c.dt_max) && c.end_time >= 0))
    return fail(ELMM_ERR_INVALID_CONFIG, "variable time steps need CFL > 0, dt_max > 0 and end_time >= 0");
  if (c.max_refine_sweeps < 0 || c.max_refine_sweeps > 3) return fail(ELMM_ERR_INVALID_CONFIG, "max_refine_sweeps in 0..3");
  if (c.wallmodeltype > 0 && c.molecular_viscosity <= 0) {
    for (int s = 0; s < 6; s++)
      if (c.Btype[s] == ELMM_BC_NOSLIP && !(c.z0[s] > 0))
        return fail(ELMM_ERR_INVALID_CONFIG, "The wall model requires positive viscosity or roughness length.");
  }
  if (c.wallmodeltype > 0)
    for (int s = 0; s < 6; s++)
      if (c.Btype[s] == ELMM_BC_NOSLIP && !(c.z0[s] >= 0))
        return fail(ELMM_ERR_INVALID_CONFIG, "z0 must be zero (smooth wall) or positive (rough wall)");
  if (c.enable_buoyancy) {
    for (int s = 0; s < 6; s++) {
      const bool per = c.Btype[s] == ELMM_BC_PERIODIC;
      if (per && c.TempBtype[s] != ELMM_BC_PERIODIC)
        return fail(ELMM_ERR_INVALID_CONFIG, "the temperature must be periodic where the flow is");
      // a surface flux at a wall in z is carried by its wall-model points,
      // the other kinds and sides by the ghost rules of CommonBase
      if (!per && (!scalar_bc_kind(c.TempBtype[s]) || !std::isfinite(c.sideTemp[s])))
        return fail(ELMM_ERR_INVALID_CONFIG,
                    "temperature sides: ELMM_BC_CONSTFLUX, ELMM_BC_DIRICHLET or ELMM_BC_NEUMANN with a finite sideTemp");
    }
    if (c.zW) return fail(ELMM_ERR_INVALID_CONFIG, "the temperature field needs a uniform z grid");
    if (c.Btype[ELMM_BO] == ELMM_BC_PERIODIC)
      return fail(ELMM_ERR_INVALID_CONFIG, "the temperature field needs walls at the bottom and top");
    if (!(c.temperature_ref > 0) || !(c.molecular_diffusivity >= 0))
      return fail(ELMM_ERR_INVALID_CONFIG, "temperature_ref must be positive and molecular_diffusivity non-negative");
  }
  if (c.num_scalars < 0 || c.num_scalars > ELMM_MAX_SCALARS)
    return fail(ELMM_ERR_INVALID_CONFIG, "num_scalars in 0.." + std::to_string(ELMM_MAX_SCALARS));
  if (c.num_scalars > 0) {
    for (int s = 0; s < 6; s++) {
      const bool per = c.Btype[s] == ELMM_BC_PERIODIC;
      if (per && c.ScalBtype[s] != ELMM_BC_PERIODIC)
        return fail(ELMM_ERR_INVALID_CONFIG, "the scalars must be periodic where the flow is");
      if (!per && (!scalar_bc_kind(c.ScalBtype[s]) || !std::isfinite(c.sideScal[s])))
        return fail(ELMM_ERR_INVALID_CONFIG,
                    "scalar sides: ELMM_BC_CONSTFLUX, ELMM_BC_DIRICHLET or ELMM_BC_NEUMANN with a finite sideScal");
    }
    if (c.zW) return fail(ELMM_ERR_INVALID_CONFIG, "the scalar fields need a uniform z grid");
    if (!(c.molecular_diffusivity >= 0)) return fail(ELMM_ERR_INVALID_CONFIG, "molecular_diffusivity must be non-negative");
  }
  if (c.num_point_sources < 0 || c.num_point_sources > ELMM_MAX_POINT_SOURCES)
    return fail(ELMM_ERR_INVALID_CONFIG, "num_point_sources in 0.." + std::to_string(ELMM_MAX_POINT_SOURCES));
  for (int q = 0; q < c.num_point_sources; q++) {
    const elmm_point_source &p = c.point_sources[q];
    if (p.scalar_number < 1 || p.scalar_number > c.num_scalars)
      return fail(ELMM_ERR_INVALID_CONFIG, "point source " + std::to_string(q) + ": scalar_number outside 1..num_scalars");
    if (!std::isfinite(p.flux) || !std::isfinite(p.position[0]) || !std::isfinite(p.position[1]) ||
        !std::isfinite(p.position[2]))
      return fail(ELMM_ERR_INVALID_CONFIG, "point source " + std::to_string(q) + ": non-finite position or flux");
  }
  if (c.avg_slice_k < 0 || c.avg_slice_k > c.Prnz || c.avg_slice_j < 0 || c.avg_slice_j > c.Prny)
    return fail(ELMM_ERR_INVALID_CONFIG, "avg_slice_k in 0..Prnz and avg_slice_j in 0..Prny");
  if (!std::isfinite(c.avg_weight)) return fail(ELMM_ERR_INVALID_CONFIG, "avg_weight must be finite");
  return ELMM_OK;
}

// InDomain (src/boundaries.f90:163-168) and GridCoords_scalar
// (src/boundaries.f90:54-97) on a uniform grid: the cell that holds a point
// source, or false when the point lies outside the domain.  nint rounds half
// away from zero.
static bool point_cell(const elmm_config &c, const double *r, int *ip) {
  const double lo[3] = {c.xmin, c.ymin, c.zmin}, h[3] = {c.dxmin, c.dymin, c.dzmin};
  const int n[3] = {c.Prnx, c.Prny, c.Prnz};
  for (int a = 0; a < 3; a++)
    if (!(r[a] >= lo[a] && r[a] <= n[a] * h[a] + lo[a])) return false;
  for (int a = 0; a < 3; a++) ip[a] = std::min(std::max((int)std::lround((r[a] - lo[a]) / h[a] + 0.5), 1), n[a]);
  return true;
}

// ---------------------------------------------------------------- launches
struct LaunchSet {
  int *starts = nullptr;  // device
  int total = 0;
  int nd = 0;
  Launch l() const { return Launch{starts, nd, total}; }
};

enum { LK_CELLS = 0, LK_BOX, LK_ROWS, LK_YCOLS, LK_TRI, LK_MOM, LK_SHELL, LK_XREG, LK_YREG, LK_TRIT, LK_TCOL, LK_DCOL,
       LK_AVG, LK_COMMIT, LK_TPAIR, LK_PROJ, LK_PROJ2, LK_DCOL2, LK_MOMT, LK_SGST, LK_WM, LK_N };

// the z-chunk lengths (planes of a tile's column) the autotuner tries for
// the momentum and SGS kernels
constexpr int kChunks[3] = {8, 16, 32};

// blocks of the host-layout pack / unpack kernels (8 per SM)
constexpr int kPackBlocks = 148 * 8;

// -------------------------------------------------------------------- batch
template <typename T>
struct BatchT {
  typedef typename Vec2<T>::type T2;
  int nd = 0;
  int device = 0;
  cudaStream_t stream = nullptr, side = nullptr;
  std::vector<elmm_config> cfg;
  std::vector<HostGrid> grid;
  std::vector<Dom<T>> hdom;     // host copies of the descriptors
  std::vector<PoisPlan> hplan;
  Dom<T> *ddom = nullptr;       // device descriptors
  PoisPlan *dplan = nullptr;
  std::vector<void *> allocs;
  LaunchSet ls[LK_N];
  size_t smem_x = 0, smem_y = 0, smem_tri = 0;
  // register FFTs / tiled z solve when every domain of the batch allows them
  bool reg_x = false, reg_y = false, tri_tile = false;
  size_t smem_xr = 0, smem_yr = 0, smem_trit = 0, smem_trit32 = 0;
  struct RegSet {
    const FFTRegKernels<T> *k = nullptr;
    LaunchSet ls;
    size_t smem = 0;
    int cap_fwd = 1, cap_inv = 1;
  };
  std::vector<RegSet> xreg, yreg;
  size_t smem_mom = (size_t)MomShape<T>::slots * SlotLayout<T, 5, MomShape<T>::nnf>::BYTES;
  size_t smem_sgs = (size_t)kRingSlots * SlotLayout<T, 3, 0>::BYTES;
  int grid_cap[16] = {};
  // host-layout staging (double), max over domains of the largest host array
  double *dstage = nullptr;
  size_t stage_elems = 0;
  // a second staging buffer (single-domain handles, allocated at the first
  // state transfer): the host copy of one field overlaps the pack or unpack
  // of the next on the side stream
  double *dstage2 = nullptr;
  cudaEvent_t ev_stage[2][2] = {};  // [buffer][0: filled on its producer, 1: drained by its consumer]
  cudaEvent_t ev_pr = nullptr;      // the host copy of Pr into its image has landed
  std::vector<double *> pr_image;  // per domain: last host Pr image (device)
  int *dbad = nullptr;
  // single-precision host arrays (the *_float entry points): hostf is set for
  // the duration of such a call; fstage holds the floats on the device
  int hostf = 0;
  float *fstage = nullptr;
  // the float side of the pipelined host transfers (upload_all /
  // download_all with hostf): one buffer per double staging buffer
  float *fpipe[2] = {nullptr, nullptr};
  cudaGraphExec_t step_exec = nullptr;
  bool step_has_cfl = false;
  double time = 0;
  // frames
  double *frame_host = nullptr;    // pinned
  double *frame_dev = nullptr;
  size_t frame_elems = 0;
  cudaEvent_t ev_ready = nullptr, ev_packed = nullptr, ev_done = nullptr;
  bool frame_pending = false;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  long long cells = 0;
  int step_kernels = 0;  // kernel launches of one captured step
  int nlaunch = 0;       // running count while enqueuing
  // device memory from a serving loop's budget instead of cudaMalloc
  Arena *arena = nullptr;
  size_t arena_bytes = 0;
  // a view steps domains whose fields other batches own, on a borrowed stream
  bool is_view = false;
  // shell cells per thread of the ghost passes: 4 for several domains, 1 for one
  int shell_per = 1;
  // one z-slab of a split domain (SlabsT): its configuration carries
  // BC_HALO on the shared faces (checked as the whole domain's beforehand),
  // and its z grid is the whole domain's from level zk0 on
  bool slab_mode = false;
  const HostGrid *zparent = nullptr;
  int zk0 = 0;
  // tile shapes chosen by the autotuner at the first step: rows of a tile of
  // the FP32 scalar stage, spectral columns of a tile of the z solve
  int tune_rows = 8, tune_cols = 16;
  int tune_mom_kc = MKC, tune_sgs_kc = MKC;  // z chunks of k_momentum and k_sgs
  int cap_mom[3] = {1, 1, 1}, cap_sgs[3] = {1, 1, 1};  // resident-block grids per chunk choice
  bool tuned = false;
  // parallel branches for the independent per-length launches of one
  // transform phase (a batch with several x or y lengths); joined back into
  // the stream before the next phase, captured as graph branches
  static constexpr int kBranches = 4;
  cudaStream_t branch[kBranches] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[kBranches] = {};
  float tune_ms[10] = {};  // rows 8, rows 4, cols 16, cols 32, momentum chunks 8/16/32, SGS chunks 8/16/32
  // immersed solid bodies per domain (elmm_set_solids): the gathers of the
  // velocity IB points followed by the nullified points, the gathers of the
  // ScalFl viscosity, the solid-face wall-model points and their u* state
  struct SolidSet {
    IBGather *vel = nullptr, *visc = nullptr;
    int nvel = 0, nib = 0, nvisc = 0;
    long long *null = nullptr;  // box indices of the nullified points of U, then V, then W
    NullCounts nnull{{0, 0, 0}};
    WMSolid *wm = nullptr;
    double *wm_ustar = nullptr;
    int nwm = 0;
    unsigned char *bskip[3] = {nullptr, nullptr, nullptr};
    unsigned char *pmask = nullptr;  // the scalars' cell mask (Dom::pmask)
    // the temperature's fill of the solid cells (k_theta_fill)
    FillCell *fill = nullptr;
    int nfill = 0;
    // the heated Pr wall-model points at solid faces (k_heat_add)
    HeatPoint *heat = nullptr;
    int nheat = 0;
    bool on = false, primed = false;
  };
  std::vector<SolidSet> sol;
  bool any_solids() const {
    for (auto &x : sol) if (x.on) return true;
    return false;
  }
  bool solids_on(int d) const { return d < (int)sol.size() && sol[d].on; }
  // Mixed path: the per-level offsets of velocity component c (0: U, 1: V)
  // of domain d from the host-layout array staged in stg (zero for a domain
  // with solid bodies), on the stream; returns the offsets for k_unpack, or
  // null for the FP64 path and for W.
  const float *stage_offsets(int d, int c, const double *stg, const HostBox &hb) {
    const Dom<T> &h = hdom[d];
    if (sizeof(T) != 4 || c > 1 || !h.voff) return nullptr;
    float *off = h.voff + c * (h.nz + 2);
    if (solids_on(d)) cudaMemsetAsync(off, 0, sizeof(float) * (h.nz + 2), stream);
    else k_level_offsets<T><<<h.nz + 2, 256, 0, stream>>>(ddom + d, stg, hb, c, h.voff);
    return off;
  }
  // One host-layout array of n elements into the double staging buffer stg
  // on stream st: a double host array is copied as it is, a float one (hostf)
  // through fstage and widened.
  int h2d(double *stg, const void *host, size_t n, cudaStream_t st) {
    if (!hostf) {
      CU(cudaMemcpyAsync(stg, host, n * sizeof(double), cudaMemcpyHostToDevice, st));
      return ELMM_OK;
    }
    int r = ensure_fstage();
    if (r) return r;
    CU(cudaMemcpyAsync(fstage, host, n * sizeof(float), cudaMemcpyHostToDevice, st));
    k_widen<<<kPackBlocks, 256, 0, st>>>(stg, fstage, (long long)n);
    return ELMM_OK;
  }
  // the staged double array back to a host array of the call's type
  int d2h(void *host, const double *stg, size_t n, cudaStream_t st) {
    if (!hostf) {
      CU(cudaMemcpyAsync(host, stg, n * sizeof(double), cudaMemcpyDeviceToHost, st));
      return ELMM_OK;
    }
    int r = ensure_fstage();
    if (r) return r;
    k_narrow<<<kPackBlocks, 256, 0, st>>>(fstage, stg, (long long)n);
    CU(cudaMemcpyAsync(host, fstage, n * sizeof(float), cudaMemcpyDeviceToHost, st));
    return ELMM_OK;
  }
  int ensure_fstage() {
    if (fstage) return ELMM_OK;
    size_t n = stage_elems;
    for (int d = 0; d < nd; d++) {  // the Pr image and the Poisson arrays fit the velocity boxes' staging
      const size_t pe = (size_t)(hdom[d].nx + 4) * (hdom[d].ny + 4) * (hdom[d].nz + 4);
      n = std::max(n, pe);
    }
    return dalloc((void **)&fstage, n * sizeof(float));
  }
  int ensure_fpipe() {
    for (auto &f : fpipe)
      if (!f) {
        int r = dalloc((void **)&f, stage_elems * sizeof(float));
        if (r) return r;
      }
    return ELMM_OK;
  }
  // Pipelined host copy of n elements of a host array of the call's type
  // into staging buffer b (on the side stream), then made double in dstage
  // / dstage2 on the stream: returns the double buffer
  int h2d_pipe(int b, const void *host, size_t n, double **out) {
    double *stg = b ? dstage2 : dstage;
    CU(cudaStreamWaitEvent(side, ev_stage[b][1], 0));
    if (!hostf) {
      CU(cudaMemcpyAsync(stg, host, n * sizeof(double), cudaMemcpyHostToDevice, side));
      CU(cudaEventRecord(ev_stage[b][0], side));
      CU(cudaStreamWaitEvent(stream, ev_stage[b][0], 0));
    } else {
      CU(cudaMemcpyAsync(fpipe[b], host, n * sizeof(float), cudaMemcpyHostToDevice, side));
      CU(cudaEventRecord(ev_stage[b][0], side));
      CU(cudaStreamWaitEvent(stream, ev_stage[b][0], 0));
      k_widen<<<kPackBlocks, 256, 0, stream>>>(stg, fpipe[b], (long long)n);
    }
    *out = stg;
    return ELMM_OK;
  }
  // the packed double buffer b to a host array of the call's type, the host
  // copy on the side stream
  int d2h_pipe(int b, void *host, size_t n) {
    const double *stg = b ? dstage2 : dstage;
    if (hostf) k_narrow<<<kPackBlocks, 256, 0, stream>>>(fpipe[b], stg, (long long)n);
    CU(cudaEventRecord(ev_stage[b][0], stream));
    CU(cudaStreamWaitEvent(side, ev_stage[b][0], 0));
    if (hostf) CU(cudaMemcpyAsync(host, fpipe[b], n * sizeof(float), cudaMemcpyDeviceToHost, side));
    else CU(cudaMemcpyAsync(host, stg, n * sizeof(double), cudaMemcpyDeviceToHost, side));
    CU(cudaEventRecord(ev_stage[b][1], side));
    return ELMM_OK;
  }
  // the offsets the pack of velocity component comp of domain d adds back, or null
  const float *pack_offsets(int d, int comp) const {
    const Dom<T> &h = hdom[d];
    return (sizeof(T) == 4 && comp < 2 && h.voff) ? h.voff + comp * (h.nz + 2) : nullptr;
  }

  ~BatchT() { release(); }

  void release() {
    if (step_exec) cudaGraphExecDestroy(step_exec);
    step_exec = nullptr;
    for (void *p : allocs) {
      if (arena) arena->release(p);
      else cudaFree(p);
    }
    allocs.clear();
    arena_bytes = 0;
    if (frame_host) cudaFreeHost(frame_host);
    frame_host = nullptr;
    for (cudaEvent_t *e : {&ev_ready, &ev_packed, &ev_done, &t0, &t1})
      if (*e) { cudaEventDestroy(*e); *e = nullptr; }
    if (!is_view) {
      if (stream) cudaStreamDestroy(stream);
      if (side) cudaStreamDestroy(side);
    }
    stream = side = nullptr;
    for (int b = 0; b < kBranches; b++) {
      if (branch[b]) cudaStreamDestroy(branch[b]);
      if (ev_join[b]) cudaEventDestroy(ev_join[b]);
      branch[b] = nullptr;
      ev_join[b] = nullptr;
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    ev_fork = nullptr;
    for (auto &pair : ev_stage)
      for (auto &e : pair)
        if (e) { cudaEventDestroy(e); e = nullptr; }
    if (ev_pr) cudaEventDestroy(ev_pr);
    ev_pr = nullptr;
  }
  // the second staging buffer and its events, or false (views, serving
  // requests and batches keep one buffer and copy field by field)
  int stage_state = 0;  // 0 untried, 1 two buffers, -1 one buffer
  bool two_stages() {
    if (is_view || arena || nd != 1 || !dstage) return false;
    if (stage_state == 0) {
      stage_state = -1;
      if (dalloc((void **)&dstage2, stage_elems * sizeof(double))) { dstage2 = nullptr; return false; }
      for (auto &pair : ev_stage)
        for (auto &e : pair)
          if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return false;
      if (cudaEventCreateWithFlags(&ev_pr, cudaEventDisableTiming) != cudaSuccess) return false;
      for (int b = 0; b < 2; b++) {  // both buffers start free
        if (cudaEventRecord(ev_stage[b][1], stream) != cudaSuccess) return false;
        if (cudaEventRecord(ev_stage[b][0], side) != cudaSuccess) return false;
      }
      stage_state = 1;
    }
    return stage_state == 1;
  }

  int dalloc(void **p, size_t bytes) {
    bytes = std::max<size_t>(bytes, 256);
    if (arena) {
      *p = arena->alloc(bytes);
      if (!*p) return fail(ELMM_ERR_ADMISSION, "the serving loop's HBM budget has no room for the request now");
      arena_bytes += Arena::round(bytes);
    } else {
      cudaError_t e = cudaMalloc(p, bytes);
      if (e != cudaSuccess) return fail(e == cudaErrorMemoryAllocation ? ELMM_ERR_OOM : ELMM_ERR_CUDA,
                                        std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    allocs.push_back(*p);
    return cudaMemset(*p, 0, bytes) == cudaSuccess ? ELMM_OK : fail(ELMM_ERR_CUDA, "cudaMemset");
  }
  // returns one allocation early (the host-layout staging of a serving
  // request after its upload)
  void dfree(void *p) {
    auto it = std::find(allocs.begin(), allocs.end(), p);
    if (it == allocs.end()) return;
    allocs.erase(it);
    if (arena) {
      const size_t before = arena->in_use();
      arena->release(p);
      arena_bytes -= before - arena->in_use();
    } else {
      cudaFree(p);
    }
  }

  template <typename X>
  int upload_table(const X **dst, const std::vector<X> &v) {
    void *p;
    int r = dalloc(&p, v.size() * sizeof(X));
    if (r) return r;
    CU(cudaMemcpy(p, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice));
    *dst = (const X *)p;
    return ELMM_OK;
  }

  int init(const elmm_config *cfgs, int n) {
    nd = n;
    device = cfgs[0].device;
    for (int d = 0; d < n; d++) {
      int r = slab_mode ? ELMM_OK : check_config(cfgs[d]);
      if (r) return r;
      if (cfgs[d].device != device) return fail(ELMM_ERR_INVALID_CONFIG, "all domains of a batch share one device");
      if (cfgs[d].precision != cfgs[0].precision) return fail(ELMM_ERR_INVALID_CONFIG, "all domains of a batch share one precision");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device) return fail(ELMM_ERR_CUDA, "no CUDA device");
    CU(cudaSetDevice(device));
    CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    CU(cudaEventCreateWithFlags(&ev_ready, cudaEventDisableTiming));
    CU(cudaEventCreateWithFlags(&ev_packed, cudaEventDisableTiming));
    CU(cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming));
    CU(cudaEventCreate(&t0));
    CU(cudaEventCreate(&t1));
    cfg.assign(cfgs, cfgs + n);
    grid.resize(n);
    hdom.resize(n);
    hplan.resize(n);
    pr_image.assign(n, nullptr);
    for (int d = 0; d < n; d++) {
      int r = init_domain(d);
      if (r) return r;
    }
    return init_tables();
  }

  // A batch over domains that other single-domain batches own (the active
  // requests of a serving loop), launched on `on_stream`; its own memory is
  // only the tables, from the same budget.
  int init_view(const std::vector<BatchT<T> *> &members, cudaStream_t on_stream, Arena *budget) {
    is_view = true;
    arena = budget;
    nd = (int)members.size();
    device = members[0]->device;
    stream = on_stream;
    CU(cudaEventCreate(&t0));
    CU(cudaEventCreate(&t1));
    for (BatchT<T> *m : members) {
      cfg.push_back(m->cfg[0]);
      grid.push_back(m->grid[0]);
      hdom.push_back(m->hdom[0]);
      hplan.push_back(m->hplan[0]);
      pr_image.push_back(nullptr);
    }
    return init_tables();
  }

  // device tables of the domains, launch maps and kernel attributes
  int init_tables() {
    const int n = nd;
    shell_per = n > 1 ? 4 : 1;
    CU(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    for (int b = 1; b < kBranches; b++) {
      CU(cudaStreamCreateWithFlags(&branch[b], cudaStreamNonBlocking));
      CU(cudaEventCreateWithFlags(&ev_join[b], cudaEventDisableTiming));
    }
    void *p;
    int r = dalloc(&p, sizeof(Dom<T>) * n);
    if (r) return r;
    ddom = (Dom<T> *)p;
    CU(cudaMemcpy(ddom, hdom.data(), sizeof(Dom<T>) * n, cudaMemcpyHostToDevice));
    r = dalloc(&p, sizeof(PoisPlan) * n);
    if (r) return r;
    dplan = (PoisPlan *)p;
    CU(cudaMemcpy(dplan, hplan.data(), sizeof(PoisPlan) * n, cudaMemcpyHostToDevice));
    r = dalloc((void **)&dbad, sizeof(int));
    if (r) return r;
    // launch maps
    for (int k = 0; k < LK_N; k++) {
      std::vector<int> st(n + 1, 0);
      for (int d = 0; d < n; d++) st[d + 1] = st[d] + tiles(k, hdom[d]);
      ls[k].nd = n;
      ls[k].total = st[n];
      r = dalloc((void **)&ls[k].starts, sizeof(int) * (n + 1));
      if (r) return r;
      CU(cudaMemcpy(ls[k].starts, st.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    }
    int maxnx = 0, maxny = 0, maxnz = 0, anyzper = 0;
    for (auto &h : hdom) { maxnx = std::max(maxnx, h.nx); maxny = std::max(maxny, h.ny); maxnz = std::max(maxnz, h.nz); anyzper |= h.zper; }
    smem_x = sizeof(T2) * 2 * (kRowsX / 2) * maxnx;
    smem_y = sizeof(T2) * 2 * TyOf<T>::v * maxny;
    smem_tri = sizeof(double) * kTriThreads * maxnz * (anyzper ? 2 : 1);
    // the opt-in maximum, so that handles of different sizes never lower the
    // limit under each other's launches
    int optin = 0;
    CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    if (smem_x > (size_t)optin || smem_y > (size_t)optin || smem_tri > (size_t)optin)
      return fail(ELMM_ERR_INVALID_CONFIG, "grid too large for the shared-memory transforms");
    CU(cudaFuncSetAttribute(k_fftx_fwd<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    CU(cudaFuncSetAttribute(k_fftx_inv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    CU(cudaFuncSetAttribute(k_ffty<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    CU(cudaFuncSetAttribute(k_tri<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    CU(cudaFuncSetAttribute(k_momentum<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 1024));
    CU(cudaFuncSetAttribute(k_momentum<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 1024));
    CU(cudaFuncSetAttribute(k_momentum<T, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 1024));
    CU(cudaFuncSetAttribute(k_sgs<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 1024));
    CU(cudaFuncSetAttribute(k_sgs<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 1024));
    CU(cudaFuncSetAttribute(k_sgs<T, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 1024));
    for (auto &h : hdom) {
      reg_x |= fft_reg_supported(h.nx);
      reg_y |= fft_reg_supported(h.ny);
      tri_tile |= tri_tiled(h);
      if (fft_reg_supported(h.nx))
        smem_xr = std::max(smem_xr, sizeof(T2) * fft_reg_batch(h.nx) * fft_reg_seq(h.nx));
      if (fft_reg_supported(h.ny))
        smem_yr = std::max(smem_yr, sizeof(T2) * fft_reg_batch(h.ny) * fft_reg_seq(h.ny));
      if (tri_tiled(h)) {
        smem_trit = std::max(smem_trit, tri_tile_smem<T, 16>(h.nz));
        smem_trit32 = std::max(smem_trit32, tri_tile_smem<T, 32>(h.nz));
      }
    }
    if (smem_xr > (size_t)optin || smem_yr > (size_t)optin || smem_trit32 > (size_t)optin)
      return fail(ELMM_ERR_INVALID_CONFIG, "shared memory of the register transforms exceeds the device limit");
    CU(cudaFuncSetAttribute(k_tri_tile<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    CU(cudaFuncSetAttribute(k_tri_tile<T, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    int nsm = 0;
    CU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    auto cap = [&](const void *f, int threads, size_t sm) {
      int b = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, threads, sm) != cudaSuccess || b < 1) b = 1;
      return b * nsm;
    };
    grid_cap[0] = cap((const void *)k_sgs<T>, SgsShape<T>::threads, smem_sgs);
    grid_cap[1] = cap((const void *)k_momentum<T>, MomShape<T>::threads, smem_mom);
    {
      const void *fm[3] = {(const void *)k_momentum<T, 8>, (const void *)k_momentum<T, 16>,
                           (const void *)k_momentum<T, 32>};
      const void *fs[3] = {(const void *)k_sgs<T, 8>, (const void *)k_sgs<T, 16>, (const void *)k_sgs<T, 32>};
      for (int q = 0; q < 3; q++) {
        cap_mom[q] = cap(fm[q], MomShape<T>::threads, smem_mom);
        cap_sgs[q] = cap(fs[q], SgsShape<T>::threads, smem_sgs);
      }
    }
    grid_cap[2] = cap((const void *)k_fftx_fwd<T>, kFFTThreads, smem_x);
    grid_cap[3] = cap((const void *)k_ffty<T>, kFFTThreads, smem_y);
    grid_cap[4] = cap((const void *)k_tri<T>, kTriThreads, smem_tri);
    grid_cap[5] = cap((const void *)k_fftx_inv<T>, kFFTThreads, smem_x);
    grid_cap[6] = cap((const void *)k_project<T>, MX * MY, 0);
    grid_cap[10] = std::is_same<T, float>::value ? cap((const void *)k_project_pair, MX * MY / 2, 0) : 1;
    grid_cap[7] = cap((const void *)k_divres<T>, TX * TY, 0);
    grid_cap[8] = cap((const void *)k_cfl<T>, TX * TY, 0);
    grid_cap[9] = shell_per == 4 ? cap((const void *)k_ghosts<T, 4>, kShellThreads, 0)
                                 : cap((const void *)k_ghosts<T>, kShellThreads, 0);
    grid_cap[13] = cap((const void *)k_tri_tile<T, 16>, tri_tile_threads<16>(), smem_trit);
    grid_cap[15] = cap((const void *)k_tri_tile<T, 32>, tri_tile_threads<32>(), smem_trit32);
    grid_cap[11] = cap((const void *)k_scalar<T>, TX * TY, 0);
    grid_cap[12] = std::is_same<T, float>::value ? cap((const void *)k_scalar_pair<8>, SPX * 8, 0) : 1;
    grid_cap[14] = std::is_same<T, float>::value ? cap((const void *)k_scalar_pair<4>, SPX * 4, 0) : 1;
    // one launch set per distinct x (y) length, holding only its domains
    auto reg_sets = [&](bool use, bool ydir, std::vector<RegSet> &out) -> int {
      if (!use) return ELMM_OK;
      std::vector<int> lens;
      for (auto &h : hdom) {
        const int n = ydir ? h.ny : h.nx;
        if (fft_reg_supported(n) && std::find(lens.begin(), lens.end(), n) == lens.end()) lens.push_back(n);
      }
      for (int n : lens) {
        RegSet r;
        r.k = fft_reg_kernels<T>(n);
        r.smem = sizeof(T2) * fft_reg_batch(n) * fft_reg_seq(n);
        std::vector<int> st(nd + 1, 0);
        for (int d = 0; d < nd; d++)
          st[d + 1] = st[d] + ((ydir ? hdom[d].ny : hdom[d].nx) == n ? tiles(ydir ? LK_YREG : LK_XREG, hdom[d]) : 0);
        r.ls.nd = nd;
        r.ls.total = st[nd];
        int rr = dalloc((void **)&r.ls.starts, sizeof(int) * (nd + 1));
        if (rr) return rr;
        CU(cudaMemcpy(r.ls.starts, st.data(), sizeof(int) * (nd + 1), cudaMemcpyHostToDevice));
        const void *f1 = ydir ? (const void *)r.k->yf : (const void *)r.k->fwd;
        const void *f2 = ydir ? (const void *)r.k->yi : (const void *)r.k->inv;
        // the dynamic maximum leaves room for the kernel's static shared memory
        for (const void *f : {f1, f2}) {
          cudaFuncAttributes fa;
          CU(cudaFuncGetAttributes(&fa, f));
          if (r.smem + fa.sharedSizeBytes > (size_t)optin)
            return fail(ELMM_ERR_INVALID_CONFIG, "shared memory of the register transforms exceeds the device limit");
          CU(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes));
        }
        r.cap_fwd = cap(f1, kRegThreads, r.smem);
        r.cap_inv = cap(f2, kRegThreads, r.smem);
        out.push_back(r);
      }
      return ELMM_OK;
    };
    if ((r = reg_sets(reg_x, false, xreg))) return r;
    if ((r = reg_sets(reg_y, true, yreg))) return r;
    // staging for host-layout copies (a view copies nothing to the host)
    stage_elems = 0;
    for (int d = 0; d < n && !is_view; d++) {
      const Dom<T> &h = hdom[d];
      size_t e = (size_t)(h.nx + 6) * (h.ny + 6) * (h.nz + 6);
      stage_elems = std::max(stage_elems, e);
    }
    if (!is_view && (r = dalloc((void **)&dstage, stage_elems * sizeof(double)))) return r;
    for (int d = 0; d < n; d++) cells += (long long)hdom[d].nx * hdom[d].ny * hdom[d].nz;
    return ELMM_OK;
  }

  // after the upload of a serving request: the host-layout staging and the
  // Pr image serve only copies to and from the host
  void drop_host_staging() {
    dfree(dstage);
    dstage = nullptr;
    if (dstage2) dfree(dstage2);
    dstage2 = nullptr;
    stage_state = -1;
    stage_elems = 0;
    for (auto &pi : pr_image) { dfree(pi); pi = nullptr; }
  }

  // whether a domain's transforms / z solve use the register FFTs and the
  // tiled Thomas kernel (decided per domain, so that a domain gives the same
  // result alone and in any batch)
  static bool tri_tiled(const Dom<T> &h) { return !h.zper && h.nz <= kTriTileMaxNz; }
  // the FP32 scalar stage runs two cells per thread when the pairs tile the
  // periodic x axis
  static bool scalar_pairs(const Dom<T> &h) { return sizeof(T) == 4 && h.nx % 2 == 0; }
  // the same for the projection (the velocity is periodic in x for every domain)
  static bool fp32_pairs(const Dom<T> &h) { return sizeof(T) == 4 && h.nx % 2 == 0 && h.bt[SIDE_WE] == BC_PERIODIC; }

  int tiles(int kind, const Dom<T> &h) const {
    int ntx = (h.nx + TX - 1) / TX, nty = (h.ny + TY - 1) / TY;
    switch (kind) {
      case LK_CELLS: return ntx * nty * h.nz;
      case LK_BOX: return ((h.nx + 2 + TX - 1) / TX) * ((h.ny + 2 + TY - 1) / TY) * (h.nz + 2);
      case LK_ROWS: return fft_reg_supported(h.nx) ? 0 : (h.ny * h.nz + kRowsX - 1) / kRowsX;
      case LK_YCOLS: return fft_reg_supported(h.ny) ? 0 : ((h.nxh + TyOf<T>::v - 1) / TyOf<T>::v) * h.nz;
      case LK_MOM: return ((h.nx + MX - 1) / MX) * ((h.ny + MY - 1) / MY) * ((h.nz + MKC - 1) / MKC);
      case LK_MOMT: return ((h.nx + MX - 1) / MX) * ((h.ny + MY - 1) / MY) * ((h.nz + tune_mom_kc - 1) / tune_mom_kc);
      case LK_SGST: return ((h.nx + MX - 1) / MX) * ((h.ny + MY - 1) / MY) * ((h.nz + tune_sgs_kc - 1) / tune_sgs_kc);
      case LK_WM: return (int)((wm_points_of(h) + kWmThreads - 1) / kWmThreads);
      case LK_PROJ: return fp32_pairs(h) && !slab_mode ? 0 : tiles(LK_MOM, h);
      case LK_PROJ2: return fp32_pairs(h) && !slab_mode ? tiles(LK_MOM, h) : 0;
      case LK_SHELL: return (int)((shell_cells(h.nx, h.ny, h.nz) + kShellThreads * shell_per - 1) / (kShellThreads * shell_per));
      case LK_XREG: {
        if (!fft_reg_supported(h.nx)) return 0;
        const int rows = 2 * fft_reg_batch(h.nx);
        return (h.ny * h.nz + rows - 1) / rows;
      }
      case LK_YREG: {
        if (!fft_reg_supported(h.ny)) return 0;
        const int C = fft_reg_batch(h.ny);
        return ((h.nxh + C - 1) / C) * h.nz;
      }
      case LK_TRIT: return tri_tiled(h) ? (h.ny * h.spitch + tune_cols - 1) / tune_cols : 0;
      case LK_TCOL: return scalar_pairs(h) ? 0 : ntx * nty * ((h.nz + TMKC - 1) / TMKC) * h.nslot;
      case LK_TPAIR:
        return scalar_pairs(h) ? ((h.nx + 2 * SPX - 1) / (2 * SPX)) * ((h.ny + tune_rows - 1) / tune_rows) *
                                     ((h.nz + TMKC - 1) / TMKC) * h.nslot
                               : 0;
      case LK_DCOL: return scalar_pairs(h) ? 0 : ntx * nty * ((h.nz + kDivChunk - 1) / kDivChunk);
      case LK_DCOL2:
        return scalar_pairs(h) ? ((h.nx + 2 * TX - 1) / (2 * TX)) * nty * ((h.nz + kDivChunk - 1) / kDivChunk) : 0;
      case LK_AVG: return (h.nslot - (h.buoy ? 1 : 0)) * ((h.avg_k > 0 ? h.ny : 0) + (h.avg_j > 0 ? h.nz : 0));
      case LK_COMMIT: {
        const long long nvec = h.plane * h.nz * (long long)sizeof(T) / 16;
        return h.nslot * (int)((nvec + kCommitVecs - 1) / kCommitVecs);
      }
      default: return tri_tiled(h) ? 0 : (h.ny * h.spitch + kTriThreads - 1) / kTriThreads;
    }
  }

  int init_domain(int di) {
    const elmm_config &c = cfg[di];
    HostGrid &g = grid[di];
    make_grid(c, g);
    if (zparent) {  // a slab: the levels of the whole domain from zk0 on, ghosts included
      const HostGrid &G = *zparent;
      for (int k = -2; k <= g.nz + 3; k++) {
        g.zW[k + 2] = G.zW[zk0 + k + 2];
        g.zPr[k + 2] = G.zPr[zk0 + k + 2];
        g.dzPr[k + 2] = G.dzPr[zk0 + k + 2];
      }
      for (int k = -2; k <= g.nz + 2; k++) g.dzW[k + 2] = G.dzW[zk0 + k + 2];
      for (int k = 1; k <= g.nz; k++) g.width[k] = G.width[zk0 + k];
      g.dzmin = G.dzmin;
    }
    Dom<T> h;
    memset(&h, 0, sizeof(h));
    h.nx = c.Prnx; h.ny = c.Prny; h.nz = c.Prnz;
    const int *b = c.Btype;
    int Unx = b[ELMM_EA] == ELMM_BC_PERIODIC ? h.nx : h.nx - 1;
    int Vny = b[ELMM_NO] == ELMM_BC_PERIODIC ? h.ny : h.ny - 1;
    int Wnz = b[ELMM_TO] == ELMM_BC_PERIODIC || b[ELMM_TO] == BC_HALO ? h.nz : h.nz - 1;
    int ext[3][3] = {{Unx, h.ny, h.nz}, {h.nx, Vny, h.nz}, {h.nx, h.ny, Wnz}};
    memcpy(h.ext, ext, sizeof(ext));
    h.aln = 128 / (int)sizeof(T);
    h.pitch = round_up(h.aln + h.nx + 1, h.aln);
    h.plane = (long long)h.pitch * (h.ny + 2);
    for (int s = 0; s < 6; s++) h.bt[s] = b[s];
    h.vz = c.zW ? 1 : 0;
    for (int s = 0; s < 6; s++) h.wall[s] = (c.wallmodeltype > 0 && b[s] == ELMM_BC_NOSLIP) ? 1 : 0;
    h.sgs = c.sgstype == 1;
    h.prgx_on = c.enable_pr_gradient_x_uniform; h.prgy_on = c.enable_pr_gradient_y_uniform;
    h.prgx = c.pr_gradient_x; h.prgy = c.pr_gradient_y;
    h.dx = c.dxmin; h.dy = c.dymin; h.dz = g.dzmin;
    h.xmin = c.xmin; h.ymin = c.ymin;
    h.dt = c.dt;
    h.dt0 = c.dt;
    h.vdt = c.variable_time_steps ? 1 : 0;
    h.cfl_target = c.CFL;
    h.dt_max = c.dt_max;
    h.end_time = c.end_time;
    h.nu_mol = c.molecular_viscosity;
    {
      const double dd[3] = {c.dxmin, c.dymin, g.dzmin};
      for (int a = 0; a < 3; a++) {
        h.cA[a] = 0.25 / dd[a];
        h.rec2[a] = 1.0 / (dd[a] * dd[a]);
        for (int comp = 0; comp < 3; comp++) h.cB[comp][a] = (comp == a ? 0.5 : 0.125) / dd[a];
      }
    }
    h.cs = c.C_Smagorinsky;
    if (!g.uniform_xy) return fail(ELMM_ERR_INVALID_CONFIG, "dxPr/dyPr must be uniform");
    size_t box = (size_t)h.plane * (h.nz + 2);
    // a margin of two rows past the box
    const size_t alloc_elems = box + 2 * (size_t)h.pitch + 64;
    T **fields[12] = {&h.U, &h.V, &h.W, &h.U2, &h.V2, &h.W2, &h.Us, &h.Vs, &h.Ws, &h.P, &h.nu, &h.Phi};
    for (T **f : fields) {
      int r = dalloc((void **)f, alloc_elems * sizeof(T));
      if (r) return r;
    }
    {
      // tensor maps of the box fields for the plane rings (wide: tile plus
      // halo, narrow: tile alone), in field order F_U..F_PHI
      typedef SlotLayout<T, 5, MomShape<T>::nnf> Lay;
      std::vector<CUtensorMap> maps(2 * F_COUNT);
      for (int f = 0; f < F_COUNT; f++) {
        int r = encode_box_map(&maps[BOX_WIDE * F_COUNT + f], *fields[f], h.pitch, h.ny, h.nz, Lay::SPW, Lay::WROWS);
        if (!r) r = encode_box_map(&maps[BOX_NARROW * F_COUNT + f], *fields[f], h.pitch, h.ny, h.nz, MX, MY);
        if (r) return r;
      }
      void *p;
      int r = dalloc(&p, maps.size() * sizeof(CUtensorMap));
      if (r) return r;
      CU(cudaMemcpy(p, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
      h.tmaps = p;
    }
    h.nxh = h.nx / 2 + 1;
    h.spitch = round_up(h.nxh, TyOf<T>::v);
    int r = dalloc((void **)&h.S, (size_t)h.nz * h.ny * h.spitch * sizeof(T2));
    if (r) return r;
    // FFT
    PoisPlan pl;
    factorize(h.nx, pl.fx);
    factorize(h.ny, pl.fy);
    hplan[di] = pl;
    auto twiddles = [](int n) {
      std::vector<T2> w(n);
      for (int m = 0; m < n; m++) {
        double a = -2.0 * M_PI * (double)m / (double)n;
        w[m].x = (T)std::cos(a);
        w[m].y = (T)std::sin(a);
      }
      return w;
    };
    if ((r = upload_table(&h.twx, twiddles(h.nx)))) return r;
    if ((r = upload_table(&h.twy, twiddles(h.ny)))) return r;
    std::vector<double> lx(h.nx), ly(h.ny);
    double rx = 1 / (c.dxmin * c.dxmin), ry = 1 / (c.dymin * c.dymin);
    for (int m = 0; m < h.nx; m++) { double s = std::sin(M_PI * m / h.nx); lx[m] = -4.0 * s * s * rx; }
    for (int m = 0; m < h.ny; m++) { double s = std::sin(M_PI * m / h.ny); ly[m] = -4.0 * s * s * ry; }
    if ((r = upload_table(&h.lamx, lx))) return r;
    if ((r = upload_table(&h.lamy, ly))) return r;
    h.zper = b[ELMM_BO] == ELMM_BC_PERIODIC;
    std::vector<double> Ab(h.nz + 2, 0.0), At(h.nz + 2, 0.0), dzc(h.nz + 2, 0.0), dzf(h.nz + 2, 0.0);
    auto zP = [&](int k) { return g.zPr[k + 2]; };
    auto zWf = [&](int k) { return g.zW[k + 2]; };
    for (int k = 1; k <= h.nz; k++) {
      Ab[k] = 1 / ((zP(k) - zP(k - 1)) * (zWf(k) - zWf(k - 1)));
      At[k] = 1 / ((zP(k + 1) - zP(k)) * (zWf(k) - zWf(k - 1)));
      dzc[k] = zWf(k) - zWf(k - 1);
      dzf[k] = zP(k + 1) - zP(k);
    }
    if (!h.zper && b[ELMM_BO] != BC_HALO) Ab[1] = 0;  // a slab face couples to the next slab
    if (!h.zper && b[ELMM_TO] != BC_HALO) At[h.nz] = 0;
    if ((r = upload_table(&h.Ab, Ab))) return r;
    if ((r = upload_table(&h.At, At))) return r;
    if ((r = upload_table(&h.dzc, dzc))) return r;
    if ((r = upload_table(&h.dzf, dzf))) return r;
    if (tri_tiled(h)) {  // pivot carries of the tiled z solve at its segment starts, once per domain
      const int ncol = h.ny * h.spitch;
      double *c0;
      if ((r = dalloc((void **)&c0, (size_t)kTriPivSegs * ncol * sizeof(double)))) return r;
      k_tri_factors<<<(ncol + 255) / 256, 256, 0, stream>>>(c0, h.lamx, h.lamy, h.Ab, h.At, h.nxh, h.spitch, h.ny, h.nz);
      CU(cudaStreamSynchronize(stream));
      CU(cudaGetLastError());
      h.tri_c0 = c0;
    }
    if ((r = upload_table(&h.zPr, g.zPr))) return r;
    if ((r = upload_table(&h.dzPr, g.dzPr))) return r;
    if ((r = upload_table(&h.zW, g.zW))) return r;
    if ((r = upload_table(&h.dzW, g.dzW))) return r;
    if ((r = upload_table(&h.width, g.width))) return r;
    {
      std::vector<double> rdz(h.nz + 1, 0.0), r2zz(h.nz + 1, 0.0), wc2(h.nz + 1, 0.0);
      for (int k = 1; k <= h.nz; k++) {
        rdz[k] = 1.0 / g.dzPr[k + 2];
        r2zz[k] = 1.0 / (2 * (g.zPr[k + 1 + 2] - g.zPr[k - 1 + 2]));
        double wc = g.width[k] * c.C_Smagorinsky;
        wc2[k] = wc * wc;
      }
      if ((r = upload_table(&h.sgs_rdz, rdz))) return r;
      if ((r = upload_table(&h.sgs_r2zz, r2zz))) return r;
      if ((r = upload_table(&h.sgs_wc2, wc2))) return r;
    }
    if (h.vz && sizeof(T) == 4) {  // per-level factors of the packed FP32 momentum path
      const int nzp = h.nz + 2;
      std::vector<float> kz((size_t)kZ2 * nzp, 0.f);
      auto zP = [&](int k) { return g.zPr[k + 2]; };
      auto zWv = [&](int k) { return g.zW[k + 2]; };
      auto dP = [&](int k) { return g.dzPr[k + 2]; };
      auto dW = [&](int k) { return g.dzW[k + 2]; };
      for (int k = 1; k <= h.nz; k++) {
        kz[KZ_AUV * nzp + k] = (float)(1.0 / (4.0 * dP(k)));
        kz[KZ_BUV * nzp + k] = (float)(1.0 / (4.0 * (zP(k + 1) - zP(k - 1))));
        kz[KZ_D1UV * nzp + k] = (float)(1.0 / (dW(k) * dP(k)));
        kz[KZ_D2UV * nzp + k] = (float)(1.0 / (dW(k - 1) * dP(k)));
        kz[KZ_AW * nzp + k] = (float)(1.0 / (4.0 * dW(k)));
        kz[KZ_BW * nzp + k] = (float)(1.0 / (zWv(k + 1) - zWv(k - 1)));
        kz[KZ_D1W * nzp + k] = (float)(1.0 / (dP(k + 1) * dW(k)));
        kz[KZ_D2W * nzp + k] = (float)(1.0 / (dP(k) * dW(k)));
        kz[KZ_RDZW * nzp + k] = (float)(1.0 / dW(k));
      }
      if ((r = upload_table(&h.kz2, kz))) return r;
    }
    // wall-model planes
    for (int s = 0; s < 6; s++) h.z0[s] = c.z0[s];
    for (int comp = 0; comp < 3; comp++)
      for (int s = 0; s < 6; s++) {
        if (!h.wall[s]) continue;
        int axis = s >> 1;
        int a0 = axis == 0 ? 1 : 0, a1 = axis == 2 ? 1 : 2;
        size_t np = (size_t)ext[comp][a0] * ext[comp][a1];
        int f = comp * 6 + s;
        if ((r = dalloc((void **)&h.wm_fluxp[f], np * sizeof(T)))) return r;
        if ((r = dalloc((void **)&h.wm_fluxm[f], np * sizeof(T)))) return r;
        if ((r = dalloc((void **)&h.wm_ustar[f], np * sizeof(double)))) return r;
        std::vector<double> ones(np, 1.0);  // WMPointUVW%ustar = 1 initially (wallmodels.f90:80)
        CU(cudaMemcpy(h.wm_ustar[f], ones.data(), np * sizeof(double), cudaMemcpyHostToDevice));
        if (c.enable_buoyancy && (s == ELMM_BO || s == ELMM_TO) && c.TempBtype[s] == ELMM_BC_DIRICHLET) {
          // a prescribed surface temperature: the points' temperature_flux, 0 initially
          if ((r = dalloc((void **)&h.wm_tfl[f], np * sizeof(double)))) return r;
          CU(cudaMemset(h.wm_tfl[f], 0, np * sizeof(double)));
        }
      }
    if (c.enable_buoyancy) {
      h.buoy = 1;
      for (int s2 = 0; s2 < 6; s2++) h.tbt[s2] = c.TempBtype[s2];
      h.tref = c.temperature_ref;
      h.grav = c.grav_acc;
      h.kappa_mol = c.molecular_diffusivity;
      h.toff = sizeof(T) == 4 ? c.temperature_ref : 0.0;  // FP32 stores theta - T_ref
      ScalSlot<T> &sl = h.slot[h.nslot++];
      for (T **f : {&sl.buf[0], &sl.buf[1], &sl.buf[2], &sl.adv})
        if ((r = dalloc((void **)f, alloc_elems * sizeof(T)))) return r;
      h.Tm = sl.buf[0];
      h.Tadv = sl.adv;
      if (MomShape<T>::nnf == 4) {  // the temperature's planes for the momentum ring
        std::vector<CUtensorMap> tm(3);
        for (int b2 = 0; b2 < 3; b2++)
          if ((r = encode_box_map(&tm[b2], sl.buf[b2], h.pitch, h.ny, h.nz, MX, MY))) return r;
        void *p;
        if ((r = dalloc(&p, tm.size() * sizeof(CUtensorMap)))) return r;
        CU(cudaMemcpy(p, tm.data(), tm.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
        h.tmapT = p;
      }
      for (int s2 = 0; s2 < 6; s2++) sl.bt[s2] = c.TempBtype[s2];
      sl.off = h.toff;
      // a surface heat flux at a wall-model wall: the temperature_flux of the
      // side's wall-model points (src/wallmodels.f90:590-596, 650-656), and
      // its term in the cells next to the wall with ComputeAreaFactor's
      // boundary area over cell volume (src/wallmodels.f90:173-203)
      const double dq = sqrt(h.dx * h.dy), area_factor = dq * (dq / 1.0) / (h.dx * h.dy * h.dz);
      for (int side : {ELMM_BO, ELMM_TO})
        if (h.wall[side] && c.TempBtype[side] == ELMM_BC_CONSTFLUX) {
          h.tflux[side] = side == ELMM_BO ? c.sideTemp[side] : -c.sideTemp[side];
          sl.wflux[side == ELMM_BO ? 0 : 1] = h.tflux[side] * area_factor;
        } else if (h.wall[side] && c.TempBtype[side] == ELMM_BC_DIRICHLET) {
          // a prescribed surface temperature (WM_MO_Dirichlet): the Pr points
          // next to the wall with u* = 1 and no flux initially
          // (src/wallmodels.f90:570-627)
          const int hh = side == ELMM_BO ? 0 : 1;
          const size_t np = (size_t)h.nx * h.ny;
          h.tdir[side] = 1;
          h.tsurf[side] = c.sideTemp[side];
          if ((r = dalloc((void **)&h.wm_pr_us[hh], np * sizeof(double)))) return r;
          if ((r = dalloc((void **)&h.wm_pr_tf[hh], np * sizeof(double)))) return r;
          std::vector<double> ones(np, 1.0);
          CU(cudaMemcpy(h.wm_pr_us[hh], ones.data(), np * sizeof(double), cudaMemcpyHostToDevice));
          CU(cudaMemset(h.wm_pr_tf[hh], 0, np * sizeof(double)));
        }
      h.wm_af = area_factor;
      set_zghosts(sl, c.TempBtype, c.sideTemp, h.wall);
      h.tdiff_live = 1;
    }
    h.kappa_mol = c.molecular_diffusivity;
    for (int sc = 0; sc < c.num_scalars; sc++) {
      ScalSlot<T> &sl = h.slot[h.nslot++];
      for (T **f : {&sl.buf[0], &sl.buf[1], &sl.buf[2], &sl.adv})
        if ((r = dalloc((void **)f, alloc_elems * sizeof(T)))) return r;
      for (int s2 = 0; s2 < 6; s2++) sl.bt[s2] = c.ScalBtype[s2];
      sl.off = 0;
      set_zghosts(sl, c.ScalBtype, c.sideScal, nullptr);  // no wall-model points for a passive scalar
      if (c.avg_slice_k > 0 && (r = dalloc((void **)&sl.acc_xy, sizeof(double) * h.nx * h.ny))) return r;
      if (c.avg_slice_j > 0 && (r = dalloc((void **)&sl.acc_xz, sizeof(double) * h.nx * h.nz))) return r;
    }
    // a slab: the second halo planes of every scalar slot beyond its BC_HALO faces
    for (int s = 0; s < h.nslot; s++)
      for (int side = 0; side < 2; side++)
        if (h.slot[s].bt[side ? SIDE_TO : SIDE_BO] == BC_HALO &&
            (r = dalloc((void **)&h.slot[s].h2[side], (size_t)h.plane * sizeof(T))))
          return r;
    h.avg_k = c.avg_slice_k;
    h.avg_j = c.avg_slice_j;
    h.avg_w = c.avg_weight;
    // point sources -> volume sources of one cell each (ScalarPointSource's
    // point_source, src/pointsources.f90:24-39): flux / volumePr
    for (int q = 0; q < c.num_point_sources; q++) {
      const elmm_point_source &p = c.point_sources[q];
      int ip[3];
      if (!point_cell(c, p.position, ip)) continue;  // outside the domain: no volume
      const int e = h.nsrc++;
      h.src_slot[e] = (h.buoy ? 1 : 0) + p.scalar_number - 1;
      h.src_i[e] = ip[0]; h.src_j[e] = ip[1]; h.src_k[e] = ip[2];
      h.src_q[e] = p.flux / (g.dxPr[ip[0]] * g.dyPr[ip[1]] * g.dzPr[ip[2] + 2]);
    }
    if (c.enable_buoyancy || c.num_scalars > 0) {
      if ((r = dalloc((void **)&h.TDiff, alloc_elems * sizeof(T)))) return r;
      // TDiff starts at the molecular diffusivity (src/initial.f90:4262-4268)
      if (c.molecular_viscosity > 0) {
        std::vector<T> kv(alloc_elems, (T)c.molecular_diffusivity);
        CU(cudaMemcpy(h.TDiff, kv.data(), alloc_elems * sizeof(T), cudaMemcpyHostToDevice));
      }
    }
    // mixed path: the per-level offsets of U and V (zero until the first
    // upload; see Dom::voff)
    if (sizeof(T) == 4 && (r = dalloc((void **)&h.voff, sizeof(float) * 2 * (h.nz + 2)))) return r;
    if ((r = dalloc((void **)&h.prm, sizeof(double)))) return r;
    h.nprpart = ((h.nx + MX - 1) / MX) * ((h.ny + MY - 1) / MY);
    if ((r = dalloc((void **)&h.prpart, sizeof(double) * h.nprpart))) return r;
    if ((r = dalloc((void **)&h.maxdiv_bits, sizeof(unsigned long long)))) return r;
    if ((r = dalloc((void **)&h.cfl_bits, sizeof(unsigned long long)))) return r;
    {
      const double ts[2] = {0.0, c.dt};  // time 0, no step yet
      if ((r = dalloc((void **)&h.tstate, sizeof(ts)))) return r;
      CU(cudaMemcpy(h.tstate, ts, sizeof(ts), cudaMemcpyHostToDevice));
    }
    if ((r = dalloc((void **)&h.flags, 4 * sizeof(int)))) return r;
    h.wait_limit = kWaitLimit;
    h.skip_plane = -1;
    if ((r = dalloc((void **)&h.refine_flag, sizeof(int)))) return r;
    if ((r = dalloc((void **)&h.refine_count, 2 * sizeof(int)))) return r;
    h.refine_tol = c.refine_tol;
    h.max_refine = c.max_refine_sweeps;
    size_t pe = (size_t)(h.nx + 4) * (h.ny + 4) * (h.nz + 4);
    if ((r = dalloc((void **)&pr_image[di], pe * sizeof(double)))) return r;
    // viscosity starts at the molecular value (src/initial.f90:4275)
    std::vector<T> nuv(box, (T)c.molecular_viscosity);
    CU(cudaMemcpy(h.nu, nuv.data(), box * sizeof(T), cudaMemcpyHostToDevice));
    hdom[di] = h;
    return ELMM_OK;
  }

  int gsz(int which, int total) const { return std::max(1, std::min(total, grid_cap[which])); }

  // ------------------------------------------------------------ stages
  // ghost shells of the listed fields after the kernel that wrote them
  // prref: the launch also reduces the pressure reference (after the projection)
  void launch_ghosts(std::initializer_list<int> fields, int gate, int prref = 0) {
    unsigned packed = 0;
    int nf = 0;
    for (int f : fields) packed |= (unsigned)f << (8 * nf++);
    nlaunch++;
    if (shell_per == 4)
      k_ghosts<T, 4><<<gsz(9, ls[LK_SHELL].total * nf), kShellThreads, 0, stream>>>(ddom, ls[LK_SHELL].l(), packed, nf,
                                                                                    gate, prref);
    else
      k_ghosts<T><<<gsz(9, ls[LK_SHELL].total * nf), kShellThreads, 0, stream>>>(ddom, ls[LK_SHELL].l(), packed, nf,
                                                                                 gate, prref);
  }
  static int chunk_index(int kc) { return kc == 8 ? 0 : kc == 16 ? 1 : 2; }
  // k_sgs with the tuned z chunk; init: 0 a stage, 1 the initial viscosity
  // and diffusivity, 2 the autotuner's timing mode (k_sgs)
  void sgs_kernel(int init) {
    const int q = chunk_index(tune_sgs_kc), g = std::max(1, std::min(ls[LK_SGST].total, cap_sgs[q]));
    if (tune_sgs_kc == 8) k_sgs<T, 8><<<g, SgsShape<T>::threads, smem_sgs, stream>>>(ddom, ls[LK_SGST].l(), init);
    else if (tune_sgs_kc == 16) k_sgs<T, 16><<<g, SgsShape<T>::threads, smem_sgs, stream>>>(ddom, ls[LK_SGST].l(), init);
    else k_sgs<T, 32><<<g, SgsShape<T>::threads, smem_sgs, stream>>>(ddom, ls[LK_SGST].l(), init);
  }
  // the wall model of a stage (k_wm_points) from the state at its start, on
  // stream s; stage 1 outside a step (the initial fields).  Returns 1 if it
  // launched.
  int wm_kernel(int stage, cudaStream_t s) {
    if (ls[LK_WM].total == 0) return 0;
    k_wm_points<T><<<std::min(ls[LK_WM].total, 148 * 16), kWmThreads, 0, s>>>(ddom, ls[LK_WM].l(), (stage - 1) % 3);
    return 1;
  }
  void momentum_kernel(const StageCoef &sc) {
    const int q = chunk_index(tune_mom_kc), g = std::max(1, std::min(ls[LK_MOMT].total, cap_mom[q]));
    if (tune_mom_kc == 8) k_momentum<T, 8><<<g, MomShape<T>::threads, smem_mom, stream>>>(ddom, ls[LK_MOMT].l(), sc);
    else if (tune_mom_kc == 16) k_momentum<T, 16><<<g, MomShape<T>::threads, smem_mom, stream>>>(ddom, ls[LK_MOMT].l(), sc);
    else k_momentum<T, 32><<<g, MomShape<T>::threads, smem_mom, stream>>>(ddom, ls[LK_MOMT].l(), sc);
  }
  int launch_sgs(int stage) {
    nlaunch++;
    // the wall model on a branch beside k_sgs (a graph branch when
    // captured): neither reads what the other writes
    const bool wm = ls[LK_WM].total > 0 && branch[1];
    if (wm) {
      CU(cudaEventRecord(ev_fork, stream));
      CU(cudaStreamWaitEvent(branch[1], ev_fork, 0));
      nlaunch += wm_kernel(stage, branch[1]);
      CU(cudaEventRecord(ev_join[1], branch[1]));
    }
    sgs_kernel(0);
    if (wm) CU(cudaStreamWaitEvent(stream, ev_join[1], 0));
    launch_ghosts({F_NU}, 0);
    return ELMM_OK;
  }
  int launch_momentum(int stage) {
    StageCoef sc{kRho[stage - 1], kBeta[stage - 1], 2 * kAlpha[stage - 1], stage};
    nlaunch++;
    // no ghost pass for U2, V2, W2: their only reader, the divergence of the
    // forward x transform, folds its neighbours on the box faces itself
    momentum_kernel(sc);
    return ELMM_OK;
  }
  void launch_project(double coef_alpha2, int use_dt, int in_place, int gate) {
    k_project_any(coef_alpha2, use_dt, in_place, gate);
    launch_ghosts({F_U, F_V, F_W, F_P}, gate, 1);  // and the pressure reference of k_prref
  }
  // k_project for the domains that take it, k_project_pair (FP32, even Prnx) for the others
  void k_project_any(double coef_alpha2, int use_dt, int in_place, int gate) {
    if (ls[LK_PROJ].total > 0) {
      nlaunch++;
      if (slab_mode)
        k_project<T, true><<<gsz(6, ls[LK_PROJ].total), MX * MY, 0, stream>>>(ddom, ls[LK_PROJ].l(), coef_alpha2,
                                                                             use_dt, in_place, gate);
      else
        k_project<T><<<gsz(6, ls[LK_PROJ].total), MX * MY, 0, stream>>>(ddom, ls[LK_PROJ].l(), coef_alpha2, use_dt,
                                                                         in_place, gate);
    }
    if constexpr (std::is_same<T, float>::value) {
      if (ls[LK_PROJ2].total > 0) {
        nlaunch++;
        k_project_pair<<<gsz(10, ls[LK_PROJ2].total), MX * MY / 2, 0, stream>>>(ddom, ls[LK_PROJ2].l(), coef_alpha2,
                                                                               use_dt, in_place, gate);
      }
    }
  }
  // one ScalarRK3 stage of every transported scalar; the new values then
  // become the current ones (the stage reads the old value at neighbours
  // while writing).  accumulate: the last stage of a step, which also feeds
  // the time-averaged slices.
  // standalone: a stage run on its own (elmm_run_stage), whose new value is
  // copied to buf[0] where the host reads it
  void launch_scalars(int stage, int accumulate, bool standalone = false) {
    if (ls[LK_TCOL].total == 0 && ls[LK_TPAIR].total == 0) return;
    bool zghost = false;
    for (int d = 0; d < nd; d++)
      for (int s = 0; s < hdom[d].nslot; s++) zghost |= hdom[d].slot[s].zg[0] || hdom[d].slot[s].zg[1];
    if (zghost) {  // BoundTemperature / BoundScalar at the start of the stage, after the stage's TDiff
      nlaunch++;
      k_scalar_zghost<T><<<2 * 148, 256, 0, stream>>>(ddom, nd, stage);
    }
    if (ls[LK_TCOL].total > 0) {
      nlaunch++;
      if (scalar_bcs())
        k_scalar<T, true><<<gsz(11, ls[LK_TCOL].total), TX * TY, 0, stream>>>(ddom, ls[LK_TCOL].l(), kRho[stage - 1],
                                                                             kBeta[stage - 1], stage);
      else
        k_scalar<T><<<gsz(11, ls[LK_TCOL].total), TX * TY, 0, stream>>>(ddom, ls[LK_TCOL].l(), kRho[stage - 1],
                                                                       kBeta[stage - 1], stage);
    }
    if constexpr (std::is_same<T, float>::value) {
      if (ls[LK_TPAIR].total > 0) {
        nlaunch++;
        launch_scalar_pair(stage);
      }
    }
    // the heat flux of the solid faces, then the fill of the solid cells
    // (src/scalars.f90:129-198)
    for (int d = 0; d < nd && d < (int)sol.size(); d++)
      if (sol[d].on && sol[d].nheat > 0) {
        nlaunch++;
        k_heat_add<T><<<std::min((sol[d].nheat + 255) / 256, 148 * 4), 256, 0, stream>>>(ddom, d, sol[d].heat,
                                                                                        sol[d].nheat, stage,
                                                                                        kBeta[stage - 1]);
      }
    for (int d = 0; d < nd && d < (int)sol.size(); d++)
      if (sol[d].on && sol[d].nfill > 0) {
        nlaunch++;
        k_theta_fill<T><<<std::min((sol[d].nfill + 255) / 256, 148 * 4), 256, 0, stream>>>(ddom, d, sol[d].fill,
                                                                                          sol[d].nfill, stage % 3);
      }
    bool puffs = false;
    for (int d = 0; d < nd; d++) puffs |= hdom[d].npv > 0;
    if (puffs) {
      nlaunch++;
      k_puff_add<T><<<1, kMaxPuffVols, 0, stream>>>(ddom, nd, stage, kBeta[stage - 1]);
    }
    if (standalone && stage % 3 != 0)
      k_scalar_commit<T><<<std::min(ls[LK_COMMIT].total, 16 * 148), kCommitThreads, 0, stream>>>(
          ddom, ls[LK_COMMIT].l(), stage % 3);
    if (accumulate && ls[LK_AVG].total > 0) {
      nlaunch++;
      k_scalar_avg<T><<<std::min(ls[LK_AVG].total, 8 * 148), 128, 0, stream>>>(ddom, ls[LK_AVG].l());
    }
  }
  // PressureCorrection on U2 (in_place = 0) or on U itself (initial projection)
  int launch_projection(double coef_alpha2, int use_dt, int in_place) {
    launch_poisson(coef_alpha2, use_dt, 0, 0);
    launch_project(coef_alpha2, use_dt, in_place, 0);
    return ELMM_OK;
  }
  // the pieces of the Poisson solve: register FFTs (one launch per distinct
  // length) and the tiled z solve where the whole batch allows them, the
  // generic kernels otherwise
  // n independent launches, launch(q, s) for q < n, spread over the branches
  // and joined back into the stream
  template <typename F>
  void fan_out(int n, F launch) {
    if (n <= 1 || !ev_fork) {
      for (int q = 0; q < n; q++) launch(q, stream);
      return;
    }
    const int nb = std::min(n, kBranches);
    cudaEventRecord(ev_fork, stream);
    for (int b = 1; b < nb; b++) cudaStreamWaitEvent(branch[b], ev_fork, 0);
    for (int q = 0; q < n; q++) launch(q, q % nb ? branch[q % nb] : stream);
    for (int b = 1; b < nb; b++) {
      cudaEventRecord(ev_join[b], branch[b]);
      cudaStreamWaitEvent(stream, ev_join[b], 0);
    }
  }
  void launch_fftx_fwd(double coef_alpha2, int use_dt, int rhs_from_phi, int gate) {
    const int nr = (int)xreg.size(), ng = ls[LK_ROWS].total > 0 ? 1 : 0;
    nlaunch += nr + ng;
    fan_out(nr + ng, [&](int q, cudaStream_t s) {
      if (q < nr) {
        const RegSet &r = xreg[q];
        r.k->fwd<<<std::max(1, std::min(r.ls.total, r.cap_fwd)), kRegThreads, r.smem, s>>>(ddom, r.ls.l(), coef_alpha2,
                                                                                           use_dt, rhs_from_phi, gate);
      } else {
        k_fftx_fwd<T><<<gsz(2, ls[LK_ROWS].total), kFFTThreads, smem_x, s>>>(ddom, ls[LK_ROWS].l(), dplan, coef_alpha2,
                                                                             use_dt, rhs_from_phi, gate);
      }
    });
  }
  void launch_ffty(int inverse, int gate) {
    const int nr = (int)yreg.size(), ng = ls[LK_YCOLS].total > 0 ? 1 : 0;
    nlaunch += nr + ng;
    fan_out(nr + ng, [&](int q, cudaStream_t s) {
      if (q < nr) {
        const RegSet &r = yreg[q];
        (inverse ? r.k->yi : r.k->yf)<<<std::max(1, std::min(r.ls.total, inverse ? r.cap_inv : r.cap_fwd)),
                                         kRegThreads, r.smem, s>>>(ddom, r.ls.l(), gate);
      } else {
        k_ffty<T><<<gsz(3, ls[LK_YCOLS].total), kFFTThreads, smem_y, s>>>(ddom, ls[LK_YCOLS].l(), dplan, inverse,
                                                                         gate);
      }
    });
  }
  // some slot of the batch has a stored z ghost plane, a surface flux or a
  // surface temperature: the scalar kernels' instantiation with those terms
  bool scalar_bcs() const {
    for (int d = 0; d < nd; d++) {
      const Dom<T> &h = hdom[d];
      if (h.tdir[ELMM_BO] || h.tdir[ELMM_TO] || h.pmask) return true;
      for (int s = 0; s < h.nslot; s++)
        if (h.slot[s].zg[0] || h.slot[s].zg[1] || h.slot[s].wflux[0] != 0 || h.slot[s].wflux[1] != 0 ||
            h.slot[s].bt[SIDE_BO] == BC_HALO || h.slot[s].bt[SIDE_TO] == BC_HALO)
          return true;
    }
    return false;
  }
  void launch_scalar_pair(int stage) {
    if constexpr (std::is_same<T, float>::value) {
      const Launch l = ls[LK_TPAIR].l();
      const double rho = kRho[stage - 1], beta = kBeta[stage - 1];
      const bool bc = scalar_bcs();
      if (tune_rows == 8) {
        if (bc) k_scalar_pair<8, true><<<gsz(12, ls[LK_TPAIR].total), SPX * 8, 0, stream>>>(ddom, l, rho, beta, stage);
        else k_scalar_pair<8><<<gsz(12, ls[LK_TPAIR].total), SPX * 8, 0, stream>>>(ddom, l, rho, beta, stage);
      } else {
        if (bc) k_scalar_pair<4, true><<<gsz(14, ls[LK_TPAIR].total), SPX * 4, 0, stream>>>(ddom, l, rho, beta, stage);
        else k_scalar_pair<4><<<gsz(14, ls[LK_TPAIR].total), SPX * 4, 0, stream>>>(ddom, l, rho, beta, stage);
      }
    }
  }
  void launch_tri(int gate) {
    if (ls[LK_TRIT].total > 0) {
      nlaunch++;
      if (tune_cols == 16)
        k_tri_tile<T, 16><<<gsz(13, ls[LK_TRIT].total), tri_tile_threads<16>(), smem_trit, stream>>>(
            ddom, ls[LK_TRIT].l(), gate);
      else
        k_tri_tile<T, 32><<<gsz(15, ls[LK_TRIT].total), tri_tile_threads<32>(), smem_trit32, stream>>>(
            ddom, ls[LK_TRIT].l(), gate);
    }
    if (ls[LK_TRI].total > 0) {
      nlaunch++;
      k_tri<T><<<gsz(4, ls[LK_TRI].total), kTriThreads, smem_tri, stream>>>(ddom, ls[LK_TRI].l(), gate);
    }
  }
  void launch_fftx_inv(int gate) {
    const int nr = (int)xreg.size(), ng = ls[LK_ROWS].total > 0 ? 1 : 0;
    nlaunch += nr + ng;
    fan_out(nr + ng, [&](int q, cudaStream_t s) {
      if (q < nr) {
        const RegSet &r = xreg[q];
        r.k->inv<<<std::max(1, std::min(r.ls.total, r.cap_inv)), kRegThreads, r.smem, s>>>(ddom, r.ls.l(), gate);
      } else {
        k_fftx_inv<T><<<gsz(5, ls[LK_ROWS].total), kFFTThreads, smem_x, s>>>(ddom, ls[LK_ROWS].l(), dplan, gate);
      }
    });
  }
  // the five transform kernels; rhs_from_phi: the right-hand side is in Phi.
  // Phi gets no ghost pass: its only reader, k_project, folds the i+1, j+1,
  // k+1 neighbours on the box faces itself.
  void launch_poisson(double coef_alpha2, int use_dt, int rhs_from_phi, int gate) {
    launch_fftx_fwd(coef_alpha2, use_dt, rhs_from_phi, gate);
    launch_ffty(0, gate);
    launch_tri(gate);
    launch_ffty(1, gate);
    launch_fftx_inv(gate);
  }
  int max_refine() const {
    int m = 0;
    for (auto &c : cfg) m = std::max(m, c.max_refine_sweeps);
    return m;
  }
  // Defect correction after a projection (mixed path): FP64 divergence
  // residual -> correction solve -> velocity / pressure update, at most
  // max_refine_sweeps times; the kernels of a sweep return at once for a
  // domain that does not need it, so the sweep stays inside the step graph.
  void launch_refine(double coef_alpha2, int use_dt) {
    const int R = max_refine();
    if (R == 0) return;
    for (int d = 0; d < nd; d++) cudaMemsetAsync(hdom[d].maxdiv_bits, 0, sizeof(unsigned long long), stream);
    k_divres<T><<<gsz(7, ls[LK_CELLS].total), TX * TY, 0, stream>>>(ddom, ls[LK_CELLS].l(), 0);
    nlaunch++;
    for (int sw = 0; sw < R; sw++) {
      k_refine_decide<T><<<(nd + 127) / 128, 128, 0, stream>>>(ddom, nd, sw == 0);
      launch_poisson(coef_alpha2, use_dt, 1, 1);
      launch_project(coef_alpha2, use_dt, 1, 1);
      k_divres<T><<<gsz(7, ls[LK_CELLS].total), TX * TY, 0, stream>>>(ddom, ls[LK_CELLS].l(), 1);
      nlaunch += 2;
    }
  }
  int launch_divmax() {
    nlaunch++;
    for (int d = 0; d < nd; d++) cudaMemsetAsync(hdom[d].maxdiv_bits, 0, sizeof(unsigned long long), stream);
    if (ls[LK_DCOL].total > 0)
      k_divmax<T><<<gsz(7, ls[LK_DCOL].total), TX * TY, 0, stream>>>(ddom, ls[LK_DCOL].l());
    if constexpr (std::is_same<T, float>::value) {
      if (ls[LK_DCOL2].total > 0) {
        nlaunch += ls[LK_DCOL].total > 0 ? 1 : 0;
        k_divmax_pair<<<gsz(7, ls[LK_DCOL2].total), TX * TY, 0, stream>>>(ddom, ls[LK_DCOL2].l());
      }
    }
    return ELMM_OK;
  }
  int launch_cfl() {
    nlaunch++;
    for (int d = 0; d < nd; d++) cudaMemsetAsync(hdom[d].cfl_bits, 0, sizeof(unsigned long long), stream);
    k_cfl<T><<<gsz(8, ls[LK_CELLS].total), TX * TY, 0, stream>>>(ddom, ls[LK_CELLS].l());
    return ELMM_OK;
  }
  // the solid-body launches of one stage phase (no-ops without bodies)
  // which: 0 viscosity of the ScalFl points, 1 wall-model corrections and the
  // IB points of U2 zeroed, 2 NullInterior + IBMomentum on the new velocity
  void launch_ib(int which, int stage) {
    for (int d = 0; d < nd && d < (int)sol.size(); d++) {
      const SolidSet &x = sol[d];
      if (!x.on) continue;
      if (which == 0 && x.nvisc > 0) {
        nlaunch++;
        k_ib_gather<T><<<std::min((x.nvisc + 255) / 256, 148 * 8), 256, 0, stream>>>(ddom, d, x.visc, x.nvisc, 0);
      }
      if (which == 1) {
        if (x.nwm > 0) {
          nlaunch++;
          k_ib_wm<T><<<std::min((x.nwm + 127) / 128, 148 * 8), 128, 0, stream>>>(ddom, d, x.wm, x.wm_ustar, x.nwm,
                                                                               kBeta[stage - 1], 0);
        }
        if (x.nib > 0) {
          nlaunch++;
          k_ib_gather<T><<<std::min((x.nib + 255) / 256, 148 * 8), 256, 0, stream>>>(ddom, d, x.vel, x.nib, 1);
        }
      }
      const int nnull = x.nnull.n[0] + x.nnull.n[1] + x.nnull.n[2];
      if (which == 2 && x.nib + nnull > 0) {
        nlaunch++;
        k_ib_gather<T><<<std::min((x.nib + nnull + 255) / 256, 148 * 8), 256, 0, stream>>>(ddom, d, x.vel, x.nib, 0,
                                                                                         x.null, x.nnull);
      }
    }
  }
  // div: the divergence check of the step, taken on the projected field before
  // IBMomentum replaces the IB points (the check of PostPoisson,
  // src/pressure.f90:884-989, is div U - Q on that field)
  int run_stage(int stage, int stop, int accumulate = 0, bool standalone = false, bool div = false) {
    launch_sgs(stage);
    if (any_solids()) launch_ib(0, stage);  // after BoundViscosity (src/dynamics.f90:896-902)
    if (stop == 1) return ELMM_OK;
    launch_momentum(stage);
    launch_scalars(stage, accumulate, standalone);  // ScalarRK3 between Convection and the projection (tsteps.f90:132-135)
    if (any_solids()) launch_ib(1, stage);
    if (stop == 2) return ELMM_OK;
    // the projection writes the new velocity into U itself, which takes the
    // place of the U <-> U2 pointer exchange (exchange_alloc, tsteps.f90:211-213)
    launch_projection(2 * kAlpha[stage - 1], 1, 0);
    launch_refine(2 * kAlpha[stage - 1], 1);
    if (any_solids()) {
      if (div) launch_divmax();
      launch_ib(2, stage);  // NullInterior, BoundUVW, IBMomentum, BoundUVW (tsteps.f90:201-206)
      launch_ghosts({F_U, F_V, F_W}, 0);
    }
    return ELMM_OK;
  }
  // PreparePuffs before the first stage's scalars (src/scalars.f90:217),
  // and the clearing of the scalars a restarting puff asks for
  void launch_puff_prep() {
    bool puffs = false, clear = false;
    for (int d = 0; d < nd; d++) {
      puffs |= hdom[d].npuff > 0;
      clear |= hdom[d].puff_clear_any != 0;
    }
    if (!puffs) return;
    nlaunch++;
    k_puff_step<T><<<(nd + 127) / 128, 128, 0, stream>>>(ddom, nd);
    if (clear) {
      nlaunch++;
      k_puff_clear<T><<<148 * 4, 256, 0, stream>>>(ddom, nd);
    }
  }
  int enqueue_step(bool cfl, bool div) {
    if (cfl) launch_cfl();
    bool vdt = false;
    for (int d = 0; d < nd; d++) vdt |= hdom[d].vdt != 0;
    if (vdt) {  // the variable steps' length, before any kernel reads dt
      nlaunch++;
      k_dt<T><<<(nd + 127) / 128, 128, 0, stream>>>(ddom, nd);
    }
    launch_puff_prep();
    for (int s = 1; s <= 3; s++) run_stage(s, 3, s == 3, false, div && s == 3);
    if (div && !any_solids()) launch_divmax();
    return ELMM_OK;
  }
  // the first TMarchRK3 call after the bodies were set: IBMomentum on the
  // state, the ghosts left as they are (src/tsteps.f90:44-48)
  void prime_solids() {
    for (int d = 0; d < nd && d < (int)sol.size(); d++) {
      SolidSet &x = sol[d];
      if (!x.on || x.primed) continue;
      if (x.nib > 0)
        k_ib_gather<T><<<std::min((x.nib + 255) / 256, 148 * 8), 256, 0, stream>>>(ddom, d, x.vel, x.nib, 0);
      x.primed = true;
    }
  }

  int step(int nsteps, elmm_stats *st) {
    int r = step_launch(nsteps);
    if (r) return r;
    return step_finish(nsteps, st);
  }

  // the launch map of one kind after a change of tile shape
  int rebuild_ls(int kind) {
    std::vector<int> st(nd + 1, 0);
    for (int d = 0; d < nd; d++) st[d + 1] = st[d] + tiles(kind, hdom[d]);
    CU(cudaMemcpy(ls[kind].starts, st.data(), sizeof(int) * (nd + 1), cudaMemcpyHostToDevice));
    ls[kind].total = st[nd];
    return ELMM_OK;
  }

  // The autotuner: before the first step of a batch (or view), times each
  // candidate shape on the batch's own domains (a warm-up and ten launches
  // each, three for the views of a serving loop, which are rebuilt often;
  // CUDA events) and keeps the fastest: the spectral columns of a tile of
  // the z solve (16, 32), the rows of a tile of the FP32 scalar stage (8, 4),
  // and the z chunk of the momentum and SGS kernels (8, 16, 32 planes).  A
  // view may be built between the steps of a running request, so the
  // launches it times only write what the next step rewrites before reading
  // it: the spectral buffer, the new value and tendency of a scalar stage,
  // the momentum tendency (a function of the state alone) and U2, and the
  // viscosity and live diffusivity of the SGS kernel's timing mode (which
  // leaves the wall-model points, and the u* a smooth wall carries from
  // stage to stage, alone).  No shape
  // changes any result: every cell's arithmetic is the same for every
  // partition.
  int autotune() {
    tuned = true;
    cudaEvent_t a, b;
    CU(cudaEventCreate(&a));
    CU(cudaEventCreate(&b));
    const int reps = is_view ? 3 : 10;
    auto time10 = [&](auto launch) -> float {
      launch();  // warm
      cudaEventRecord(a, stream);
      for (int r = 0; r < reps; r++) launch();
      cudaEventRecord(b, stream);
      cudaEventSynchronize(b);
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      return ms;
    };
    int r = ELMM_OK;
    if (ls[LK_TRIT].total > 0) {
      for (int v = 0; v < 2 && !r; v++) {
        tune_cols = v ? 32 : 16;
        if ((r = rebuild_ls(LK_TRIT))) break;
        tune_ms[2 + v] = time10([&] { launch_tri(0); });
      }
      tune_cols = tune_ms[3] < tune_ms[2] ? 32 : 16;
      if (!r) r = rebuild_ls(LK_TRIT);
    }
    if (!r && ls[LK_TPAIR].total > 0) {
      for (int v = 0; v < 2 && !r; v++) {
        tune_rows = v ? 4 : 8;
        if ((r = rebuild_ls(LK_TPAIR))) break;
        tune_ms[v] = time10([&] { launch_scalar_pair(1); });
      }
      tune_rows = tune_ms[1] < tune_ms[0] ? 4 : 8;
      if (!r) r = rebuild_ls(LK_TPAIR);
    }
    // the z chunks of the momentum kernel (timed as a second stage, which
    // also reads the old tendency) and of the SGS kernel (its stage mode)
    const StageCoef sc1{kRho[1], kBeta[1], 2 * kAlpha[1], 2};
    int best_m = 1, best_s = 1;
    for (int q = 0; q < 3 && !r; q++) {
      tune_mom_kc = kChunks[q];
      if ((r = rebuild_ls(LK_MOMT))) break;
      tune_ms[4 + q] = time10([&] { momentum_kernel(sc1); });
      if (tune_ms[4 + q] < tune_ms[4 + best_m]) best_m = q;
    }
    for (int q = 0; q < 3 && !r; q++) {
      tune_sgs_kc = kChunks[q];
      if ((r = rebuild_ls(LK_SGST))) break;
      tune_ms[7 + q] = time10([&] { sgs_kernel(2); });
      if (tune_ms[7 + q] < tune_ms[7 + best_s]) best_s = q;
    }
    tune_mom_kc = kChunks[best_m];
    tune_sgs_kc = kChunks[best_s];
    if (!r) r = rebuild_ls(LK_MOMT);
    if (!r) r = rebuild_ls(LK_SGST);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (r) return r;
    CU(cudaGetLastError());
    return ELMM_OK;
  }
  // the shapes set by the caller instead of the autotuner (elmm_batch_set_tuning):
  // out-of-set values are refused; nothing is timed
  int set_tuning(const int32_t *v, int n) {
    auto in = [](int x, std::initializer_list<int> set) {
      for (int y : set) if (x == y) return true;
      return false;
    };
    if (n > 0 && !in(v[0], {4, 8})) return fail(ELMM_ERR_INVALID_ARG, "scalar tile rows: 4 or 8");
    if (n > 1 && !in(v[1], {16, 32})) return fail(ELMM_ERR_INVALID_ARG, "z-solve tile columns: 16 or 32");
    if (n > 2 && !in(v[2], {8, 16, 32})) return fail(ELMM_ERR_INVALID_ARG, "momentum z chunk: 8, 16 or 32");
    if (n > 3 && !in(v[3], {8, 16, 32})) return fail(ELMM_ERR_INVALID_ARG, "SGS z chunk: 8, 16 or 32");
    CU(cudaSetDevice(device));
    CU(cudaStreamSynchronize(stream));
    if (n > 0) tune_rows = v[0];
    if (n > 1) tune_cols = v[1];
    if (n > 2) tune_mom_kc = v[2];
    if (n > 3) tune_sgs_kc = v[3];
    for (int kind : {LK_TPAIR, LK_TRIT, LK_MOMT, LK_SGST}) {
      int r = rebuild_ls(kind);
      if (r) return r;
    }
    if (step_exec) {  // the step graph holds the old launch shapes
      cudaGraphExecDestroy(step_exec);
      step_exec = nullptr;
    }
    tuned = true;
    return ELMM_OK;
  }

  // ------------------------------------------------------------ puffs
  // elmm_set_puffs: windows and volumes into the descriptor, the state (last
  // release -huge, as PuffSource%last_start starts) and the clock on the device
  // cvol, ncv: the volumes whose puffs' clear flags pick the scalars a
  // restart clears (a slab of a split domain: the whole domain's volumes,
  // its own ones elsewhere); the volumes' own list by default
  int set_puffs(int d, const elmm_puff *pf, int np, const elmm_puff_volume *vol, int nv,
                const elmm_puff_volume *cvol = nullptr, int ncv = 0) {
    CU(cudaSetDevice(device));
    CU(cudaStreamSynchronize(stream));
    Dom<T> &h = hdom[d];
    const elmm_config &c = cfg[d];
    if (np < 0 || np > kMaxPuffs || nv < 0 || nv > kMaxPuffVols || (np > 0 && !pf) || (nv > 0 && !vol))
      return fail(ELMM_ERR_INVALID_ARG, "puffs: at most ELMM_MAX_PUFFS puffs and ELMM_MAX_PUFF_VOLUMES volumes");
    for (int q = 0; q < np; q++)
      if (!std::isfinite(pf[q].start_time) || !std::isfinite(pf[q].end_time) || !std::isfinite(pf[q].period) ||
          !std::isfinite(pf[q].duration))
        return fail(ELMM_ERR_INVALID_ARG, "puffs: non-finite window");
    for (int q = 0; q < nv; q++) {
      const elmm_puff_volume &v = vol[q];
      if (v.puff < 0 || v.puff >= np || v.scalar_number < 1 || v.scalar_number > c.num_scalars || v.xi < 1 ||
          v.xi > h.nx || v.yj < 1 || v.yj > h.ny || v.zk < 1 || v.zk > h.nz || !std::isfinite(v.flux))
        return fail(ELMM_ERR_INVALID_ARG, "puff volume: puff index, scalar or cell out of range");
    }
    if (step_exec) { cudaGraphExecDestroy(step_exec); step_exec = nullptr; }
    if (!h.puff_state) {
      double *st;
      int r = dalloc((void **)&st, (4 * kMaxPuffs + 1) * sizeof(double));
      if (r) return r;
      h.puff_state = st;
    }
    std::vector<double> st(4 * kMaxPuffs + 1, 0.0);
    h.npuff = np;
    h.puff_clear_any = 0;
    for (int q = 0; q < np; q++) {
      st[4 * q] = -std::numeric_limits<double>::max();
      h.puff_start[q] = pf[q].start_time;
      h.puff_end[q] = pf[q].end_time;
      h.puff_period[q] = pf[q].period;
      h.puff_dur[q] = pf[q].duration;
      h.puff_clear_slots[q] = 0;
    }
    st[4 * kMaxPuffs] = time;
    h.npv = nv;
    for (int q = 0; q < nv; q++) {
      const int slot = (h.buoy ? 1 : 0) + vol[q].scalar_number - 1;
      h.pv_puff[q] = vol[q].puff;
      h.pv_slot[q] = slot;
      h.pv_i[q] = vol[q].xi;
      h.pv_j[q] = vol[q].yj;
      h.pv_k[q] = vol[q].zk;
      h.pv_q[q] = vol[q].flux;
    }
    if (!cvol) {
      cvol = vol;
      ncv = nv;
    }
    for (int q = 0; q < ncv; q++) {
      const elmm_puff_volume &v = cvol[q];
      if (v.puff < 0 || v.puff >= np || v.scalar_number < 1 || v.scalar_number > c.num_scalars)
        return fail(ELMM_ERR_INVALID_ARG, "puff volume: puff index or scalar out of range");
      if (pf[v.puff].clear) {
        h.puff_clear_slots[v.puff] |= 1u << ((h.buoy ? 1 : 0) + v.scalar_number - 1);
        h.puff_clear_any = 1;
      }
    }
    CU(cudaMemcpy(h.puff_state, st.data(), st.size() * sizeof(double), cudaMemcpyHostToDevice));
    return push_dom(d);
  }

  // ------------------------------------------------------------ solids
  void drop_solids(int d) {
    if (d >= (int)sol.size()) return;
    SolidSet &x = sol[d];
    for (void *p : {(void *)x.vel, (void *)x.visc, (void *)x.wm, (void *)x.wm_ustar, (void *)x.bskip[0],
                    (void *)x.bskip[1], (void *)x.bskip[2], (void *)x.null, (void *)x.pmask, (void *)x.fill, (void *)x.heat})
      if (p) dfree(p);
    x = SolidSet();
    for (int c = 0; c < 3; c++) hdom[d].bskip[c] = nullptr;
    hdom[d].pmask = nullptr;
  }
  // elmm_set_solids: checks the lists, turns (i, j, k) into box indices with
  // the ghost folds applied, uploads them and marks the step graph stale.
  // On any error the domain is left without bodies.
  int set_solids(int d, const elmm_solids *s) {
    CU(cudaSetDevice(device));
    CU(cudaStreamSynchronize(stream));
    if ((int)sol.size() < nd) sol.resize(nd);
    drop_solids(d);
    if (step_exec) { cudaGraphExecDestroy(step_exec); step_exec = nullptr; }
    int r = push_dom(d);
    if (r || !s) return r;
    r = install_solids(d, s);
    if (r) {
      drop_solids(d);
      push_dom(d);
      return r;
    }
    // the immersed-boundary kernels work on full velocities: the mixed
    // path's stored deviations become full values and its offsets zero
    if (sizeof(T) == 4 && hdom[d].voff) {
      k_drop_offsets<T><<<148 * 4, 256, 0, stream>>>(ddom + d);
      CU(cudaMemsetAsync(hdom[d].voff, 0, sizeof(float) * 2 * (hdom[d].nz + 2), stream));
      CU(cudaStreamSynchronize(stream));
      CU(cudaGetLastError());
    }
    return ELMM_OK;
  }
  // The cells of the temperature's fill of the solid cells (k_theta_fill)
  // from the solid Pr cells of s: the interior solid cells with a fluid
  // 6-neighbour in range -1..n+2, each with its fluid neighbours' cells, a
  // ghost cell through the rules of BoundTemperature for adiabatic sides
  // (x, y periodic; z mirrored at a wall-model wall, the first level
  // otherwise).  A body whose fill reads the ghost cell of a side with a
  // heat flux or a prescribed value and no wall-model points is refused.
  int build_fill(int d, const elmm_solids *s) {
    Dom<T> &h = hdom[d];
    const elmm_config &cf = cfg[d];
    SolidSet &x = sol[d];
    const int nx = h.nx, ny = h.ny, nz = h.nz, ex = nx + 4, ey = ny + 4, ez = nz + 4;
    auto at = [&](int i, int j, int k) { return (size_t)(i + 1) + (size_t)ex * ((size_t)(j + 1) + (size_t)ey * (k + 1)); };
    std::vector<char> solid((size_t)ex * ey * ez, 0);
    for (int64_t q = 0; q < s->n_solid_pr; q++) {
      const int32_t *t = s->solid_pr_ijk + 3 * q;
      for (int oi : {-nx, 0, nx})
        for (int oj : {-ny, 0, ny}) {
          const int i = t[0] + oi, j = t[1] + oj;
          if (i >= -1 && i <= nx + 2 && j >= -1 && j <= ny + 2) solid[at(i, j, t[2])] = 1;
        }
    }
    const bool mlo = h.wall[SIDE_BO] != 0, mhi = h.wall[SIDE_TO] != 0;
    auto fold = [&](int i, int j, int k, int o[3]) {
      o[0] = i < 1 ? i + nx : i > nx ? i - nx : i;
      o[1] = j < 1 ? j + ny : j > ny ? j - ny : j;
      o[2] = k < 1 ? (mlo ? 1 - k : 1) : k > nz ? (mhi ? 2 * nz + 1 - k : nz) : k;
    };
    static const int nb[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    std::vector<FillCell> fc;
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          if (!solid[at(i, j, k)]) continue;
          FillCell c{};
          c.box = bidx(h, i, j, k);
          for (auto &o : nb) {
            const int a = i + o[0], b = j + o[1], e = k + o[2];
            if (solid[at(a, b, e)]) continue;
            const int zs = e < 1 ? ELMM_BO : e > nz ? ELMM_TO : -1;
            if (zs >= 0 && !h.wall[zs] && (cf.TempBtype[zs] != ELMM_BC_CONSTFLUX || cf.sideTemp[zs] != 0))
              return fail(ELMM_ERR_INVALID_ARG,
                          "a body next to a side with a heat flux or a prescribed temperature and no wall-model points");
            int g[3];
            fold(a, b, e, g);
            if (solid[at(g[0], g[1], g[2])])
              return fail(ELMM_ERR_INVALID_ARG, "a fluid ghost cell next to a body copies a solid cell");
            c.ref[c.n++] = bidx(h, g[0], g[1], g[2]);
          }
          if (c.n > 0) fc.push_back(c);
        }
    if (fc.empty()) return ELMM_OK;
    int rr = dalloc((void **)&x.fill, fc.size() * sizeof(FillCell));
    if (rr) return rr;
    CU(cudaMemcpy(x.fill, fc.data(), fc.size() * sizeof(FillCell), cudaMemcpyHostToDevice));
    x.nfill = (int)fc.size();
    return ELMM_OK;
  }
  int install_solids(int d, const elmm_solids *s) {
    Dom<T> &h = hdom[d];
    const elmm_config &c = cfg[d];
    if (!h.wall[SIDE_BO] || h.bt[SIDE_BO] != BC_NOSLIP)
      return fail(ELMM_ERR_INVALID_ARG, "solid bodies need the wall model on a no-slip bottom");
    const bool per[3] = {h.bt[SIDE_WE] == BC_PERIODIC, h.bt[SIDE_SO] == BC_PERIODIC, h.bt[SIDE_BO] == BC_PERIODIC};
    // extents: 0..2 velocity components, 3 the pressure grid (viscosity)
    auto ext = [&](int comp, int a) { return comp < 3 ? h.ext[comp][a] : (a == 0 ? h.nx : a == 1 ? h.ny : h.nz); };
    auto in_target = [&](int comp, int i, int j, int k) {
      const int v[3] = {i, j, k};
      for (int a = 0; a < 3; a++) {
        const int lo = per[a] ? 2 : 1, hi = per[a] ? ext(comp, a) - 1 : ext(comp, a);
        if (v[a] < lo || v[a] > hi) return false;
      }
      return true;
    };
    // a source one cell into the ghosts -> the interior cell its ghost copies
    auto fold = [&](int comp, int i, int j, int k, long long &idx, double &sign) {
      const int v[3] = {i, j, k};
      int o[3];
      sign = 1;
      for (int a = 0; a < 3; a++) {
        const int n = ext(comp, a);
        if (v[a] < 0 || v[a] > n + 1) return false;
        if (comp < 3) {
          Fold f = fold_vel(v[a], n, h.bt[2 * a], h.bt[2 * a + 1], a == comp);
          o[a] = f.src;
          if (f.zero) sign = 0;
          else sign *= f.sign;
        } else {
          o[a] = fold_rep(v[a], n, per[a]);
        }
      }
      idx = bidx(h, o[0], o[1], o[2]);
      return true;
    };
    std::vector<IBGather> vel, visc;
    std::vector<long long> targets[4];
    auto add_points = [&](int comp, const elmm_ib_point *pts, int64_t n, std::vector<IBGather> &out) {
      for (int64_t q = 0; q < n; q++) {
        const elmm_ib_point &p = pts[q];
        if (!in_target(comp, p.xi, p.yj, p.zk) || p.interp < 0 || p.interp > ELMM_IB_MAX_INTERP) return false;
        IBGather g{};
        g.tgt = bidx(h, p.xi, p.yj, p.zk);
        g.comp = comp;
        g.n = p.interp;
        for (int m = 0; m < p.interp; m++) {
          double sg;
          if (!fold(comp, p.ii[m], p.jj[m], p.kk[m], g.src[m], sg) || !std::isfinite(p.coef[m])) return false;
          g.coef[m] = p.coef[m] * sg;
        }
        targets[comp].push_back(g.tgt);
        out.push_back(g);
      }
      return true;
    };
    for (int comp = 0; comp < 3; comp++)
      if (s->n_ib[comp] < 0 || (s->n_ib[comp] > 0 && !s->ib[comp]) ||
          !add_points(comp, s->ib[comp], s->n_ib[comp], vel))
        return fail(ELMM_ERR_INVALID_ARG, "IB point out of range (or within one cell of a periodic boundary)");
    const int nib = (int)vel.size();
    std::vector<long long> nulls;
    int ncomp_null[3] = {0, 0, 0};
    for (int comp = 0; comp < 3; comp++) {
      if (s->n_null[comp] < 0 || (s->n_null[comp] > 0 && !s->null_ijk[comp]))
        return fail(ELMM_ERR_INVALID_ARG, "nullified points");
      for (int64_t q = 0; q < s->n_null[comp]; q++) {
        const int32_t *t = s->null_ijk[comp] + 3 * q;
        if (!in_target(comp, t[0], t[1], t[2]))
          return fail(ELMM_ERR_INVALID_ARG, "nullified point out of range (or within one cell of a periodic boundary)");
        const long long idx = bidx(h, t[0], t[1], t[2]);
        targets[comp].push_back(idx);
        nulls.push_back(idx);
        ncomp_null[comp]++;
      }
    }
    if (s->n_scalfl < 0 || (s->n_scalfl > 0 && !s->scalfl) || !add_points(3, s->scalfl, s->n_scalfl, visc))
      return fail(ELMM_ERR_INVALID_ARG, "ScalFl point out of range (or within one cell of a periodic boundary)");
    // one parallel pass is exact only if no point reads a value the pass writes
    for (int comp = 0; comp < 4; comp++) std::sort(targets[comp].begin(), targets[comp].end());
    auto is_target = [&](int comp, long long i) {
      return std::binary_search(targets[comp].begin(), targets[comp].end(), i);
    };
    for (auto *list : {&vel, &visc})
      for (auto &g : *list)
        for (int m = 0; m < g.n; m++)
          if (g.coef[m] != 0 && is_target(g.comp, g.src[m]))
            return fail(ELMM_ERR_INVALID_ARG, "an interpolation point is itself a forcing or nullified point");
    std::vector<WMSolid> wm;
    if (s->n_wm < 0 || (s->n_wm > 0 && !s->wm)) return fail(ELMM_ERR_INVALID_ARG, "wall-model points");
    for (int64_t q = 0; q < s->n_wm; q++) {
      const elmm_wm_point &p = s->wm[q];
      const int comp = p.component - 1;
      if (comp < 0 || comp > 2 || p.direction < 1 || p.direction > 6 || !(p.z0 > 0 || (p.z0 == 0 && h.nu_mol > 0)) ||
          p.xi < 1 || p.xi > h.ext[comp][0] || p.yj < 1 || p.yj > h.ext[comp][1] || p.zk < 1 || p.zk > h.ext[comp][2])
        return fail(ELMM_ERR_INVALID_ARG,
                    "solid-face wall-model point out of range (or smooth, z0 = 0, without molecular viscosity)");
      WMSolid w{};
      w.c = bidx(h, p.xi, p.yj, p.zk);
      w.comp = comp;
      w.dir = p.direction;
      w.k = p.zk;
      for (int a = 0; a < 3; a++) w.dist[a] = p.dist[a];
      w.z0 = p.z0;
      w.tflux = p.temperature_flux;
      if (!std::isfinite(w.tflux) || (w.tflux != 0 && !c.enable_buoyancy))
        return fail(ELMM_ERR_INVALID_ARG, "a solid face's heat flux needs the temperature field");
      if (!(norm_host(w.dist) > 0)) return fail(ELMM_ERR_INVALID_ARG, "wall-model point on the wall");
      wm.push_back(w);
    }
    SolidSet &x = sol[d];
    int r;
    auto up = [&](void **dst, const void *src, size_t bytes) {
      if (bytes == 0) return (int)ELMM_OK;
      int rr = dalloc(dst, bytes);
      if (rr) return rr;
      return cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess ? (int)ELMM_OK
                                                                                 : fail(ELMM_ERR_CUDA, "cudaMemcpy");
    };
    if ((r = up((void **)&x.vel, vel.data(), vel.size() * sizeof(IBGather)))) return r;
    if ((r = up((void **)&x.null, nulls.data(), nulls.size() * sizeof(long long)))) return r;
    for (int comp = 0; comp < 3; comp++) x.nnull.n[comp] = ncomp_null[comp];
    if ((r = up((void **)&x.visc, visc.data(), visc.size() * sizeof(IBGather)))) return r;
    if ((r = up((void **)&x.wm, wm.data(), wm.size() * sizeof(WMSolid)))) return r;
    std::vector<double> us(wm.size(), 1.0);  // WMPointUVW%ustar starts at 1 (immersedboundary.f90:235)
    if ((r = up((void **)&x.wm_ustar, us.data(), us.size() * sizeof(double)))) return r;
    x.nvel = (int)vel.size();
    x.nib = nib;
    x.nvisc = (int)visc.size();
    x.nwm = (int)wm.size();
    for (int comp = 0; comp < 3; comp++) {
      const int e0 = h.ext[comp][0], e1 = h.ext[comp][1];
      std::vector<unsigned char> m((size_t)e0 * e1, 0);
      if (s->n_bottom_skip[comp] < 0 || (s->n_bottom_skip[comp] > 0 && !s->bottom_skip_ij[comp]))
        return fail(ELMM_ERR_INVALID_ARG, "bottom skip list");
      for (int64_t q = 0; q < s->n_bottom_skip[comp]; q++) {
        const int32_t *t = s->bottom_skip_ij[comp] + 2 * q;
        if (t[0] < 1 || t[0] > e0 || t[1] < 1 || t[1] > e1) return fail(ELMM_ERR_INVALID_ARG, "bottom skip point");
        m[(size_t)(t[0] - 1) + (size_t)e0 * (t[1] - 1)] = 1;
      }
      if (s->n_bottom_skip[comp] > 0) {
        if ((r = up((void **)&x.bskip[comp], m.data(), m.size()))) return r;
        h.bskip[comp] = x.bskip[comp];
      }
    }
    if (c.num_scalars > 0 || c.enable_buoyancy) {
      // the scalars' cell mask: bit 0 the solid Pr cells with their periodic
      // x and y images in the ghost columns (and the z ghost planes), bit 1
      // the Pr wall-model points of the scalar equations
      if (s->n_solid_pr < 0 || (s->n_solid_pr > 0 && !s->solid_pr_ijk) || s->n_wm_pr < 0 ||
          (s->n_wm_pr > 0 && !s->wm_pr_ijk))
        return fail(ELMM_ERR_INVALID_ARG, "solid Pr cells or Pr wall-model points");
      std::vector<unsigned char> m((size_t)h.plane * (h.nz + 2), 0);
      auto in = [&](const int32_t *t) {
        return t[0] >= 1 && t[0] <= h.nx && t[1] >= 1 && t[1] <= h.ny && t[2] >= 1 && t[2] <= h.nz;
      };
      for (int64_t q = 0; q < s->n_solid_pr; q++) {
        const int32_t *t = s->solid_pr_ijk + 3 * q;
        if (t[0] < 1 || t[0] > h.nx || t[1] < 1 || t[1] > h.ny || t[2] < -1 || t[2] > h.nz + 2)
          return fail(ELMM_ERR_INVALID_ARG, "solid Pr cell out of range");
        if (t[2] < 0 || t[2] > h.nz + 1) continue;
        for (int oi : {-h.nx, 0, h.nx})
          for (int oj : {-h.ny, 0, h.ny}) {
            const int i = t[0] + oi, j = t[1] + oj;
            if (i >= 0 && i <= h.nx + 1 && j >= 0 && j <= h.ny + 1) m[bidx(h, i, j, t[2])] |= 1;
          }
      }
      for (int64_t q = 0; q < s->n_wm_pr; q++) {
        const int32_t *t = s->wm_pr_ijk + 3 * q;
        if (!in(t)) return fail(ELMM_ERR_INVALID_ARG, "Pr wall-model point out of range");
        m[bidx(h, t[0], t[1], t[2])] |= 2;
      }
      // bit 2: the wall points the deduplication keeps (they carry the wall's flux)
      if (s->n_wall_pr < 0 || (s->n_wall_pr > 0 && !s->wall_pr_ijk))
        return fail(ELMM_ERR_INVALID_ARG, "wall points");
      for (int64_t q = 0; q < s->n_wall_pr; q++) {
        const int32_t *t = s->wall_pr_ijk + 3 * q;
        if (!in(t) || (t[2] != 1 && t[2] != h.nz)) return fail(ELMM_ERR_INVALID_ARG, "wall point out of range");
        m[bidx(h, t[0], t[1], t[2])] |= 4;
      }
      if ((r = up((void **)&x.pmask, m.data(), m.size()))) return r;
      h.pmask = x.pmask;
    }
    if (c.enable_buoyancy && (r = build_fill(d, s))) return r;
    if (s->n_heat_pr < 0 || (s->n_heat_pr > 0 && (!s->heat_pr_ijk || !s->heat_pr_q)) ||
        (s->n_heat_pr > 0 && !c.enable_buoyancy))
      return fail(ELMM_ERR_INVALID_ARG, "heated Pr wall-model points (they need the temperature field)");
    if (s->n_heat_pr > 0) {
      std::vector<HeatPoint> hp;
      for (int64_t q = 0; q < s->n_heat_pr; q++) {
        const int32_t *t = s->heat_pr_ijk + 3 * q;
        if (t[0] < 1 || t[0] > h.nx || t[1] < 1 || t[1] > h.ny || t[2] < 1 || t[2] > h.nz ||
            !std::isfinite(s->heat_pr_q[q]))
          return fail(ELMM_ERR_INVALID_ARG, "heated Pr wall-model point out of range");
        hp.push_back(HeatPoint{bidx(h, t[0], t[1], t[2]), s->heat_pr_q[q]});
      }
      if ((r = up((void **)&x.heat, hp.data(), hp.size() * sizeof(HeatPoint)))) return r;
      x.nheat = (int)hp.size();
    }
    x.on = true;
    x.primed = false;
    return push_dom(d);
  }
  static double norm_host(const double *v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
  // elmm_set_fault_injection: the wait limit and the skipped plane of every
  // domain (read by the kernels from the device descriptors, so the captured
  // step graph stays valid)
  int set_fault_injection(int wait_limit, int skip_plane) {
    CU(cudaSetDevice(device));
    CU(cudaStreamSynchronize(stream));
    for (int d = 0; d < nd; d++) {
      hdom[d].wait_limit = wait_limit;
      hdom[d].skip_plane = skip_plane;
      int r = push_dom(d);
      if (r) return r;
    }
    return ELMM_OK;
  }
  int push_dom(int d) {
    CU(cudaMemcpy(ddom + d, &hdom[d], sizeof(Dom<T>), cudaMemcpyHostToDevice));
    return ELMM_OK;
  }

  // enqueues nsteps replays of the step graph (captured on first use) without
  // waiting for them
  int step_launch(int nsteps) {
    CU(cudaSetDevice(device));
    if (!tuned) {
      int r = autotune();
      if (r) return r;
    }
    if (frame_pending) CU(cudaStreamWaitEvent(stream, ev_packed, 0));
    bool cfl = false;
    for (auto &c : cfg) cfl |= c.enable_CFL_check != 0 || c.variable_time_steps != 0;
    if (!step_exec || step_has_cfl != cfl) {
      if (step_exec) { cudaGraphExecDestroy(step_exec); step_exec = nullptr; }
      cudaGraph_t g;
      CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      nlaunch = 0;
      enqueue_step(cfl, true);
      step_kernels = nlaunch;
      CU(cudaStreamEndCapture(stream, &g));
      cudaError_t e = cudaGraphInstantiate(&step_exec, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return fail(ELMM_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      step_has_cfl = cfl;
    }
    for (int d = 0; d < nd; d++) CU(cudaMemsetAsync(hdom[d].refine_count, 0, sizeof(int), stream));
    if (nsteps > 0) prime_solids();
    CU(cudaEventRecord(t0, stream));
    for (int s = 0; s < nsteps; s++) CU(cudaGraphLaunch(step_exec, stream));
    CU(cudaEventRecord(t1, stream));
    return ELMM_OK;
  }

  // waits for the steps of step_launch and reports them
  int step_finish(int nsteps, elmm_stats *st) {
    CU(cudaStreamSynchronize(stream));
    CU(cudaGetLastError());
    if (hdom[0].vdt) {  // the device clock of variable steps
      double ts[2];
      CU(cudaMemcpy(ts, hdom[0].tstate, sizeof(ts), cudaMemcpyDeviceToHost));
      time = ts[0];
    } else {
      time += nsteps * cfg[0].dt;
    }
    int r = fill_stats(st, nsteps);
    if (st) {
      st->kernels = nsteps * step_kernels;
      int tot = 0;
      for (int d = 0; d < nd; d++) {
        int c0 = 0;
        CU(cudaMemcpy(&c0, hdom[d].refine_count, sizeof(int), cudaMemcpyDeviceToHost));
        tot = std::max(tot, c0);
      }
      st->refine_sweeps = tot;
    }
    return r;
  }

  int fill_stats(elmm_stats *st, int nsteps) {
    double md = 0, cf = 0, dt0 = cfg[0].dt;
    int gave_up = 0, past_end = 0;
    for (int d = 0; d < nd; d++) {
      int fl[3] = {0, 0, 0};
      CU(cudaMemcpy(fl, hdom[d].flags, sizeof(fl), cudaMemcpyDeviceToHost));
      if (fl[1]) {  // a bounded device-side wait gave up: report it once
        gave_up = 1;
        CU(cudaMemset(hdom[d].flags + 1, 0, sizeof(int)));
      }
      if (fl[2]) {  // a variable step started at end_time
        past_end = 1;
        CU(cudaMemset(hdom[d].flags + 2, 0, sizeof(int)));
      }
      unsigned long long b1 = 0, b2 = 0;
      CU(cudaMemcpy(&b1, hdom[d].maxdiv_bits, sizeof(b1), cudaMemcpyDeviceToHost));
      CU(cudaMemcpy(&b2, hdom[d].cfl_bits, sizeof(b2), cudaMemcpyDeviceToHost));
      double a, c2;
      memcpy(&a, &b1, 8);
      memcpy(&c2, &b2, 8);
      if (!(a <= md)) md = a;
      double dtd = cfg[d].dt;
      if (hdom[d].vdt) {  // the length of the last variable step
        double ts[2];
        CU(cudaMemcpy(ts, hdom[d].tstate, sizeof(ts), cudaMemcpyDeviceToHost));
        dtd = ts[1];
        if (d == 0) dt0 = dtd;
      }
      c2 = c2 * dtd;
      if (!(c2 <= cf)) cf = c2;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    if (st) {
      memset(st, 0, sizeof(*st));
      st->steps_done = nsteps;
      st->time = time;
      st->dt = dt0;
      st->cfl = cf;
      st->max_div = md;
      st->nan_detected = !std::isfinite(md) || !std::isfinite(cf);
      st->elapsed_ms = ms;
    }
    if (gave_up) return fail(ELMM_ERR_TIMEOUT, "a device-side wait for a plane copy gave up; the step is incomplete");
    if (past_end)
      return fail(ELMM_ERR_INVALID_ARG, "a variable time step started at end_time (the run was over; it took the "
                                        "step length of its CFL limit)");
    if (!std::isfinite(md) || !std::isfinite(cf)) return fail(ELMM_ERR_NAN, "NaN or Inf in the velocity field");
    return ELMM_OK;
  }

  int project(double coef, elmm_stats *st) {
    CU(cudaSetDevice(device));
    if (frame_pending) CU(cudaStreamWaitEvent(stream, ev_packed, 0));
    CU(cudaEventRecord(t0, stream));
    // the fused divergence of k_fftx_fwd reads U2: make U2 the current field
    for (int d = 0; d < nd; d++) {
      size_t box = (size_t)hdom[d].plane * (hdom[d].nz + 2) * sizeof(T);
      CU(cudaMemcpyAsync(hdom[d].U2, hdom[d].U, box, cudaMemcpyDeviceToDevice, stream));
      CU(cudaMemcpyAsync(hdom[d].V2, hdom[d].V, box, cudaMemcpyDeviceToDevice, stream));
      CU(cudaMemcpyAsync(hdom[d].W2, hdom[d].W, box, cudaMemcpyDeviceToDevice, stream));
    }
    launch_projection(coef, 0, 0);
    launch_refine(coef, 0);
    launch_divmax();
    // the end of InitialConditions (src/initial.f90:4291-4336): eddy
    // viscosity of the projected field and, with scalars, their diffusivity,
    // and the wall model once on the initial fields (the u* and fluxes its
    // points carry into the first stage; the solid-face points' u* alone)
    sgs_kernel(1);
    wm_kernel(1, stream);
    for (int d = 0; d < nd && d < (int)sol.size(); d++)
      if (sol[d].on && sol[d].nwm > 0)
        k_ib_wm<T><<<std::min((sol[d].nwm + 127) / 128, 148 * 8), 128, 0, stream>>>(ddom, d, sol[d].wm,
                                                                                   sol[d].wm_ustar, sol[d].nwm, 0.0, 1);
    launch_ghosts({F_NU}, 0);
    CU(cudaEventRecord(t1, stream));
    CU(cudaStreamSynchronize(stream));
    CU(cudaGetLastError());
    return fill_stats(st, 0);
  }

  // per-kernel timing of one stage (CUDA events on the launching stream);
  // the ghost-shell launches of the stage are summed into the last slot
  int profile_stage(int stage, int reps, double *ms) {
    CU(cudaSetDevice(device));
    const int nk = ELMM_NKERNELS;
    const int kGhost = 9, nev = 2 * (nk + 3);
    std::vector<cudaEvent_t> ev(nev);
    for (auto &e : ev) CU(cudaEventCreate(&e));
    std::vector<double> acc(nk, 0.0);
    std::vector<int> slot;
    const double a2 = 2 * kAlpha[stage - 1];
    StageCoef sc{kRho[stage - 1], kBeta[stage - 1], a2, stage};
    for (int r = 0; r < reps; r++) {
      slot.clear();
      auto timed = [&](int k, auto launch) {
        cudaEventRecord(ev[2 * slot.size()], stream);
        launch();
        cudaEventRecord(ev[2 * slot.size() + 1], stream);
        slot.push_back(k);
      };
      timed(0, [&] {
        sgs_kernel(0);
        wm_kernel(stage, stream);
      });
      timed(kGhost, [&] { launch_ghosts({F_NU}, 0); });
      timed(1, [&] {
        momentum_kernel(sc);
      });
      timed(2, [&] { launch_fftx_fwd(a2, 1, 0, 0); });
      timed(3, [&] { launch_ffty(0, 0); });
      timed(4, [&] { launch_tri(0); });
      timed(5, [&] { launch_ffty(1, 0); });
      timed(6, [&] { launch_fftx_inv(0); });
      timed(7, [&] { k_project_any(a2, 1, 0, 0); });
      timed(kGhost, [&] { launch_ghosts({F_U, F_V, F_W, F_P}, 0); });
      timed(8, [&] { k_prref<T><<<std::min(nd, 1024), 256, 0, stream>>>(ddom, nd, 0); });
      timed(10, [&] { launch_scalars(stage, 0); });
      CU(cudaStreamSynchronize(stream));
      CU(cudaGetLastError());
      for (size_t q = 0; q < slot.size(); q++) {
        float t = 0;
        CU(cudaEventElapsedTime(&t, ev[2 * q], ev[2 * q + 1]));
        acc[slot[q]] += t;
      }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    for (int k = 0; k < nk; k++) ms[k] = acc[k] / reps;
    return ELMM_OK;
  }

  // --------------------------------------------------------- host copies
  HostBox hbox_vel(int d, int comp) const {
    const Dom<T> &h = hdom[d];
    return HostBox{-2, h.ext[comp][0] + 6, h.ext[comp][1] + 6, h.ext[comp][2] + 6};
  }
  HostBox hbox_p(int d) const {
    const Dom<T> &h = hdom[d];
    return HostBox{-1, h.nx + 4, h.ny + 4, h.nz + 4};
  }

  // The state and the temperature in one pipelined pass (elmm_march_host):
  // every host copy runs on the side stream into a staging buffer (Pr into
  // its own image) while the stream unpacks the field before it.  Needs the
  // two staging buffers; otherwise the field-by-field calls.
  // U..Th: host arrays of the call's type (double, or float with hostf)
  int upload_all(int d, const void *U, const void *V, const void *W, const void *Pr, const void *Th) {
    if (!two_stages() || !ev_pr || (hostf && ensure_fpipe())) {
      int r = upload(d, U, V, W, Pr);
      if (r || !Th) return r;
      return upload_temperature(d, Th);
    }
    if (!U || !V || !W) return fail(ELMM_ERR_INVALID_ARG, "NULL velocity array");
    if (Th && !hdom[d].buoy) return fail(ELMM_ERR_INVALID_ARG, "no temperature field (enable_buoyancy is 0)");
    CU(cudaSetDevice(device));
    if (frame_pending) CU(cudaStreamWaitEvent(stream, ev_packed, 0));
    const Dom<T> &h = hdom[d];
    CU(cudaMemsetAsync(dbad, 0, sizeof(int), stream));
    const void *src[4] = {U, V, W, Th};
    int b = 0;
    for (int f = 0; f < 5; f++) {
      if (f == 3) {  // Pr into its own image, no staging buffer (a float Pr through a staging buffer)
        HostBox hp = hbox_p(d);
        size_t np = (size_t)hp.n0 * hp.n1 * hp.n2;
        if (Pr && hostf) {
          double *stg;
          if (int r = h2d_pipe(b, Pr, np, &stg)) return r;
          CU(cudaMemcpyAsync(pr_image[d], stg, np * sizeof(double), cudaMemcpyDeviceToDevice, stream));
          CU(cudaEventRecord(ev_stage[b][1], stream));
          b ^= 1;
          k_unpack<T><<<kPackBlocks, 256, 0, stream>>>(ddom + d, h.P, pr_image[d], hp, h.nx, h.ny, h.nz, dbad);
        } else if (Pr) {
          CU(cudaMemcpyAsync(pr_image[d], Pr, np * sizeof(double), cudaMemcpyHostToDevice, side));
          CU(cudaEventRecord(ev_pr, side));
          CU(cudaStreamWaitEvent(stream, ev_pr, 0));
          k_unpack<T><<<kPackBlocks, 256, 0, stream>>>(ddom + d, h.P, pr_image[d], hp, h.nx, h.ny, h.nz, dbad);
        } else {
          CU(cudaMemsetAsync(pr_image[d], 0, np * sizeof(double), stream));
          CU(cudaMemsetAsync(h.P, 0, (size_t)h.plane * (h.nz + 2) * sizeof(T), stream));
        }
        continue;
      }
      const int c = f < 3 ? f : 3;
      if (c == 3 && !Th) continue;
      const size_t n = c < 3 ? (size_t)hbox_vel(d, c).n0 * hbox_vel(d, c).n1 * hbox_vel(d, c).n2
                             : (size_t)(h.nx + 6) * (h.ny + 6) * (h.nz + 6);
      double *stg;
      if (int r = h2d_pipe(b, src[c], n, &stg)) return r;
      if (c < 3) {
        HostBox hb = hbox_vel(d, c);
        const float *off = stage_offsets(d, c, stg, hb);
        k_unpack<T><<<kPackBlocks, 256, 0, stream>>>(ddom + d, c == 0 ? h.U : c == 1 ? h.V : h.W, stg, hb,
                                                     h.ext[c][0], h.ext[c][1], h.ext[c][2], dbad, off);
        k_halo_vel<T><<<256, 256, 0, stream>>>(ddom + d, c);
      } else {
        k_unpack_scalar<T><<<kPackBlocks, 256, 0, stream>>>(ddom + d, 0, stg, dbad);
      }
      CU(cudaEventRecord(ev_stage[b][1], stream));
      b ^= 1;
    }
    k_halo_p<T><<<256, 256, 0, stream>>>(ddom + d);
    CU(cudaMemsetAsync(hdom[d].prm, 0, sizeof(double), stream));
    int bad = 0;
    CU(cudaMemcpyAsync(&bad, dbad, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    CU(cudaStreamSynchronize(side));
    CU(cudaGetLastError());
    if (bad) return fail(ELMM_ERR_NAN, "non-finite value in the uploaded state");
    return ELMM_OK;
  }
  // the state and the temperature back to the host, the pack of one field
  // overlapping the host copy of the one before
  int download_all(int d, void *U, void *V, void *W, void *Pr, void *Th) {
    if (Th && !hdom[d].buoy) return fail(ELMM_ERR_INVALID_ARG, "no temperature field (enable_buoyancy is 0)");
    if (!two_stages() || (hostf && ensure_fpipe())) {
      int r = download(d, U, V, W, Pr);
      if (r || !Th) return r;
      return download_field(d, ELMM_FIELD_TEMPERATURE, Th);
    }
    CU(cudaSetDevice(device));
    void *dst[5] = {U, V, W, Pr, Th};
    const int fid[5] = {ELMM_FIELD_U, ELMM_FIELD_V, ELMM_FIELD_W, ELMM_FIELD_PR, ELMM_FIELD_TEMPERATURE};
    int b = 0;
    for (int f = 0; f < 5; f++) {
      if (!dst[f]) continue;
      double *stg = b ? dstage2 : dstage;
      CU(cudaStreamWaitEvent(stream, ev_stage[b][1], 0));
      size_t n = pack(d, fid[f], stg, stream);
      if (int r = d2h_pipe(b, dst[f], n)) return r;
      b ^= 1;
    }
    CU(cudaStreamSynchronize(side));
    CU(cudaStreamSynchronize(stream));
    CU(cudaGetLastError());
    return ELMM_OK;
  }
  // TMarchRK3 on host arrays: upload, nsteps steps, download
  int march_host(void *U, void *V, void *W, void *Pr, void *Th, int nsteps, elmm_stats *st) {
    if (nd != 1) return fail(ELMM_ERR_INVALID_ARG, "host-array steps are per single-domain handle");
    int r = upload_all(0, U, V, W, Pr, Th);
    if (r) return r;
    r = step(nsteps, st);
    if (r) return r;
    return download_all(0, U, V, W, Pr, Th);
  }

  int upload(int d, const void *U, const void *V, const void *W, const void *Pr) {
    if (d < 0 || d >= nd) return fail(ELMM_ERR_INVALID_ARG, "domain index");
    if (!U || !V || !W) return fail(ELMM_ERR_INVALID_ARG, "NULL velocity array");
    CU(cudaSetDevice(device));
    if (frame_pending) CU(cudaStreamWaitEvent(stream, ev_packed, 0));
    const Dom<T> &h = hdom[d];
    CU(cudaMemsetAsync(dbad, 0, sizeof(int), stream));
    const void *src[3] = {U, V, W};
    T *dst[3] = {h.U, h.V, h.W};
    const bool two = !hostf && two_stages();
    for (int c = 0; c < 3; c++) {
      HostBox hb = hbox_vel(d, c);
      size_t n = (size_t)hb.n0 * hb.n1 * hb.n2;
      double *stg = dstage;
      if (two) {  // copy on the side stream once the buffer's last unpack is done
        const int b = c & 1;
        stg = b ? dstage2 : dstage;
        CU(cudaStreamWaitEvent(side, ev_stage[b][1], 0));
        CU(cudaMemcpyAsync(stg, src[c], n * sizeof(double), cudaMemcpyHostToDevice, side));
        CU(cudaEventRecord(ev_stage[b][0], side));
        CU(cudaStreamWaitEvent(stream, ev_stage[b][0], 0));
      } else {
        int r = h2d(stg, src[c], n, stream);
        if (r) return r;
      }
      const float *off = stage_offsets(d, c, stg, hb);
      k_unpack<T><<<kPackBlocks, 256, 0, stream>>>(ddom + d, dst[c], stg, hb, h.ext[c][0], h.ext[c][1], h.ext[c][2], dbad,
                                                   off);
      k_halo_vel<T><<<256, 256, 0, stream>>>(ddom + d, c);
      if (two) CU(cudaEventRecord(ev_stage[c & 1][1], stream));
    }
    HostBox hp = hbox_p(d);
    size_t np = (size_t)hp.n0 * hp.n1 * hp.n2;
    if (Pr) {
      int r = h2d(pr_image[d], Pr, np, stream);
      if (r) return r;
      k_unpack<T><<<kPackBlocks, 256, 0, stream>>>(ddom + d, h.P, pr_image[d], hp, h.nx, h.ny, h.nz, dbad);
    } else {
      CU(cudaMemsetAsync(pr_image[d], 0, np * sizeof(double), stream));
      CU(cudaMemsetAsync(h.P, 0, (size_t)h.plane * (h.nz + 2) * sizeof(T), stream));
    }
    k_halo_p<T><<<256, 256, 0, stream>>>(ddom + d);
    CU(cudaMemsetAsync(h.prm, 0, sizeof(double), stream));
    int bad = 0;
    CU(cudaMemcpyAsync(&bad, dbad, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    CU(cudaGetLastError());
    if (bad) return fail(ELMM_ERR_NAN, "non-finite value in the uploaded state");
    return ELMM_OK;
  }

  int upload_temperature(int d, const void *Th) {
    if (d < 0 || d >= nd) return fail(ELMM_ERR_INVALID_ARG, "domain index");
    if (!Th) return fail(ELMM_ERR_INVALID_ARG, "NULL temperature array");
    if (!hdom[d].buoy) return fail(ELMM_ERR_INVALID_ARG, "no temperature field (enable_buoyancy is 0)");
    CU(cudaSetDevice(device));
    if (frame_pending) CU(cudaStreamWaitEvent(stream, ev_packed, 0));
    const Dom<T> &h = hdom[d];
    const size_t n = (size_t)(h.nx + 6) * (h.ny + 6) * (h.nz + 6);
    CU(cudaMemsetAsync(dbad, 0, sizeof(int), stream));
    if (int r = h2d(dstage, Th, n, stream)) return r;
    k_unpack_scalar<T><<<kPackBlocks, 256, 0, stream>>>(ddom + d, 0, dstage, dbad);
    int bad = 0;
    CU(cudaMemcpyAsync(&bad, dbad, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    CU(cudaGetLastError());
    if (bad) return fail(ELMM_ERR_NAN, "non-finite value in the uploaded temperature");
    return ELMM_OK;
  }

  int upload_scalar(int d, int sc, const void *S) {
    if (d < 0 || d >= nd) return fail(ELMM_ERR_INVALID_ARG, "domain index");
    if (!S) return fail(ELMM_ERR_INVALID_ARG, "NULL scalar array");
    if (sc < 1 || sc > cfg[d].num_scalars) return fail(ELMM_ERR_INVALID_ARG, "scalar number outside 1..num_scalars");
    CU(cudaSetDevice(device));
    if (frame_pending) CU(cudaStreamWaitEvent(stream, ev_packed, 0));
    const Dom<T> &h = hdom[d];
    const size_t n = (size_t)(h.nx + 6) * (h.ny + 6) * (h.nz + 6);
    CU(cudaMemsetAsync(dbad, 0, sizeof(int), stream));
    if (int r = h2d(dstage, S, n, stream)) return r;
    k_unpack_scalar<T><<<kPackBlocks, 256, 0, stream>>>(ddom + d, (h.buoy ? 1 : 0) + sc - 1, dstage, dbad);
    int bad = 0;
    CU(cudaMemcpyAsync(&bad, dbad, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    CU(cudaGetLastError());
    if (bad) return fail(ELMM_ERR_NAN, "non-finite value in the uploaded scalar");
    return ELMM_OK;
  }

  int download_scalar_slices(int d, int sc, double *xy, double *xz) {
    if (d < 0 || d >= nd) return fail(ELMM_ERR_INVALID_ARG, "domain index");
    if (sc < 1 || sc > cfg[d].num_scalars) return fail(ELMM_ERR_INVALID_ARG, "scalar number outside 1..num_scalars");
    const Dom<T> &h = hdom[d];
    const ScalSlot<T> &sl = h.slot[(h.buoy ? 1 : 0) + sc - 1];
    if ((xy && !sl.acc_xy) || (xz && !sl.acc_xz))
      return fail(ELMM_ERR_INVALID_ARG, "no such slice (avg_slice_k / avg_slice_j is 0)");
    CU(cudaSetDevice(device));
    if (xy) CU(cudaMemcpyAsync(xy, sl.acc_xy, sizeof(double) * h.nx * h.ny, cudaMemcpyDeviceToHost, stream));
    if (xz) CU(cudaMemcpyAsync(xz, sl.acc_xz, sizeof(double) * h.nx * h.nz, cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    CU(cudaGetLastError());
    return ELMM_OK;
  }

  int reset_scalar_averages() {
    CU(cudaSetDevice(device));
    for (auto &h : hdom)
      for (int q = 0; q < h.nslot; q++) {
        if (h.slot[q].acc_xy) CU(cudaMemsetAsync(h.slot[q].acc_xy, 0, sizeof(double) * h.nx * h.ny, stream));
        if (h.slot[q].acc_xz) CU(cudaMemsetAsync(h.slot[q].acc_xz, 0, sizeof(double) * h.nx * h.nz, stream));
      }
    CU(cudaStreamSynchronize(stream));
    return ELMM_OK;
  }

  // pack one field into dst (device, host layout); returns elements
  size_t pack(int d, int field, double *dst, cudaStream_t s) {
    const Dom<T> &h = hdom[d];
    const T *F;
    switch (field) {
      case ELMM_FIELD_U: case ELMM_FIELD_V: case ELMM_FIELD_W:
      case ELMM_FIELD_U2: case ELMM_FIELD_V2: case ELMM_FIELD_W2: {
        int comp = (field == ELMM_FIELD_U || field == ELMM_FIELD_U2) ? 0 : (field == ELMM_FIELD_V || field == ELMM_FIELD_V2) ? 1 : 2;
        F = field <= ELMM_FIELD_W ? (comp == 0 ? h.U : comp == 1 ? h.V : h.W) : (comp == 0 ? h.U2 : comp == 1 ? h.V2 : h.W2);
        HostBox hb = hbox_vel(d, comp);
        k_pack_vel<T><<<kPackBlocks, 256, 0, s>>>(ddom + d, F, comp, dst, hb, pack_offsets(d, comp));
        return (size_t)hb.n0 * hb.n1 * hb.n2;
      }
      case ELMM_FIELD_USTAR: case ELMM_FIELD_VSTAR: case ELMM_FIELD_WSTAR: {
        int comp = field - ELMM_FIELD_USTAR;
        F = comp == 0 ? h.Us : comp == 1 ? h.Vs : h.Ws;
        HostBox hb = hbox_vel(d, comp);
        size_t n = (size_t)hb.n0 * hb.n1 * hb.n2;
        cudaMemsetAsync(dst, 0, n * sizeof(double), s);
        k_pack_scalar<T><<<kPackBlocks, 256, 0, s>>>(ddom + d, F, dst, hb, 0, 0, h.ext[comp][0], h.ext[comp][1], h.ext[comp][2]);
        return n;
      }
      case ELMM_FIELD_PR: {
        HostBox hb = hbox_p(d);
        size_t n = (size_t)hb.n0 * hb.n1 * hb.n2;
        cudaMemcpyAsync(dst, pr_image[d], n * sizeof(double), cudaMemcpyDeviceToDevice, s);
        k_pack_scalar<T><<<kPackBlocks, 256, 0, s>>>(ddom + d, h.P, dst, hb, 1, 1, h.nx, h.ny, h.nz);
        return n;
      }
      case ELMM_FIELD_TEMPERATURE: case ELMM_FIELD_TDIFF: case ELMM_FIELD_TEMPERATURE_ADV: {
        const int lo = field == ELMM_FIELD_TDIFF ? -1 : -2;
        const size_t n = (size_t)(h.nx + 2 * (1 - lo)) * (h.ny + 2 * (1 - lo)) * (h.nz + 2 * (1 - lo));
        const T *Fs = field == ELMM_FIELD_TEMPERATURE ? h.Tm : field == ELMM_FIELD_TDIFF ? h.TDiff : h.Tadv;
        // TDiff folds like the viscosity: periodic where the flow is
        const int *bt = field == ELMM_FIELD_TDIFF ? h.bt : h.tbt;
        k_pack_scalar_box<T><<<kPackBlocks, 256, 0, s>>>(ddom + d, Fs, dst, lo, field == ELMM_FIELD_TEMPERATURE ? h.toff : 0.0,
                                                 field == ELMM_FIELD_TEMPERATURE_ADV, bt[0] == BC_PERIODIC,
                                                 bt[2] == BC_PERIODIC, bt[4] == BC_PERIODIC);
        return n;
      }
      case ELMM_FIELD_VISCOSITY: case ELMM_FIELD_PHI: {
        HostBox hb = hbox_p(d);
        size_t n = (size_t)hb.n0 * hb.n1 * hb.n2;
        cudaMemsetAsync(dst, 0, n * sizeof(double), s);
        k_pack_scalar<T><<<kPackBlocks, 256, 0, s>>>(ddom + d, field == ELMM_FIELD_PHI ? h.Phi : h.nu, dst, hb,
                                              field == ELMM_FIELD_PHI ? 2 : 3, 0, h.nx, h.ny, h.nz);
        return n;
      }
    }
    if (field >= ELMM_FIELD_SCALAR && field < ELMM_FIELD_SCALAR_ADV + ELMM_MAX_SCALARS) {
      const bool adv = field >= ELMM_FIELD_SCALAR_ADV;
      const ScalSlot<T> &sl = h.slot[(h.buoy ? 1 : 0) + field - (adv ? ELMM_FIELD_SCALAR_ADV : ELMM_FIELD_SCALAR)];
      const size_t n = (size_t)(h.nx + 6) * (h.ny + 6) * (h.nz + 6);
      k_pack_scalar_box<T><<<kPackBlocks, 256, 0, s>>>(ddom + d, adv ? sl.adv : sl.buf[0], dst, -2, sl.off, adv,
                                               sl.bt[0] == BC_PERIODIC, sl.bt[2] == BC_PERIODIC, sl.bt[4] == BC_PERIODIC);
      return n;
    }
    return 0;
  }

  int download_field(int d, int field, void *host) {
    if (d < 0 || d >= nd) return fail(ELMM_ERR_INVALID_ARG, "domain index");
    const int nsc = cfg[d].num_scalars;
    const bool scal = (field >= ELMM_FIELD_SCALAR && field < ELMM_FIELD_SCALAR + nsc) ||
                      (field >= ELMM_FIELD_SCALAR_ADV && field < ELMM_FIELD_SCALAR_ADV + nsc);
    if (!scal && (field < 0 || field > ELMM_FIELD_TEMPERATURE_ADV)) return fail(ELMM_ERR_INVALID_ARG, "field id");
    if (field == ELMM_FIELD_TDIFF && !hdom[d].TDiff)
      return fail(ELMM_ERR_INVALID_ARG, "no diffusivity field (no temperature and no scalars)");
    if ((field == ELMM_FIELD_TEMPERATURE || field == ELMM_FIELD_TEMPERATURE_ADV) && !hdom[d].buoy)
      return fail(ELMM_ERR_INVALID_ARG, "no temperature field (enable_buoyancy is 0)");
    if (!host) return fail(ELMM_ERR_INVALID_ARG, "NULL host array");
    CU(cudaSetDevice(device));
    size_t n = pack(d, field, dstage, stream);
    if (int r = d2h(host, dstage, n, stream)) return r;
    CU(cudaStreamSynchronize(stream));
    CU(cudaGetLastError());
    return ELMM_OK;
  }

  int download(int d, void *U, void *V, void *W, void *Pr) {
    void *dst[4] = {U, V, W, Pr};
    if (d < 0 || d >= nd) return fail(ELMM_ERR_INVALID_ARG, "domain index");
    CU(cudaSetDevice(device));
    if (hostf || !two_stages()) {
      for (int f = 0; f < 4; f++)
        if (dst[f]) {
          int r = download_field(d, f, dst[f]);
          if (r) return r;
        }
      return ELMM_OK;
    }
    // pack field f into one buffer while the other is copied to the host
    int b = 0;
    for (int f = 0; f < 4; f++) {
      if (!dst[f]) continue;
      double *stg = b ? dstage2 : dstage;
      CU(cudaStreamWaitEvent(stream, ev_stage[b][1], 0));  // its last host copy is done
      size_t n = pack(d, f, stg, stream);
      CU(cudaEventRecord(ev_stage[b][0], stream));
      CU(cudaStreamWaitEvent(side, ev_stage[b][0], 0));
      CU(cudaMemcpyAsync(dst[f], stg, n * sizeof(double), cudaMemcpyDeviceToHost, side));
      CU(cudaEventRecord(ev_stage[b][1], side));
      b ^= 1;
    }
    CU(cudaStreamSynchronize(side));
    CU(cudaStreamSynchronize(stream));
    CU(cudaGetLastError());
    return ELMM_OK;
  }

  // ----------------------------------------------------- async frames
  size_t frame_offsets(int d, size_t off[5]) {
    off[0] = 0;
    for (int c = 0; c < 3; c++) {
      HostBox hb = hbox_vel(d, c);
      off[c + 1] = off[c] + (size_t)hb.n0 * hb.n1 * hb.n2;
    }
    HostBox hp = hbox_p(d);
    off[4] = off[3] + (size_t)hp.n0 * hp.n1 * hp.n2;
    return off[4];
  }

  int frame_begin() {
    if (nd != 1) return fail(ELMM_ERR_INVALID_ARG, "frames are per single-domain handle");
    CU(cudaSetDevice(device));
    if (frame_pending) {
      CU(cudaEventSynchronize(ev_done));
      frame_pending = false;
    }
    size_t off[5];
    size_t need = frame_offsets(0, off);
    if (need > frame_elems) {
      if (frame_host) cudaFreeHost(frame_host);
      frame_host = nullptr;
      CU(cudaMallocHost((void **)&frame_host, need * sizeof(double)));
      int r = dalloc((void **)&frame_dev, need * sizeof(double));
      if (r) return r;
      frame_elems = need;
    }
    CU(cudaEventRecord(ev_ready, stream));
    CU(cudaStreamWaitEvent(side, ev_ready, 0));
    for (int f = 0; f < 4; f++) pack(0, f, frame_dev + off[f], side);
    CU(cudaEventRecord(ev_packed, side));
    CU(cudaMemcpyAsync(frame_host, frame_dev, need * sizeof(double), cudaMemcpyDeviceToHost, side));
    CU(cudaEventRecord(ev_done, side));
    frame_pending = true;
    return ELMM_OK;
  }

  int frame_wait(double *U, double *V, double *W, double *Pr) {
    if (!frame_pending) return fail(ELMM_ERR_INVALID_ARG, "no frame in flight");
    CU(cudaEventSynchronize(ev_done));
    frame_pending = false;
    size_t off[5];
    frame_offsets(0, off);
    double *dst[4] = {U, V, W, Pr};
    for (int f = 0; f < 4; f++)
      if (dst[f]) memcpy(dst[f], frame_host + off[f], (off[f + 1] - off[f]) * sizeof(double));
    return ELMM_OK;
  }
};

// ------------------------------------------------------------ handle types
struct elmm_batch {
  int precision = 0;
  std::unique_ptr<BatchT<double>> b64;
  std::unique_ptr<BatchT<float>> b32;
};

struct elmm_handle {
  elmm_batch b;
};

struct elmm_poisson {
  elmm_batch b;
  int nx, ny, nz;
};

#define DISPATCH(B, EXPR) ((B).precision == ELMM_PREC_MIXED ? (B).b32->EXPR : (B).b64->EXPR)

static int batch_init(elmm_batch &B, const elmm_config *cfgs, int n) {
  if (!cfgs || n < 1) return fail(ELMM_ERR_INVALID_ARG, "no configuration");
  B.precision = cfgs[0].precision;
  int r;
  if (B.precision == ELMM_PREC_MIXED) {
    B.b32.reset(new BatchT<float>());
    r = B.b32->init(cfgs, n);
  } else {
    B.b64.reset(new BatchT<double>());
    r = B.b64->init(cfgs, n);
  }
  return r;
}

// Phi and RHS are double host arrays, or float ones when B.hostf is set
template <typename T>
static int poisson_exec(BatchT<T> &B, void *Phi, const void *RHS) {
  CU(cudaSetDevice(B.device));
  const Dom<T> &h = B.hdom[0];
  // RHS(0:n+1)^3 -> box field (Phi is free until the inverse transform) -> transforms
  HostBox hb{0, h.nx + 2, h.ny + 2, h.nz + 2};
  size_t n = (size_t)hb.n0 * hb.n1 * hb.n2;
  if (int r = B.h2d(B.dstage, RHS, n, B.stream)) return r;
  CU(cudaMemsetAsync(B.dbad, 0, sizeof(int), B.stream));
  k_unpack<T><<<kPackBlocks, 256, 0, B.stream>>>(B.ddom, h.Phi, B.dstage, hb, h.nx, h.ny, h.nz, B.dbad);
  B.launch_poisson(1.0, 0, 1, 0);
  HostBox hp = B.hbox_p(0);
  size_t np = (size_t)hp.n0 * hp.n1 * hp.n2;
  if (int r = B.h2d(B.dstage, Phi, np, B.stream)) return r;  // the host's ghosts stay as they are
  k_pack_scalar<T><<<kPackBlocks, 256, 0, B.stream>>>(B.ddom, h.Phi, B.dstage, hp, 0, 0, h.nx, h.ny, h.nz);
  if (int r = B.d2h(Phi, B.dstage, np, B.stream)) return r;
  CU(cudaStreamSynchronize(B.stream));
  CU(cudaGetLastError());
  int bad = 0;
  CU(cudaMemcpy(&bad, B.dbad, sizeof(int), cudaMemcpyDeviceToHost));
  if (bad) return fail(ELMM_ERR_NAN, std::to_string(bad) + " non-finite right-hand-side value(s)");
  return ELMM_OK;
}


// Runs f on the batch with its host arrays taken as float (the *_float entry
// points of a single-precision host).
template <typename F>
static int with_float_host(elmm_batch &B, F f) {
  if (B.precision == ELMM_PREC_MIXED) {
    B.b32->hostf = 1;
    const int r = f(*B.b32);
    B.b32->hostf = 0;
    return r;
  }
  B.b64->hostf = 1;
  const int r = f(*B.b64);
  B.b64->hostf = 0;
  return r;
}

#include "elmm_server.inl"
#include "elmm_slabs.inl"

extern "C" {

const char *elmm_version(void) { return "elmm-b200 1.0 (sm_100a)"; }

const char *elmm_last_error(void) { return g_err.c_str(); }

int elmm_config_defaults(elmm_config *c, int32_t Prnx, int32_t Prny, int32_t Prnz) {
  if (!c) return fail(ELMM_ERR_INVALID_ARG, "NULL config");
  memset(c, 0, sizeof(*c));
  c->abi_version = ELMM_ABI_VERSION;
  c->Prnx = Prnx; c->Prny = Prny; c->Prnz = Prnz;
  int bt[6] = {ELMM_BC_PERIODIC, ELMM_BC_PERIODIC, ELMM_BC_PERIODIC, ELMM_BC_PERIODIC, ELMM_BC_NOSLIP, ELMM_BC_FREESLIP};
  memcpy(c->Btype, bt, sizeof(bt));
  c->dxmin = c->dymin = c->dzmin = 1.0;
  c->dt = 0.02;
  c->CFL = 0.3;     // time_step_control%CFL (src/parameters.f90:110); used with variable steps
  c->dt_max = 0.02;
  c->molecular_viscosity = 1.0 / 70000;
  c->C_Smagorinsky = 0.122;
  c->filter_ratio = 1.0;
  c->sgstype = 1;
  c->wallmodeltype = 1;
  for (int s = 0; s < 6; s++) c->z0[s] = 0.01;
  c->precision = ELMM_PREC_FP64;
  c->refine_tol = 1e-6;
  for (int s = 0; s < 6; s++) c->TempBtype[s] = bt[s] == ELMM_BC_PERIODIC ? ELMM_BC_PERIODIC : ELMM_BC_CONSTFLUX;
  c->temperature_ref = 295;                             // src/parameters.f90:220
  c->grav_acc = 9.81;                                   // src/parameters.f90:146
  c->molecular_diffusivity = c->molecular_viscosity / 0.7;  // src/parameters.f90:129
  return ELMM_OK;
}

int elmm_create(const elmm_config *cfg, elmm_handle **out) {
  if (!cfg || !out) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  elmm_handle *h = new elmm_handle();
  int r = batch_init(h->b, cfg, 1);
  if (r) { delete h; return r; }
  *out = h;
  return ELMM_OK;
}

int elmm_destroy(elmm_handle *h) {
  delete h;
  return ELMM_OK;
}

int elmm_upload_state(elmm_handle *h, const double *U, const double *V, const double *W, const double *Pr) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return DISPATCH(h->b, upload(0, U, V, W, Pr));
}

int elmm_download_state(elmm_handle *h, double *U, double *V, double *W, double *Pr) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return DISPATCH(h->b, download(0, U, V, W, Pr));
}

int elmm_download_field(elmm_handle *h, int32_t field, double *host) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return DISPATCH(h->b, download_field(0, field, host));
}

int elmm_upload_temperature(elmm_handle *h, const double *T) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return DISPATCH(h->b, upload_temperature(0, T));
}

int elmm_upload_scalar(elmm_handle *h, int32_t sc, const double *S) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return DISPATCH(h->b, upload_scalar(0, sc, S));
}

int elmm_download_scalar_slices(elmm_handle *h, int32_t sc, double *xy, double *xz) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return DISPATCH(h->b, download_scalar_slices(0, sc, xy, xz));
}

int elmm_reset_scalar_averages(elmm_handle *h) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return DISPATCH(h->b, reset_scalar_averages());
}

int elmm_frame_begin(elmm_handle *h) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return DISPATCH(h->b, frame_begin());
}

int elmm_frame_wait(elmm_handle *h, double *U, double *V, double *W, double *Pr) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return DISPATCH(h->b, frame_wait(U, V, W, Pr));
}

int elmm_project(elmm_handle *h, double coef, elmm_stats *st) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  if (!(coef > 0)) return fail(ELMM_ERR_INVALID_ARG, "coef must be positive");
  return DISPATCH(h->b, project(coef, st));
}

int elmm_step(elmm_handle *h, int32_t nsteps, elmm_stats *st) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  if (nsteps < 0) return fail(ELMM_ERR_INVALID_ARG, "nsteps < 0");
  return DISPATCH(h->b, step(nsteps, st));
}

int elmm_march_host(elmm_handle *h, double *U, double *V, double *W, double *Pr, double *Temperature,
                    int32_t nsteps, elmm_stats *stats) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  if (nsteps < 0) return fail(ELMM_ERR_INVALID_ARG, "nsteps < 0");
  return DISPATCH(h->b, march_host(U, V, W, Pr, Temperature, nsteps, stats));
}

int elmm_set_fault_injection(elmm_handle *h, int32_t wait_limit, int32_t skip_plane) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  if (wait_limit < 1) return fail(ELMM_ERR_INVALID_ARG, "wait_limit < 1");
  return DISPATCH(h->b, set_fault_injection(wait_limit, skip_plane));
}

int elmm_upload_state_float(elmm_handle *h, const float *U, const float *V, const float *W, const float *Pr) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return with_float_host(h->b, [&](auto &b) { return b.upload(0, U, V, W, Pr); });
}

int elmm_download_state_float(elmm_handle *h, float *U, float *V, float *W, float *Pr) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return with_float_host(h->b, [&](auto &b) { return b.download(0, U, V, W, Pr); });
}

int elmm_download_field_float(elmm_handle *h, int32_t field, float *host) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return with_float_host(h->b, [&](auto &b) { return b.download_field(0, field, host); });
}

int elmm_upload_temperature_float(elmm_handle *h, const float *T) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return with_float_host(h->b, [&](auto &b) { return b.upload_temperature(0, T); });
}

int elmm_upload_scalar_float(elmm_handle *h, int32_t sc, const float *S) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return with_float_host(h->b, [&](auto &b) { return b.upload_scalar(0, sc, S); });
}

int elmm_march_host_float(elmm_handle *h, float *U, float *V, float *W, float *Pr, float *Temperature, int32_t nsteps,
                          elmm_stats *stats) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  if (nsteps < 0) return fail(ELMM_ERR_INVALID_ARG, "nsteps < 0");
  return with_float_host(h->b, [&](auto &b) { return b.march_host(U, V, W, Pr, Temperature, nsteps, stats); });
}

int elmm_set_puffs(elmm_handle *h, const elmm_puff *puffs, int32_t npuffs, const elmm_puff_volume *volumes,
                   int32_t nvolumes) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return DISPATCH(h->b, set_puffs(0, puffs, npuffs, volumes, nvolumes));
}

int elmm_set_solids(elmm_handle *h, const elmm_solids *s) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return DISPATCH(h->b, set_solids(0, s));
}

int elmm_run_stage(elmm_handle *h, int32_t stage, int32_t stop) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  if (stage < 1 || stage > 3 || stop < 1 || stop > 3) return fail(ELMM_ERR_INVALID_ARG, "stage 1..3, stop 1..3");
  int r = DISPATCH(h->b, run_stage(stage, stop, 0, true));
  if (r) return r;
  cudaStream_t s = h->b.precision == ELMM_PREC_MIXED ? h->b.b32->stream : h->b.b64->stream;
  CU(cudaStreamSynchronize(s));
  CU(cudaGetLastError());
  return ELMM_OK;
}

int elmm_profile_stage(elmm_handle *h, int32_t stage, int32_t reps, double *ms) {
  if (!h || !ms) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  if (stage < 1 || stage > 3 || reps < 1) return fail(ELMM_ERR_INVALID_ARG, "stage 1..3, reps >= 1");
  return DISPATCH(h->b, profile_stage(stage, reps, ms));
}

// ------------------------------------------------------------- batches
int elmm_batch_create(const elmm_config *cfgs, int32_t n, elmm_batch **out) {
  if (!cfgs || !out || n < 1) return fail(ELMM_ERR_INVALID_ARG, "bad arguments");
  *out = nullptr;
  elmm_batch *b = new elmm_batch();
  int r = batch_init(*b, cfgs, n);
  if (r) { delete b; return r; }
  *out = b;
  return ELMM_OK;
}

int elmm_batch_destroy(elmm_batch *b) {
  delete b;
  return ELMM_OK;
}

int elmm_batch_upload_state(elmm_batch *b, int32_t d, const double *U, const double *V, const double *W,
                            const double *Pr) {
  if (!b) return fail(ELMM_ERR_INVALID_ARG, "NULL batch");
  return DISPATCH(*b, upload(d, U, V, W, Pr));
}

int elmm_batch_download_state(elmm_batch *b, int32_t d, double *U, double *V, double *W, double *Pr) {
  if (!b) return fail(ELMM_ERR_INVALID_ARG, "NULL batch");
  return DISPATCH(*b, download(d, U, V, W, Pr));
}

// ------------------------------------------------------------- serving
int elmm_server_create(const elmm_server_config *cfg, elmm_server **out) {
  if (!cfg || !out) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  if (cfg->precision != ELMM_PREC_FP64 && cfg->precision != ELMM_PREC_MIXED)
    return fail(ELMM_ERR_INVALID_CONFIG, "unknown precision");
  if (cfg->max_active < 1 || cfg->max_active > ELMM_SERVER_MAX_ACTIVE)
    return fail(ELMM_ERR_INVALID_CONFIG, "max_active in 1.." + std::to_string(ELMM_SERVER_MAX_ACTIVE));
  if (cfg->chunk_steps < 1) return fail(ELMM_ERR_INVALID_CONFIG, "chunk_steps must be positive");
  if (cfg->policy != ELMM_SERVE_FIFO && cfg->policy != ELMM_SERVE_SHORTEST_FIRST)
    return fail(ELMM_ERR_INVALID_CONFIG, "unknown admission policy");
  if (cfg->hbm_budget_bytes < (1 << 20)) return fail(ELMM_ERR_INVALID_CONFIG, "hbm_budget_bytes below 1 MiB");
  elmm_server *s = new elmm_server();
  s->precision = cfg->precision;
  int r;
  if (s->precision == ELMM_PREC_MIXED) {
    s->s32.reset(new ServerT<float>());
    r = s->s32->init(*cfg);
  } else {
    s->s64.reset(new ServerT<double>());
    r = s->s64->init(*cfg);
  }
  if (r) { delete s; return r; }
  *out = s;
  return ELMM_OK;
}

int elmm_server_destroy(elmm_server *s) {
  delete s;
  return ELMM_OK;
}

#define SDISPATCH(S, EXPR) ((S)->precision == ELMM_PREC_MIXED ? (S)->s32->EXPR : (S)->s64->EXPR)

int elmm_server_submit(elmm_server *s, const elmm_config *cfg, const double *U, const double *V, const double *W,
                       const double *Pr, const double *S0, int32_t nsteps, int64_t *id) {
  if (!s || !cfg || !id) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  return SDISPATCH(s, submit(*cfg, U, V, W, Pr, S0, nsteps, id));
}

int elmm_server_wait_any(elmm_server *s, int32_t timeout_ms, elmm_request_info *info) {
  if (!s || !info) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  return SDISPATCH(s, wait_any(std::max(0, (int)timeout_ms), info));
}

int elmm_server_collect(elmm_server *s, int64_t id, double *xy, double *xz) {
  if (!s) return fail(ELMM_ERR_INVALID_ARG, "NULL server");
  return SDISPATCH(s, collect(id, xy, xz));
}

int elmm_server_stats_get(elmm_server *s, elmm_server_stats *st) {
  if (!s || !st) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  SDISPATCH(s, stats(st));
  return ELMM_OK;
}

double elmm_server_now(const elmm_server *s) {
  if (!s) return 0;
  return s->precision == ELMM_PREC_MIXED ? s->s32->now() : s->s64->now();
}

int elmm_batch_profile_stage(elmm_batch *b, int32_t stage, int32_t reps, double *ms) {
  if (!b || !ms) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  if (stage < 1 || stage > 3 || reps < 1) return fail(ELMM_ERR_INVALID_ARG, "stage 1..3, reps >= 1");
  return DISPATCH(*b, profile_stage(stage, reps, ms));
}

int elmm_batch_tuning(const elmm_batch *b, int32_t out[2]) {
  if (!b || !out) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  out[0] = b->precision == ELMM_PREC_MIXED ? b->b32->tune_rows : b->b64->tune_rows;
  out[1] = b->precision == ELMM_PREC_MIXED ? b->b32->tune_cols : b->b64->tune_cols;
  return ELMM_OK;
}

int elmm_batch_get_tuning(const elmm_batch *b, int32_t *out, int32_t n) {
  if (!b || !out || n < 0) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  int32_t v[ELMM_TUNE_KNOBS];
  if (b->precision == ELMM_PREC_MIXED) {
    v[0] = b->b32->tune_rows; v[1] = b->b32->tune_cols; v[2] = b->b32->tune_mom_kc; v[3] = b->b32->tune_sgs_kc;
  } else {
    v[0] = b->b64->tune_rows; v[1] = b->b64->tune_cols; v[2] = b->b64->tune_mom_kc; v[3] = b->b64->tune_sgs_kc;
  }
  for (int q = 0; q < n && q < ELMM_TUNE_KNOBS; q++) out[q] = v[q];
  return ELMM_OK;
}

int elmm_get_tuning(const elmm_handle *h, int32_t *out, int32_t n) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return elmm_batch_get_tuning(&h->b, out, n);
}

int elmm_set_tuning(elmm_handle *h, const int32_t *vals, int32_t n) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return elmm_batch_set_tuning(&h->b, vals, n);
}

int elmm_batch_set_tuning(elmm_batch *b, const int32_t *vals, int32_t n) {
  if (!b || !vals || n < 0 || n > ELMM_TUNE_KNOBS) return fail(ELMM_ERR_INVALID_ARG, "NULL argument or n out of range");
  return DISPATCH(*b, set_tuning(vals, n));
}

static int batch_domain_ok(const elmm_batch *b, int32_t d) {
  const int nd = b->precision == ELMM_PREC_MIXED ? b->b32->nd : b->b64->nd;
  return d >= 0 && d < nd;
}

int elmm_batch_set_solids(elmm_batch *b, int32_t d, const elmm_solids *s) {
  if (!b) return fail(ELMM_ERR_INVALID_ARG, "NULL batch");
  if (!batch_domain_ok(b, d)) return fail(ELMM_ERR_INVALID_ARG, "domain index");
  return DISPATCH(*b, set_solids(d, s));
}

int elmm_batch_set_puffs(elmm_batch *b, int32_t d, const elmm_puff *puffs, int32_t npuffs,
                         const elmm_puff_volume *volumes, int32_t nvolumes) {
  if (!b) return fail(ELMM_ERR_INVALID_ARG, "NULL batch");
  if (!batch_domain_ok(b, d)) return fail(ELMM_ERR_INVALID_ARG, "domain index");
  return DISPATCH(*b, set_puffs(d, puffs, npuffs, volumes, nvolumes));
}

int elmm_batch_upload_scalar(elmm_batch *b, int32_t d, int32_t sc, const double *S) {
  if (!b) return fail(ELMM_ERR_INVALID_ARG, "NULL batch");
  return DISPATCH(*b, upload_scalar(d, sc, S));
}

int elmm_batch_download_field(elmm_batch *b, int32_t d, int32_t field, double *host) {
  if (!b) return fail(ELMM_ERR_INVALID_ARG, "NULL batch");
  return DISPATCH(*b, download_field(d, field, host));
}

int elmm_batch_download_scalar_slices(elmm_batch *b, int32_t d, int32_t sc, double *xy, double *xz) {
  if (!b) return fail(ELMM_ERR_INVALID_ARG, "NULL batch");
  return DISPATCH(*b, download_scalar_slices(d, sc, xy, xz));
}

int elmm_batch_project(elmm_batch *b, double coef) {
  if (!b) return fail(ELMM_ERR_INVALID_ARG, "NULL batch");
  return DISPATCH(*b, project(coef, nullptr));
}

int elmm_batch_step(elmm_batch *b, int32_t nsteps, elmm_stats *st) {
  if (!b) return fail(ELMM_ERR_INVALID_ARG, "NULL batch");
  return DISPATCH(*b, step(nsteps, st));
}

int64_t elmm_batch_cells(const elmm_batch *b) {
  if (!b) return 0;
  return b->precision == ELMM_PREC_MIXED ? b->b32->cells : b->b64->cells;
}

// ---------------------------------------------------- PoisSolver interface
static int poisson_new(elmm_poisson **out, const int32_t n[3], double Lx, double Ly, const double *zW, double Lz,
                       const int32_t bcs[6], int32_t precision, int32_t device) {
  if (!out || !n || !bcs) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  elmm_config c;
  elmm_config_defaults(&c, n[0], n[1], n[2]);
  for (int s = 0; s < 6; s++) {
    if (bcs[s] != ELMM_BC_PERIODIC && bcs[s] != ELMM_BC_NEUMANN)
      return fail(ELMM_ERR_INVALID_CONFIG, "Poisson BCs must be periodic or staggered Neumann");
    c.Btype[s] = bcs[s] == ELMM_BC_PERIODIC ? ELMM_BC_PERIODIC : ELMM_BC_NEUMANN;
  }
  c.dxmin = Lx / n[0];
  c.dymin = Ly / n[1];
  c.dzmin = zW ? (zW[n[2]] - zW[0]) / n[2] : Lz / n[2];
  c.zW = zW;
  c.sgstype = 0;
  c.wallmodeltype = 0;
  c.precision = precision;
  c.device = device;
  elmm_poisson *p = new elmm_poisson();
  p->nx = n[0]; p->ny = n[1]; p->nz = n[2];
  int r = batch_init(p->b, &c, 1);
  if (r) { delete p; return r; }
  *out = p;
  return ELMM_OK;
}

int elmm_poisson_solver_new(elmm_poisson **out, const int32_t n[3], const double L[3], const int32_t bcs[6],
                            int32_t precision, int32_t device) {
  if (!L) return fail(ELMM_ERR_INVALID_ARG, "NULL L");
  return poisson_new(out, n, L[0], L[1], nullptr, L[2], bcs, precision, device);
}

int elmm_poisson_solver_nonuniform_z_new(elmm_poisson **out, const int32_t n[3], const double Lxy[2],
                                         const double *zPr, const double *zW, const int32_t bcs[6],
                                         int32_t precision, int32_t device) {
  (void)zPr;  // zPr(k) = (zW(k-1) + zW(k)) / 2 is recomputed from zW
  if (!Lxy || !zW) return fail(ELMM_ERR_INVALID_ARG, "NULL grid");
  return poisson_new(out, n, Lxy[0], Lxy[1], zW, 0.0, bcs, precision, device);
}

int elmm_poisson_solver_execute(elmm_poisson *s, double *Phi, const double *RHS) {
  if (!s || !Phi || !RHS) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  return s->b.precision == ELMM_PREC_MIXED ? poisson_exec(*s->b.b32, Phi, RHS) : poisson_exec(*s->b.b64, Phi, RHS);
}

int elmm_poisson_solver_finalize(elmm_poisson *s) {
  delete s;
  return ELMM_OK;
}

// ---- single-precision host arrays (prec=sp hosts) -------------------------
int elmm_poisson_solver_new_float(elmm_poisson **out, const int32_t n[3], const float L[3], const int32_t bcs[6],
                                  int32_t precision, int32_t device) {
  if (!L) return fail(ELMM_ERR_INVALID_ARG, "NULL L");
  return poisson_new(out, n, (double)L[0], (double)L[1], nullptr, (double)L[2], bcs, precision, device);
}

int elmm_poisson_solver_nonuniform_z_new_float(elmm_poisson **out, const int32_t n[3], const float Lxy[2],
                                               const float *zPr, const float *zW, const int32_t bcs[6],
                                               int32_t precision, int32_t device) {
  (void)zPr;  // zPr(k) = (zW(k-1) + zW(k)) / 2 is recomputed from zW
  if (!Lxy || !zW || !n) return fail(ELMM_ERR_INVALID_ARG, "NULL grid");
  if (n[2] < 1) return fail(ELMM_ERR_INVALID_CONFIG, "nz < 1");
  std::vector<double> zw(zW, zW + n[2] + 1);
  return poisson_new(out, n, (double)Lxy[0], (double)Lxy[1], zw.data(), 0.0, bcs, precision, device);
}

int elmm_poisson_solver_execute_float(elmm_poisson *s, float *Phi, const float *RHS) {
  if (!s || !Phi || !RHS) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  return with_float_host(s->b, [&](auto &b) { return poisson_exec(b, Phi, RHS); });
}

int elmm_poisson_solver_finalize_float(elmm_poisson *s) { return elmm_poisson_solver_finalize(s); }

}  // extern "C"

// ============================================================================
// elmm_poisson_solve_noalloc: the solve of elmm_poisson_solver_execute on
// device arrays, for callers that cannot allocate device memory (a host
// whose pool already owns the GPU, or a path where cudaMalloc/cudaFree would
// synchronise the device).  All working memory sits in noalloc_scratch, a
// fixed array in this library's device image; nothing here calls cudaMalloc,
// cudaFree or any other allocating routine.  The kernels are the generic-length
// kernels of the handle-based solver; only their descriptors and buffers live
// elsewhere.

// Every GPU that loads the library holds this array until the process exits.
static __device__ __align__(256) unsigned char noalloc_scratch[ELMM_NOALLOC_SCRATCH_BYTES];

// byte offsets of the pieces carved out of noalloc_scratch (256-aligned)
struct NoAllocLayout {
  size_t dom, plan, starts, bad, twx, twy, lamx, lamy, Ab, At, dzc, dzf, box, S, total;
};

static NoAllocLayout noalloc_layout(int nx, int ny, int nz, size_t box_elems, size_t s_elems) {
  NoAllocLayout l;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t at = o;
    o += (bytes + 255) / 256 * 256;
    return at;
  };
  l.dom = take(sizeof(Dom<double>));
  l.plan = take(sizeof(PoisPlan));
  l.starts = take(2 * sizeof(int));
  l.bad = take(sizeof(int));
  l.twx = take(sizeof(double2) * nx);
  l.twy = take(sizeof(double2) * ny);
  l.lamx = take(sizeof(double) * nx);
  l.lamy = take(sizeof(double) * ny);
  l.Ab = take(sizeof(double) * (nz + 2));
  l.At = take(sizeof(double) * (nz + 2));
  l.dzc = take(sizeof(double) * (nz + 2));
  l.dzf = take(sizeof(double) * (nz + 2));
  l.box = take(sizeof(double) * box_elems);
  l.S = take(sizeof(double2) * s_elems);
  l.total = o;
  return l;
}

// Writes the descriptors and the FFT / tridiagonal tables of one solve into
// the scratch array and zeroes its one accumulator (the count of non-finite
// right-hand-side values).  Nothing else in the array needs to start at zero:
// every other element a solve reads is written earlier in the same solve.
// The tables follow the handle-based set-up: twiddles exp(-2 pi i m / n), the
// eigenvalues -4 sin^2(pi m / n) / d^2, and the z coefficients of a uniform
// grid with zW(k) = k dz (src/poisson.f90:23-60 for the discrete problem).
static __global__ void k_noalloc_setup(Dom<double> h, PoisPlan pl, NoAllocLayout lay, unsigned char *base) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  if (tid == 0) {
    *reinterpret_cast<Dom<double> *>(base + lay.dom) = h;
    *reinterpret_cast<PoisPlan *>(base + lay.plan) = pl;
    int *st = reinterpret_cast<int *>(base + lay.starts);
    st[0] = 0;
    st[1] = 0;
    *reinterpret_cast<int *>(base + lay.bad) = 0;
  }
  double2 *twx = reinterpret_cast<double2 *>(base + lay.twx), *twy = reinterpret_cast<double2 *>(base + lay.twy);
  double *lamx = reinterpret_cast<double *>(base + lay.lamx), *lamy = reinterpret_cast<double *>(base + lay.lamy);
  const double rx = 1.0 / (h.dx * h.dx), ry = 1.0 / (h.dy * h.dy);
  for (int m = tid; m < h.nx; m += nth) {
    const double a = __ddiv_rn(__dmul_rn(-2.0 * M_PI, (double)m), (double)h.nx);
    twx[m] = make_double2(cos(a), sin(a));
    const double sn = sin(__ddiv_rn(__dmul_rn(M_PI, (double)m), (double)h.nx));
    lamx[m] = -4.0 * sn * sn * rx;
  }
  for (int m = tid; m < h.ny; m += nth) {
    const double a = __ddiv_rn(__dmul_rn(-2.0 * M_PI, (double)m), (double)h.ny);
    twy[m] = make_double2(cos(a), sin(a));
    const double sn = sin(__ddiv_rn(__dmul_rn(M_PI, (double)m), (double)h.ny));
    lamy[m] = -4.0 * sn * sn * ry;
  }
  double *Ab = reinterpret_cast<double *>(base + lay.Ab), *At = reinterpret_cast<double *>(base + lay.At);
  double *dzc = reinterpret_cast<double *>(base + lay.dzc), *dzf = reinterpret_cast<double *>(base + lay.dzf);
  auto zW = [&](int k) { return __dmul_rn((double)k, h.dz); };
  auto zP = [&](int k) { return __dmul_rn(__dadd_rn(zW(k - 1), zW(k)), 0.5); };
  for (int k = tid; k <= h.nz + 1; k += nth) {
    double ab = 0, at = 0, c = 0, f = 0;
    if (k >= 1 && k <= h.nz) {
      const double w = __dsub_rn(zW(k), zW(k - 1));
      ab = 1.0 / __dmul_rn(__dsub_rn(zP(k), zP(k - 1)), w);
      at = 1.0 / __dmul_rn(__dsub_rn(zP(k + 1), zP(k)), w);
      c = w;
      f = __dsub_rn(zP(k + 1), zP(k));
      if (!h.zper && k == 1) ab = 0;
      if (!h.zper && k == h.nz) at = 0;
    }
    Ab[k] = ab; At[k] = at; dzc[k] = c; dzf[k] = f;
  }
}

static std::mutex noalloc_mu;
// per device: the context the set-up ran in, the device address of
// noalloc_scratch in that context, and the kernels' limits
struct NoAllocDev {
  unsigned long long ctx_id = 0;  // 0: no set-up yet
  unsigned char *base = nullptr;
  int optin = 0, nsm = 0;
};
static NoAllocDev noalloc_dev[64];

// The unique id of the current context (cuCtxGetCurrent + cuCtxGetId from
// the driver the runtime already loaded, as for cuTensorMapEncodeTiled), or
// 0 if it cannot be had.  A context that was destroyed and created again
// (cudaDeviceReset, a torn-down primary context) has a new id, and the
// module holding noalloc_scratch may then sit at a new address.
static unsigned long long current_ctx_id() {
  typedef CUresult (*GetCurrent)(CUcontext *);
  typedef CUresult (*GetId)(CUcontext, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool looked = false;
  if (!looked) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (GetCurrent)p;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (GetId)p;
    looked = true;
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

// With `device` current: the device address of the scratch array (host code
// only holds a stand-in for it) and the kernels' shared-memory limit, once
// per context.  A call in a context other than the one of the stored set-up
// (or when the context id is unknown) repeats the set-up, so a stale address
// of an earlier context is never used.
static int noalloc_setup(int device, NoAllocDev *out) {
  std::lock_guard<std::mutex> lock(noalloc_mu);
  // the caller's cudaSetDevice made the device's primary context current
  // (CUDA 12 creates it there), so it has an id
  const unsigned long long id = current_ctx_id();
  NoAllocDev &nd = noalloc_dev[device];
  if (id != 0 && nd.ctx_id == id) {
    *out = nd;
    return ELMM_OK;
  }
  unsigned char *ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void **)&ptr, noalloc_scratch);
  if (e == cudaErrorMemoryAllocation)
    return fail(ELMM_ERR_OOM, "elmm_poisson_solve_noalloc: loading the library's device image, which holds the fixed " +
                                  std::to_string((size_t)ELMM_NOALLOC_SCRATCH_BYTES) +
                                  "-byte scratch array, ran out of device memory (make the first call on a device "
                                  "before the host's memory pool reserves the GPU's memory)");
  if (e != cudaSuccess)
    return fail(ELMM_ERR_CUDA, std::string("cudaGetSymbolAddress(noalloc_scratch): ") + cudaGetErrorString(e));
  int optin = 0, nsm = 0;
  CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  CU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  CU(cudaFuncSetAttribute(k_fftx_fwd<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  CU(cudaFuncSetAttribute(k_fftx_inv<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  CU(cudaFuncSetAttribute(k_ffty<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  CU(cudaFuncSetAttribute(k_tri<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  nd.base = ptr;
  nd.optin = optin;
  nd.nsm = nsm;
  nd.ctx_id = id;  // 0 (id unknown) keeps the next call doing the set-up again
  *out = nd;
  return ELMM_OK;
}

// The caller's current device, made current again when the call returns.
struct KeepDevice {
  int dev = -1;
  KeepDevice() {
    if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
  }
  ~KeepDevice() {
    if (dev >= 0) cudaSetDevice(dev);
  }
};

extern "C" int elmm_poisson_solve_noalloc(const int32_t n[3], const double L[3], const int32_t bcs[6], int32_t device,
                                          double *Phi, const double *RHS, void *stream) {
  if (!n || !L || !bcs || !Phi || !RHS) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  // the same problem as elmm_poisson_solver_new (uniform z)
  elmm_config c;
  elmm_config_defaults(&c, n[0], n[1], n[2]);
  for (int s = 0; s < 6; s++) {
    if (bcs[s] != ELMM_BC_PERIODIC && bcs[s] != ELMM_BC_NEUMANN)
      return fail(ELMM_ERR_INVALID_CONFIG, "Poisson BCs must be periodic or staggered Neumann");
    c.Btype[s] = bcs[s];
  }
  c.dxmin = L[0] / n[0];
  c.dymin = L[1] / n[1];
  c.dzmin = L[2] / n[2];
  c.sgstype = 0;
  c.wallmodeltype = 0;
  c.precision = ELMM_PREC_FP64;
  c.device = device;
  int r = check_config(c);
  if (r) return r;
  const int nx = n[0], ny = n[1], nz = n[2];
  const int aln = 128 / (int)sizeof(double);
  const int pitch = round_up(aln + nx + 1, aln);
  const long long plane = (long long)pitch * (ny + 2);
  const int nxh = nx / 2 + 1, spitch = round_up(nxh, TyOf<double>::v);
  const size_t box_elems = (size_t)plane * (nz + 2) + 2 * (size_t)pitch + 64;
  const NoAllocLayout lay = noalloc_layout(nx, ny, nz, box_elems, (size_t)nz * ny * spitch);
  if (lay.total > ELMM_NOALLOC_SCRATCH_BYTES)
    return fail(ELMM_ERR_INVALID_ARG, "elmm_poisson_solve_noalloc: a " + std::to_string(nx) + "x" + std::to_string(ny) +
                                          "x" + std::to_string(nz) + " grid needs " + std::to_string(lay.total) +
                                          " bytes of scratch, more than the fixed " +
                                          std::to_string((size_t)ELMM_NOALLOC_SCRATCH_BYTES) + " bytes");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev || device >= 64)
    return fail(ELMM_ERR_INVALID_ARG, "no CUDA device " + std::to_string(device));
  KeepDevice keep;
  CU(cudaSetDevice(device));
  NoAllocDev nd;
  if ((r = noalloc_setup(device, &nd))) return r;
  unsigned char *base = nd.base;
  const size_t smem_x = sizeof(double2) * 2 * (kRowsX / 2) * nx, smem_y = sizeof(double2) * 2 * TyOf<double>::v * ny;
  const int zper = bcs[ELMM_BO] == ELMM_BC_PERIODIC;
  const size_t smem_tri = sizeof(double) * kTriThreads * nz * (zper ? 2 : 1);
  const size_t optin = (size_t)nd.optin;
  if (smem_x > optin || smem_y > optin || smem_tri > optin)
    return fail(ELMM_ERR_INVALID_CONFIG, "grid too large for the shared-memory transforms");

  Dom<double> h;
  memset(&h, 0, sizeof(h));
  h.nx = nx; h.ny = ny; h.nz = nz;
  h.aln = aln; h.pitch = pitch; h.plane = plane;
  for (int s = 0; s < 6; s++) h.bt[s] = bcs[s];
  h.dx = c.dxmin; h.dy = c.dymin; h.dz = c.dzmin;
  h.dt = 1.0;
  h.zper = zper;
  h.nxh = nxh; h.spitch = spitch;
  h.Phi = reinterpret_cast<double *>(base + lay.box);
  h.S = reinterpret_cast<double2 *>(base + lay.S);
  h.twx = reinterpret_cast<const double2 *>(base + lay.twx);
  h.twy = reinterpret_cast<const double2 *>(base + lay.twy);
  h.lamx = reinterpret_cast<const double *>(base + lay.lamx);
  h.lamy = reinterpret_cast<const double *>(base + lay.lamy);
  h.Ab = reinterpret_cast<const double *>(base + lay.Ab);
  h.At = reinterpret_cast<const double *>(base + lay.At);
  h.dzc = reinterpret_cast<const double *>(base + lay.dzc);
  h.dzf = reinterpret_cast<const double *>(base + lay.dzf);
  PoisPlan pl;
  factorize(nx, pl.fx);
  factorize(ny, pl.fy);
  const Dom<double> *ddom = reinterpret_cast<const Dom<double> *>(base + lay.dom);
  const PoisPlan *dplan = reinterpret_cast<const PoisPlan *>(base + lay.plan);
  const int *starts = reinterpret_cast<const int *>(base + lay.starts);
  int *bad = reinterpret_cast<int *>(base + lay.bad);
  const int nsm = nd.nsm;
  auto blocks = [&](const void *f, int threads, size_t smem, int total) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, threads, smem) != cudaSuccess || b < 1) b = 1;
    return std::max(1, std::min(total, b * nsm));
  };
  const Launch rows{starts, 1, (ny * nz + kRowsX - 1) / kRowsX};
  const Launch ycols{starts, 1, ((nxh + TyOf<double>::v - 1) / TyOf<double>::v) * nz};
  const Launch tri{starts, 1, (ny * spitch + kTriThreads - 1) / kTriThreads};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int gset = std::max(1, std::min(64, (std::max(std::max(nx, ny), nz + 2) + 255) / 256));
  k_noalloc_setup<<<gset, 256, 0, st>>>(h, pl, lay, base);
  // `bad` counts non-finite right-hand-side values; this asynchronous entry
  // point never reads it back (it would have to synchronise), so non-finite
  // input is not reported, as the header states
  k_unpack<double><<<256, 256, 0, st>>>(ddom, h.Phi, RHS, HostBox{0, nx + 2, ny + 2, nz + 2}, nx, ny, nz, bad);
  k_fftx_fwd<double><<<blocks((const void *)k_fftx_fwd<double>, kFFTThreads, smem_x, rows.total), kFFTThreads, smem_x,
                       st>>>(ddom, rows, dplan, 1.0, 0, 1, 0);
  const int gy = blocks((const void *)k_ffty<double>, kFFTThreads, smem_y, ycols.total);
  k_ffty<double><<<gy, kFFTThreads, smem_y, st>>>(ddom, ycols, dplan, 0, 0);
  k_tri<double><<<blocks((const void *)k_tri<double>, kTriThreads, smem_tri, tri.total), kTriThreads, smem_tri, st>>>(
      ddom, tri, 0);
  k_ffty<double><<<gy, kFFTThreads, smem_y, st>>>(ddom, ycols, dplan, 1, 0);
  k_fftx_inv<double><<<blocks((const void *)k_fftx_inv<double>, kFFTThreads, smem_x, rows.total), kFFTThreads, smem_x,
                       st>>>(ddom, rows, dplan, 0);
  k_pack_scalar<double><<<256, 256, 0, st>>>(ddom, h.Phi, Phi, HostBox{-1, nx + 4, ny + 4, nz + 4}, 0, 0, nx, ny, nz);
  CU(cudaGetLastError());
  return ELMM_OK;
}
