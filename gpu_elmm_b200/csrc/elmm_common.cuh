// elmm_common.cuh -- device-side data layout of one ELMM domain on the B200.
//
// Every field of a domain lives in one "box" that covers the pressure grid
// plus a one-cell shell of ghost cells, i in [0, Prnx+1], j in [0, Prny+1],
// k in [0, Prnz+1], x contiguous.  The first interior column (i = 1) is
// aligned to 128 bytes, so a warp that reads 32 consecutive interior cells of
// a row touches whole 32-byte sectors.  The second-order stencils of the
// reference (advection.f90, subgrid.f90, momentum_diffusion.f90, pressure.f90)
// read at most one cell beyond the interior, so one ghost layer suffices;
// the three-deep ghost layers of the reference's host arrays are produced
// only when a field is copied back to the host.
//
// Staggered components use the same box with their own extents:
// U(1:Unx,1:Uny,1:Unz) etc. (src/initial.f90:871-896).
#pragma once

#include <cstddef>
#include <cstdint>

#define ELMM_HD __host__ __device__ __forceinline__

namespace elmm {

enum { BC_NOSLIP = 1, BC_FREESLIP = 2, BC_PERIODIC = 3, BC_DIRICHLET = 4, BC_NEUMANN = 5, BC_CONSTFLUX = 6 };
// The z face a slab of a split domain shares with the next slab (never a
// user code): its ghost plane holds the neighbour's plane, copied in by the
// slab exchange, and no kernel folds onto it.
enum { BC_HALO = 9 };
enum { SIDE_WE = 0, SIDE_EA = 1, SIDE_SO = 2, SIDE_NO = 3, SIDE_BO = 4, SIDE_TO = 5 };

// box fields of a domain, the order of the tensor maps
enum { F_U = 0, F_V, F_W, F_U2, F_V2, F_W2, F_US, F_VS, F_WS, F_P, F_NU, F_PHI, F_COUNT };
// tensor-map box shapes: the tile with its one-cell halo, and the tile alone
enum { BOX_WIDE = 0, BOX_NARROW = 1 };

// wall-model face planes: index = comp*6 + side
constexpr int kFaces = 18;

template <typename T> struct Vec2;
template <> struct Vec2<double> { typedef double2 type; };
template <> struct Vec2<float> { typedef float2 type; };

// One transported scalar of ScalarRK3 (src/scalars.f90:233-299): the
// potential temperature or a passive scalar.  Box fields in the layout of
// the velocity boxes.
constexpr int kMaxSlots = 5;    // temperature + ELMM_MAX_SCALARS passive scalars
constexpr int kMaxSources = 8;  // ELMM_MAX_POINT_SOURCES
constexpr int kMaxPuffs = 4;    // ELMM_MAX_PUFFS
constexpr int kMaxPuffVols = 16;  // ELMM_MAX_PUFF_VOLUMES
template <typename T>
struct ScalSlot {
  // three value buffers in rotation: stage s of a step reads buf[(s-1) % 3]
  // and writes buf[s % 3], so the value is in buf[0] again after the third
  // stage and between steps (no copy-back), and one graph serves every step
  T *buf[3];
  T *adv;                // the stage tendency
  int bt[6];             // BC per side (TempBtype / ScalBtype)
  double off;            // the box stores value - off
  // surface flux term of the wall-model points at k = 1 and k = nz:
  // temperature_flux * area_factor (src/scalars.f90:323-327); 0 for the
  // passive scalars and adiabatic walls
  double wflux[2];
  double *acc_xy, *acc_xz;  // time-averaged slices (FP64, [j][i] and [k][i]) or null
  // z sides whose ghost plane holds CommonBase's value (BC_DIRICHLET,
  // BC_NEUMANN, or a non-zero BC_CONSTFLUX the rules of the ghost carry),
  // written by k_scalar_zghost before each stage: [0] the plane below
  // k = 1, [1] the plane above k = nz; zside: the BC value of the side
  int zg[2];
  double zside[2];
  // a slab of a split domain: the second planes beyond its BC_HALO faces
  // (level -1 below, nz + 2 above; the slab exchange fills them after each
  // stage) for the two-deep z stencil of KappaScalar, one plane each in the
  // in-plane layout of a box plane; null elsewhere
  T *h2[2];
};

// Domain descriptor, copied to device memory once at creation.  Coefficients
// are kept in FP64 and converted to the kernel's arithmetic type on use.
template <typename T>
struct Dom {
  typedef typename Vec2<T>::type T2;
  int nx, ny, nz;        // Prnx, Prny, Prnz
  int ext[3][3];         // ext[c][d]: extent of component c (U,V,W) along dim d
  int aln;               // column of i = 1 in a row
  int pitch;             // row pitch in elements
  long long plane;       // plane stride in elements = pitch * (ny + 2)
  int bt[6];             // velocity BC per side
  int vz;                // 1: stretched z (GRID_VARIABLE_Z)
  int wall[6];           // 1: wall-model face planes active for this side
  int sgs;               // 1: Smagorinsky
  int prgx_on, prgy_on;
  double prgx, prgy;
  double dx, dy, dz;     // dxmin, dymin, dzmin
  double xmin, ymin;     // xU(0), yV(0)
  double dt;             // the current step's length (rewritten on the device by k_dt with variable steps)
  double nu_mol, cs;
  // variable time steps (TimeStepLength, src/dynamics.f90:517-548): target
  // CFL, longest step, end time (0: none), the configured dt; tstate on the
  // device holds the time after the last step and that step's length
  int vdt;
  double cfl_target, dt_max, end_time, dt0;
  double *tstate;
  // coefficients computed once on the host as the reference computes them
  // once per call (advection.f90: Ax = 0.25/dxmin etc.; momentum_diffusion.f90:
  // recdxmin2 = 1/dxmin**2)
  double cA[3];          // 0.25 / dxmin, dymin, dzmin
  double cB[3][3];       // advective-form factors of component c: 0.5 along c, 0.125 across
  double rec2[3];        // 1 / dxmin**2, ...
  // fields (box layout)
  T *U, *V, *W, *U2, *V2, *W2, *Us, *Vs, *Ws, *P, *nu, *Phi;
  // spectral data S[k][ky][kx], row pitch spitch (complex elements)
  T2 *S;
  int nxh, spitch;
  // FFT tables: exp(-2 pi i m / n) for m < n, in T
  const T2 *twx, *twy;
  // Poisson tables (FP64): eigenvalues and z-operator rows, index 1..nz
  const double *lamx, *lamy, *Ab, *At, *dzc, *dzf;
  const double *tri_c0;  // [piece][ny * spitch]: carry of the pivot recurrence at each piece start (tiled z solve)
  int zper;
  // grid tables (FP64), index k + 2 for k in [-2, nz + 3]
  const double *zPr, *dzPr, *zW, *dzW;
  const double *width;   // Smagorinsky filter width per k, index k (1..nz)
  // per-k factors of NuSmag (index k, 1..nz): 1/dzPr(k), 1/(2 (zPr(k+1)-zPr(k-1))), (width Cs)^2
  const double *sgs_rdz, *sgs_r2zz, *sgs_wc2;
  // wall model: per face plane fluxp/fluxm/ustar, plane dims from ext[]
  T *wm_fluxp[kFaces], *wm_fluxm[kFaces];
  double *wm_ustar[kFaces];
  // a prescribed surface temperature at a wall-model wall (tdir[side], the
  // value tsurf[side]): the temperature_flux state of the face's velocity
  // points (as wm_ustar), the u* and flux of the Pr points next to the
  // bottom [0] and top [1] per (i, j), and ComputeAreaFactor of the points
  int tdir[6];
  double tsurf[6];
  double *wm_tfl[kFaces];
  double *wm_pr_us[2], *wm_pr_tf[2];
  double wm_af;
  // stretched z, packed FP32 momentum path: per-level factors kz2[q * (nz + 2) + k]
  // (q: kZ2 entries, see elmm_packed.cuh)
  const float *kz2;
  // per component: 1 marks a bottom-plane point without a wall-model point
  // (next to or under a solid body), or null for none
  const unsigned char *bskip[3];
  // solid bodies with passive scalars: per box cell, bit 0 a solid Pr cell
  // (Prtype > 0; x and y ghost images too), bit 1 a Pr wall-model point of
  // the scalar equations; null without bodies or scalars
  const unsigned char *pmask;
  double z0[6];
  // pressure reference: stored P = true Pr + prm; top-layer partial sums
  double *prm;           // 1 value
  double *prpart;        // partial sums of the top layer of P
  int nprpart;
  // Mixed path: U and V are stored as deviations from a per-level offset,
  // value = stored + voff[c * (nz + 2) + k] for c = 0 (U), 1 (V) and k in
  // [0, nz + 1].  With a mean velocity of several m/s, FP32 rounding of the
  // full value leaves noise whose divergence every projection then turns
  // into pressure; the deviations round ~10-50x finer.  The offset is
  // constant over each level, so every x and y difference (divergence,
  // projection, ghost images) works on the stored values unchanged; the
  // ghost levels 0 and nz+1 follow the BoundUVW fold of their source level
  // (odd at a no-slip wall, even at a free-slip one, periodic copies), so a
  // fold of stored values is the fold of full values.  Null on the FP64
  // path; zero on a domain with solid bodies.
  float *voff;
  // diagnostics
  unsigned long long *maxdiv_bits;  // max |div u| as the bits of a positive double
  unsigned long long *cfl_bits;
  int *flags;            // [0]: NaN seen, [1]: a bounded wait gave up
  // the bounded plane waits of k_momentum / k_sgs: tries before giving up,
  // and the plane whose copies are not issued (-1: none; fault injection by
  // elmm_set_fault_injection for tests of the timeout path)
  int wait_limit, skip_plane;
  const void *tmaps;     // CUtensorMap[2][F_COUNT] (device memory, 64-byte aligned)
  const void *tmapT;     // FP32 with buoyancy: CUtensorMap[3], narrow boxes of the temperature's value buffers
  // defect correction of the mixed path
  int *refine_flag;      // 1: the next correction sweep runs for this domain
  int *refine_count;     // sweeps run since the counter was reset
  double refine_tol;
  int max_refine;
  // potential temperature (enable_buoyancy): box fields of the current and
  // the next value, the stage tendency and the diffusivity.  Stored as
  // theta - toff: toff = temperature_ref on the mixed path (FP32 keeps the
  // perturbations' digits), 0 on the FP64 path.
  int buoy;
  int tbt[6];            // temperature BC per side
  T *Tm, *Tadv, *TDiff;
  double toff, tref, grav, kappa_mol;
  // temperature_flux of the wall-model points per side: sideTemp at the
  // bottom, -sideTemp at the top (src/wallmodels.f90:819-827, 870-878)
  double tflux[6];
  // scalar slots of the ScalarRK3 kernel: slot 0 is the temperature when
  // buoy is set (Tm aliases its buf[0], Tadv its tendency), then the passive
  // scalars
  int nslot;
  ScalSlot<T> slot[kMaxSlots];
  int tdiff_live;        // 1: TDiff follows the viscosity every stage (buoyancy)
  // volume sources of the point sources, in the order of the configuration:
  // slot, cell, flux / volume of the cell
  int nsrc;
  int src_slot[kMaxSources], src_i[kMaxSources], src_j[kMaxSources], src_k[kMaxSources];
  double src_q[kMaxSources];
  // puffs (src/puffs.f90): windows and volumes; puff_state on the device holds
  // per puff {last_start, dt_fraction, restart, -} and, after them, the time
  // of the next step
  int npuff, puff_clear_any;
  double puff_start[kMaxPuffs], puff_end[kMaxPuffs], puff_period[kMaxPuffs], puff_dur[kMaxPuffs];
  unsigned puff_clear_slots[kMaxPuffs];  // bit s: slot s is cleared at a release of the puff
  double *puff_state;
  int npv;
  int pv_puff[kMaxPuffVols], pv_slot[kMaxPuffVols], pv_i[kMaxPuffVols], pv_j[kMaxPuffVols], pv_k[kMaxPuffVols];
  double pv_q[kMaxPuffVols];
  // time-averaged slices: plane k, plane j (0: none), weight of one step
  int avg_k, avg_j;
  double avg_w;
};

template <typename T>
ELMM_HD long long bidx(const Dom<T> &d, int i, int j, int k) {
  return (long long)(d.aln - 1 + i) + (long long)d.pitch * (long long)(j + (long long)(d.ny + 2) * k);
}

// ---------------------------------------------------------------- BC folds
// Ghost cell g of a velocity component along one dimension (n = extent of
// the component, `normal` = the component points along this dimension).
// Rules of BoundUVW_do_BC (src/boundaries.f90:398-1791); the sequential
// x, y, z passes of that routine make the three dimensions independent.
struct Fold {
  int src;    // source index in [1, n]
  int sign;   // +1 / -1
  int zero;   // 1: the ghost is a constant 0
};

ELMM_HD Fold fold_vel(int g, int n, int blo, int bhi, bool normal) {
  Fold f{g, 1, 0};
  if (g >= 1 && g <= n) return f;
  if (g < 1) {
    switch (blo) {
      case BC_PERIODIC: f.src = n + g; break;
      case BC_NOSLIP:
        if (normal) { if (g == 0) { f.src = 1; f.zero = 1; } else { f.src = -g; f.sign = -1; } }
        else { f.src = 1 - g; f.sign = -1; }
        break;
      case BC_FREESLIP:
        if (normal) { if (g == 0) { f.src = 1; f.zero = 1; } else { f.src = -g; f.sign = -1; } }
        else f.src = 1;
        break;
      case BC_HALO: f.src = 0; break;  // the exchanged plane (deeper ghosts clamp onto it)
      default: f.src = 1; break;  // NEUMANN
    }
  } else {
    switch (bhi) {
      case BC_PERIODIC: f.src = g - n; break;
      case BC_NOSLIP:
        if (normal) { if (g == n + 1) { f.src = n; f.zero = 1; } else { f.src = 2 * n + 2 - g; f.sign = -1; } }
        else { f.src = 2 * n + 1 - g; f.sign = -1; }
        break;
      case BC_FREESLIP:
        if (normal) { if (g == n + 1) { f.src = n; f.zero = 1; } else { f.src = 2 * n + 2 - g; f.sign = -1; } }
        else f.src = n;
        break;
      case BC_HALO: f.src = n + 1; break;
      default: f.src = n; break;
    }
  }
  return f;
}

// whether z index k of a field with n interior levels lies in the ghost
// plane of a slab face (filled by the exchange, skipped by the ghost passes)
ELMM_HD bool halo_plane(int k, int n, const int *bt) {
  return (k < 1 && bt[4] == BC_HALO) || (k > n && bt[5] == BC_HALO);
}

// Ghosts of Viscosity (BoundViscosity, src/scalarboundaries.f90:326-431) and
// of Phi one cell deep (Bound_Phi, src/boundaries.f90:1817-1948): periodic
// copy, otherwise a copy of the adjacent interior cell.
ELMM_HD int fold_rep(int g, int n, bool periodic) {
  if (g >= 1 && g <= n) return g;
  if (periodic) return g < 1 ? n + g : g - n;
  return g < 1 ? 1 : n;
}

// The ghost images of interior index t along one dimension for a one-deep
// shell: the producer of cell t also writes the ghosts that fold onto it.
// Only t == 1 and t == n can have images; fixed slots keep everything in
// registers.
struct Images {
  int t, n1;            // the index itself and the hi ghost index n + 1
  int lo_ok, hi_ok;     // ghost 0 / ghost n+1 fold onto t
  int lo_sign, hi_sign;
  int lo_zero, hi_zero; // the ghost is a constant 0 written by this cell
};

ELMM_HD Images images_none(int t, int n) { return Images{t, n + 1, 0, 0, 1, 1, 0, 0}; }

ELMM_HD Images images_vel(int t, int n, int blo, int bhi, bool normal) {
  Images im = images_none(t, n);
  if (t != 1 && t != n) return im;
  Fold lo = fold_vel(0, n, blo, bhi, normal);
  if (lo.zero ? (t == 1) : (lo.src == t)) { im.lo_ok = 1; im.lo_sign = lo.zero ? 1 : lo.sign; im.lo_zero = lo.zero; }
  Fold hi = fold_vel(n + 1, n, blo, bhi, normal);
  if (hi.zero ? (t == n) : (hi.src == t)) { im.hi_ok = 1; im.hi_sign = hi.zero ? 1 : hi.sign; im.hi_zero = hi.zero; }
  return im;
}

ELMM_HD Images images_rep(int t, int n, bool periodic) {
  Images im = images_none(t, n);
  if (fold_rep(0, n, periodic) == t) im.lo_ok = 1;
  if (fold_rep(n + 1, n, periodic) == t) im.hi_ok = 1;
  return im;
}

// Only periodic copies (pressure: its non-periodic ghosts are never read by
// the second-order kernels).
ELMM_HD Images images_per(int t, int n, bool periodic) {
  Images im = images_none(t, n);
  if (periodic) { im.lo_ok = (t == n); im.hi_ok = (t == 1); }
  return im;
}

// Writes value v of interior cell (i,j,k) to all of its ghost images.
template <typename T>
__device__ __forceinline__ void push_ghosts(const Dom<T> &d, T *F, const Images &ix, const Images &iy,
                                            const Images &iz, T v) {
  if (!(ix.lo_ok | ix.hi_ok | iy.lo_ok | iy.hi_ok | iz.lo_ok | iz.hi_ok)) return;
  const int xi[3] = {ix.t, 0, ix.n1}, yi[3] = {iy.t, 0, iy.n1}, zi[3] = {iz.t, 0, iz.n1};
  const int xo[3] = {1, ix.lo_ok, ix.hi_ok}, yo[3] = {1, iy.lo_ok, iy.hi_ok}, zo[3] = {1, iz.lo_ok, iz.hi_ok};
  const int xs[3] = {1, ix.lo_sign, ix.hi_sign}, ys[3] = {1, iy.lo_sign, iy.hi_sign}, zs[3] = {1, iz.lo_sign, iz.hi_sign};
  const int xz[3] = {0, ix.lo_zero, ix.hi_zero}, yz[3] = {0, iy.lo_zero, iy.hi_zero}, zz[3] = {0, iz.lo_zero, iz.hi_zero};
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int b = 0; b < 3; b++)
#pragma unroll
      for (int a = 0; a < 3; a++) {
        if (a == 0 && b == 0 && c == 0) continue;
        if (!(xo[a] && yo[b] && zo[c])) continue;
        const int s = xs[a] * ys[b] * zs[c];
        const bool z = xz[a] | yz[b] | zz[c];
        const T w = z ? T(0) : (s > 0 ? v : -v);
        F[bidx(d, xi[a], yi[b], zi[c])] = w;
      }
}

template <typename T>
__device__ __forceinline__ void push_vel(const Dom<T> &d, T *F, int comp, int i, int j, int k, T v) {
  // cells off every face of the box have no ghost images (the extents of a
  // component are nx-1..nx etc., so i in [2, nx-2] is interior for all)
  if (i > 1 && i < d.nx - 1 && j > 1 && j < d.ny - 1 && k > 1 && k < d.nz - 1) return;
  const int *e = d.ext[comp];
  if (i != 1 && i != e[0] && j != 1 && j != e[1] && k != 1 && k != e[2]) return;
  Images ix = images_vel(i, e[0], d.bt[0], d.bt[1], comp == 0);
  Images iy = images_vel(j, e[1], d.bt[2], d.bt[3], comp == 1);
  Images iz = images_vel(k, e[2], d.bt[4], d.bt[5], comp == 2);
  push_ghosts(d, F, ix, iy, iz, v);
}

// Velocity component comp at any index of its one-deep shell, read from the
// interior: a ghost index folds onto its source by the BoundUVW rules.
// Kernels use it for the few neighbours on a box face instead of relying on
// the device ghost cells.
template <typename T>
__device__ __forceinline__ T vel_folded(const Dom<T> &d, const T *F, int comp, int i, int j, int k) {
  const int *e = d.ext[comp];
  const Fold fx = fold_vel(i, e[0], d.bt[0], d.bt[1], comp == 0);
  const Fold fy = fold_vel(j, e[1], d.bt[2], d.bt[3], comp == 1);
  const Fold fz = fold_vel(k, e[2], d.bt[4], d.bt[5], comp == 2);
  if (fx.zero | fy.zero | fz.zero) return (T)0;
  const T v = __ldg(F + bidx(d, fx.src, fy.src, fz.src));
  return fx.sign * fy.sign * fz.sign < 0 ? -v : v;
}

// The offset of velocity component c (0: U, 1: V, 2: W, which has none) at
// level k in [0, nz + 1]; zero on the FP64 path.
template <typename T>
__device__ __forceinline__ T vel_off(const Dom<T> &d, int c, int k) {
  if constexpr (sizeof(T) == 4) {
    return c < 2 ? __ldg(d.voff + c * (d.nz + 2) + k) : 0.f;
  } else {
    return (T)0;
  }
}

// Domain lookup of a flattened tile index (batched launches).
__device__ __forceinline__ int find_dom(const int *starts, int nd, int t) {
  int lo = 0, hi = nd - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(starts + mid) <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

}  // namespace elmm
