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

enum { BC_NOSLIP = 1, BC_FREESLIP = 2, BC_PERIODIC = 3, BC_NEUMANN = 5 };
enum { SIDE_WE = 0, SIDE_EA = 1, SIDE_SO = 2, SIDE_NO = 3, SIDE_BO = 4, SIDE_TO = 5 };

// wall-model face planes: index = comp*6 + side
constexpr int kFaces = 18;

template <typename T> struct Vec2;
template <> struct Vec2<double> { typedef double2 type; };
template <> struct Vec2<float> { typedef float2 type; };

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
  double dt;
  double nu_mol, cs;
  // fields (box layout)
  T *U, *V, *W, *U2, *V2, *W2, *Us, *Vs, *Ws, *P, *nu, *Phi;
  // spectral data S[k][ky][kx], row pitch spitch (complex elements)
  T2 *S;
  int nxh, spitch;
  // FFT tables: exp(-2 pi i m / n) for m < n, in T
  const T2 *twx, *twy;
  // Poisson tables (FP64): eigenvalues and z-operator rows, index 1..nz
  const double *lamx, *lamy, *Ab, *At, *dzc, *dzf;
  int zper;
  // grid tables (FP64), index k + 2 for k in [-2, nz + 3]
  const double *zPr, *dzPr, *zW, *dzW;
  const double *width;   // Smagorinsky filter width per k, index k (1..nz)
  // wall model: per face plane fluxp/fluxm/ustar, plane dims from ext[]
  T *wm_fluxp[kFaces], *wm_fluxm[kFaces];
  double *wm_ustar[kFaces];
  double z0[6];
  // pressure reference: stored P = true Pr + prm; top-layer partial sums
  double *prm;           // 1 value
  double *prpart;        // partial sums of the top layer of P
  int nprpart;
  // diagnostics
  unsigned long long *maxdiv_bits;  // max |div u| as the bits of a positive double
  unsigned long long *cfl_bits;
  int *flags;            // [0]: NaN seen
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
      default: f.src = n; break;
    }
  }
  return f;
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
struct Images {
  int n;
  int idx[3];
  int sign[3];
  int zero[3];
};

ELMM_HD Images images_vel(int t, int n, int blo, int bhi, bool normal) {
  Images im;
  im.n = 1; im.idx[0] = t; im.sign[0] = 1; im.zero[0] = 0;
  Fold lo = fold_vel(0, n, blo, bhi, normal);
  if (lo.zero ? (t == 1) : (lo.src == t)) {
    im.idx[im.n] = 0; im.sign[im.n] = lo.zero ? 1 : lo.sign; im.zero[im.n] = lo.zero; im.n++;
  }
  Fold hi = fold_vel(n + 1, n, blo, bhi, normal);
  if (hi.zero ? (t == n) : (hi.src == t)) {
    im.idx[im.n] = n + 1; im.sign[im.n] = hi.zero ? 1 : hi.sign; im.zero[im.n] = hi.zero; im.n++;
  }
  return im;
}

ELMM_HD Images images_rep(int t, int n, bool periodic) {
  Images im;
  im.n = 1; im.idx[0] = t; im.sign[0] = 1; im.zero[0] = 0;
  if (fold_rep(0, n, periodic) == t) { im.idx[im.n] = 0; im.sign[im.n] = 1; im.zero[im.n] = 0; im.n++; }
  if (fold_rep(n + 1, n, periodic) == t) { im.idx[im.n] = n + 1; im.sign[im.n] = 1; im.zero[im.n] = 0; im.n++; }
  return im;
}

// Only periodic copies (pressure: its non-periodic ghosts are never read by
// the second-order kernels).
ELMM_HD Images images_per(int t, int n, bool periodic) {
  Images im;
  im.n = 1; im.idx[0] = t; im.sign[0] = 1; im.zero[0] = 0;
  if (periodic) {
    if (t == n) { im.idx[im.n] = 0; im.sign[im.n] = 1; im.zero[im.n] = 0; im.n++; }
    if (t == 1) { im.idx[im.n] = n + 1; im.sign[im.n] = 1; im.zero[im.n] = 0; im.n++; }
  }
  return im;
}

// Writes value v of interior cell (i,j,k) to all of its ghost images.
template <typename T>
__device__ __forceinline__ void push_ghosts(const Dom<T> &d, T *F, const Images &ix, const Images &iy,
                                            const Images &iz, T v) {
  if (ix.n == 1 && iy.n == 1 && iz.n == 1) return;
  for (int c = 0; c < iz.n; c++)
    for (int b = 0; b < iy.n; b++)
      for (int a = 0; a < ix.n; a++) {
        if (a == 0 && b == 0 && c == 0) continue;
        int s = ix.sign[a] * iy.sign[b] * iz.sign[c];
        bool z = ix.zero[a] | iy.zero[b] | iz.zero[c];
        T w = z ? T(0) : (s > 0 ? v : -v);
        F[bidx(d, ix.idx[a], iy.idx[b], iz.idx[c])] = w;
      }
}

template <typename T>
__device__ __forceinline__ void push_vel(const Dom<T> &d, T *F, int comp, int i, int j, int k, T v) {
  const int *e = d.ext[comp];
  Images ix = images_vel(i, e[0], d.bt[0], d.bt[1], comp == 0);
  Images iy = images_vel(j, e[1], d.bt[2], d.bt[3], comp == 1);
  Images iz = images_vel(k, e[2], d.bt[4], d.bt[5], comp == 2);
  push_ghosts(d, F, ix, iy, iz, v);
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

// Order-preserving bits of a non-negative double for atomicMax.
__device__ __forceinline__ void atomic_max_pos(unsigned long long *a, double v) {
  if (!(v >= 0)) v = __longlong_as_double(0x7ff8000000000000ULL);  // NaN wins
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

}  // namespace elmm
