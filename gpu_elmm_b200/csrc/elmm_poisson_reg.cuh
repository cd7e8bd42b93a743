// elmm_poisson_reg.cuh -- the transforms and the z solve of the Poisson
// problem (src/poisson.f90:23-60, the PoisFFT replacement) for the common
// case: x and y lengths with a register FFT (ELMM_FFT_SIZES) and a
// non-periodic z axis of at most kTriTileMaxNz cells.  Other grids use the
// generic kernels of elmm_kernels.cuh / elmm_kernels2.cuh; both compute the
// same discrete solution.
#pragma once

#include "elmm_fftreg.cuh"
#include "elmm_stream.cuh"

namespace elmm {

constexpr int kRegThreads = 256;
// resident blocks per SM the x-transform kernels are compiled for: for up to
// 16 elements per thread three (FP32, 80 registers) or two (FP64, 128
// registers) fit without spills; longer FP32 sequences (24 elements: lengths
// 192, 384) two blocks of 128 registers, faster than one block of ~200 (the
// y transform of those lengths spills at 128 and keeps the compiler's choice)
template <typename T, int N>
constexpr int fft_reg_min_blocks() { return N / fplan_P(N) <= 16 ? (sizeof(T) == 4 ? 3 : 2) : (sizeof(T) == 4 ? 2 : 1); }
// the forward x transform (with the fused divergence) of FP32 lengths up to
// 16 elements per thread: four resident blocks (64 registers) measured
// faster than three (0.050 -> 0.043 ms at 256 x 256 x 128); the inverse
// keeps three
template <typename T, int N>
constexpr int fft_reg_min_blocks_fwd() { return N / fplan_P(N) <= 16 && sizeof(T) == 4 ? 4 : fft_reg_min_blocks<T, N>(); }

// The reads of the divergence stencil of one x row (j, k) of the x
// transforms.  Away from the box faces the neighbours are the adjacent box
// cells; on a face a neighbour folds onto an interior cell as BoundUVW fills
// the ghost, so each read is scale * F[c + offset] with scale in {1, -1, 0}
// (exact).  x and y are periodic (the FFT solve requires it), so only the
// i = 0 column folds in x.
template <typename T>
struct RhsRow {
  long long o_uw1, o_vs, o_wc, o_wb;  // offsets: U2 at i - 1 for i = 1, V2 at j - 1, W2 at k, W2 at k - 1
  T s_uw1, s_vs, s_wc, s_wb;
};

template <typename T>
__device__ __forceinline__ RhsRow<T> rhs_row(const Dom<T> &d, int j, int k) {
  RhsRow<T> r;
  const long long pitch = d.pitch, plane = d.plane;
  auto fold = [&](int comp, int axis, int g, long long stride, long long &off, T &scale) {
    const int *e = d.ext[comp];
    const Fold f = fold_vel(g, e[axis], d.bt[2 * axis], d.bt[2 * axis + 1], comp == axis);
    const int own = axis == 0 ? 1 : axis == 1 ? j : k;  // the interior index the row itself sits at
    off = f.zero ? 0 : (long long)(f.src - own) * stride;
    scale = f.zero ? (T)0 : (T)f.sign;
  };
  fold(0, 0, 0, 1, r.o_uw1, r.s_uw1);
  fold(1, 1, j - 1, pitch, r.o_vs, r.s_vs);
  fold(2, 2, k, plane, r.o_wc, r.s_wc);
  fold(2, 2, k - 1, plane, r.o_wb, r.s_wb);
  return r;
}

// right-hand side at interior cell i of a row, box index c: the divergence
// of (U2, V2, W2) / coef, or the value already stored in Phi (PoisSolver
// interface, defect correction)
template <typename T>
__device__ __forceinline__ T poisson_rhs(const Dom<T> &d, const RhsRow<T> &r, long long c, int i, T rdx, T rdy,
                                         T rdzk, T rdt2, int rhs_from_phi) {
  if (rhs_from_phi) return ld((const T *)d.Phi, c) * rdt2;
  const T *U2 = d.U2, *V2 = d.V2, *W2 = d.W2;
  const long long ouw = i == 1 ? r.o_uw1 : -1;
  const T suw = i == 1 ? r.s_uw1 : (T)1;
  const T uc = ld(U2, c), uw = suw * ld(U2, c + ouw);
  const T vc = ld(V2, c), vs = r.s_vs * ld(V2, c + r.o_vs);
  const T wc = r.s_wc * ld(W2, c + r.o_wc), wb = r.s_wb * ld(W2, c + r.o_wb);
  const T div = (uc - uw) * rdx + (vc - vs) * rdy + (wc - wb) * rdzk;
  return div * rdt2;
}

// ------------------------------------------------------------ x forward
// 16-byte vectors of a row: four floats or two doubles (rows start on a
// 128-byte boundary and every register-FFT length is a multiple of 16)
template <typename T> struct Row16;
template <> struct Row16<float> {
  static constexpr int n = 4;
  static __device__ __forceinline__ void ld(const float *p, float (&v)[4]) {
    const float4 q = __ldg(reinterpret_cast<const float4 *>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
  }
};
template <> struct Row16<double> {
  static constexpr int n = 2;
  static __device__ __forceinline__ void ld(const double *p, double (&v)[2]) {
    const double2 q = __ldg(reinterpret_cast<const double2 *>(p));
    v[0] = q.x; v[1] = q.y;
  }
};

// Divergence + real FFT along x of 2 * NS rows (two real rows per complex
// sequence), split into the half spectra of the two rows: S[row][0..nx/2].
// The divergence is formed from 16-byte row vectors (a thread takes one
// chunk of both rows of a sequence) into shared memory, from where each FFT
// thread picks its strided elements; the arithmetic per cell is that of
// poisson_rhs.
template <typename T, int N>
__device__ __forceinline__ void fftx_fwd_tile(const Dom<T> &d, int lt, typename Vec2<T>::type *smem, double coef,
                                              int rhs_from_phi) {
  typedef typename Vec2<T>::type T2;
  typedef FPlan<N> Pl;
  typedef Row16<T> RV;
  constexpr int P = Pl::P, E = Pl::E, NS = kRegThreads / P;
  constexpr int VE = RV::n, NCH = N / VE;
  __shared__ RhsRow<T> rinfo[2 * NS];
  const int s = threadIdx.x / P, t = threadIdx.x - s * P;
  const int ny = d.ny, nrows = ny * d.nz;
  const int r0 = 2 * lt * NS;  // first row of the tile; sequence q holds rows r0 + 2q, r0 + 2q + 1
  const T rdt2 = (T)(1.0 / coef);
  const T rdx = (T)(1.0 / d.dx), rdy = (T)(1.0 / d.dy), rdz = (T)(1.0 / d.dz);
  if (threadIdx.x < 2 * NS) {
    const int q = min(r0 + (int)threadIdx.x, nrows - 1);
    const int k = q / ny + 1;
    rinfo[threadIdx.x] = rhs_row(d, q - (k - 1) * ny + 1, k);
  }
  __syncthreads();
  for (int task = threadIdx.x; task < NS * NCH; task += kRegThreads) {
    const int sq = task / NCH, c = task - sq * NCH;
    T va[VE], vb[VE];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      T *out = h ? vb : va;
      const int q = r0 + 2 * sq + h;
#pragma unroll
      for (int e = 0; e < VE; e++) out[e] = (T)0;
      if (q >= nrows) continue;  // rows past the end are not read
      const int k = q / ny + 1, j = q - (k - 1) * ny + 1;
      const long long c0 = bidx(d, 1, j, k) + (long long)c * VE;
      if (rhs_from_phi) {
        T p[VE];
        RV::ld(d.Phi + c0, p);
#pragma unroll
        for (int e = 0; e < VE; e++) out[e] = p[e] * rdt2;
        continue;
      }
      const RhsRow<T> &r = rinfo[2 * sq + h];
      const T rdzk = d.vz ? (T)d.sgs_rdz[k] : rdz;
      T uc[VE], vc[VE], vs[VE], wc[VE], wb[VE];
      RV::ld(d.U2 + c0, uc);
      RV::ld(d.V2 + c0, vc);
      RV::ld(d.V2 + c0 + r.o_vs, vs);
      RV::ld(d.W2 + c0 + r.o_wc, wc);
      RV::ld(d.W2 + c0 + r.o_wb, wb);
      const T uw0 = c == 0 ? r.s_uw1 * ld((const T *)d.U2, c0 + r.o_uw1) : ld((const T *)d.U2, c0 - 1);
#pragma unroll
      for (int e = 0; e < VE; e++) {
        const T uw = e == 0 ? uw0 : uc[e - 1];
        const T vse = r.s_vs * vs[e];
        const T wce = r.s_wc * wc[e], wbe = r.s_wb * wb[e];
        const T div = (uc[e] - uw) * rdx + (vc[e] - vse) * rdy + (wce - wbe) * rdzk;
        out[e] = div * rdt2;
      }
    }
    T2 *dst = smem + sq * Pl::SEQ + c * VE;
#pragma unroll
    for (int e = 0; e < VE; e++) dst[e] = T2{va[e], vb[e]};
  }
  __syncthreads();
  T2 *sh = smem + s * Pl::SEQ;
  T2 v[E];
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = sh[t + P * e];
  __syncthreads();  // fft_reg writes sh
  fft_reg<T, T2, N, false>(v, sh, t, d.twx);
  // Z = FFT(a + i b): A_m = (Z_m + conj Z_{N-m}) / 2, B_m = (Z_m - conj Z_{N-m}) / 2i
  const int ra = r0 + 2 * s, rb = ra + 1;
  const bool va_ok = ra < nrows, vb_ok = rb < nrows;
  constexpr int nxh = N / 2 + 1;
  T2 *Sa = d.S + (long long)(va_ok ? ra : 0) * d.spitch, *Sb = d.S + (long long)(vb_ok ? rb : 0) * d.spitch;
#pragma unroll
  for (int m = t; m < nxh; m += P) {
    const T2 zk = sh[m], zc = sh[m == 0 ? 0 : N - m];
    T2 A, B;
    A.x = (zk.x + zc.x) * (T)0.5;
    A.y = (zk.y - zc.y) * (T)0.5;
    B.x = (zk.y + zc.y) * (T)0.5;
    B.y = (zc.x - zk.x) * (T)0.5;
    if (va_ok) Sa[m] = A;
    if (vb_ok) Sb[m] = B;
  }
  __syncthreads();  // the next tile reuses sh and rinfo
}

// One launch per x length N: the launch set holds only the domains with
// nx == N.
template <typename T, int N>
__global__ void __launch_bounds__(kRegThreads, fft_reg_min_blocks_fwd<T, N>()) k_fftx_fwd_reg(const Dom<T> *__restrict__ doms, Launch L,
                                                              double coef_alpha2, int use_dt, int rhs_from_phi,
                                                              int gate) {
  typedef typename Vec2<T>::type T2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T2 *sm = reinterpret_cast<T2 *>(smem_raw);
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    if (gate && !*d.refine_flag) continue;
    const double coef = use_dt ? coef_alpha2 * d.dt : coef_alpha2;
    fftx_fwd_tile<T, N>(d, t - __ldg(L.starts + di), sm, coef, rhs_from_phi);
  }
}

// --------------------------------------------------------------- y (both)
// Complex FFT along y of C = kRegThreads / P consecutive kx columns of one
// k plane of S, in place.
template <typename T, int N, bool INV>
__device__ __forceinline__ void ffty_tile(const Dom<T> &d, int lt, typename Vec2<T>::type *smem) {
  typedef typename Vec2<T>::type T2;
  typedef FPlan<N> Pl;
  constexpr int P = Pl::P, E = Pl::E, C = kRegThreads / P;
  const int c = threadIdx.x % C, t = threadIdx.x / C;
  const int nxh = d.nxh, ncx = (nxh + C - 1) / C;
  const int k = lt / ncx, kx = (lt - k * ncx) * C + c;
  const bool ok = kx < nxh;
  const long long sp = d.spitch;
  T2 *S = d.S + (long long)k * N * sp + kx;
  T2 v[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    if (ok) v[e] = S[(long long)(t + P * e) * sp];
    else { v[e].x = 0; v[e].y = 0; }
  }
  T2 *sh = smem + c * Pl::SEQ;
  fft_reg<T, T2, N, INV>(v, sh, t, d.twy);
#pragma unroll
  for (int e = 0; e < E; e++)
    if (ok) S[(long long)(t + P * e) * sp] = sh[t + P * e];
  __syncthreads();
}

template <typename T, int N, bool INV>
__global__ void __launch_bounds__(kRegThreads) k_ffty_reg(const Dom<T> *__restrict__ doms, Launch L, int gate) {
  typedef typename Vec2<T>::type T2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T2 *sm = reinterpret_cast<T2 *>(smem_raw);
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    if (gate && !*d.refine_flag) continue;
    ffty_tile<T, N, INV>(d, t - __ldg(L.starts + di), sm);
  }
}

// ------------------------------------------------------------ x inverse
// Two rows per complex sequence: Z_m = A_m + i B_m with the Hermitian
// completion A_{N-m} = conj(A_m); the real and imaginary parts of the
// inverse transform are the two rows of Phi (interior only).
template <typename T, int N>
__device__ __forceinline__ void fftx_inv_tile(const Dom<T> &d, int lt, typename Vec2<T>::type *smem) {
  typedef typename Vec2<T>::type T2;
  typedef FPlan<N> Pl;
  constexpr int P = Pl::P, E = Pl::E, NS = kRegThreads / P;
  constexpr int nxh = N / 2 + 1;
  const int s = threadIdx.x / P, t = threadIdx.x - s * P;
  const int ny = d.ny, nrows = ny * d.nz;
  const int ra = 2 * (lt * NS + s), rb = ra + 1;
  const bool va = ra < nrows, vb = rb < nrows;
  const int qa = va ? ra : 0, qb = vb ? rb : 0;  // rows past the end are not read
  const T2 *Sa = d.S + (long long)qa * d.spitch, *Sb = d.S + (long long)qb * d.spitch;
  T2 v[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int m = t + P * e;
    const int mm = m < nxh ? m : N - m;
    T2 A, B;
    A.x = 0; A.y = 0; B.x = 0; B.y = 0;
    if (va) A = Sa[mm];
    if (vb) B = Sb[mm];
    if (mm == 0 || 2 * mm == N) { A.y = 0; B.y = 0; }
    if (m >= nxh) { A.y = -A.y; B.y = -B.y; }
    v[e].x = A.x - B.y;
    v[e].y = A.y + B.x;
  }
  T2 *sh = smem + s * Pl::SEQ;
  fft_reg<T, T2, N, true>(v, sh, t, d.twx);
  const int ka = qa / ny + 1, kb = qb / ny + 1;
  T *Pa = d.Phi + bidx(d, 1, qa - (ka - 1) * ny + 1, ka), *Pb = d.Phi + bidx(d, 1, qb - (kb - 1) * ny + 1, kb);
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int i0 = t + P * e;
    const T2 z = sh[i0];
    if (va) Pa[i0] = z.x;
    if (vb) Pb[i0] = z.y;
  }
  __syncthreads();
}

template <typename T, int N>
__global__ void __launch_bounds__(kRegThreads, fft_reg_min_blocks<T, N>()) k_fftx_inv_reg(const Dom<T> *__restrict__ doms, Launch L, int gate) {
  typedef typename Vec2<T>::type T2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T2 *sm = reinterpret_cast<T2 *>(smem_raw);
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    if (gate && !*d.refine_flag) continue;
    fftx_inv_tile<T, N>(d, t - __ldg(L.starts + di), sm);
  }
}

// The kernels of one length, for the host's dispatch table.
template <typename T>
struct FFTRegKernels {
  int n;
  void (*fwd)(const Dom<T> *, Launch, double, int, int, int);
  void (*inv)(const Dom<T> *, Launch, int);
  void (*yf)(const Dom<T> *, Launch, int);
  void (*yi)(const Dom<T> *, Launch, int);
};

template <typename T>
inline const FFTRegKernels<T> *fft_reg_kernels(int n) {
#define ELMM_REG_ENTRY(n_) {n_, k_fftx_fwd_reg<T, n_>, k_fftx_inv_reg<T, n_>, k_ffty_reg<T, n_, false>, k_ffty_reg<T, n_, true>},
  static const FFTRegKernels<T> table[] = {ELMM_FFT_SIZES(ELMM_REG_ENTRY)};
#undef ELMM_REG_ENTRY
  for (const auto &e : table)
    if (e.n == n) return &e;
  return nullptr;
}

// sequences (x) or columns (y) one block of the register kernels handles
__host__ __device__ constexpr int fft_reg_batch(int n) { return kRegThreads / fplan_P(n); }

// ------------------------------------------------- tiled tridiagonal solve
// The z solve of every (kx, ky) mode (Thomas algorithm, non-periodic z) for
// kTriCols consecutive spectral columns.  The pivots of the forward sweep
// depend on the grid only: k_tri_factors stores, once per domain, the pivot
// recurrence's carry at the first level of each segment, from which the
// tile rebuilds the reciprocals iv(k) of its segment in shared memory (the
// same operations, so the same values).  With them both sweeps are first-order linear
// recurrences,
//   forward   y(k) = r(k) iv(k) - Ab(k) iv(k) y(k-1),
//   backward  x(k) = y(k) - At(k) iv(k) x(k+1),
// which a block solves for the real and imaginary part of each column with
// kTriSegs threads per part: each thread composes the affine map of its
// segment of k, the segment maps are chained through shared memory, and each
// thread then replays its segment from the exact entry value.  The tile of S
// is copied into shared memory with cp.async (while the pivots are rebuilt)
// and written back at the end.  The (0,0) mode is the zero-mean prefix-sum solution of
// the generic kernel, k_tri.
#ifndef ELMM_TRI_COLS
#define ELMM_TRI_COLS 16
#endif
#ifndef ELMM_TRI_SEGS
#define ELMM_TRI_SEGS 8
#endif
constexpr int kTriCols = ELMM_TRI_COLS;
constexpr int kTriSegs = ELMM_TRI_SEGS;
constexpr int kTriTileMaxNz = 256;

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// tile of S, reciprocal pivots, and the (A, B) maps of the segments, for a
// tile of COLS spectral columns
template <typename T, int COLS = kTriCols>
__host__ __device__ constexpr size_t tri_tile_smem(int nz) {
  return (size_t)nz * COLS * (2 * sizeof(T) + sizeof(double)) + 2 * sizeof(double) * kTriSegs * 2 * COLS;
}
// threads of a tile of COLS columns: kTriSegs per real or imaginary part
template <int COLS>
constexpr int tri_tile_threads() { return 2 * COLS * kTriSegs; }

// One step of the pivot recurrence of the forward sweep: the reciprocal
// pivot iv(k) of a mode with eigenvalue lam, and c(k) = At(k) iv(k) carried
// to k + 1.
__device__ __forceinline__ double tri_pivot(const double *__restrict__ Ab, const double *__restrict__ At, int k,
                                            double lam, double &cprev) {
  const double den = (-(Ab[k] + At[k]) + lam) - (k > 1 ? Ab[k] * cprev : 0.0);
  const double v = 1.0 / den;
  cprev = At[k] * v;
  return v;
}

// the first level of segment seg of the tiled z solve (segments of
// ceil(nz / kTriSegs) levels)
__host__ __device__ __forceinline__ int tri_seg_begin(int nz, int seg) {
  return 1 + seg * ((nz + kTriSegs - 1) / kTriSegs);
}
// the pivots are rebuilt in twice as many pieces: both threads of a column
// and segment take one half
constexpr int kTriPivSegs = 2 * kTriSegs;
__host__ __device__ __forceinline__ int tri_piv_begin(int nz, int p) {
  return 1 + p * ((nz + kTriPivSegs - 1) / kTriPivSegs);
}

// c0[p * ncol + col]: c(kb - 1) of mode col = ky * spitch + kx at the first
// level kb of each pivot piece p (0 for the first); the tiled solve rebuilds
// the reciprocal pivots of its pieces from it
__global__ void k_tri_factors(double *c0, const double *__restrict__ lamx, const double *__restrict__ lamy,
                              const double *__restrict__ Ab, const double *__restrict__ At, int nxh, int spitch, int ny,
                              int nz) {
  const int ncol = ny * spitch;
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < ncol; col += gridDim.x * blockDim.x) {
    const int ky = col / spitch, kx = col - ky * spitch;
    const bool mode = kx < nxh && !(kx == 0 && ky == 0);
    const double lam = mode ? lamx[kx] + lamy[ky] : 0.0;
    double cprev = 0;
    int p = 0;
    for (int k = 1; k <= nz; k++) {
      while (p < kTriPivSegs && tri_piv_begin(nz, p) == k) c0[(long long)(p++) * ncol + col] = mode ? cprev : 0.0;
      if (mode) tri_pivot(Ab, At, k, lam, cprev);
    }
    for (; p < kTriPivSegs; p++) c0[(long long)p * ncol + col] = 0.0;  // empty pieces
  }
}

// COLS: the tile width, a tuning choice (every column is solved alone, so
// the result does not depend on it)
template <typename T, int COLS = kTriCols>
__global__ void __launch_bounds__(tri_tile_threads<COLS>()) k_tri_tile(const Dom<T> *__restrict__ doms, Launch L,
                                                                      int gate) {
  constexpr int kTriCols = COLS, kTriTileThreads = tri_tile_threads<COLS>();  // this tile's shape
  typedef typename Vec2<T>::type T2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int kChunk = 16 / (int)sizeof(T2), kPerRow = kTriCols / kChunk, XS = 2 * kTriCols;
  constexpr int NP = 2 * kTriCols;         // systems (column parts) per tile
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    if (gate && !*d.refine_flag) continue;
    const int lt = t - __ldg(L.starts + di);
    const int nz = d.nz, ncol = d.ny * d.spitch;
    const long long ps = ncol;
    const int col0 = lt * kTriCols;
    T2 *tile = reinterpret_cast<T2 *>(smem_raw);                                            // [nz][kTriCols]
    double *ivs = reinterpret_cast<double *>(smem_raw + (size_t)nz * kTriCols * sizeof(T2));  // [nz][kTriCols]
    double *mapA = ivs + (size_t)nz * kTriCols;                                              // [kTriSegs][NP]
    double *mapB = mapA + kTriSegs * NP;
    const double *Ab = d.Ab, *At = d.At;
    for (int q = threadIdx.x; q < nz * kPerRow; q += kTriTileThreads) {
      const int k = q / kPerRow, c = (q - k * kPerRow) * kChunk;
      if (col0 + c < ncol) cp_async16(tile + k * kTriCols + c, d.S + k * ps + col0 + c);
    }
    const int sys = threadIdx.x % NP, seg = threadIdx.x / NP;
    const int c = sys >> 1;  // column; sys & 1 selects the real or imaginary part
    const int col = col0 + c, ky = col / d.spitch, kx = col - ky * d.spitch;
    const bool active = col < ncol && kx < d.nxh;
    const bool zero_mode = kx == 0 && ky == 0;
    const bool solve = active && !zero_mode;
    const int len = (nz + kTriSegs - 1) / kTriSegs;
    const int kb = tri_seg_begin(nz, seg), ke = min(nz, kb + len - 1);  // this thread's segment, kb > ke if empty
    // the reciprocal pivots of the column, rebuilt piece by piece from the
    // stored carries (each thread of the column takes one piece) while the
    // tile of S lands
    if (col < ncol) {
      const int p = 2 * seg + (sys & 1);
      const int pl = (nz + kTriPivSegs - 1) / kTriPivSegs;
      const int pb = tri_piv_begin(nz, p), pe = min(nz, pb + pl - 1);
      double cprev = d.tri_c0[(long long)p * ncol + col];
      const double lam = solve ? d.lamx[kx] + d.lamy[ky] : 0.0;
      for (int k = pb; k <= pe; k++) ivs[(k - 1) * kTriCols + c] = solve ? tri_pivot(Ab, At, k, lam, cprev) : 0.0;
    }
    cp_async_wait_all();
    __syncthreads();
    T *x = reinterpret_cast<T *>(tile) + sys;  // element k - 1 at x[(k - 1) * XS]
    const double *iv = ivs + c;                // element k - 1 at iv[(k - 1) * kTriCols]
    const double norm = 1.0 / ((double)d.nx * (double)d.ny);
    // forward: y(k) = a(k) + b(k) y(k-1), a = r norm iv, b = -Ab iv (b(1) = 0)
    double A = 0, B = 1;
    if (solve)
      for (int k = kb; k <= ke; k++) {
        const double ivk = iv[(k - 1) * kTriCols];
        const double a = (double)x[(k - 1) * XS] * norm * ivk, b = -Ab[k] * ivk;
        A = a + b * A;
        B = b * B;
      }
    mapA[seg * NP + sys] = A;
    mapB[seg * NP + sys] = B;
    __syncthreads();
    if (solve) {
      double y = 0;  // y(kb - 1), y(0) = 0
      for (int s2 = 0; s2 < seg; s2++) y = mapA[s2 * NP + sys] + mapB[s2 * NP + sys] * y;
      for (int k = kb; k <= ke; k++) {
        const double ivk = iv[(k - 1) * kTriCols];
        y = (double)x[(k - 1) * XS] * norm * ivk - Ab[k] * ivk * y;
        x[(k - 1) * XS] = (T)y;
      }
    }
    __syncthreads();
    // backward: x(k) = y(k) + g(k) x(k+1), g = -At iv (g(nz) = 0); segments
    // run from their top end down
    A = 0;
    B = 1;
    if (solve)
      for (int k = ke; k >= kb; k--) {
        const double g = -At[k] * iv[(k - 1) * kTriCols];
        A = (double)x[(k - 1) * XS] + g * A;
        B = g * B;
      }
    __syncthreads();  // every thread has read the forward maps
    mapA[seg * NP + sys] = A;
    mapB[seg * NP + sys] = B;
    __syncthreads();
    if (solve) {
      double xv = 0;  // x(ke + 1), x(nz + 1) = 0
      for (int s2 = kTriSegs - 1; s2 > seg; s2--) xv = mapA[s2 * NP + sys] + mapB[s2 * NP + sys] * xv;
      for (int k = ke; k >= kb; k--) {
        xv = (double)x[(k - 1) * XS] - At[k] * iv[(k - 1) * kTriCols] * xv;
        x[(k - 1) * XS] = (T)xv;
      }
    }
    if (active && zero_mode && seg == 0) {
      // F(k) = F(k-1) + dzc(k) r(k) is the flux (x(k+1) - x(k)) / dzf(k)
      double F = 0, xx = 0, sx = 0;
      for (int k = 1; k <= nz - 1; k++) {
        F = F + ((double)x[(k - 1) * XS] * norm) * d.dzc[k];
        x[(k - 1) * XS] = (T)xx;
        sx += xx;
        xx = xx + F * d.dzf[k];
      }
      sx += xx;
      sx = sx / nz;
      for (int k = 0; k < nz - 1; k++) x[k * XS] = (T)((double)x[k * XS] - sx);
      x[(nz - 1) * XS] = (T)(xx - sx);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nz * kPerRow; q += kTriTileThreads) {
      const int k = q / kPerRow, c2 = (q - k * kPerRow) * kChunk;
      if (col0 + c2 < ncol)
        *reinterpret_cast<int4 *>(d.S + k * ps + col0 + c2) = *reinterpret_cast<const int4 *>(tile + k * kTriCols + c2);
    }
    __syncthreads();  // the tile is free for the next one
  }
}

}  // namespace elmm
