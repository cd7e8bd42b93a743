// elmm_slabs.cuh -- the z solve of a domain split into z-slabs.
//
// After the x and y transforms every slab holds its levels of each (kx, ky)
// column of the tridiagonal system of src/poisson.f90:23-60.  Instead of a
// transpose to whole columns, the slabs run the Thomas algorithm as the
// affine-map recurrences of the tiled solve (elmm_poisson_reg.cuh), with
// the slab as the segment:
//
//   forward   y(k) = r(k) iv(k) - Ab(k) iv(k) y(k-1):  slab s maps its entry
//             y(k0) to its last y by y_last = A_s + B_s y(k0)
//   backward  x(k) = y(k) - At(k) iv(k) x(k+1):         slab s maps the first x
//             of the slab above to its own first x by x(k0+1) = A'_s + B'_s x_in
//
// so one exchange of three numbers per column and slab follows each sweep
// (k_slab_tri_fmap, then k_slab_tri_fwd, then k_slab_tri_bwd) and nothing
// of the spectral buffer crosses between GPUs.  The reciprocal pivots iv(k)
// depend on the grid only: k_slab_tri_pivots runs the pivot recurrence of
// the whole column once at creation and keeps the slab's levels, with the
// operations of tri_pivot (so the values of a single-domain solve).  The
// (0,0) mode is singular: its right-hand side is gathered whole into every
// slab, and each slab runs the zero-mean prefix-sum solution of k_tri_tile
// and keeps its own levels.
#pragma once

#include "elmm_common.cuh"
#include "elmm_poisson_reg.cuh"

namespace elmm {

// iv[(k - 1) * ncol + col], k = 1..nzl: the reciprocal pivots of levels
// k0 + 1 .. k0 + nzl of the whole column (Abg, Atg: the whole domain's
// coefficients, index 1..nz); 0 for the (0,0) mode and the padding columns
__global__ void k_slab_tri_pivots(double *iv, const double *__restrict__ lamx, const double *__restrict__ lamy,
                                  const double *__restrict__ Abg, const double *__restrict__ Atg, int nxh, int spitch,
                                  int ny, int k0, int nzl) {
  const int ncol = ny * spitch;
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < ncol; col += gridDim.x * blockDim.x) {
    const int ky = col / spitch, kx = col - ky * spitch;
    const bool mode = kx < nxh && !(kx == 0 && ky == 0);
    const double lam = mode ? lamx[kx] + lamy[ky] : 0.0;
    double cprev = 0;
    for (int k = 1; k <= k0 + nzl; k++) {
      double v = 0;
      if (mode) {
        const double den = (-(Abg[k] + Atg[k]) + lam) - (k > 1 ? Abg[k] * cprev : 0.0);
        v = 1.0 / den;
        cprev = Atg[k] * v;
      }
      if (k > k0) iv[(long long)(k - k0 - 1) * ncol + col] = v;
    }
  }
}

// The maps of a slab's forward sweep with entry y(k0) = 0:
// fmap[part * ncol + col] = A (part 0 real, 1 imaginary), fmap[2 * ncol + col] = B.
// The (0,0) mode's right-hand side goes to zcol[part * nzg + k0 + k - 1].
template <typename T>
__global__ void k_slab_tri_fmap(const Dom<T> *__restrict__ dom, const double *__restrict__ iv, double *fmap,
                                double *zcol, int k0, int nzg) {
  const Dom<T> &d = *dom;
  const int ncol = d.ny * d.spitch, nz = d.nz;
  const long long ks = 2LL * ncol;  // T elements per level of S
  const double norm = 1.0 / ((double)d.nx * (double)d.ny);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * ncol; t += gridDim.x * blockDim.x) {
    const int col = t >> 1, part = t & 1;
    const int ky = col / d.spitch, kx = col - ky * d.spitch;
    if (kx >= d.nxh) continue;
    const T *x = reinterpret_cast<const T *>(d.S) + 2LL * col + part;  // level k at x[(k - 1) * ks]
    if (kx == 0 && ky == 0) {
      for (int k = 1; k <= nz; k++) zcol[(long long)part * nzg + k0 + k - 1] = (double)x[(k - 1) * ks];
      continue;
    }
    double A = 0, B = 1;
    for (int k = 1; k <= nz; k++) {
      const double ivk = iv[(long long)(k - 1) * ncol + col];
      const double a = (double)x[(k - 1) * ks] * norm * ivk, b = -d.Ab[k] * ivk;
      A = a + b * A;
      B = b * B;
    }
    fmap[(long long)part * ncol + col] = A;
    if (part == 0) fmap[2LL * ncol + col] = B;
  }
}

// The forward sweep of slab s from its exact entry (the maps of the slabs
// below, fmaps[q * 3 * ncol ...] for q < s, composed from y(0) = 0), written
// into S, and the map of the slab's backward sweep into bmap (layout of
// fmap): x(k0 + 1) = A' + B' x(k0 + nzl + 1), accumulated upwards as
// A' = sum_k y(k) prod_{j<k} g(j), B' = prod g, g = -At iv.  The (0,0)
// mode: the zero-mean solution of the whole column from zcol (every slab
// computes the same column; dzc, dzf are the whole domain's, index 1..nzg),
// this slab's levels written.
template <typename T>
__global__ void k_slab_tri_fwd(const Dom<T> *__restrict__ dom, const double *__restrict__ iv,
                               const double *__restrict__ fmaps, double *bmap, const double *__restrict__ zcol,
                               const double *__restrict__ dzc, const double *__restrict__ dzf, int k0, int nzg, int s) {
  const Dom<T> &d = *dom;
  const int ncol = d.ny * d.spitch, nz = d.nz;
  const long long ks = 2LL * ncol, ms = 3LL * ncol;
  const double norm = 1.0 / ((double)d.nx * (double)d.ny);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * ncol; t += gridDim.x * blockDim.x) {
    const int col = t >> 1, part = t & 1;
    const int ky = col / d.spitch, kx = col - ky * d.spitch;
    if (kx >= d.nxh) continue;
    T *x = reinterpret_cast<T *>(d.S) + 2LL * col + part;
    if (kx == 0 && ky == 0) {
      // F(k) = F(k-1) + dzc(k) r(k) is the flux (x(k+1) - x(k)) / dzf(k)
      const double *r = zcol + (long long)part * nzg;
      double F = 0, xx = 0, sx = 0;
      for (int k = 1; k <= nzg - 1; k++) {
        F = F + (r[k - 1] * norm) * dzc[k];
        if (k > k0 && k <= k0 + nz) x[(k - k0 - 1) * ks] = (T)xx;
        sx += xx;
        xx = xx + F * dzf[k];
      }
      sx += xx;
      sx = sx / nzg;
      for (int k = k0 + 1; k <= k0 + nz; k++) {
        T &e = x[(k - k0 - 1) * ks];
        e = k < nzg ? (T)((double)e - sx) : (T)(xx - sx);
      }
      continue;
    }
    double y = 0;  // y(k0)
    for (int q = 0; q < s; q++) y = fmaps[q * ms + (long long)part * ncol + col] + fmaps[q * ms + 2LL * ncol + col] * y;
    double A = 0, G = 1;
    for (int k = 1; k <= nz; k++) {
      const double ivk = iv[(long long)(k - 1) * ncol + col];
      y = (double)x[(k - 1) * ks] * norm * ivk - d.Ab[k] * ivk * y;
      const T yt = (T)y;
      x[(k - 1) * ks] = yt;
      A = A + G * (double)yt;
      G = G * (-d.At[k] * ivk);
    }
    bmap[(long long)part * ncol + col] = A;
    if (part == 0) bmap[2LL * ncol + col] = G;
  }
}

// The backward sweep of slab s from its exact entry x(k0 + nzl + 1) (the
// maps of the slabs above, composed downwards from x(nzg + 1) = 0).
template <typename T>
__global__ void k_slab_tri_bwd(const Dom<T> *__restrict__ dom, const double *__restrict__ iv,
                               const double *__restrict__ bmaps, int s, int ns) {
  const Dom<T> &d = *dom;
  const int ncol = d.ny * d.spitch, nz = d.nz;
  const long long ks = 2LL * ncol, ms = 3LL * ncol;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * ncol; t += gridDim.x * blockDim.x) {
    const int col = t >> 1, part = t & 1;
    const int ky = col / d.spitch, kx = col - ky * d.spitch;
    if (kx >= d.nxh || (kx == 0 && ky == 0)) continue;
    T *x = reinterpret_cast<T *>(d.S) + 2LL * col + part;
    double xv = 0;
    for (int q = ns - 1; q > s; q--) xv = bmaps[q * ms + (long long)part * ncol + col] + bmaps[q * ms + 2LL * ncol + col] * xv;
    for (int k = nz; k >= 1; k--) {
      xv = (double)x[(k - 1) * ks] - d.At[k] * iv[(long long)(k - 1) * ncol + col] * xv;
      x[(k - 1) * ks] = (T)xv;
    }
  }
}

// ------------------------------------------------ tiled form of the sweeps
// The kernels above walk a column with one thread.  For slabs of up to
// kTriTileMaxNz levels the tiled form splits each column's levels into
// kTriSegs segments (one thread each, per real or imaginary part), as
// k_tri_tile does: a block stages COLS columns of S and of the pivots in
// shared memory with cp.async, each thread composes the affine map of its
// segment, and the segment maps are chained in shared memory to the slab's
// map or to each segment's exact entry.  Same recurrences, a different
// grouping of the map compositions.
template <typename T, int COLS>
struct SlabTile {
  typedef typename Vec2<T>::type T2;
  static constexpr int NP = 2 * COLS;              // systems (column parts) of a tile
  static constexpr int THREADS = NP * kTriSegs;    // one per segment of each system
  static constexpr int XS = 2 * COLS;              // T elements per level of the tile
  static __host__ __device__ size_t smem(int nz) {
    return (size_t)nz * COLS * (sizeof(T2) + sizeof(double)) + 2 * sizeof(double) * kTriSegs * NP;
  }
  T2 *tile;
  double *ivs, *mapA, *mapB;
  int col0, ncol, nz, sys, seg, c, part, col, kb, ke;
  bool active, zero, solve;
  __device__ SlabTile(const Dom<T> &d, const double *__restrict__ iv, int lt, unsigned char *smem_raw) {
    ncol = d.ny * d.spitch;
    nz = d.nz;
    col0 = lt * COLS;
    tile = reinterpret_cast<T2 *>(smem_raw);
    ivs = reinterpret_cast<double *>(smem_raw + (size_t)nz * COLS * sizeof(T2));
    mapA = ivs + (size_t)nz * COLS;
    mapB = mapA + kTriSegs * NP;
    constexpr int kS = 16 / (int)sizeof(T2), kI = 2;  // columns per 16-byte chunk of S and of iv
    for (int q = threadIdx.x; q < nz * (COLS / kS); q += THREADS) {
      const int k = q / (COLS / kS), cc = (q - k * (COLS / kS)) * kS;
      if (col0 + cc < ncol) cp_async16(tile + k * COLS + cc, d.S + (long long)k * ncol + col0 + cc);
    }
    for (int q = threadIdx.x; q < nz * (COLS / kI); q += THREADS) {
      const int k = q / (COLS / kI), cc = (q - k * (COLS / kI)) * kI;
      if (col0 + cc < ncol) cp_async16(ivs + k * COLS + cc, iv + (long long)k * ncol + col0 + cc);
    }
    sys = threadIdx.x % NP;
    seg = threadIdx.x / NP;
    c = sys >> 1;
    part = sys & 1;
    col = col0 + c;
    const int ky = col / d.spitch, kx = col - ky * d.spitch;
    active = col < ncol && kx < d.nxh;
    zero = kx == 0 && ky == 0;
    solve = active && !zero;
    const int len = (nz + kTriSegs - 1) / kTriSegs;
    kb = 1 + seg * len;
    ke = min(nz, kb + len - 1);  // kb > ke: an empty segment
    cp_async_wait_all();
    __syncthreads();
  }
  __device__ T &x(int k) const { return reinterpret_cast<T *>(tile)[(k - 1) * XS + sys]; }
  __device__ double iv(int k) const { return ivs[(k - 1) * COLS + c]; }
  // this segment's forward map y(ke) = A + B y(kb - 1)
  __device__ void fwd_map(const double *__restrict__ Ab, double norm, double &A, double &B) const {
    A = 0;
    B = 1;
    if (solve)
      for (int k = kb; k <= ke; k++) {
        const double ivk = iv(k);
        const double a = (double)x(k) * norm * ivk, b = -Ab[k] * ivk;
        A = a + b * A;
        B = b * B;
      }
  }
  // this segment's backward map x(kb) = A + B x(ke + 1)
  __device__ void bwd_map(const double *__restrict__ At, double &A, double &B) const {
    A = 0;
    B = 1;
    if (solve)
      for (int k = ke; k >= kb; k--) {
        const double g = -At[k] * iv(k);
        A = (double)x(k) + g * A;
        B = g * B;
      }
  }
  __device__ void put_maps(double A, double B) {
    mapA[seg * NP + sys] = A;
    mapB[seg * NP + sys] = B;
  }
  __device__ void store(const Dom<T> &d) {
    __syncthreads();
    constexpr int kS = 16 / (int)sizeof(T2);
    for (int q = threadIdx.x; q < nz * (COLS / kS); q += THREADS) {
      const int k = q / (COLS / kS), cc = (q - k * (COLS / kS)) * kS;
      if (col0 + cc < ncol)
        *reinterpret_cast<int4 *>(d.S + (long long)k * ncol + col0 + cc) = *reinterpret_cast<const int4 *>(tile + k * COLS + cc);
    }
    __syncthreads();  // the shared memory is free for the next tile
  }
};

// tiled k_slab_tri_fmap
template <typename T, int COLS>
__global__ void __launch_bounds__(SlabTile<T, COLS>::THREADS)
    k_slab_tri_fmap_tile(const Dom<T> *__restrict__ dom, const double *__restrict__ iv, double *fmap, double *zcol,
                         int k0, int nzg) {
  typedef SlabTile<T, COLS> Tl;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Dom<T> &d = *dom;
  const int ncol = d.ny * d.spitch, ntile = (ncol + COLS - 1) / COLS;
  const double norm = 1.0 / ((double)d.nx * (double)d.ny);
  for (int lt = blockIdx.x; lt < ntile; lt += gridDim.x) {
    Tl t(d, iv, lt, smem_raw);
    double A, B;
    t.fwd_map(d.Ab, norm, A, B);
    t.put_maps(A, B);
    __syncthreads();
    if (t.seg == 0 && t.solve) {
      A = t.mapA[t.sys];
      B = t.mapB[t.sys];
      for (int s2 = 1; s2 < kTriSegs; s2++) {
        A = t.mapA[s2 * Tl::NP + t.sys] + t.mapB[s2 * Tl::NP + t.sys] * A;
        B = t.mapB[s2 * Tl::NP + t.sys] * B;
      }
      fmap[(long long)t.part * ncol + t.col] = A;
      if (t.part == 0) fmap[2LL * ncol + t.col] = B;
    }
    if (t.seg == 0 && t.active && t.zero)
      for (int k = 1; k <= t.nz; k++) zcol[(long long)t.part * nzg + k0 + k - 1] = (double)t.x(k);
    __syncthreads();  // the shared memory is free for the next tile
  }
}

// tiled k_slab_tri_fwd
template <typename T, int COLS>
__global__ void __launch_bounds__(SlabTile<T, COLS>::THREADS)
    k_slab_tri_fwd_tile(const Dom<T> *__restrict__ dom, const double *__restrict__ iv, const double *__restrict__ fmaps,
                        double *bmap, const double *__restrict__ zcol, const double *__restrict__ dzc,
                        const double *__restrict__ dzf, int k0, int nzg, int s) {
  typedef SlabTile<T, COLS> Tl;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Dom<T> &d = *dom;
  const int ncol = d.ny * d.spitch, ntile = (ncol + COLS - 1) / COLS;
  const long long ms = 3LL * ncol;
  const double norm = 1.0 / ((double)d.nx * (double)d.ny);
  for (int lt = blockIdx.x; lt < ntile; lt += gridDim.x) {
    Tl t(d, iv, lt, smem_raw);
    double A, B;
    t.fwd_map(d.Ab, norm, A, B);
    t.put_maps(A, B);
    __syncthreads();
    if (t.solve) {
      double y = 0;  // y(k0): the maps of the slabs below
      for (int q = 0; q < s; q++)
        y = fmaps[q * ms + (long long)t.part * ncol + t.col] + fmaps[q * ms + 2LL * ncol + t.col] * y;
      for (int s2 = 0; s2 < t.seg; s2++) y = t.mapA[s2 * Tl::NP + t.sys] + t.mapB[s2 * Tl::NP + t.sys] * y;
      for (int k = t.kb; k <= t.ke; k++) {
        const double ivk = t.iv(k);
        y = (double)t.x(k) * norm * ivk - d.Ab[k] * ivk * y;
        t.x(k) = (T)y;
      }
    }
    if (t.seg == 0 && t.active && t.zero) {
      // the zero-mean solution of the whole (0,0) column (k_slab_tri_fwd)
      const double *r = zcol + (long long)t.part * nzg;
      double F = 0, xx = 0, sx = 0;
      for (int k = 1; k <= nzg - 1; k++) {
        F = F + (r[k - 1] * norm) * dzc[k];
        if (k > k0 && k <= k0 + t.nz) t.x(k - k0) = (T)xx;
        sx += xx;
        xx = xx + F * dzf[k];
      }
      sx += xx;
      sx = sx / nzg;
      for (int k = k0 + 1; k <= k0 + t.nz; k++) {
        T &e = t.x(k - k0);
        e = k < nzg ? (T)((double)e - sx) : (T)(xx - sx);
      }
    }
    __syncthreads();  // the forward maps are read, the segments replayed
    t.bwd_map(d.At, A, B);
    t.put_maps(A, B);
    __syncthreads();
    if (t.seg == 0 && t.solve) {
      A = t.mapA[(kTriSegs - 1) * Tl::NP + t.sys];
      B = t.mapB[(kTriSegs - 1) * Tl::NP + t.sys];
      for (int s2 = kTriSegs - 2; s2 >= 0; s2--) {
        A = t.mapA[s2 * Tl::NP + t.sys] + t.mapB[s2 * Tl::NP + t.sys] * A;
        B = t.mapB[s2 * Tl::NP + t.sys] * B;
      }
      bmap[(long long)t.part * ncol + t.col] = A;
      if (t.part == 0) bmap[2LL * ncol + t.col] = B;
    }
    t.store(d);
  }
}

// tiled k_slab_tri_bwd
template <typename T, int COLS>
__global__ void __launch_bounds__(SlabTile<T, COLS>::THREADS)
    k_slab_tri_bwd_tile(const Dom<T> *__restrict__ dom, const double *__restrict__ iv, const double *__restrict__ bmaps,
                        int s, int ns) {
  typedef SlabTile<T, COLS> Tl;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Dom<T> &d = *dom;
  const int ncol = d.ny * d.spitch, ntile = (ncol + COLS - 1) / COLS;
  const long long ms = 3LL * ncol;
  for (int lt = blockIdx.x; lt < ntile; lt += gridDim.x) {
    Tl t(d, iv, lt, smem_raw);
    double A, B;
    t.bwd_map(d.At, A, B);
    t.put_maps(A, B);
    __syncthreads();
    if (t.solve) {
      double xv = 0;  // x(k0 + nzl + 1): the maps of the slabs above
      for (int q = ns - 1; q > s; q--)
        xv = bmaps[q * ms + (long long)t.part * ncol + t.col] + bmaps[q * ms + 2LL * ncol + t.col] * xv;
      for (int s2 = kTriSegs - 1; s2 > t.seg; s2--) xv = t.mapA[s2 * Tl::NP + t.sys] + t.mapB[s2 * Tl::NP + t.sys] * xv;
      for (int k = t.ke; k >= t.kb; k--) {
        xv = (double)t.x(k) - d.At[k] * t.iv(k) * xv;
        t.x(k) = (T)xv;
      }
    }
    t.store(d);
  }
}

}  // namespace elmm
