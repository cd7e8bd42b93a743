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

}  // namespace elmm
