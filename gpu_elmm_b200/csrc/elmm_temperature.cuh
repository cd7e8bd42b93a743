// elmm_temperature.cuh -- one stage of ScalarRK3 for the potential
// temperature (src/scalars.f90:88-299): KappaScalar advection
// (src/scalar_advection.f90:102-272), ScalarDiffusion_nobranch
// (src/scalar_diffusion.f90:404-507), the wall-model point term of
// TemperatureExtra (src/scalars.f90:301-334, DivergenceWM
// src/wallmodels.f90:1150-1166) and the RK combine, one cell per thread.
//
// The stencil reaches two cells in each direction.  Instead of a two-deep
// ghost shell the kernel folds every neighbour index onto the interior as
// BoundTemperature (src/scalarboundaries.f90:12-300) fills it for the
// supported conditions: periodic copies, and the first interior cell for a
// zero-flux (constant-flux 0) side at every ghost depth.  The diffusivity
// folds by BoundViscosity (periodic copy or adjacent cell), the same map.
// Without solid bodies every face carries flux (src/wallmodels.f90:910-950).
#pragma once

#include "elmm_common.cuh"

namespace elmm {

// index fold of a scalar neighbour along one axis: periodic wrap, else the
// nearest interior cell
__device__ __forceinline__ int scal_fold(int g, int n, bool periodic) {
  if (g >= 1 && g <= n) return g;
  if (periodic) return g < 1 ? g + n : g - n;
  return g < 1 ? 1 : n;
}

// FluxLimiter of KappaScalar (src/scalar_advection.f90:262-270)
template <typename T>
__device__ __forceinline__ T kappa_limiter(T r) {
  return fmax((T)0, fmin((T)2 * r, fmin((T)2, ((T)1 + (T)2 * r) / (T)3)));
}

// the flux through the face between cells b and c, with a the cell before b
// and e the cell after c along the face normal, velocity vel on the face
template <typename T>
__device__ __forceinline__ T kappa_flux(T vel, T a, T b, T c, T e) {
  const T eps = (T)1e-8;
  T sr, sl;
  if (vel > 0) { sr = c - b; sl = b - a; }
  else { sr = b - c; sl = c - e; }
  const T sg = signbit(sl) ? (T)-1 : (T)1;
  const T slope = kappa_limiter<T>((sr + eps * sg) / (sl + eps * sg));
  return vel > 0 ? vel * (b + (b - a) * slope / (T)2) : vel * (c + (c - e) * slope / (T)2);
}

template <typename T>
__global__ void __launch_bounds__(TX *TY) k_temperature(const Dom<T> *__restrict__ doms, Launch L, double rho,
                                                        double beta, int stage1) {
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    if (!d.buoy) continue;
    int lt = t - __ldg(L.starts + di);
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const int ntx = (nx + TX - 1) / TX, nty = (ny + TY - 1) / TY;
    const int tx = lt % ntx; lt /= ntx;
    const int ty = lt % nty;
    const int k = lt / nty + 1;
    const int i = tx * TX + (threadIdx.x % TX) + 1;
    const int j = ty * TY + (threadIdx.x / TX) + 1;
    if (i > nx || j > ny) continue;
    const bool px = d.tbt[SIDE_WE] == BC_PERIODIC, py = d.tbt[SIDE_SO] == BC_PERIODIC,
               pz = d.tbt[SIDE_BO] == BC_PERIODIC;
    const T *__restrict__ S = d.Tm;
    const T *__restrict__ K = d.TDiff;
    // folded coordinates of the neighbours i-2..i+2 (index 0..4)
    int xs[5], ys[5], zs[5];
#pragma unroll
    for (int q = 0; q < 5; q++) {
      xs[q] = scal_fold(i - 2 + q, nx, px);
      ys[q] = scal_fold(j - 2 + q, ny, py);
      zs[q] = scal_fold(k - 2 + q, nz, pz);
    }
    auto s_at = [&](int a, int b, int c) { return ld(S, bidx(d, xs[a], ys[b], zs[c])); };
    auto k_at = [&](int a, int b, int c) { return ld(K, bidx(d, xs[a], ys[b], zs[c])); };
    const long long cc = bidx(d, i, j, k);
    // velocities on the six faces (their ghosts are filled)
    const T ue = ld(d.U, cc), uw = ld(d.U, cc - 1);
    const T vn = ld(d.V, cc), vs = ld(d.V, cc - d.pitch);
    const T wt = ld(d.W, cc), wb = ld(d.W, cc - d.plane);
    const T s0 = s_at(2, 2, 2);
    const T Ax = (T)(1.0 / d.dx), Ay = (T)(1.0 / d.dy), Az = (T)(1.0 / d.dz);
    // advection: the loop order of KappaScalar gives each cell +A f(low face)
    // then -A f(high face) in x and y; in z the even faces come first
    T a = (T)0;
    a = a + Ax * kappa_flux<T>(uw, s_at(0, 2, 2), s_at(1, 2, 2), s0, s_at(3, 2, 2));
    a = a - Ax * kappa_flux<T>(ue, s_at(1, 2, 2), s0, s_at(3, 2, 2), s_at(4, 2, 2));
    a = a + Ay * kappa_flux<T>(vs, s_at(2, 0, 2), s_at(2, 1, 2), s0, s_at(2, 3, 2));
    a = a - Ay * kappa_flux<T>(vn, s_at(2, 1, 2), s0, s_at(2, 3, 2), s_at(2, 4, 2));
    const T fzb = kappa_flux<T>(wb, s_at(2, 2, 0), s_at(2, 2, 1), s0, s_at(2, 2, 3));
    const T fzt = kappa_flux<T>(wt, s_at(2, 2, 1), s0, s_at(2, 2, 3), s_at(2, 2, 4));
    if (((k - 1) & 1) == 0) {  // face k-1 is even
      a = a + Az * fzb;
      a = a - Az * fzt;
    } else {
      a = a - Az * fzt;
      a = a + Az * fzb;
    }
    // diffusion, in the order of ScalarDiffusion_nobranch
    const T Dx = (T)(1.0 / (2 * d.dx * d.dx)), Dy = (T)(1.0 / (2 * d.dy * d.dy)), Dz = (T)(1.0 / (2 * d.dz * d.dz));
    const T k0 = k_at(2, 2, 2);
    a = a + (k_at(3, 2, 2) + k0) * (s_at(3, 2, 2) - s0) * Dx;
    a = a - (k0 + k_at(1, 2, 2)) * (s0 - s_at(1, 2, 2)) * Dx;
    a = a + (k_at(2, 3, 2) + k0) * (s_at(2, 3, 2) - s0) * Dy;
    a = a - (k0 + k_at(2, 1, 2)) * (s0 - s_at(2, 1, 2)) * Dy;
    a = a + (k_at(2, 2, 3) + k0) * (s_at(2, 2, 3) - s0) * Dz;
    a = a - (k0 + k_at(2, 2, 1)) * (s0 - s_at(2, 2, 1)) * Dz;
    // wall-model point next to a wall-model side: + div * theta (the surface
    // flux is zero); div as DivergenceWM with dzPr(k)
    if ((k == 1 && d.wall[SIDE_BO]) || (k == nz && d.wall[SIDE_TO])) {
      const T dzk = (T)d.dzPr[k + 2];
      T div = (T)0;
      div = div + ue / (T)d.dx;
      div = div - uw / (T)d.dx;
      div = div + vn / (T)d.dy;
      div = div - vs / (T)d.dy;
      div = div + wt / dzk;
      div = div - wb / dzk;
      a = a + div * s0;
    }
    // RK combine of the stage: T2 = Tadv_old * (rho dt) + Tadv * (beta dt)
    T t2 = stage1 ? (T)0 : ld((const T *)d.Tadv, cc) * (T)(rho * d.dt);
    t2 = t2 + a * (T)(beta * d.dt);
    d.Tadv[cc] = a;
    d.Tn[cc] = s0 + t2;
  }
}

// interior of Temperature(-2:n+3) (host, double) -> device box, minus toff
template <typename T>
__global__ void k_unpack_temperature(const Dom<T> *__restrict__ dom, const double *__restrict__ src, int *bad) {
  const Dom<T> &d = *dom;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const long long total = (long long)nx * ny * nz;
  const long long n0 = nx + 6, n1 = ny + 6;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total; w += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(w % nx) + 1;
    const long long r = w / nx;
    const int j = (int)(r % ny) + 1, k = (int)(r / ny) + 1;
    const double v = src[(i + 2) + n0 * ((j + 2) + n1 * (k + 2))];
    if (!isfinite(v)) atomicAdd(bad, 1);
    d.Tm[bidx(d, i, j, k)] = (T)(v - d.toff);
  }
}

// box field F with lower bound lo (-2: Temperature, Temperature_adv; -1:
// TDiff) -> host array, every ghost folded onto the interior (periodic copy,
// else the nearest interior cell), plus add.  interior_only: ghosts are 0.
template <typename T>
__global__ void k_pack_temperature(const Dom<T> *__restrict__ dom, const T *F, double *dst, int lo, double add,
                                   int interior_only) {
  const Dom<T> &d = *dom;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const int n0 = nx + 2 * (1 - lo), n1 = ny + 2 * (1 - lo), n2 = nz + 2 * (1 - lo);
  const bool px = d.tbt[SIDE_WE] == BC_PERIODIC, py = d.tbt[SIDE_SO] == BC_PERIODIC,
             pz = d.tbt[SIDE_BO] == BC_PERIODIC;
  const long long total = (long long)n0 * n1 * n2;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total; w += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(w % n0) + lo;
    const long long r = w / n0;
    const int j = (int)(r % n1) + lo, k = (int)(r / n1) + lo;
    const bool ghost = i < 1 || i > nx || j < 1 || j > ny || k < 1 || k > nz;
    if (ghost && interior_only) { dst[w] = 0; continue; }
    const T v = F[bidx(d, scal_fold(i, nx, px), scal_fold(j, ny, py), scal_fold(k, nz, pz))];
    dst[w] = (double)v + add;
  }
}

}  // namespace elmm
