// elmm_temperature.cuh -- one stage of ScalarRK3 (src/scalars.f90:88-299)
// for every transported scalar of a domain, the potential temperature and the
// passive scalars: KappaScalar advection (src/scalar_advection.f90:102-272),
// ScalarDiffusion_nobranch (src/scalar_diffusion.f90:404-507), the volume
// sources of the point sources (ScalarExtra -> ScalarVolumeSources,
// src/scalars.f90:364-379, src/volumesources.f90:741-771), the wall-model
// point term (TemperatureExtra / ScalarExtra, DivergenceWM
// src/wallmodels.f90:1150-1166) and the RK combine, one cell per thread; in
// the last stage of a step the new value also enters the time-averaged
// slices (Scalar_avg, src/outputs.f90:1043-1045).
//
// The stencil reaches two cells in each direction.  Instead of a two-deep
// ghost shell the kernel folds every neighbour index onto the interior as
// BoundTemperature / BoundScalar (src/scalarboundaries.f90:12-308) fill it
// for the supported conditions: periodic copies, and the first interior cell
// for a zero-flux (constant-flux 0) side at every ghost depth.  The
// diffusivity folds by BoundViscosity (periodic copy or adjacent cell), the
// same map.  Without solid bodies every face carries flux
// (src/wallmodels.f90:910-950).
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

// FluxLimiter of KappaScalar (src/scalar_advection.f90:262-270).  The FP32
// path of the mixed precision mode divides by 3 as a multiplication by 1/3
// and forms the slope ratio with the fast division (both within a few ulp);
// the FP64 path keeps the reference's divisions.
template <typename T>
__device__ __forceinline__ T kappa_limiter(T r) {
  return fmax((T)0, fmin((T)2 * r, fmin((T)2, ((T)1 + (T)2 * r) / (T)3)));
}
template <>
__device__ __forceinline__ float kappa_limiter<float>(float r) {
  return fmaxf(0.f, fminf(2.f * r, fminf(2.f, (1.f + 2.f * r) * (1.f / 3.f))));
}
template <typename T>
__device__ __forceinline__ T kappa_ratio(T num, T den) { return num / den; }
template <>
__device__ __forceinline__ float kappa_ratio<float>(float num, float den) { return __fdividef(num, den); }

// the flux through the face between cells b and c, with a the cell before b
// and e the cell after c along the face normal, velocity vel on the face
template <typename T>
__device__ __forceinline__ T kappa_flux(T vel, T a, T b, T c, T e) {
  const T eps = (T)1e-8;
  T sr, sl;
  if (vel > 0) { sr = c - b; sl = b - a; }
  else { sr = b - c; sl = c - e; }
  const T sg = signbit(sl) ? (T)-1 : (T)1;
  const T slope = kappa_limiter<T>(kappa_ratio<T>(sr + eps * sg, sl + eps * sg));
  return vel > 0 ? vel * (b + (b - a) * slope / (T)2) : vel * (c + (c - e) * slope / (T)2);
}

// BoundTemperature / BoundScalar on the z sides with a stored ghost plane
// (CommonBase, src/scalarboundaries.f90:203-288), before the stage reads
// them: the plane below k = 1 or above k = nz of the stage's input buffer
// from the first interior level and, for a flux, the diffusivity, whose
// ghost is its interior value (BoundViscosity, :403-425).  FP64 arithmetic
// on the full values (the stored value plus the slot's offset).
template <typename T>
__global__ void k_scalar_zghost(const Dom<T> *__restrict__ doms, int nd, int stage) {
  for (int di = 0; di < nd; di++) {
    const Dom<T> &d = doms[di];
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    for (int s = 0; s < d.nslot; s++) {
      const ScalSlot<T> &sl = d.slot[s];
#pragma unroll 1
      for (int h = 0; h < 2; h++) {
        if (!sl.zg[h]) continue;
        T *S = sl.buf[(stage - 1) % 3];
        const int kin = h ? nz : 1, kg = h ? nz + 1 : 0, kind = sl.bt[h ? SIDE_TO : SIDE_BO];
        const double side = sl.zside[h], off = sl.off;
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nx * ny; q += gridDim.x * blockDim.x) {
          const int i = q % nx + 1, j = q / nx + 1;
          const double t = (double)S[bidx(d, i, j, kin)] + off;
          double g;
          if (kind == BC_DIRICHLET) {
            g = side - (t - side);
          } else if (kind == BC_NEUMANN) {
            g = h ? t + side * d.dzW[nz + 1 + 2] : t - side * d.dzW[0 + 2];
          } else {  // BC_CONSTFLUX
            const double kd = (double)d.TDiff[bidx(d, i, j, kin)];
            g = h ? t - side * d.dzW[nz + 2] / ((kd + kd) / 2.0) : t + side * d.dzW[0 + 2] / ((kd + kd) / 2.0);
          }
          S[bidx(d, i, j, kg)] = (T)(g - off);
        }
      }
    }
  }
}

// A block owns a TX x TY column of cells of one scalar slot and marches up a
// chunk of TMKC planes; the scalar (k-2..k+2), the diffusivity (k-1..k+1)
// and W(k-1) ride along in registers, x and y neighbours come from offsets
// folded once per thread.  Tiles: (slot, column, chunk) per domain.
#ifndef ELMM_SCALAR_CHUNK
#define ELMM_SCALAR_CHUNK 16
#endif
constexpr int TMKC = ELMM_SCALAR_CHUNK;

// BC: some slot has a stored z ghost plane, a surface flux or a surface
// temperature (the launch picks the plain instantiation otherwise)
template <typename T, bool BC = false>
__global__ void __launch_bounds__(TX *TY, sizeof(T) == 4 ? 6 : 3)
    k_scalar(const Dom<T> *__restrict__ doms, Launch L, double rho, double beta, int stage) {
  const int stage1 = stage == 1;
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    int lt = t - __ldg(L.starts + di);
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const int ntx = (nx + TX - 1) / TX, nty = (ny + TY - 1) / TY, nkc = (nz + TMKC - 1) / TMKC;
    const int tx = lt % ntx; lt /= ntx;
    const int ty = lt % nty; lt /= nty;
    const int kc = lt % nkc;
    const int s = lt / nkc;
    const ScalSlot<T> &sl = d.slot[s];
    const int k0 = kc * TMKC + 1, k1 = min(k0 + TMKC - 1, nz);
    const int i = tx * TX + (threadIdx.x % TX) + 1;
    const int j = ty * TY + (threadIdx.x / TX) + 1;
    if (i > nx || j > ny) continue;
    const bool px = sl.bt[SIDE_WE] == BC_PERIODIC, py = sl.bt[SIDE_SO] == BC_PERIODIC,
               pz = sl.bt[SIDE_BO] == BC_PERIODIC;
    const long long pitch = d.pitch, plane = d.plane;
    // folded offsets of the x and y neighbours -2..+2 (index 0..4); a plane
    // holds fewer than 2^31 elements
    int ox[5], oy[5];
#pragma unroll
    for (int q = 0; q < 5; q++) {
      ox[q] = scal_fold(i - 2 + q, nx, px) - i;
      oy[q] = (scal_fold(j - 2 + q, ny, py) - j) * (int)pitch;
    }
    auto zoff = [&](int kk) { return (long long)(scal_fold(kk, nz, pz) - kk) * plane; };  // fold of plane kk
    const T *__restrict__ S = sl.buf[(stage - 1) % 3];
    // the scalar's planes: a stored ghost plane (k_scalar_zghost, or a slab's
    // halo) is read as it is; a slab's second halo planes live in h2
    const bool hlo = BC && sl.bt[SIDE_BO] == BC_HALO, hhi = BC && sl.bt[SIDE_TO] == BC_HALO;
    const int zs0 = sl.zg[0] || hlo, zs1 = sl.zg[1] || hhi;
    auto szoff = [&](int kk) { return BC && ((kk == 0 && zs0) || (kk == nz + 1 && zs1)) ? 0LL : zoff(kk); };
    auto kzoff = [&](int kk) { return (kk == 0 && hlo) || (kk == nz + 1 && hhi) ? 0LL : zoff(kk); };
    // the scalar at level kk of this column, o its unfolded box index
    auto lds = [&](int kk, long long o) -> T {
      if constexpr (BC) {
        if (kk == -1 && hlo) return ld(sl.h2[0], o + plane);
        if (kk == nz + 2 && hhi) return ld(sl.h2[1], o - (long long)(nz + 2) * plane);
      }
      return ld(S, o + szoff(kk));
    };
    // volume sources of this slot in this column, in configuration order
    unsigned srcm = 0;
    for (int q = 0; q < d.nsrc; q++)
      if (d.src_slot[q] == s && d.src_i[q] == i && d.src_j[q] == j) srcm |= 1u << q;
    const T *__restrict__ K = d.TDiff;
    const T *__restrict__ U = d.U;
    const T *__restrict__ V = d.V;
    const T *__restrict__ W = d.W;
    T *__restrict__ Sadv = sl.adv;
    T *__restrict__ Snew = sl.buf[stage % 3];
    const T Ax = (T)(1.0 / d.dx), Ay = (T)(1.0 / d.dy), Az = (T)(1.0 / d.dz);
    const T Dx = (T)(1.0 / (2 * d.dx * d.dx)), Dy = (T)(1.0 / (2 * d.dy * d.dy)), Dz = (T)(1.0 / (2 * d.dz * d.dz));
    const T rdx = (T)d.dx, rdy = (T)d.dy;
    const T rdt = (T)(rho * d.dt), bdt = (T)(beta * d.dt);
    const bool wm_lo = d.wall[SIDE_BO] != 0, wm_hi = d.wall[SIDE_TO] != 0;
    long long cc = bidx(d, i, j, k0);
    // column windows: the scalar at k-2..k+2, diffusivity at k-1..k+1, W at k-1
    T sz[5], kz[3];
#pragma unroll
    for (int q = 0; q < 5; q++) sz[q] = lds(k0 - 2 + q, cc + (long long)(q - 2) * plane);
#pragma unroll
    for (int q = 0; q < 3; q++) kz[q] = ld(K, cc + (long long)(q - 1) * plane + kzoff(k0 - 1 + q));
    T wb = ld(W, cc - plane);
    // the bottom-face flux of plane k is the top-face flux of plane k-1
    T fzb = kappa_flux<T>(wb, sz[0], sz[1], sz[2], sz[3]);
    for (int k = k0; k <= k1; k++) {
      const T s0 = sz[2];
      const T ue = ld(U, cc), uw = ld(U, cc - 1);
      const T vn = ld(V, cc), vs = ld(V, cc - pitch);
      const T wt = ld(W, cc);
      const T sxm2 = ld(S, cc + ox[0]), sxm1 = ld(S, cc + ox[1]), sxp1 = ld(S, cc + ox[3]), sxp2 = ld(S, cc + ox[4]);
      const T sym2 = ld(S, cc + oy[0]), sym1 = ld(S, cc + oy[1]), syp1 = ld(S, cc + oy[3]), syp2 = ld(S, cc + oy[4]);
      const T k0v = kz[1];
      const T kxm = ld(K, cc + ox[1]), kxp = ld(K, cc + ox[3]), kym = ld(K, cc + oy[1]), kyp = ld(K, cc + oy[3]);
      const T told = stage1 ? (T)0 : ld((const T *)Sadv, cc);
      // advection: the loop order of KappaScalar gives each cell +A f(low
      // face) then -A f(high face) in x and y; in z the even faces come first
      T a = (T)0;
      // the face velocities in full (the mixed path stores U and V as
      // deviations from a per-level offset; the FP64 path has none)
      T uwf = uw, uef = ue, vsf = vs, vnf = vn;
      if constexpr (sizeof(T) == 4) {
        const T uo = vel_off(d, 0, k), vo = vel_off(d, 1, k);
        uwf = uw + uo; uef = ue + uo; vsf = vs + vo; vnf = vn + vo;
      }
      a = a + Ax * kappa_flux<T>(uwf, sxm2, sxm1, s0, sxp1);
      a = a - Ax * kappa_flux<T>(uef, sxm1, s0, sxp1, sxp2);
      a = a + Ay * kappa_flux<T>(vsf, sym2, sym1, s0, syp1);
      a = a - Ay * kappa_flux<T>(vnf, sym1, s0, syp1, syp2);
      const T fzt = kappa_flux<T>(wt, sz[1], s0, sz[3], sz[4]);
      if (((k - 1) & 1) == 0) {  // face k-1 is even
        a = a + Az * fzb;
        a = a - Az * fzt;
      } else {
        a = a - Az * fzt;
        a = a + Az * fzb;
      }
      // a solid cell keeps no advection tendency (src/scalars.f90:259-268)
      if constexpr (BC) {
        if (d.pmask && (d.pmask[cc] & 1)) a = (T)0;
      }
      // diffusion, in the order of ScalarDiffusion_nobranch
      a = a + (kxp + k0v) * (sxp1 - s0) * Dx;
      a = a - (k0v + kxm) * (s0 - sxm1) * Dx;
      a = a + (kyp + k0v) * (syp1 - s0) * Dy;
      a = a - (k0v + kym) * (s0 - sym1) * Dy;
      a = a + (kz[2] + k0v) * (sz[3] - s0) * Dz;
      a = a - (k0v + kz[0]) * (s0 - sz[1]) * Dz;
      // volume sources (FluxKernel: + flux / volume of the cell)
      if (srcm) {
        for (int q = 0; q < d.nsrc; q++)
          if (((srcm >> q) & 1u) && d.src_k[q] == k) a = a + (T)d.src_q[q];
      }
      // wall-model point next to a wall-model side (with solid bodies, a
      // point of the mask): + the surface flux term, then + div * value; div
      // as DivergenceWM with dzPr(k), without the faces towards solid cells
      bool wmc = (k == 1 && wm_lo) || (k == nz && wm_hi);
      if constexpr (BC) {
        if (d.pmask) wmc = (d.pmask[cc] & 2) != 0;
      }
      if (wmc) {
        if constexpr (BC) {
          // the wall's surface flux at a wall point (with solid bodies, one
          // the deduplication kept, bit 2 of the mask)
          if (!d.pmask || (d.pmask[cc] & 4)) {
            a = a + (T)sl.wflux[k == 1 ? 0 : 1];
            // a prescribed surface temperature: the flux of the point from
            // the wall model of this stage (temperature slot only)
            const double *tpr = s == 0 ? d.wm_pr_tf[k == 1 ? 0 : 1] : nullptr;
            if (tpr) a = a + (T)(tpr[(i - 1) + (long long)nx * (j - 1)] * d.wm_af);
          }
        }
        const T dzk = (T)d.dzPr[k + 2];
        T div = (T)0;
        if (BC && d.pmask) {  // the offsets are zero with solid bodies: stored values are full ones
          const unsigned char *pm = d.pmask;
          if (!(pm[cc + 1] & 1)) div = div + ue / rdx;
          if (!(pm[cc - 1] & 1)) div = div - uw / rdx;
          if (!(pm[cc + pitch] & 1)) div = div + vn / rdy;
          if (!(pm[cc - pitch] & 1)) div = div - vs / rdy;
          if (!(pm[cc + plane] & 1)) div = div + wt / dzk;
          if (!(pm[cc - plane] & 1)) div = div - wb / dzk;
        } else {
          div = div + ue / rdx;
          div = div - uw / rdx;
          div = div + vn / rdy;
          div = div - vs / rdy;
          div = div + wt / dzk;
          div = div - wb / dzk;
        }
        a = a + div * s0;
      }
      // RK combine of the stage: S2 = Sadv_old * (rho dt) + Sadv * (beta dt)
      T t2 = stage1 ? (T)0 : told * rdt;
      t2 = t2 + a * bdt;
      Sadv[cc] = a;
      Snew[cc] = s0 + t2;
      // shift the windows up one plane
      if (k < k1) {
        const long long cn = cc + plane;
#pragma unroll
        for (int q = 0; q < 4; q++) sz[q] = sz[q + 1];
        sz[4] = lds(k + 3, cn + 2 * plane);
        kz[0] = kz[1];
        kz[1] = kz[2];
        kz[2] = ld(K, cn + plane + kzoff(k + 2));
        wb = wt;
        fzb = fzt;
        cc = cn;
      }
    }
  }
}

// The FP32 stage with two x-adjacent cells per thread (domains with an even
// Prnx; x is periodic for every scalar): the pair's x faces are three fluxes
// for two cells, every load and store is a float2, and the per-plane
// bookkeeping of the column march is shared by the pair.  Same operations in
// the same order as k_scalar.  A block is 16 x 8 threads, a tile 32 x 8 cells.
constexpr int SPX = 16;
#ifndef ELMM_SCALAR_PAIR_MIN_BLOCKS
#define ELMM_SCALAR_PAIR_MIN_BLOCKS 3
#endif

__device__ __forceinline__ float2 ld2(const float *p, long long o) {
  return __ldg(reinterpret_cast<const float2 *>(p + o));
}

// the in-plane inputs of a cell pair at one level (k_scalar_pair loads those
// of level k + 1 while it computes level k)
struct PairPlane {
  float2 sm, sp, km, kp, um, u0, vs, vn, wt, sym2, sym1, syp1, syp2, kym, kyp, told;
};

// SPY: the rows of a tile, a tuning choice (8 or 4; the arithmetic of a
// cell does not depend on it)
template <int SPY, bool BC = false>
__global__ void __launch_bounds__(SPX *SPY, ELMM_SCALAR_PAIR_MIN_BLOCKS * 8 / SPY)
    k_scalar_pair(const Dom<float> *__restrict__ doms, Launch L, double rho, double beta, int stage) {
  typedef float T;
  const int stage1 = stage == 1;
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    int lt = t - __ldg(L.starts + di);
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const int ntx = (nx + 2 * SPX - 1) / (2 * SPX), nty = (ny + SPY - 1) / SPY, nkc = (nz + TMKC - 1) / TMKC;
    const int tx = lt % ntx; lt /= ntx;
    const int ty = lt % nty; lt /= nty;
    const int kc = lt % nkc;
    const int s = lt / nkc;
    const ScalSlot<T> &sl = d.slot[s];
    const int k0 = kc * TMKC + 1, k1 = min(k0 + TMKC - 1, nz);
    const int i = tx * 2 * SPX + 2 * (threadIdx.x % SPX) + 1;  // odd: the pair is 8-byte aligned
    const int j = ty * SPY + (threadIdx.x / SPX) + 1;
    if (i > nx || j > ny) continue;
    const bool py = sl.bt[SIDE_SO] == BC_PERIODIC, pz = sl.bt[SIDE_BO] == BC_PERIODIC;
    const long long pitch = d.pitch, plane = d.plane;
    // the aligned pairs (i-2, i-1) and (i+2, i+3), periodic in x (nx even
    // keeps them aligned); rows j-2..j+2 folded
    const int oxm = (i - 2 >= 1 ? i - 2 : i - 2 + nx) - i, oxp = (i + 2 <= nx ? i + 2 : i + 2 - nx) - i;
    int oy[5];
#pragma unroll
    for (int q = 0; q < 5; q++) oy[q] = (scal_fold(j - 2 + q, ny, py) - j) * (int)pitch;
    auto zoff = [&](int kk) { return (long long)(scal_fold(kk, nz, pz) - kk) * plane; };
    const T *__restrict__ S = sl.buf[(stage - 1) % 3];
    const bool hlo = BC && sl.bt[SIDE_BO] == BC_HALO, hhi = BC && sl.bt[SIDE_TO] == BC_HALO;
    const int zs0 = sl.zg[0] || hlo, zs1 = sl.zg[1] || hhi;
    auto szoff = [&](int kk) { return BC && ((kk == 0 && zs0) || (kk == nz + 1 && zs1)) ? 0LL : zoff(kk); };
    auto kzoff = [&](int kk) { return (kk == 0 && hlo) || (kk == nz + 1 && hhi) ? 0LL : zoff(kk); };
    auto lds2 = [&](int kk, long long o) -> float2 {
      if constexpr (BC) {
        if (kk == -1 && hlo) return ld2(sl.h2[0], o + plane);
        if (kk == nz + 2 && hhi) return ld2(sl.h2[1], o - (long long)(nz + 2) * plane);
      }
      return ld2(S, o + szoff(kk));
    };
    unsigned srcm = 0;  // volume sources of this slot in this pair's columns
    for (int q = 0; q < d.nsrc; q++)
      if (d.src_slot[q] == s && (d.src_i[q] == i || d.src_i[q] == i + 1) && d.src_j[q] == j) srcm |= 1u << q;
    const T *__restrict__ K = d.TDiff;
    const T *__restrict__ U = d.U;
    const T *__restrict__ V = d.V;
    const T *__restrict__ W = d.W;
    T *__restrict__ Sadv = sl.adv;
    T *__restrict__ Snew = sl.buf[stage % 3];
    const T Ax = (T)(1.0 / d.dx), Ay = (T)(1.0 / d.dy), Az = (T)(1.0 / d.dz);
    const T Dx = (T)(1.0 / (2 * d.dx * d.dx)), Dy = (T)(1.0 / (2 * d.dy * d.dy)), Dz = (T)(1.0 / (2 * d.dz * d.dz));
    const T rdx = (T)d.dx, rdy = (T)d.dy;
    const T rdt = (T)(rho * d.dt), bdt = (T)(beta * d.dt);
    const bool wm_lo = d.wall[SIDE_BO] != 0, wm_hi = d.wall[SIDE_TO] != 0;
    long long cc = bidx(d, i, j, k0);
    float2 sz[5], kz[3];
#pragma unroll
    for (int q = 0; q < 5; q++) sz[q] = lds2(k0 - 2 + q, cc + (long long)(q - 2) * plane);
#pragma unroll
    for (int q = 0; q < 3; q++) kz[q] = ld2(K, cc + (long long)(q - 1) * plane + kzoff(k0 - 1 + q));
    float2 wb = ld2(W, cc - plane);
    float2 fzb = make_float2(kappa_flux<T>(wb.x, sz[0].x, sz[1].x, sz[2].x, sz[3].x),
                             kappa_flux<T>(wb.y, sz[0].y, sz[1].y, sz[2].y, sz[3].y));
    auto load_plane = [&](long long c) {
      PairPlane p;
      p.sm = ld2(S, c + oxm); p.sp = ld2(S, c + oxp);  // S(i-2, i-1), S(i+2, i+3)
      p.km = ld2(K, c + oxm); p.kp = ld2(K, c + oxp);  // .y = K(i-1), .x = K(i+2)
      p.um = ld2(U, c - 2); p.u0 = ld2(U, c);          // .y = U(i-1); U(i), U(i+1)
      p.vs = ld2(V, c - pitch); p.vn = ld2(V, c);
      p.wt = ld2(W, c);
      p.sym2 = ld2(S, c + oy[0]); p.sym1 = ld2(S, c + oy[1]); p.syp1 = ld2(S, c + oy[3]); p.syp2 = ld2(S, c + oy[4]);
      p.kym = ld2(K, c + oy[1]); p.kyp = ld2(K, c + oy[3]);
      p.told = stage1 ? make_float2(0.f, 0.f) : ld2(Sadv, c);
      return p;
    };
    PairPlane cur = load_plane(cc);
    for (int k = k0; k <= k1; k++) {
      // the next level's inputs are requested before this level's arithmetic
      PairPlane nxt = cur;
      float2 sz_n = sz[4], kz_n = kz[2];
      if (k < k1) {
        nxt = load_plane(cc + plane);
        sz_n = lds2(k + 3, cc + 3 * plane);
        kz_n = ld2(K, cc + 2 * plane + kzoff(k + 2));
      }
      const float2 s0 = sz[2];
      const float2 sm = cur.sm, sp = cur.sp, km = cur.km, kp = cur.kp, um = cur.um, u0 = cur.u0;
      const float2 vs = cur.vs, vn = cur.vn, wt = cur.wt;
      const float2 sym2 = cur.sym2, sym1 = cur.sym1, syp1 = cur.syp1, syp2 = cur.syp2;
      const float2 kym = cur.kym, kyp = cur.kyp, told = cur.told;
      // x faces: low face of cell i, the face between the pair, high face of
      // i+1, with the full face velocities (stored deviation + level offset)
      const T uo = vel_off(d, 0, k), vo = vel_off(d, 1, k);
      const T f0 = kappa_flux<T>(um.y + uo, sm.x, sm.y, s0.x, s0.y);
      const T f1 = kappa_flux<T>(u0.x + uo, sm.y, s0.x, s0.y, sp.x);
      const T f2 = kappa_flux<T>(u0.y + uo, s0.x, s0.y, sp.x, sp.y);
      const float2 fzt = make_float2(kappa_flux<T>(wt.x, sz[1].x, s0.x, sz[3].x, sz[4].x),
                                     kappa_flux<T>(wt.y, sz[1].y, s0.y, sz[3].y, sz[4].y));
      const bool even = ((k - 1) & 1) == 0;  // face k-1 is even
      const bool wmk = (k == 1 && wm_lo) || (k == nz && wm_hi);
      float2 out_a, out_n;
#pragma unroll
      for (int c = 0; c < 2; c++) {
        // the pair's lanes: x neighbours, y and z neighbours of cell i + c
        const T sc = c ? s0.y : s0.x;
        const T sxm1 = c ? s0.x : sm.y, sxp1 = c ? sp.x : s0.y;
        const T kxm = c ? kz[1].x : km.y, kxp = c ? kp.x : kz[1].y, k0v = c ? kz[1].y : kz[1].x;
        const T fl = c ? f1 : f0, fh = c ? f2 : f1;
        const T vsc = (c ? vs.y : vs.x) + vo, vnc = (c ? vn.y : vn.x) + vo;
        const T a2 = c ? sym2.y : sym2.x, a1 = c ? sym1.y : sym1.x, b1 = c ? syp1.y : syp1.x, b2 = c ? syp2.y : syp2.x;
        T a = (T)0;
        a = a + Ax * fl;
        a = a - Ax * fh;
        a = a + Ay * kappa_flux<T>(vsc, a2, a1, sc, b1);
        a = a - Ay * kappa_flux<T>(vnc, a1, sc, b1, b2);
        const T fb = c ? fzb.y : fzb.x, ft = c ? fzt.y : fzt.x;
        if (even) {
          a = a + Az * fb;
          a = a - Az * ft;
        } else {
          a = a - Az * ft;
          a = a + Az * fb;
        }
        const T kym_c = c ? kym.y : kym.x, kyp_c = c ? kyp.y : kyp.x;
        const T zp = c ? sz[3].y : sz[3].x, zm = c ? sz[1].y : sz[1].x;
        const T kzp = c ? kz[2].y : kz[2].x, kzm = c ? kz[0].y : kz[0].x;
        if constexpr (BC) {  // a solid cell keeps no advection tendency
          if (d.pmask && (d.pmask[cc + c] & 1)) a = (T)0;
        }
        a = a + (kxp + k0v) * (sxp1 - sc) * Dx;
        a = a - (k0v + kxm) * (sc - sxm1) * Dx;
        a = a + (kyp_c + k0v) * (b1 - sc) * Dy;
        a = a - (k0v + kym_c) * (sc - a1) * Dy;
        a = a + (kzp + k0v) * (zp - sc) * Dz;
        a = a - (k0v + kzm) * (sc - zm) * Dz;
        if (srcm) {
          for (int q = 0; q < d.nsrc; q++)
            if (((srcm >> q) & 1u) && d.src_i[q] == i + c && d.src_k[q] == k) a = a + (T)d.src_q[q];
        }
        bool wmc = wmk;
        if constexpr (BC) {
          if (d.pmask) wmc = (d.pmask[cc + c] & 2) != 0;
        }
        if (wmc) {
          if constexpr (BC) {
            if (!d.pmask || (d.pmask[cc + c] & 4)) {
              a = a + (T)sl.wflux[k == 1 ? 0 : 1];
              const double *tpr = s == 0 ? d.wm_pr_tf[k == 1 ? 0 : 1] : nullptr;
              if (tpr) a = a + (T)(tpr[(i + c - 1) + (long long)nx * (j - 1)] * d.wm_af);
            }
          }
          const T dzk = (T)d.dzPr[k + 2];
          const T ue = c ? u0.y : u0.x, uw = c ? u0.x : um.y;
          const T wtc = c ? wt.y : wt.x, wbc = c ? wb.y : wb.x;
          T div = (T)0;
          if (BC && d.pmask) {  // the offsets are zero with solid bodies
            const unsigned char *pm = d.pmask + cc + c;
            if (!(pm[1] & 1)) div = div + ue / rdx;
            if (!(pm[-1] & 1)) div = div - uw / rdx;
            if (!(pm[pitch] & 1)) div = div + (c ? vn.y : vn.x) / rdy;
            if (!(pm[-pitch] & 1)) div = div - (c ? vs.y : vs.x) / rdy;
            if (!(pm[plane] & 1)) div = div + wtc / dzk;
            if (!(pm[-plane] & 1)) div = div - wbc / dzk;
          } else {
            div = div + ue / rdx;
            div = div - uw / rdx;
            div = div + (c ? vn.y : vn.x) / rdy;  // stored values: the level offset cancels
            div = div - (c ? vs.y : vs.x) / rdy;
            div = div + wtc / dzk;
            div = div - wbc / dzk;
          }
          a = a + div * sc;
        }
        T t2 = stage1 ? (T)0 : (c ? told.y : told.x) * rdt;
        t2 = t2 + a * bdt;
        if (c) { out_a.y = a; out_n.y = sc + t2; } else { out_a.x = a; out_n.x = sc + t2; }
      }
      *reinterpret_cast<float2 *>(Sadv + cc) = out_a;
      *reinterpret_cast<float2 *>(Snew + cc) = out_n;
      if (k < k1) {
#pragma unroll
        for (int q = 0; q < 4; q++) sz[q] = sz[q + 1];
        sz[4] = sz_n;
        kz[0] = kz[1];
        kz[1] = kz[2];
        kz[2] = kz_n;
        wb = wt;
        fzb = fzt;
        cc += plane;
        cur = nxt;
      }
    }
  }
}

// PreparePuffs (src/puffs.f90:30-84) at the start of a step, one thread per
// domain: whether each puff restarts in this step, the fraction of the step
// its window covers (the restart branch keeps the reference's
// `time + dt - max(...) / dt`), the time of its last release (updated at the
// last stage there; nothing reads it in between), and the clock.
template <typename T>
__global__ void k_puff_step(const Dom<T> *__restrict__ doms, int nd) {
  const int di = blockIdx.x * blockDim.x + threadIdx.x;
  if (di >= nd) return;
  const Dom<T> &d = doms[di];
  if (d.npuff == 0) return;
  double *st = d.puff_state;
  const double time = st[4 * kMaxPuffs], dt = d.dt;
  for (int p = 0; p < d.npuff; p++) {
    double last = st[4 * p];
    const double start = d.puff_start[p], end = d.puff_end[p], period = d.puff_period[p], dur = d.puff_dur[p];
    const bool restart = time + dt > last + period && time + dt >= start && time <= end;
    double f;
    if (!restart && time <= last + dur && time >= start)
      f = fmax(fmin(fmin(last + dur, time + dt), end) - time, 0.0) / dt;
    else if (restart)
      f = time + dt - fmax(fmax(last + period, time), start) / dt;
    else
      f = 0;
    st[4 * p + 1] = f;
    st[4 * p + 2] = restart ? 1.0 : 0.0;
    if (restart) last = last >= start ? last + period : start;
    st[4 * p] = last;
  }
  st[4 * kMaxPuffs] = time + dt;
}

// DoPuffs (src/puffs.f90:86-126) after a scalar stage, one thread per puff
// volume: the volume's fraction x flux joins the stage tendency of its cell,
// and beta dt of it the new value (the RK combine is linear in the
// tendency; in the reference the term comes after the point sources,
// src/scalars.f90:366-372).  Kept out of the stencil kernels, whose
// registers are spoken for.
template <typename T>
__global__ void k_puff_add(const Dom<T> *__restrict__ doms, int nd, int stage, double beta) {
  for (int di = 0; di < nd; di++) {
    const Dom<T> &d = doms[di];
    const int q = threadIdx.x;
    if (q >= d.npv) continue;
    const double f = d.puff_state[4 * d.pv_puff[q] + 1];
    if (!(f > 0)) continue;
    const ScalSlot<T> &sl = d.slot[d.pv_slot[q]];
    const long long c = bidx(d, d.pv_i[q], d.pv_j[q], d.pv_k[q]);
    const double add = f * d.pv_q[q];
    atomicAdd(sl.adv + c, (T)add);
    atomicAdd(sl.buf[stage % 3] + c, (T)(beta * d.dt * add));
  }
}

// The `clear` of a releasing puff: its scalars are set to zero, ghosts
// included, before the first stage reads them (src/puffs.f90:66-74).
template <typename T>
__global__ void k_puff_clear(const Dom<T> *__restrict__ doms, int nd) {
  for (int di = 0; di < nd; di++) {
    const Dom<T> &d = doms[di];
    if (!d.puff_clear_any) continue;
    unsigned slots = 0;
    for (int p = 0; p < d.npuff; p++)
      if (d.puff_state[4 * p + 2] != 0) slots |= d.puff_clear_slots[p];
    if (!slots) continue;
    const long long n = d.plane * (long long)(d.nz + 2);
    for (int s = 0; s < d.nslot; s++) {
      if (!((slots >> s) & 1u)) continue;
      T *F = d.slot[s].buf[0];
      for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        F[q] = (T)(0.0 - d.slot[s].off);
      for (int side = 0; side < 2; side++) {  // a slab's second halo planes (every slab clears at once)
        T *H = d.slot[s].h2[side];
        if (!H) continue;
        for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.plane;
             q += (long long)gridDim.x * blockDim.x)
          H[q] = (T)(0.0 - d.slot[s].off);
      }
    }
  }
}

// A stage run on its own (elmm_run_stage) leaves the new value in buf[from];
// this copies planes 1..nz of every slot of every domain into buf[0], where
// the host reads it, in 16-byte vectors (a box starts on a 256-byte boundary
// and a plane is a whole number of 128-byte rows).  Tiles: (slot, chunk of
// kCommitVecs vectors); a thread moves kCommitPer vectors with all its loads
// issued first.  Steps never need it: the rotation of the buffers brings the
// value back to buf[0] after the third stage.
constexpr int kCommitThreads = 256, kCommitPer = 4, kCommitVecs = kCommitThreads * kCommitPer;

template <typename T>
__global__ void k_scalar_commit(const Dom<T> *__restrict__ doms, Launch L, int from) {
  typedef typename Vec2<T>::type V2;
  typedef float4 V;  // 16 bytes: 4 floats or 2 doubles
  static_assert(sizeof(V2) * 2 == sizeof(V) || sizeof(V2) == sizeof(V), "16-byte vectors");
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    const int lt = t - __ldg(L.starts + di);
    const long long nvec = d.plane * d.nz * (long long)sizeof(T) / 16;
    const int per = (int)((nvec + kCommitVecs - 1) / kCommitVecs);
    const int s = lt / per, c = lt % per;
    const V *src = reinterpret_cast<const V *>(d.slot[s].buf[from] + d.plane);
    V *dst = reinterpret_cast<V *>(d.slot[s].buf[0] + d.plane);
    const long long v0 = (long long)c * kCommitVecs + threadIdx.x;
    V x[kCommitPer];
#pragma unroll
    for (int q = 0; q < kCommitPer; q++)
      if (v0 + q * kCommitThreads < nvec) x[q] = __ldg(src + v0 + q * kCommitThreads);
#pragma unroll
    for (int q = 0; q < kCommitPer; q++)
      if (v0 + q * kCommitThreads < nvec) dst[v0 + q * kCommitThreads] = x[q];
  }
}

// Scalar_avg = Scalar_avg + Scalar * time_weight (src/outputs.f90:1043-1045)
// on the two slice planes of every passive scalar, after the last stage of a
// step.  Tiles: (slot, row of the slice planes) per domain, rows of the xy
// plane first; one thread per cell of the row.
template <typename T>
__global__ void k_scalar_avg(const Dom<T> *__restrict__ doms, Launch L) {
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    int lt = t - __ldg(L.starts + di);
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const int rows = (d.avg_k > 0 ? ny : 0) + (d.avg_j > 0 ? nz : 0);
    const int s = (d.buoy ? 1 : 0) + lt / rows;  // the passive slots follow the temperature
    const int r = lt % rows;
    const ScalSlot<T> &sl = d.slot[s];
    const bool xy = d.avg_k > 0 && r < ny;
    const int j = xy ? r + 1 : d.avg_j, k = xy ? d.avg_k : r - (d.avg_k > 0 ? ny : 0) + 1;
    double *acc = xy ? sl.acc_xy + (size_t)(j - 1) * nx : sl.acc_xz + (size_t)(k - 1) * nx;
    const T *S = sl.buf[0] + bidx(d, 1, j, k);
    // a variable step weighs its length / dt of the configured weight
    const double w = d.vdt ? d.avg_w * (d.dt / d.dt0) : d.avg_w;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) acc[i] = acc[i] + ((double)S[i] + sl.off) * w;
  }
}

// interior of Temperature(-2:n+3) or Scalar(-2:n+3,sc) (host, double) ->
// the box of scalar slot s, minus its offset
template <typename T>
__global__ void k_unpack_scalar(const Dom<T> *__restrict__ dom, int s, const double *__restrict__ src, int *bad) {
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
    d.slot[s].buf[0][bidx(d, i, j, k)] = (T)(v - d.slot[s].off);
  }
}

// box field F with lower bound lo (-2: Temperature, Scalar and their _adv;
// -1: TDiff) -> host array, every ghost folded onto the interior (periodic
// copy where per[axis], else the nearest interior cell), plus add.
// interior_only: ghosts are 0.
template <typename T>
__global__ void k_pack_scalar_box(const Dom<T> *__restrict__ dom, const T *F, double *dst, int lo, double add,
                                  int interior_only, int px, int py, int pz) {
  const Dom<T> &d = *dom;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const int n0 = nx + 2 * (1 - lo), n1 = ny + 2 * (1 - lo), n2 = nz + 2 * (1 - lo);
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
