// elmm_kernels.cuh -- the sm_100a kernels of one RK3 stage of TMarchRK3
// (src/tsteps.f90:24-243), templated on the storage/arithmetic type T
// (double: plain FP64 path; float: mixed path, whose reductions, singular
// Poisson mode and divergence residual stay in FP64).
//
// Every kernel walks a flattened list of tiles that may span several domains
// (a batch); find_dom() maps a tile to its domain.  The grid is sized to the
// number of resident blocks and each block strides over the tiles.
//
// Per stage:
//   k_sgs       SubgridStresses: Smagorinsky viscosity (+ ghosts),
//               wall-model fluxes (dynamics.f90:869-908)
//   k_momentum  Convection + OtherTerms: CDS2 advection, diffusion with the
//               wall-flux corrections, RK combine, old-pressure gradient,
//               U2 += U; writes U2 with its ghosts (dynamics.f90:230-499,
//               tsteps.f90:263-358)
//   k_fftx_fwd  divergence RHS (pressure.f90:688-717) fused with the real
//               FFT along x
//   k_ffty      complex FFT along y (forward, then inverse)
//   k_tri       tridiagonal solve in z per wavenumber pair
//   k_fftx_inv  inverse real FFT along x -> Phi with its ghosts
//   k_project   PostPoisson (pressure.f90:728-991): U = U2 - coef grad Phi,
//               Pr += Phi, top-layer partial sums for FixPressureToReference
//   k_prref     the pressure reference (pressure.f90:1160-1220)
#pragma once

#include "elmm_common.cuh"
#include "elmm_fft.cuh"

namespace elmm {

constexpr int TX = 32, TY = 4;  // cell tile of the stencil kernels

struct Launch {
  const int *starts;  // per-domain first tile, nd + 1 entries (device)
  int nd;
  int total;          // total tiles
};

template <typename T>
__device__ __forceinline__ T ld(const T *p, long long o) { return __ldg(p + o); }

// ------------------------------------------------------------------ k_sgs
// One thread per cell of the Pr box including its one-cell ghost shell; a
// ghost cell takes the viscosity of the interior cell it folds onto
// (BoundViscosity), computed again rather than read back.
template <typename T>
__device__ __forceinline__ T nusmag(const Dom<T> &d, int i, int j, int k) {
  const T *U = d.U, *V = d.V, *W = d.W;
  const T dx = (T)d.dx, dy = (T)d.dy;
  const T dzk = (T)d.dzPr[k + 2];
  const T zz = (T)(d.zPr[k + 1 + 2] - d.zPr[k - 1 + 2]);
  const long long c = bidx(d, i, j, k);
  const long long sx = 1, sy = d.pitch, sz = d.plane;
  T D00 = (ld(U, c) - ld(U, c - sx)) / dx;
  T D11 = (ld(V, c) - ld(V, c - sy)) / dy;
  T D22 = (ld(W, c) - ld(W, c - sz)) / dzk;
  T D01 = (ld(U, c + sy) + ld(U, c - sx + sy) - ld(U, c - sy) - ld(U, c - sx - sy)) / (4 * dy);
  T D02 = (ld(U, c + sz) + ld(U, c - sx + sz) - ld(U, c - sz) - ld(U, c - sx - sz)) / (2 * zz);
  T D10 = (ld(V, c + sx) + ld(V, c + sx - sy) - ld(V, c - sx) - ld(V, c - sx - sy)) / (4 * dx);
  T D12 = (ld(V, c + sz) + ld(V, c - sy + sz) - ld(V, c - sz) - ld(V, c - sy - sz)) / (2 * zz);
  T D20 = (ld(W, c + sx) + ld(W, c + sx - sz) - ld(W, c - sx) - ld(W, c - sx - sz)) / (4 * dx);
  T D21 = (ld(W, c + sy) + ld(W, c + sy - sz) - ld(W, c - sy) - ld(W, c - sy - sz)) / (4 * dy);
  // Strainu: sum over jj (outer), ii (inner) of S(ii,jj)^2 (subgrid.f90:170-181)
  T s, S = 0;
  s = (D00 + D00) / 2; S = S + s * s;
  s = (D10 + D01) / 2; S = S + s * s;
  s = (D20 + D02) / 2; S = S + s * s;
  s = (D01 + D10) / 2; S = S + s * s;
  s = (D11 + D11) / 2; S = S + s * s;
  s = (D21 + D12) / 2; S = S + s * s;
  s = (D02 + D20) / 2; S = S + s * s;
  s = (D12 + D21) / 2; S = S + s * s;
  s = (D22 + D22) / 2; S = S + s * s;
  T Sbar = sqrt((T)2 * S);
  T wc = (T)d.width[k] * (T)d.cs;
  return Sbar * (wc * wc);
}

// gfortran's NORM2: scaled sum of squares
__device__ __forceinline__ double norm2_3(const double *x) {
  double scale = 0, ssq = 1;
#pragma unroll
  for (int m = 0; m < 3; m++) {
    if (x[m] != 0) {
      double ax = fabs(x[m]);
      if (scale < ax) { double r = scale / ax; ssq = 1 + ssq * (r * r); scale = ax; }
      else { double r = ax / scale; ssq = ssq + r * r; }
    }
  }
  return scale * sqrt(ssq);
}

// WMFlatUstar / WMRoughUstar, src/wallmodels.f90:1190-1335
__device__ inline double wm_flat_ustar(double ustar, double vel, double dist, double nu) {
  if (nu <= 0) return 0;
  double ustar_lam = sqrt(nu * vel / dist);
  if ((dist * ustar_lam / nu) < 5.0) return ustar_lam;
  for (int i = 1;; i++) {  // at most 50 iterations (wallmodels.f90:1230)
    double ustar2 = ustar;
    double z_pl = dist * ustar2 / nu;
    if (z_pl <= 5.0) ustar = sqrt(nu * vel / dist);
    else if (z_pl < 30.0) ustar = vel / (5 * log(z_pl) - (double)3.05f);
    else ustar = vel / (log(z_pl) / 0.4 + 5.5);
    if (fabs(ustar - ustar2) / fabs(ustar) < 1e-4) return ustar;
    if (i >= 50) return 0;
  }
}

__device__ inline double wm_rough_ustar(double ustar, double vel, double dist, double z0, double nu) {
  if (nu > 0) {
    ustar = sqrt(nu * vel / dist);
    if (dist * ustar / nu < 11.225 * 1.1) return ustar;
  }
  if (dist <= z0 * 2) return nu > 0 ? wm_flat_ustar(ustar, vel, dist, nu) : 0.0;
  return vel * 0.41 / log(dist / z0);
}

// ComputeUVWFluxesWM / fluxes for the point of component comp on side f at
// cell (i,j,k) (src/wallmodels.f90:2159-2338); the wall-point distance is
// the one of GetOutsideBoundariesWM_UVW (src/wallmodels.f90:690-909).
template <typename T>
__device__ void wm_point(const Dom<T> &d, int comp, int f, int i, int j, int k, long long pidx) {
  const T *U = d.U, *V = d.V, *W = d.W;
  const long long c = bidx(d, i, j, k), sx = 1, sy = d.pitch, sz = d.plane;
  double vel[3];
  if (comp == 0) {
    vel[0] = (double)ld(U, c);
    vel[1] = ((double)ld(V, c + sx) + (double)ld(V, c) + (double)ld(V, c + sx - sy) + (double)ld(V, c - sy)) / 4.0;
    vel[2] = ((double)ld(W, c + sx) + (double)ld(W, c) + (double)ld(W, c + sx - sz) + (double)ld(W, c - sz)) / 4.0;
  } else if (comp == 1) {
    vel[0] = ((double)ld(U, c + sy) + (double)ld(U, c) + (double)ld(U, c - sx + sy) + (double)ld(U, c - sx)) / 4.0;
    vel[1] = (double)ld(V, c);
    vel[2] = ((double)ld(W, c + sy) + (double)ld(W, c) + (double)ld(W, c + sy - sz) + (double)ld(W, c - sz)) / 4.0;
  } else {
    vel[0] = ((double)ld(U, c + sz) + (double)ld(U, c) + (double)ld(U, c - sx + sz) + (double)ld(U, c - sx)) / 4.0;
    vel[1] = ((double)ld(V, c + sz) + (double)ld(V, c) + (double)ld(V, c - sy + sz) + (double)ld(V, c - sy)) / 4.0;
    vel[2] = (double)ld(W, c);
  }
  // distance to the wall: xU(0) - x(1) etc. with the staggered coordinate of the component
  double dist[3] = {0, 0, 0};
  const int axis = f >> 1;
  const bool hi = f & 1;
  if (axis == 0) {
    // xU(i) = i dxmin + xmin, xPr(i) = (xU(i-1) + xU(i)) / 2 (initial.f90:4395-4450)
    double xc = comp == 0 ? (double)i * d.dx + d.xmin
                          : (((double)(i - 1) * d.dx + d.xmin) + ((double)i * d.dx + d.xmin)) / 2.0;
    double xw = hi ? (double)(d.ext[0][0] + 1) * d.dx + d.xmin : 0.0 * d.dx + d.xmin;
    dist[0] = xw - xc;
  } else if (axis == 1) {
    double yc = comp == 1 ? (double)j * d.dy + d.ymin
                          : (((double)(j - 1) * d.dy + d.ymin) + ((double)j * d.dy + d.ymin)) / 2.0;
    double yw = hi ? (double)(d.ext[1][1] + 1) * d.dy + d.ymin : 0.0 * d.dy + d.ymin;
    dist[1] = yw - yc;
  } else {
    double zc = comp == 2 ? d.zW[k + 2] : d.zPr[k + 2];
    double zw = hi ? d.zW[d.ext[2][2] + 1 + 2] : d.zW[0 + 2];
    dist[2] = zw - zc;
  }
  double dd = norm2_3(dist);
  double t[3] = {vel[0], vel[1], vel[2]};  // wall velocity 0
  double dot = t[0] * dist[0] + t[1] * dist[1] + t[2] * dist[2];
#pragma unroll
  for (int m = 0; m < 3; m++) t[m] = t[m] - dot * dist[m] / (dd * dd);
  double tv = norm2_3(t);
  const int face = comp * 6 + f;
  double ustar = d.wm_ustar[face][pidx];
  if (tv != 0) ustar = wm_rough_ustar(ustar, tv, dd, d.z0[f], d.nu_mol);
  if (ustar < 0) ustar = 0;
  d.wm_ustar[face][pidx] = ustar;
  double mag = norm2_3(t);
  double fp = 0, fm = 0;
  if (mag > 1.4901161193847656e-08) {
    if (d.vz && f == SIDE_BO) {
      fp = (t[comp] / mag) * (ustar * ustar);
      fm = fp;
      if (comp < 2) { fp = fp / d.dzPr[k + 2]; fm = fm / d.dzPr[k - 1 + 2]; }
      else { fp = fp / d.dzW[k + 2]; fm = fm / d.dzW[k - 1 + 2]; }
    } else if (d.vz && f == SIDE_TO) {
      fp = (t[comp] / mag) * (ustar * ustar);
      fm = fp;
      if (comp < 2) { fp = fp / d.dzPr[k + 1 + 2]; fm = fm / d.dzPr[k + 2]; }
      else { fp = fp / d.dzW[k + 1 + 2]; fm = fm / d.dzW[k + 2]; }
    } else {
      double drec = axis == 0 ? 1 / d.dx : axis == 1 ? 1 / d.dy : 1 / d.dz;
      fp = (t[comp] / mag) * (ustar * ustar) * drec;
      fm = fp;
    }
    if (!hi) { fp = -fp; fm = -fm; }  // MINUSX/Y/Z directions are odd
  }
  d.wm_fluxp[face][pidx] = (T)fp;
  d.wm_fluxm[face][pidx] = (T)fm;
}

// index of cell (i,j,k) in the face plane of side f for component comp, or -1
template <typename T>
__device__ __forceinline__ long long wm_plane_index(const Dom<T> &d, int comp, int f, int i, int j, int k) {
  const int *e = d.ext[comp];
  if (i < 1 || i > e[0] || j < 1 || j > e[1] || k < 1 || k > e[2]) return -1;
  switch (f) {
    case SIDE_WE: return i == 1 ? (long long)(j - 1) + (long long)e[1] * (k - 1) : -1;
    case SIDE_EA: return i == e[0] ? (long long)(j - 1) + (long long)e[1] * (k - 1) : -1;
    case SIDE_SO: return j == 1 ? (long long)(i - 1) + (long long)e[0] * (k - 1) : -1;
    case SIDE_NO: return j == e[1] ? (long long)(i - 1) + (long long)e[0] * (k - 1) : -1;
    case SIDE_BO: return k == 1 ? (long long)(i - 1) + (long long)e[0] * (j - 1) : -1;
    default: return k == e[2] ? (long long)(i - 1) + (long long)e[0] * (j - 1) : -1;
  }
}

template <typename T>
__global__ void __launch_bounds__(TX *TY) k_sgs(const Dom<T> *__restrict__ doms, Launch L) {
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    int lt = t - __ldg(L.starts + di);
    const int ntx = (d.nx + 2 + TX - 1) / TX, nty = (d.ny + 2 + TY - 1) / TY;
    const int tx = lt % ntx; lt /= ntx;
    const int ty = lt % nty;
    const int k = lt / nty;  // 0..nz+1
    const int i = tx * TX + (threadIdx.x % TX);
    const int j = ty * TY + (threadIdx.x / TX);
    if (i > d.nx + 1 || j > d.ny + 1) continue;
    const int si = fold_rep(i, d.nx, d.bt[SIDE_WE] == BC_PERIODIC);
    const int sj = fold_rep(j, d.ny, d.bt[SIDE_SO] == BC_PERIODIC);
    const int sk = fold_rep(k, d.nz, d.bt[SIDE_BO] == BC_PERIODIC);
    T nu;
    if (d.sgs) {
      nu = nusmag(d, si, sj, sk);
      if (d.nu_mol > 0) nu = nu + (T)d.nu_mol;
    } else {
      nu = (T)d.nu_mol;
    }
    d.nu[bidx(d, i, j, k)] = nu;
    if (si != i || sj != j || sk != k) continue;
    // wall-model fluxes of the velocity points at this cell
#pragma unroll 1
    for (int f = 0; f < 6; f++) {
      if (!d.wall[f]) continue;
#pragma unroll 1
      for (int comp = 0; comp < 3; comp++) {
        long long p = wm_plane_index(d, comp, f, i, j, k);
        if (p >= 0) wm_point(d, comp, f, i, j, k, p);
      }
    }
  }
}

// ------------------------------------------------------------- k_momentum
struct StageCoef {
  double rho, beta, alpha2;  // RK_rho, RK_beta, 2*RK_alpha of the stage
  int stage;
};

// advection + diffusion + wall corrections of one component at (i,j,k)
// (advection.f90:15-327, advection_variable_z.f90:15-324,
//  momentum_diffusion.f90:169-420 and the wmfluxes includes)
template <typename T>
__device__ __forceinline__ T tendency_u(const Dom<T> &d, int i, int j, int k, long long c) {
  const T *U = d.U, *V = d.V, *W = d.W, *nu = d.nu;
  const long long sx = 1, sy = d.pitch, sz = d.plane;
  const T u = ld(U, c), ue = ld(U, c + sx), uw = ld(U, c - sx), un = ld(U, c + sy), us = ld(U, c - sy);
  const T ut = ld(U, c + sz), ub = ld(U, c - sz);
  const T v = ld(V, c), ve = ld(V, c + sx), vs = ld(V, c - sy), vse = ld(V, c + sx - sy);
  const T w = ld(W, c), we = ld(W, c + sx), wb = ld(W, c - sz), wbe = ld(W, c + sx - sz);
  T a;
  if (!d.vz) {
    const T Ax = (T)(0.25 / d.dx), Ay = (T)(0.25 / d.dy), Az = (T)(0.25 / d.dz);
    a = -((Ax * (ue + u) * (ue + u) - Ax * (u + uw) * (u + uw)) + (Ay * (un + u) * (ve + v) - Ay * (u + us) * (vse + vs)) +
          (Az * (ut + u) * (we + w) - Az * (u + ub) * (wbe + wb)));
    const T Bx = (T)(0.5 / d.dx), By = (T)(0.125 / d.dy), Bz = (T)(0.125 / d.dz);
    T Vadv = (v + ve + vs + vse);
    T Wadv = (w + we + wb + wbe);
    a = a - (Bx * (ue - uw) * u + By * (un - us) * Vadv + Bz * (ut - ub) * Wadv);
  } else {
    const T Ax = (T)(0.25 / d.dx), Ay = (T)(0.25 / d.dy);
    const T dzp = (T)d.dzPr[k + 2];
    a = -((Ax * (ue + u) * (ue + u) - Ax * (u + uw) * (u + uw)) + (Ay * (un + u) * (ve + v) - Ay * (u + us) * (vse + vs)) +
          ((ut + u) * (we + w) - (u + ub) * (wbe + wb)) / dzp / 4);
    const T Bx = (T)(0.5 / d.dx), By = (T)(0.125 / d.dy);
    T Vadv = (v + ve + vs + vse);
    T Wadv = (w + we + wb + wbe) / 4;
    a = a - (Bx * (ue - uw) * u + By * (un - us) * Vadv + (ut - ub) / (T)(d.zPr[k + 1 + 2] - d.zPr[k - 1 + 2]) * Wadv);
  }
  a = a * (T)0.5;
  // diffusion
  const T rx = (T)(1.0 / (d.dx * d.dx)), ry = (T)(1.0 / (d.dy * d.dy)), rz = (T)(1.0 / (d.dz * d.dz));
  const T n0 = ld(nu, c), ne = ld(nu, c + sx), nn = ld(nu, c + sy), nne = ld(nu, c + sx + sy), ns = ld(nu, c - sy),
          nse = ld(nu, c + sx - sy), nt = ld(nu, c + sz), nte = ld(nu, c + sx + sz), nb = ld(nu, c - sz),
          nbe = ld(nu, c + sx - sz);
  a = a + ne * (ue - u) * rx;
  a = a - n0 * (u - uw) * rx;
  a = a + (T)0.25 * (nne + ne + nn + n0) * (un - u) * ry;
  a = a - (T)0.25 * (ne + nse + n0 + ns) * (u - us) * ry;
  if (!d.vz) {
    a = a + (T)0.25 * (nte + ne + nt + n0) * (ut - u) * rz;
    a = a - (T)0.25 * (ne + nbe + n0 + nb) * (u - ub) * rz;
  } else {
    T tz = (T)0.25 * (nte + ne + nt + n0) * (ut - u) / (T)d.dzW[k + 2];
    tz = tz - (T)0.25 * (ne + nbe + n0 + nb) * (u - ub) / (T)d.dzW[k - 1 + 2];
    tz = tz / (T)d.dzPr[k + 2];
    a = a + tz;
  }
  // wall-flux corrections (wmfluxes-[variable_z-]nobranch-U-inc.f90), list order xm, xp, ym, yp, zm, zp
  const int *e = d.ext[0];
  if (d.wall[SIDE_WE] && i == 1) {
    long long p = (long long)(j - 1) + (long long)e[1] * (k - 1);
    a = a + n0 * (u - uw) * rx;
    a = a + d.wm_fluxp[0 * 6 + SIDE_WE][p];
  }
  if (d.wall[SIDE_EA] && i == e[0]) {
    long long p = (long long)(j - 1) + (long long)e[1] * (k - 1);
    a = a - ne * (ue - u) * rx;
    a = a - d.wm_fluxm[0 * 6 + SIDE_EA][p];
  }
  if (d.wall[SIDE_SO] && j == 1) {
    long long p = (long long)(i - 1) + (long long)e[0] * (k - 1);
    a = a + (ne + nse + n0 + ns) * (u - us) * ry / 4;
    a = a + d.wm_fluxp[0 * 6 + SIDE_SO][p];
  }
  if (d.wall[SIDE_NO] && j == e[1]) {
    long long p = (long long)(i - 1) + (long long)e[0] * (k - 1);
    a = a - (nne + ne + nn + n0) * (un - u) * ry / 4;
    a = a - d.wm_fluxm[0 * 6 + SIDE_NO][p];
  }
  if (d.wall[SIDE_BO] && k == 1) {
    long long p = (long long)(i - 1) + (long long)e[0] * (j - 1);
    T s = ne + nbe + n0 + nb;
    if (d.vz) a = a + s * (u - ub) / (T)d.dzW[k - 1 + 2] / 4 / (T)d.dzPr[k + 2];
    else a = a + s * (u - ub) * rz / 4;
    a = a + d.wm_fluxp[0 * 6 + SIDE_BO][p];
  }
  if (d.wall[SIDE_TO] && k == e[2]) {
    long long p = (long long)(i - 1) + (long long)e[0] * (j - 1);
    T s = nte + ne + nt + n0;
    if (d.vz) a = a - s * (ut - u) / (T)d.dzW[k + 2] / 4 / (T)d.dzPr[k + 2];
    else a = a - s * (ut - u) * rz / 4;
    a = a - d.wm_fluxm[0 * 6 + SIDE_TO][p];
  }
  return a;
}

template <typename T>
__device__ __forceinline__ T tendency_v(const Dom<T> &d, int i, int j, int k, long long c) {
  const T *U = d.U, *V = d.V, *W = d.W, *nu = d.nu;
  const long long sx = 1, sy = d.pitch, sz = d.plane;
  const T v = ld(V, c), ve = ld(V, c + sx), vw = ld(V, c - sx), vn = ld(V, c + sy), vs = ld(V, c - sy);
  const T vt = ld(V, c + sz), vb = ld(V, c - sz);
  const T u = ld(U, c), un = ld(U, c + sy), uw = ld(U, c - sx), unw = ld(U, c - sx + sy);
  const T w = ld(W, c), wn = ld(W, c + sy), wb = ld(W, c - sz), wbn = ld(W, c + sy - sz);
  T a;
  if (!d.vz) {
    const T Ax = (T)(0.25 / d.dx), Ay = (T)(0.25 / d.dy), Az = (T)(0.25 / d.dz);
    a = -((Ay * (vn + v) * (vn + v) - Ay * (v + vs) * (v + vs)) + (Ax * (ve + v) * (un + u) - Ax * (v + vw) * (unw + uw)) +
          (Az * (vt + v) * (wn + w) - Az * (v + vb) * (wbn + wb)));
    const T Bx = (T)(0.125 / d.dx), By = (T)(0.5 / d.dy), Bz = (T)(0.125 / d.dz);
    T Uadv = (u + un + uw + unw);
    T Wadv = (w + wn + wb + wbn);
    a = a - (Bx * (ve - vw) * Uadv + By * (vn - vs) * v + Bz * (vt - vb) * Wadv);
  } else {
    const T Ax = (T)(0.25 / d.dx), Ay = (T)(0.25 / d.dy);
    const T dzp = (T)d.dzPr[k + 2];
    a = -((Ay * (vn + v) * (vn + v) - Ay * (v + vs) * (v + vs)) + (Ax * (ve + v) * (un + u) - Ax * (v + vw) * (unw + uw)) +
          ((vt + v) * (wn + w) - (v + vb) * (wbn + wb)) / dzp / 4);
    const T Bx = (T)(0.125 / d.dx), By = (T)(0.5 / d.dy);
    T Uadv = (u + un + uw + unw);
    T Wadv = (w + wn + wb + wbn) / 4;
    a = a - (Bx * (ve - vw) * Uadv + By * (vn - vs) * v + (vt - vb) / (T)(d.zPr[k + 1 + 2] - d.zPr[k - 1 + 2]) * Wadv);
  }
  a = a * (T)0.5;
  const T rx = (T)(1.0 / (d.dx * d.dx)), ry = (T)(1.0 / (d.dy * d.dy)), rz = (T)(1.0 / (d.dz * d.dz));
  const T n0 = ld(nu, c), ne = ld(nu, c + sx), nn = ld(nu, c + sy), nne = ld(nu, c + sx + sy), nw = ld(nu, c - sx),
          nnw = ld(nu, c - sx + sy), nt = ld(nu, c + sz), nnt = ld(nu, c + sy + sz), nb = ld(nu, c - sz),
          nnb = ld(nu, c + sy - sz);
  a = a + (T)0.25 * (nne + ne + nn + n0) * (ve - v) * rx;
  a = a - (T)0.25 * (nn + n0 + nnw + nw) * (v - vw) * rx;
  a = a + nn * (vn - v) * ry;
  a = a - n0 * (v - vs) * ry;
  if (!d.vz) {
    a = a + (T)0.25 * (nnt + nn + nt + n0) * (vt - v) * rz;
    a = a - (T)0.25 * (nn + nnb + n0 + nb) * (v - vb) * rz;
  } else {
    T tz = (T)0.25 * (nnt + nn + nt + n0) * (vt - v) / (T)d.dzW[k + 2];
    tz = tz - (T)0.25 * (nn + nnb + n0 + nb) * (v - vb) / (T)d.dzW[k - 1 + 2];
    tz = tz / (T)d.dzPr[k + 2];
    a = a + tz;
  }
  const int *e = d.ext[1];
  if (d.wall[SIDE_WE] && i == 1) {
    long long p = (long long)(j - 1) + (long long)e[1] * (k - 1);
    a = a + (nn + n0 + nnw + nw) * (v - vw) * rx / 4;
    a = a + d.wm_fluxp[1 * 6 + SIDE_WE][p];
  }
  if (d.wall[SIDE_EA] && i == e[0]) {
    long long p = (long long)(j - 1) + (long long)e[1] * (k - 1);
    a = a - (nne + ne + nn + n0) * (ve - v) * rx / 4;
    a = a - d.wm_fluxm[1 * 6 + SIDE_EA][p];
  }
  if (d.wall[SIDE_SO] && j == 1) {
    long long p = (long long)(i - 1) + (long long)e[0] * (k - 1);
    a = a + n0 * (v - vs) * ry;
    a = a + d.wm_fluxp[1 * 6 + SIDE_SO][p];
  }
  if (d.wall[SIDE_NO] && j == e[1]) {
    long long p = (long long)(i - 1) + (long long)e[0] * (k - 1);
    a = a - nn * (vn - v) * ry;
    a = a - d.wm_fluxm[1 * 6 + SIDE_NO][p];
  }
  if (d.wall[SIDE_BO] && k == 1) {
    long long p = (long long)(i - 1) + (long long)e[0] * (j - 1);
    T s = nn + nnb + n0 + nb;
    if (d.vz) a = a + s * (v - vb) / (T)d.dzW[k - 1 + 2] / 4 / (T)d.dzPr[k + 2];
    else a = a + s * (v - vb) * rz / 4;
    a = a + d.wm_fluxp[1 * 6 + SIDE_BO][p];
  }
  if (d.wall[SIDE_TO] && k == e[2]) {
    long long p = (long long)(i - 1) + (long long)e[0] * (j - 1);
    T s = nnt + nn + nt + n0;
    if (d.vz) a = a - s * (vt - v) / (T)d.dzW[k + 2] / 4 / (T)d.dzPr[k + 2];
    else a = a - s * (vt - v) * rz / 4;
    a = a - d.wm_fluxm[1 * 6 + SIDE_TO][p];
  }
  return a;
}

template <typename T>
__device__ __forceinline__ T tendency_w(const Dom<T> &d, int i, int j, int k, long long c) {
  const T *U = d.U, *V = d.V, *W = d.W, *nu = d.nu;
  const long long sx = 1, sy = d.pitch, sz = d.plane;
  const T w = ld(W, c), we = ld(W, c + sx), ww = ld(W, c - sx), wn = ld(W, c + sy), ws = ld(W, c - sy);
  const T wt = ld(W, c + sz), wb = ld(W, c - sz);
  const T u = ld(U, c), ut = ld(U, c + sz), uw = ld(U, c - sx), utw = ld(U, c - sx + sz);
  const T v = ld(V, c), vt = ld(V, c + sz), vs = ld(V, c - sy), vts = ld(V, c - sy + sz);
  T a;
  if (!d.vz) {
    const T Ax = (T)(0.25 / d.dx), Ay = (T)(0.25 / d.dy), Az = (T)(0.25 / d.dz);
    a = -((Az * (wt + w) * (wt + w) - Az * (w + wb) * (w + wb)) + (Ay * (wn + w) * (vt + v) - Ay * (w + ws) * (vs + vts)) +
          (Ax * (we + w) * (ut + u) - Ax * (w + ww) * (utw + uw)));
    const T Bx = (T)(0.125 / d.dx), By = (T)(0.125 / d.dy), Bz = (T)(0.5 / d.dz);
    T Uadv = (u + ut + uw + utw);
    T Vadv = (v + vt + vs + vts);
    a = a - (Bx * (we - ww) * Uadv + By * (wn - ws) * Vadv + Bz * (wt - wb) * w);
  } else {
    const T Ax = (T)(0.25 / d.dx), Ay = (T)(0.25 / d.dy);
    const T dzw = (T)d.dzW[k + 2];
    a = -(((wt + w) * (wt + w) - (w + wb) * (w + wb)) / dzw / 4 + (Ay * (wn + w) * (vt + v) - Ay * (w + ws) * (vts + vs)) +
          (Ax * (we + w) * (ut + u) - Ax * (w + ww) * (utw + uw)));
    const T Bx = (T)(0.125 / d.dx), By = (T)(0.125 / d.dy);
    T Uadv = (u + ut + uw + utw);
    T Vadv = (v + vt + vs + vts);
    a = a - (Bx * (we - ww) * Uadv + By * (wn - ws) * Vadv + (wt - wb) / (T)(d.zW[k + 1 + 2] - d.zW[k - 1 + 2]) * w);
  }
  a = a * (T)0.5;
  const T rx = (T)(1.0 / (d.dx * d.dx)), ry = (T)(1.0 / (d.dy * d.dy)), rz = (T)(1.0 / (d.dz * d.dz));
  const T n0 = ld(nu, c), ne = ld(nu, c + sx), nt = ld(nu, c + sz), nte = ld(nu, c + sx + sz), nw = ld(nu, c - sx),
          ntw = ld(nu, c - sx + sz), nn = ld(nu, c + sy), ntn = ld(nu, c + sy + sz), ns = ld(nu, c - sy),
          nts = ld(nu, c - sy + sz);
  a = a + (T)0.25 * (nte + ne + nt + n0) * (we - w) * rx;
  a = a - (T)0.25 * (nt + n0 + ntw + nw) * (w - ww) * rx;
  a = a + (T)0.25 * (ntn + nt + nn + n0) * (wn - w) * ry;
  a = a - (T)0.25 * (nt + nts + n0 + ns) * (w - ws) * ry;
  if (!d.vz) {
    a = a + nt * (wt - w) * rz;
    a = a - n0 * (w - wb) * rz;
  } else {
    T tz = nt * (wt - w) / (T)d.dzPr[k + 1 + 2];
    tz = tz - n0 * (w - wb) / (T)d.dzPr[k + 2];
    tz = tz / (T)d.dzW[k + 2];
    a = a + tz;
  }
  const int *e = d.ext[2];
  if (d.wall[SIDE_WE] && i == 1) {
    long long p = (long long)(j - 1) + (long long)e[1] * (k - 1);
    a = a + (nt + n0 + ntw + nw) * (w - ww) * rx / 4;
    a = a + d.wm_fluxp[2 * 6 + SIDE_WE][p];
  }
  if (d.wall[SIDE_EA] && i == e[0]) {
    long long p = (long long)(j - 1) + (long long)e[1] * (k - 1);
    a = a - (nte + ne + nt + n0) * (we - w) * rx / 4;
    a = a - d.wm_fluxm[2 * 6 + SIDE_EA][p];
  }
  if (d.wall[SIDE_SO] && j == 1) {
    long long p = (long long)(i - 1) + (long long)e[0] * (k - 1);
    a = a + (nt + nts + n0 + ns) * (w - ws) * ry / 4;
    a = a + d.wm_fluxp[2 * 6 + SIDE_SO][p];
  }
  if (d.wall[SIDE_NO] && j == e[1]) {
    long long p = (long long)(i - 1) + (long long)e[0] * (k - 1);
    a = a - (ntn + nt + nn + n0) * (wn - w) * ry / 4;
    a = a - d.wm_fluxm[2 * 6 + SIDE_NO][p];
  }
  if (d.wall[SIDE_BO] && k == 1) {
    long long p = (long long)(i - 1) + (long long)e[0] * (j - 1);
    if (d.vz) a = a + n0 * (w - wb) / (T)d.dzPr[k + 2] / (T)d.dzW[k + 2];
    else a = a + n0 * (w - wb) * rz;
    a = a + d.wm_fluxp[2 * 6 + SIDE_BO][p];
  }
  if (d.wall[SIDE_TO] && k == e[2]) {
    long long p = (long long)(i - 1) + (long long)e[0] * (j - 1);
    if (d.vz) a = a - nt * (wt - w) / (T)d.dzPr[k + 1 + 2] / (T)d.dzW[k + 2];
    else a = a - nt * (wt - w) * rz;
    a = a - d.wm_fluxm[2 * 6 + SIDE_TO][p];
  }
  return a;
}

template <typename T>
__device__ __forceinline__ T pr_true(const T *P, long long o, T m) { return ld(P, o) - m; }

template <typename T>
__global__ void __launch_bounds__(TX *TY) k_momentum(const Dom<T> *__restrict__ doms, Launch L, StageCoef sc) {
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    int lt = t - __ldg(L.starts + di);
    const int ntx = (d.nx + TX - 1) / TX, nty = (d.ny + TY - 1) / TY;
    const int tx = lt % ntx; lt /= ntx;
    const int ty = lt % nty;
    const int k = lt / nty + 1;
    const int i = tx * TX + (threadIdx.x % TX) + 1;
    const int j = ty * TY + (threadIdx.x / TX) + 1;
    if (i > d.nx || j > d.ny) continue;
    const long long c = bidx(d, i, j, k);
    const T dt = (T)d.dt;
    const T rdt = (T)sc.rho, bdt = (T)sc.beta;
    const T coef = (T)(sc.alpha2 * d.dt);
    const T m = (T)(*d.prm);
    const T *P = d.P;
    // U component
    if (i <= d.ext[0][0] && j <= d.ext[0][1] && k <= d.ext[0][2]) {
      T ts = tendency_u(d, i, j, k, c);
      T u2 = sc.stage > 1 ? d.Us[c] * rdt * dt : (T)0;
      d.Us[c] = ts;
      u2 = u2 + ts * bdt * dt;
      if (d.prgx_on) u2 = u2 + (-coef) * (T)d.prgx;
      u2 = u2 + (-coef / (T)d.dx) * (pr_true(P, c + 1, m) - pr_true(P, c, m));
      u2 = u2 + ld(d.U, c);
      d.U2[c] = u2;
      push_vel(d, d.U2, 0, i, j, k, u2);
    }
    if (i <= d.ext[1][0] && j <= d.ext[1][1] && k <= d.ext[1][2]) {
      T ts = tendency_v(d, i, j, k, c);
      T v2 = sc.stage > 1 ? d.Vs[c] * rdt * dt : (T)0;
      d.Vs[c] = ts;
      v2 = v2 + ts * bdt * dt;
      if (d.prgy_on) v2 = v2 + (-coef) * (T)d.prgy;
      v2 = v2 + (-coef / (T)d.dy) * (pr_true(P, c + d.pitch, m) - pr_true(P, c, m));
      v2 = v2 + ld(d.V, c);
      d.V2[c] = v2;
      push_vel(d, d.V2, 1, i, j, k, v2);
    }
    if (i <= d.ext[2][0] && j <= d.ext[2][1] && k <= d.ext[2][2]) {
      T ts = tendency_w(d, i, j, k, c);
      T w2 = sc.stage > 1 ? d.Ws[c] * rdt * dt : (T)0;
      d.Ws[c] = ts;
      w2 = w2 + ts * bdt * dt;
      if (d.vz) w2 = w2 - coef * (pr_true(P, c + d.plane, m) - pr_true(P, c, m)) / (T)d.dzW[k + 2];
      else w2 = w2 + (-coef / (T)d.dz) * (pr_true(P, c + d.plane, m) - pr_true(P, c, m));
      w2 = w2 + ld(d.W, c);
      d.W2[c] = w2;
      push_vel(d, d.W2, 2, i, j, k, w2);
    }
  }
}

// ------------------------------------------------------------- Poisson
// FFT factorisations and plan of one domain, passed by value
struct PoisPlan {
  FFTFactors fx, fy;
};

constexpr int kRowsX = 8;  // real rows per block of the x transforms

// divergence RHS of PrePoisson (pressure.f90:688-717, Q = 0) fused with the
// forward real FFT along x of kRowsX rows (two real rows per complex FFT).
template <typename T>
__global__ void __launch_bounds__(128) k_fftx_fwd(const Dom<T> *__restrict__ doms, Launch L,
                                                  const PoisPlan *__restrict__ plans, double coef_alpha2,
                                                  int use_dt, const T *rhs_direct) {
  typedef typename Vec2<T>::type T2;
  extern __shared__ unsigned char smem_raw[];
  T2 *buf0 = reinterpret_cast<T2 *>(smem_raw);
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    const PoisPlan &pl = plans[di];
    const int N = d.nx;
    const int ntr = kRowsX / 2;
    T2 *buf1 = buf0 + ntr * N;
    const int lt = t - __ldg(L.starts + di);
    const int row0 = lt * kRowsX;
    const int nrows = d.ny * d.nz;
    const double coef = use_dt ? coef_alpha2 * d.dt : coef_alpha2;
    const T rdt2 = (T)(1.0 / coef);
    const T *U2 = d.U2, *V2 = d.V2, *W2 = d.W2;
    const T dx = (T)d.dx, dy = (T)d.dy, dz = (T)d.dz;
    for (int w = threadIdx.x; w < kRowsX * N; w += blockDim.x) {
      const int r = w / N, i = w - r * N + 1;
      const int row = row0 + r;
      T rhs = 0;
      if (row < nrows) {
        const int j = row % d.ny + 1, k = row / d.ny + 1;
        const long long c = bidx(d, i, j, k);
        if (rhs_direct) {  // PoisSolver interface: the RHS is given
          rhs = ld(rhs_direct, c);
        } else {
          const T dzk = d.vz ? (T)d.dzPr[k + 2] : dz;
          T div = (ld(U2, c) - ld(U2, c - 1)) / dx + (ld(V2, c) - ld(V2, c - d.pitch)) / dy +
                  (ld(W2, c) - ld(W2, c - d.plane)) / dzk - (T)0;
          rhs = div * rdt2;
        }
      }
      T2 *z = buf0 + (r >> 1) * N + (i - 1);
      if (r & 1) z->y = rhs; else z->x = rhs;
    }
    __syncthreads();
    T2 *res = fft_block<T, T2>(buf0, buf1, ntr, pl.fx, d.twx, false);
    // split Z = FFT(a + i b) into the half spectra of a and b
    const int nxh = d.nxh;
    for (int w = threadIdx.x; w < ntr * nxh; w += blockDim.x) {
      const int p = w / nxh, m = w - p * nxh;
      const T2 *Z = res + p * N;
      T2 zk = Z[m], zc = Z[m == 0 ? 0 : N - m];
      T2 A, B;
      A.x = (zk.x + zc.x) * (T)0.5;
      A.y = (zk.y - zc.y) * (T)0.5;
      B.x = (zk.y + zc.y) * (T)0.5;
      B.y = (zc.x - zk.x) * (T)0.5;
      const int ra = row0 + 2 * p, rb = ra + 1;
      if (ra < nrows) d.S[((long long)(ra / d.ny) * d.ny + ra % d.ny) * d.spitch + m] = A;
      if (rb < nrows) d.S[((long long)(rb / d.ny) * d.ny + rb % d.ny) * d.spitch + m] = B;
    }
    __syncthreads();
  }
}

// complex FFT along y of a tile of kTy columns (kx) of one k plane
template <typename T> struct TyOf;
template <> struct TyOf<double> { static constexpr int v = 8; };
template <> struct TyOf<float> { static constexpr int v = 16; };

template <typename T>
__global__ void __launch_bounds__(128) k_ffty(const Dom<T> *__restrict__ doms, Launch L,
                                              const PoisPlan *__restrict__ plans, int inverse) {
  typedef typename Vec2<T>::type T2;
  constexpr int C = TyOf<T>::v;
  extern __shared__ unsigned char smem_raw[];
  T2 *buf0 = reinterpret_cast<T2 *>(smem_raw);
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    const PoisPlan &pl = plans[di];
    const int N = d.ny;
    T2 *buf1 = buf0 + C * N;
    const int lt = t - __ldg(L.starts + di);
    const int ncx = (d.nxh + C - 1) / C;
    const int cx = lt % ncx, k = lt / ncx;
    const int kx0 = cx * C;
    T2 *S = d.S + (long long)k * d.ny * d.spitch;
    for (int w = threadIdx.x; w < C * N; w += blockDim.x) {
      const int j = w / C, c = w - j * C;
      T2 v;
      if (kx0 + c < d.nxh) v = S[(long long)j * d.spitch + kx0 + c];
      else { v.x = 0; v.y = 0; }
      buf0[c * N + j] = v;
    }
    __syncthreads();
    T2 *res = fft_block<T, T2>(buf0, buf1, C, pl.fy, d.twy, inverse != 0);
    for (int w = threadIdx.x; w < C * N; w += blockDim.x) {
      const int j = w / C, c = w - j * C;
      if (kx0 + c < d.nxh) S[(long long)j * d.spitch + kx0 + c] = res[c * N + j];
    }
    __syncthreads();
  }
}

// Tridiagonal solve in z for each (kx, ky): the Thomas algorithm in FP64 on
// the rows of Residue_variable_z (poisson.f90:23-60), Neumann rows at the
// ends or a cyclic system for periodic z; the (0,0) mode is singular and is
// solved by two prefix sums with its mean pinned to zero.
constexpr int kTriThreads = 64;

template <typename T>
__global__ void __launch_bounds__(kTriThreads) k_tri(const Dom<T> *__restrict__ doms, Launch L) {
  typedef typename Vec2<T>::type T2;
  extern __shared__ double cps[];  // [nz][kTriThreads]
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    const int lt = t - __ldg(L.starts + di);
    const int col = lt * kTriThreads + threadIdx.x;
    const int ky = col / d.spitch, kx = col - ky * d.spitch;
    if (ky >= d.ny || kx >= d.nxh) continue;
    const int nz = d.nz;
    const long long ps = (long long)d.ny * d.spitch;
    T2 *S = d.S + (long long)ky * d.spitch + kx;
    const double norm = 1.0 / ((double)d.nx * (double)d.ny);
    const double lam = d.lamx[kx] + d.lamy[ky];
    const double *Ab = d.Ab, *At = d.At;
    if (kx == 0 && ky == 0) {
      // singular mode: F(k) = F(k-1) + dzc(k) r(k) is the flux (x(k+1)-x(k))/dzf(k)
      double F0x = 0, F0y = 0;
      if (d.zper) {  // choose F(0) so that x is periodic: sum_k dzf(k) F(k) = 0
        double Fx = 0, Fy = 0, swx = 0, swy = 0, sd = 0;
        for (int k = 1; k <= nz; k++) {
          T2 r = S[(long long)(k - 1) * ps];
          Fx = Fx + ((double)r.x * norm) * d.dzc[k];
          Fy = Fy + ((double)r.y * norm) * d.dzc[k];
          swx += Fx * d.dzf[k]; swy += Fy * d.dzf[k]; sd += d.dzf[k];
        }
        F0x = -swx / sd; F0y = -swy / sd;
      }
      double Fx = 0, Fy = 0, xx = 0, xy = 0, sx = 0, sy = 0;
      for (int k = 1; k <= nz - 1; k++) {
        T2 r = S[(long long)(k - 1) * ps];
        Fx = Fx + ((double)r.x * norm) * d.dzc[k];
        Fy = Fy + ((double)r.y * norm) * d.dzc[k];
        T2 o; o.x = (T)xx; o.y = (T)xy;
        S[(long long)(k - 1) * ps] = o;  // x(k)
        sx += xx; sy += xy;
        xx = xx + (Fx + F0x) * d.dzf[k];
        xy = xy + (Fy + F0y) * d.dzf[k];
      }
      sx += xx; sy += xy;
      sx = sx / nz; sy = sy / nz;
      T2 last; last.x = (T)(xx - sx); last.y = (T)(xy - sy);
      for (int k = 0; k < nz - 1; k++) {
        T2 v = S[(long long)k * ps];
        v.x = (T)((double)v.x - sx);
        v.y = (T)((double)v.y - sy);
        S[(long long)k * ps] = v;
      }
      S[(long long)(nz - 1) * ps] = last;
      continue;
    }
    double *cp = cps + threadIdx.x;
    if (!d.zper) {
      double b = -(Ab[1] + At[1]) + lam;
      double inv = 1.0 / b;
      cp[0] = At[1] * inv;
      T2 r = S[0];
      double dx_ = (double)r.x * norm * inv, dy_ = (double)r.y * norm * inv;
      T2 o; o.x = (T)dx_; o.y = (T)dy_;
      double px = dx_, py = dy_;
      S[0] = o;
      for (int k = 2; k <= nz; k++) {
        double den = (-(Ab[k] + At[k]) + lam) - Ab[k] * cp[(k - 2) * kTriThreads];
        double iv = 1.0 / den;
        cp[(k - 1) * kTriThreads] = At[k] * iv;
        T2 rk = S[(long long)(k - 1) * ps];
        px = ((double)rk.x * norm - Ab[k] * px) * iv;
        py = ((double)rk.y * norm - Ab[k] * py) * iv;
        T2 ok; ok.x = (T)px; ok.y = (T)py;
        S[(long long)(k - 1) * ps] = ok;
      }
      // back substitution (px, py hold x(nz))
      for (int k = nz - 1; k >= 1; k--) {
        T2 dk = S[(long long)(k - 1) * ps];
        px = (double)dk.x - cp[(k - 1) * kTriThreads] * px;
        py = (double)dk.y - cp[(k - 1) * kTriThreads] * py;
        T2 ok; ok.x = (T)px; ok.y = (T)py;
        S[(long long)(k - 1) * ps] = ok;
      }
    } else {
      // cyclic system (periodic z) by Sherman-Morrison; c2 and z in shared memory
      double *zz = cps + (long long)nz * kTriThreads + threadIdx.x;
      const double alpha = At[nz], beta = Ab[1];
      const double b0 = -(Ab[1] + At[1]) + lam;
      const double gamma = -b0;
      double bb = b0 - gamma;
      double inv = 1.0 / bb;
      cp[0] = At[1] * inv;
      T2 r = S[0];
      double yx = (double)r.x * norm * inv, yy = (double)r.y * norm * inv;
      double z_ = gamma * inv;
      zz[0] = z_;
      T2 o; o.x = (T)yx; o.y = (T)yy;
      S[0] = o;
      for (int k = 2; k <= nz; k++) {
        double bk = -(Ab[k] + At[k]) + lam;
        if (k == nz) bk = bk - alpha * beta / gamma;
        double den = bk - Ab[k] * cp[(k - 2) * kTriThreads];
        double iv = 1.0 / den;
        cp[(k - 1) * kTriThreads] = At[k] * iv;
        T2 rk = S[(long long)(k - 1) * ps];
        yx = ((double)rk.x * norm - Ab[k] * yx) * iv;
        yy = ((double)rk.y * norm - Ab[k] * yy) * iv;
        double uk = (k == nz) ? alpha : 0.0;
        z_ = (uk - Ab[k] * z_) * iv;
        zz[(k - 1) * kTriThreads] = z_;
        T2 ok; ok.x = (T)yx; ok.y = (T)yy;
        S[(long long)(k - 1) * ps] = ok;
      }
      for (int k = nz - 1; k >= 1; k--) {
        T2 dk = S[(long long)(k - 1) * ps];
        yx = (double)dk.x - cp[(k - 1) * kTriThreads] * yx;
        yy = (double)dk.y - cp[(k - 1) * kTriThreads] * yy;
        z_ = zz[(k - 1) * kTriThreads] - cp[(k - 1) * kTriThreads] * z_;
        zz[(k - 1) * kTriThreads] = z_;
        T2 ok; ok.x = (T)yx; ok.y = (T)yy;
        S[(long long)(k - 1) * ps] = ok;
      }
      // now S holds y, zz holds z; x = y - fac z
      T2 y0 = S[0], yn = S[(long long)(nz - 1) * ps];
      double z0 = zz[0], zn = zz[(nz - 1) * kTriThreads];
      double den = 1.0 + z0 + beta * zn / gamma;
      double fx = ((double)y0.x + beta * (double)yn.x / gamma) / den;
      double fy = ((double)y0.y + beta * (double)yn.y / gamma) / den;
      for (int k = 0; k < nz; k++) {
        T2 v = S[(long long)k * ps];
        double zk = zz[k * kTriThreads];
        v.x = (T)((double)v.x - fx * zk);
        v.y = (T)((double)v.y - fy * zk);
        S[(long long)k * ps] = v;
      }
    }
  }
}

}  // namespace elmm
