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

// the u* of a wall point: WMRoughStress with a roughness length, else
// WMFlatStress (src/wallmodels.f90:2262-2275, 1243-1265); ustar is the
// point's value from the stage before (the start of the flat iteration)
__device__ inline double wm_ustar(double ustar, double vel, double dist, double z0, double nu) {
  return z0 > 0 ? wm_rough_ustar(ustar, vel, dist, z0, nu) : wm_flat_ustar(ustar, vel, dist, nu);
}

// PsiM_MO, the Businger-Dyer stability function of momentum
// (src/wallmodels.f90:1546-1556)
__device__ inline double psim_mo(double zeta) {
  if (zeta < 0) {
    const double x = pow(1 - 15.0 * zeta, 0.25), h = (1 + x) / 2.0;
    return log(((1 + x * x) / 2.0) * (h * h)) - 2.0 * atan(x) + 3.141592653589793 / 2;
  }
  return -4.8 * zeta;
}

// WM_MO_Flux_ustar (src/wallmodels.f90:1606-1660): u* of a rough wall under
// a prescribed surface temperature flux, the log law corrected by PsiM_MO at
// the Obukhov stability z/L, both relaxed by halves from the point's u* of
// the stage before.  The tolerances 1e-3, 1e-4 and 1e-5 are default-real
// literals in the reference (their float values widened).
__device__ inline double wm_mo_flux_ustar(double ustar, double vel, double dist, double z0, double tflux,
                                          double tref, double g, double nu) {
  if (dist <= z0) {
    if (nu <= 0) return 0;
    if ((dist * ustar / nu) < 11.225) return sqrt(nu * vel / dist);
    return vel / (log(fabs(ustar * dist / nu)) / 0.4 + 5.2);
  }
  double zL = 0, Psi = 0;
  for (int i = 1;; i++) {  // at most 50 iterations
    const double ustar2 = ustar;
    ustar = ustar + (fmax(vel * 0.4 / log(fmax((dist / z0) - Psi, (double)1e-5f)), 0.0) - ustar) / 2;
    if (ustar < (double)1e-4f) {
      zL = -10000;
    } else {  // Obukhov_zL (src/wallmodels.f90:1598-1602)
      const double zL2 = dist * (0.4 * (g / tref) * tflux) / (-(ustar * ustar * ustar));
      zL = zL + (zL2 - zL) / 2;
    }
    Psi = psim_mo(zL);
    if (fabs(ustar - ustar2) / fmax(fabs(ustar), 1e-3) < (double)1e-3f) return ustar;
    if (i >= 50) return 0;
  }
}

// PsiM_MO_mod / PsiH_MO_mod, the stability functions of Zilitinkevich and
// Esau (2006) with L defined with the von Karman constant k_U
// (src/wallmodels.f90:1572-1595)
__device__ inline double psim_mo_mod(double zeta, double kU) {
  if (zeta < 0) {
    const double x = pow(1 - 6.0 * zeta * kU, 0.25), h = (1 + x) / 2.0;
    return log(((1 + x * x) / 2.0) * (h * h)) - 2.0 * atan(x) + 3.141592653589793 / 2;
  }
  return -(3 * pow(zeta * kU, 5.0 / 6.0));
}
__device__ inline double psih_mo_mod(double zeta, double kU) {
  if (zeta < 0) {
    const double x = pow(1 - 6.0 * zeta * kU, 0.25);
    return 2.0 * log((1 + x * x) / 2.0);
  }
  return -(2.5 * pow(zeta * kU, 4.0 / 5.0));
}

// WM_MO_Dirichlet_ustar_tfl (src/wallmodels.f90:1664-1716): u* and the
// surface temperature flux of a rough wall with a prescribed surface
// temperature, tempdif = theta(point) - theta(surface).  tflux comes in as
// the point's flux of the stage before (the start of the stability
// iteration, relaxed until z/L changes by less than 1e-3); its 1.1 is a
// default-real literal in the reference.
template <typename T>
__device__ inline void wm_mo_dirichlet(const Dom<T> &d, double &ustar, double &tflux, double dist, double z0,
                                       double vel, double tempdif) {
  const double kU = 0.4, kT = 0.47, nu = d.nu_mol;
  ustar = wm_rough_ustar(ustar, vel, dist, z0, nu);
  double dist_plus = 1.7976931348623157e308;  // huge()
  if (nu > 0) dist_plus = dist * sqrt(nu * vel / dist) / nu;
  if (dist <= z0 || dist_plus < (double)1.1f * 11.225) {
    tflux = -d.kappa_mol * tempdif / dist;
    return;
  }
  double zL = 0, zL0 = -10000.0;
  int i = 0;
  for (;;) {
    i++;
    zL = -dist * d.grav * tflux / (kU * d.tref * (ustar * ustar * ustar));
    const double pm = psim_mo_mod(zL, kU), ph = psih_mo_mod(zL, kU);
    ustar = vel * kU / (log(dist / z0) - pm);
    tflux = -tempdif * ustar * kT / (log(dist / z0) - ph);  // z0H = z0
    if (i > 1 && fabs(zL - zL0) / fmax(fabs(zL), 1e-4) < 1e-3) break;
    if (i >= 50 || zL > 10000) break;
    zL0 = zL;
  }
  if (i >= 50 || zL > 10000) {
    ustar = sqrt(nu * vel / dist);
    tflux = -d.kappa_mol * tempdif / dist;
  }
}

// ComputeViscsWM for the Pr point next to side f (bottom or top) at cell
// (i, j, k) with a prescribed surface temperature (WM_MO_Dirichlet,
// src/wallmodels.f90:1858-1884, 2080-2111): the point's u* and surface
// temperature flux from the cell-centred velocity and theta at the start of
// the stage (Tm); the viscosity it forms is overwritten by SubgridModel in
// the reference and is not kept.
template <typename T>
__device__ void wm_pr_dirichlet(const Dom<T> &d, int f, int i, int j, int k, const T *Tm) {
  if (!(d.z0[f] > 0)) return;  // smooth wall: the flat branch leaves u* and the flux of a Pr point alone
  const long long c = bidx(d, i, j, k);
  double ou = 0, ov = 0;
  if constexpr (sizeof(T) == 4) { ou = (double)vel_off(d, 0, k); ov = (double)vel_off(d, 1, k); }
  const double uv[3] = {(((double)ld(d.U, c) + ou) + ((double)ld(d.U, c - 1) + ou)) / 2.0,
                        (((double)ld(d.V, c) + ov) + ((double)ld(d.V, c - d.pitch) + ov)) / 2.0,
                        ((double)ld(d.W, c) + (double)ld(d.W, c - d.plane)) / 2.0};
  const double distz = f == SIDE_BO ? d.zW[0 + 2] - d.zPr[1 + 2] : d.zW[d.ext[2][2] + 1 + 2] - d.zPr[d.nz + 2];
  const double dv[3] = {0.0, 0.0, distz};
  const double dist = sqrt((dv[0] * dv[0] + dv[1] * dv[1]) + dv[2] * dv[2]);
  const double dot = (uv[0] * dv[0] + uv[1] * dv[1]) + uv[2] * dv[2];
  double vect[3];
#pragma unroll
  for (int m = 0; m < 3; m++) vect[m] = uv[m] - dot * dv[m] / (dist * dist);
  const double vel = sqrt((vect[0] * vect[0] + vect[1] * vect[1]) + vect[2] * vect[2]);
  const double tdif = ((double)ld(Tm, c) + d.toff) - d.tsurf[f];
  const int h = f == SIDE_BO ? 0 : 1;
  const long long q = (long long)(i - 1) + (long long)d.nx * (j - 1);
  double ustar = d.wm_pr_us[h][q], tfl = d.wm_pr_tf[h][q];
  wm_mo_dirichlet(d, ustar, tfl, dist, d.z0[f], vel, tdif);
  if (ustar < 0) ustar = 0;
  d.wm_pr_us[h][q] = ustar;
  d.wm_pr_tf[h][q] = tfl;
}

// ComputeUVWFluxesWM / fluxes for the point of component comp on side f at
// cell (i,j,k) (src/wallmodels.f90:2159-2338); the wall-point distance is
// the one of GetOutsideBoundariesWM_UVW (src/wallmodels.f90:690-909).
template <typename T>
__device__ void wm_point(const Dom<T> &d, int comp, int f, int i, int j, int k, long long pidx, const T *Tm) {
  const T *U = d.U, *V = d.V, *W = d.W;
  const long long c = bidx(d, i, j, k), sx = 1, sy = d.pitch, sz = d.plane;
  // full velocities: stored values plus the per-level offsets of U and V of
  // the mixed path (the FP64 path reads the stored values alone), in FP64
  const double ou0 = (double)vel_off(d, 0, k), ov0 = (double)vel_off(d, 1, k);
  auto lu = [&](long long o, double off) {
    if constexpr (sizeof(T) == 4) return (double)ld(U, c + o) + off;
    else return (double)ld(U, c + o);
  };
  auto lv = [&](long long o, double off) {
    if constexpr (sizeof(T) == 4) return (double)ld(V, c + o) + off;
    else return (double)ld(V, c + o);
  };
  double vel[3];
  if (comp == 0) {
    vel[0] = lu(0, ou0);
    vel[1] = (lv(sx, ov0) + lv(0, ov0) + lv(sx - sy, ov0) + lv(-sy, ov0)) / 4.0;
    vel[2] = ((double)ld(W, c + sx) + (double)ld(W, c) + (double)ld(W, c + sx - sz) + (double)ld(W, c - sz)) / 4.0;
  } else if (comp == 1) {
    vel[0] = (lu(sy, ou0) + lu(0, ou0) + lu(-sx + sy, ou0) + lu(-sx, ou0)) / 4.0;
    vel[1] = lv(0, ov0);
    vel[2] = ((double)ld(W, c + sy) + (double)ld(W, c) + (double)ld(W, c + sy - sz) + (double)ld(W, c - sz)) / 4.0;
  } else {
    const double ou1 = (double)vel_off(d, 0, k + 1), ov1 = (double)vel_off(d, 1, k + 1);
    vel[0] = (lu(sz, ou1) + lu(0, ou0) + lu(-sx + sz, ou1) + lu(-sx, ou0)) / 4.0;
    vel[1] = (lv(sz, ov1) + lv(0, ov0) + lv(-sy + sz, ov1) + lv(-sy, ov0)) / 4.0;
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
  if (d.z0[f] > 0 && d.tdir[f]) {  // WM_MO_DirichletStress (src/wallmodels.f90:1922-1938, 2228-2253)
    const double vel2 = sqrt((t[0] * t[0] + t[1] * t[1]) + t[2] * t[2]);  // sqrt(sum(tan_vect**2))
    // local_value of theta at the point (src/wallmodels.f90:2340-2353), x and y periodic
    const int i2 = comp == 0 ? (i + 1 > d.nx ? 1 : i + 1) : i, j2 = comp == 1 ? (j + 1 > d.ny ? 1 : j + 1) : j;
    const double temp = (((double)ld(Tm, bidx(d, i2, j2, comp == 2 ? k + 1 : k)) + d.toff) +
                         ((double)ld(Tm, bidx(d, i, j, k)) + d.toff)) / 2;
    double tfl = d.wm_tfl[face][pidx];
    wm_mo_dirichlet(d, ustar, tfl, dd, d.z0[f], vel2, temp - d.tsurf[f]);
    d.wm_tfl[face][pidx] = tfl;
  } else if (d.z0[f] > 0 && d.tflux[f] > 0)  // WM_MO_FluxStress (src/wallmodels.f90:1836-1854, 2255-2259)
    ustar = tv != 0 ? wm_mo_flux_ustar(ustar, tv, dd, d.z0[f], d.tflux[f], d.tref, d.grav, d.nu_mol) : 0.0;
  else if (tv != 0)
    ustar = wm_ustar(ustar, tv, dd, d.z0[f], d.nu_mol);
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

// SubgridStresses' wall model (src/dynamics.f90:879-888): ComputeViscsWM
// for the Pr points with a prescribed surface temperature, and
// ComputeUVWFluxesWM for every velocity point on a wall-model face, from the
// state at the start of the stage (tb: its temperature buffer).  One thread
// a point; a domain's points in the order: the Pr points of the bottom and
// top (i + nx j), then per component and side its face plane in index
// order (x sides: j + ny k, y sides: i + nx k, z sides: i + nx j).  The
// parts touch disjoint state.  Launched after k_sgs (whose viscosity they do
// not read) and, with the initial fields, at the end of the initial
// projection.
constexpr int kWmThreads = 128;
template <typename T>
__host__ __device__ inline void wm_face_plane(const Dom<T> &d, int comp, int f, int &n0, int &n1) {
  const int *e = d.ext[comp];
  const int axis = f >> 1;
  n0 = axis == 0 ? e[1] : e[0];
  n1 = axis == 2 ? e[1] : e[2];
}
template <typename T>
__host__ __device__ inline long long wm_points_of(const Dom<T> &d) {
  long long n = 0;
  for (int f = SIDE_BO; f <= SIDE_TO; f++)
    if (d.tdir[f]) n += (long long)d.nx * d.ny;
  for (int comp = 0; comp < 3; comp++)
    for (int f = 0; f < 6; f++)
      if (d.wall[f]) {
        int n0, n1;
        wm_face_plane(d, comp, f, n0, n1);
        n += (long long)n0 * n1;
      }
  return n;
}
template <typename T>
__global__ void __launch_bounds__(kWmThreads) k_wm_points(const Dom<T> *__restrict__ doms, Launch L, int tb) {
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    long long p = (long long)(t - __ldg(L.starts + di)) * kWmThreads + threadIdx.x;
    const T *Tm = d.buoy ? d.slot[0].buf[tb] : nullptr;
    bool done = false;
#pragma unroll 1
    for (int f = SIDE_BO; f <= SIDE_TO && !done; f++) {
      if (!d.tdir[f]) continue;
      const long long np = (long long)d.nx * d.ny;
      if (p < np) {
        wm_pr_dirichlet(d, f, (int)(p % d.nx) + 1, (int)(p / d.nx) + 1, f == SIDE_BO ? 1 : d.nz, Tm);
        done = true;
      } else {
        p -= np;
      }
    }
#pragma unroll 1
    for (int comp = 0; comp < 3 && !done; comp++)
#pragma unroll 1
      for (int f = 0; f < 6 && !done; f++) {
        if (!d.wall[f]) continue;
        int n0, n1;
        wm_face_plane(d, comp, f, n0, n1);
        const long long np = (long long)n0 * n1;
        if (p >= np) {
          p -= np;
          continue;
        }
        const int *e = d.ext[comp];
        const int axis = f >> 1, hi = f & 1;
        const int a = (int)(p % n0) + 1, b = (int)(p / n0) + 1;
        const int i = axis == 0 ? (hi ? e[0] : 1) : a;
        const int j = axis == 0 ? a : axis == 1 ? (hi ? e[1] : 1) : b;
        const int k = axis == 2 ? (hi ? e[2] : 1) : b;
        wm_point(d, comp, f, i, j, k, p, Tm);
        done = true;
      }
  }
}

}  // namespace elmm

#include "elmm_momentum.cuh"

namespace elmm {

// ------------------------------------------------------------- Poisson
// FFT factorisations and plan of one domain, passed by value
struct PoisPlan {
  FFTFactors fx, fy;
};

constexpr int kRowsX = 8;  // real rows per block of the x transforms
constexpr int kFFTThreads = 256;

// divergence RHS of PrePoisson (pressure.f90:688-717, Q = 0) fused with the
// forward real FFT along x of kRowsX rows (two real rows per complex FFT).
template <typename T>
__global__ void __launch_bounds__(kFFTThreads) k_fftx_fwd(const Dom<T> *__restrict__ doms, Launch L,
                                                  const PoisPlan *__restrict__ plans, double coef_alpha2,
                                                  int use_dt, int rhs_from_phi, int gate) {
  typedef typename Vec2<T>::type T2;
  extern __shared__ unsigned char smem_raw[];
  T2 *buf0 = reinterpret_cast<T2 *>(smem_raw);
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    if (gate && !*d.refine_flag) continue;  // defect-correction sweep not needed
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
    const T rdx = (T)(1.0 / d.dx), rdy = (T)(1.0 / d.dy), rdz = (T)(1.0 / d.dz);
#pragma unroll 4
    for (int w = threadIdx.x; w < kRowsX * N; w += blockDim.x) {
      const int r = w / N, i = w - r * N + 1;
      const int row = row0 + r;
      T rhs = 0;
      if (row < nrows) {
        const int j = row % d.ny + 1, k = row / d.ny + 1;
        const long long c = bidx(d, i, j, k);
        if (rhs_from_phi) {  // the RHS was put in Phi (PoisSolver interface, defect correction)
          rhs = ld((const T *)d.Phi, c) * rdt2;
        } else {
          const T rdzk = d.vz ? (T)d.sgs_rdz[k] : rdz;
          // on a box face the neighbours fold onto the interior (BoundUVW)
          const bool face = i == 1 || i > d.ext[0][0] || j == 1 || j > d.ext[1][1] || k == 1 || k > d.ext[2][2] ||
                            j > d.ext[0][1] || j > d.ext[2][1] || k > d.ext[0][2] || k > d.ext[1][2];
          T uc, uw, vc, vs, wc, wb;
          if (!face) {
            uc = ld(U2, c); uw = ld(U2, c - 1);
            vc = ld(V2, c); vs = ld(V2, c - d.pitch);
            wc = ld(W2, c); wb = ld(W2, c - d.plane);
          } else {
            uc = vel_folded(d, U2, 0, i, j, k); uw = vel_folded(d, U2, 0, i - 1, j, k);
            vc = vel_folded(d, V2, 1, i, j, k); vs = vel_folded(d, V2, 1, i, j - 1, k);
            wc = vel_folded(d, W2, 2, i, j, k); wb = vel_folded(d, W2, 2, i, j, k - 1);
          }
          T div = (uc - uw) * rdx + (vc - vs) * rdy + (wc - wb) * rdzk;
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
#pragma unroll 4
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
__global__ void __launch_bounds__(kFFTThreads) k_ffty(const Dom<T> *__restrict__ doms, Launch L,
                                              const PoisPlan *__restrict__ plans, int inverse, int gate) {
  typedef typename Vec2<T>::type T2;
  constexpr int C = TyOf<T>::v;
  extern __shared__ unsigned char smem_raw[];
  T2 *buf0 = reinterpret_cast<T2 *>(smem_raw);
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    if (gate && !*d.refine_flag) continue;  // defect-correction sweep not needed
    const PoisPlan &pl = plans[di];
    const int N = d.ny;
    T2 *buf1 = buf0 + C * N;
    const int lt = t - __ldg(L.starts + di);
    const int ncx = (d.nxh + C - 1) / C;
    const int cx = lt % ncx, k = lt / ncx;
    const int kx0 = cx * C;
    T2 *S = d.S + (long long)k * d.ny * d.spitch;
#pragma unroll 4
    for (int w = threadIdx.x; w < C * N; w += blockDim.x) {
      const int j = w / C, c = w - j * C;
      T2 v;
      if (kx0 + c < d.nxh) v = S[(long long)j * d.spitch + kx0 + c];
      else { v.x = 0; v.y = 0; }
      buf0[c * N + j] = v;
    }
    __syncthreads();
    T2 *res = fft_block<T, T2>(buf0, buf1, C, pl.fy, d.twy, inverse != 0);
#pragma unroll 4
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
__global__ void __launch_bounds__(kTriThreads) k_tri(const Dom<T> *__restrict__ doms, Launch L, int gate) {
  typedef typename Vec2<T>::type T2;
  extern __shared__ double cps[];  // [nz][kTriThreads]
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    if (gate && !*d.refine_flag) continue;  // defect-correction sweep not needed
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
      // Thomas algorithm; rows are fetched kPre at a time so that the loads of
      // a batch are in flight together (the recurrence only needs the values)
      constexpr int kPre = 8;
      double px = 0, py = 0, cprev = 0;
      for (int kb = 1; kb <= nz; kb += kPre) {
        T2 rr[kPre];
#pragma unroll
        for (int q = 0; q < kPre; q++)
          if (kb + q <= nz) rr[q] = S[(long long)(kb + q - 1) * ps];
#pragma unroll
        for (int q = 0; q < kPre; q++) {
          const int k = kb + q;
          if (k > nz) break;
          double den = (-(Ab[k] + At[k]) + lam) - (k > 1 ? Ab[k] * cprev : 0.0);
          double iv = 1.0 / den;
          cprev = At[k] * iv;
          cp[(k - 1) * kTriThreads] = cprev;
          if (k == 1) {
            px = (double)rr[q].x * norm * iv;
            py = (double)rr[q].y * norm * iv;
          } else {
            px = ((double)rr[q].x * norm - Ab[k] * px) * iv;
            py = ((double)rr[q].y * norm - Ab[k] * py) * iv;
          }
          T2 ok; ok.x = (T)px; ok.y = (T)py;
          S[(long long)(k - 1) * ps] = ok;
        }
      }
      // back substitution (px, py hold x(nz))
      for (int kt = nz - 1; kt >= 1; kt -= kPre) {
        T2 rr[kPre];
#pragma unroll
        for (int q = 0; q < kPre; q++)
          if (kt - q >= 1) rr[q] = S[(long long)(kt - q - 1) * ps];
#pragma unroll
        for (int q = 0; q < kPre; q++) {
          const int k = kt - q;
          if (k < 1) break;
          const double c = cp[(k - 1) * kTriThreads];
          px = (double)rr[q].x - c * px;
          py = (double)rr[q].y - c * py;
          T2 ok; ok.x = (T)px; ok.y = (T)py;
          S[(long long)(k - 1) * ps] = ok;
        }
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
