// elmm_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker; never the product).
//
// A CPU, FP64 restatement of the ELMM per-timestep flow solve, written from the
// reference Fortran so that the CUDA library can be checked against it, and
// timed as the CPU baseline.  Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py load it.
//
// Parity status: the reference (Fortran 2008 + an un-vendored PoisFFT module)
// cannot be compiled in this environment, so this restatement is not pinned
// to outputs of the reference itself ("parity unpinned" w.r.t. reference
// binaries).  It is pinned to known answers derived from the mathematics:
// the analytic Taylor-Green decay, the discrete divergence after a projection,
// the residual of the Poisson operator of src/poisson.f90:23-60, and a dense
// scipy solve of the same operator (tests/test_oracle_*.py).
//
// Every routine cites the reference lines it follows.  Arrays keep the
// reference's Fortran layout and lower bounds (x fastest):
//   U,V,W(-2:n+3)^3, Pr,Viscosity,Phi(-1:n+2)^3, RHS(0:n+1)^3.
// Loops keep the reference's order of floating-point operations so that the
// CUDA kernels, which follow the same formulas, agree to rounding.
//
// Supported subset (the hot path of the configurations in scope):
//   BCs NOSLIP / FREESLIP / PERIODIC / NEUMANN on any side; uniform grid or
//   stretched z (GRID_VARIABLE_Z); CDS2 skew-symmetric advection; Smagorinsky;
//   explicit 2nd-order diffusion with the rough-wall log-law wall model at
//   no-slip sides; incremental projection with FFT(x,y) + tridiagonal(z)
//   Poisson solve; PRESSURE_REFERENCE_BOUNDARY at To; RK3.

#include <algorithm>
#include <array>
#include <limits>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/elmm_gpu.h"

namespace orc {

typedef std::complex<double> cd;

// ---------------------------------------------------------------- arrays
struct A1 {
  int lo = 0;
  std::vector<double> v;
  void init(int l, int h) { lo = l; v.assign((size_t)(h - l + 1), 0.0); }
  double &operator()(int i) { return v[(size_t)(i - lo)]; }
  double operator()(int i) const { return v[(size_t)(i - lo)]; }
};

struct A3 {
  int l0 = 0, l1 = 0, l2 = 0, n0 = 0, n1 = 0, n2 = 0;
  std::vector<double> v;
  void init(int a0, int b0, int a1, int b1, int a2, int b2) {
    l0 = a0; l1 = a1; l2 = a2;
    n0 = b0 - a0 + 1; n1 = b1 - a1 + 1; n2 = b2 - a2 + 1;
    v.assign((size_t)n0 * n1 * n2, 0.0);
  }
  double &operator()(int i, int j, int k) {
    return v[(size_t)(i - l0) + (size_t)n0 * ((size_t)(j - l1) + (size_t)n1 * (size_t)(k - l2))];
  }
  double operator()(int i, int j, int k) const {
    return v[(size_t)(i - l0) + (size_t)n0 * ((size_t)(j - l1) + (size_t)n1 * (size_t)(k - l2))];
  }
  void fill(double x) { std::fill(v.begin(), v.end(), x); }
};

// Side indices as src/parameters.f90:193 (We=1 .. To=6).
enum { We = 1, Ea = 2, So = 3, No = 4, Bo = 5, To = 6 };
enum { BC_NOSLIP = 1, BC_FREESLIP = 2, BC_PERIODIC = 3, BC_NEUMANN = 5 };
// Directions of src/wallmodels.f90:151.
enum { MINUSX = 1, PLUSX = 2, MINUSY = 3, PLUSY = 4, MINUSZ = 5, PLUSZ = 6 };

// RK3 coefficients, src/parameters.f90:317-320.
static const double RK_alpha[3] = {4.0 / 15.0, 1.0 / 15.0, 1.0 / 6.0};
static const double RK_beta[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
static const double RK_rho[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};

// WMPointUVW, src/wallmodels.f90:68-98 (fields used on the hot path).
struct WMPointUVW {
  double fluxp = 0, fluxm = 0;
  int xi = 0, yj = 0, zk = 0;
  double distx = 0, disty = 0, distz = 0;
  double z0 = 0;
  double ustar = 1;
  double wallu = 0, wallv = 0, wallw = 0;
  double temperature_flux = 0;
  double temperature = 0;
  bool prescribed_temperature = false;
};

// The WMPoint of a Pr cell next to a wall in z (src/wallmodels.f90:20-64,
// 570-685), kept for the sides with a prescribed surface temperature: the
// state of WM_MO_Dirichlet and the flux TemperatureExtra adds.
struct WMPointPr {
  int xi = 0, yj = 0, zk = 0;
  double distz = 0, z0 = 0;
  double ustar = 1, temperature_flux = 0, temperature = 0;
};

// ------------------------------------------------------------------- FFT
// Mixed-radix decimation-in-time DFT, X[m] = sum_j x[j] exp(-2 pi i j m / n).
struct FFTPlan {
  int n = 0;
  std::vector<int> fac;
  std::vector<cd> w;  // w[m] = exp(-2 pi i m / n)
  bool init(int n_) {
    n = n_;
    fac.clear();
    int r = n;
    for (int p : {4, 2, 3, 5}) {
      while (r % p == 0) { fac.push_back(p); r /= p; }
    }
    if (r != 1) return false;
    w.resize(n);
    for (int m = 0; m < n; m++) {
      double a = -2.0 * M_PI * (double)m / (double)n;
      w[m] = cd(std::cos(a), std::sin(a));
    }
    return true;
  }
  void rec(const cd *x, int xs, cd *y, int len, int fi, int wstep) const {
    if (len == 1) { y[0] = x[0]; return; }
    int p = fac[fi], m = len / p;
    for (int r = 0; r < p; r++) rec(x + (size_t)r * xs, xs * p, y + (size_t)r * m, m, fi + 1, wstep * p);
    cd t[5];
    for (int k = 0; k < m; k++) {
      for (int r = 0; r < p; r++) t[r] = y[r * m + k] * w[((size_t)r * k * wstep) % n];
      for (int q = 0; q < p; q++) {
        cd s = 0;
        for (int r = 0; r < p; r++) s += t[r] * w[((size_t)r * q * m * wstep) % n];
        y[k + q * m] = s;
      }
    }
  }
  // forward DFT of x into y (distinct buffers)
  void forward(const cd *x, cd *y) const { rec(x, 1, y, n, 0, 1); }
  // unnormalised inverse, X -> sum_m X[m] exp(+2 pi i j m / n)
  void inverse(const cd *x, cd *y, std::vector<cd> &tmp) const {
    tmp.resize(n);
    for (int i = 0; i < n; i++) tmp[i] = std::conj(x[i]);
    rec(tmp.data(), 1, y, n, 0, 1);
    for (int i = 0; i < n; i++) y[i] = std::conj(y[i]);
  }
};

// -------------------------------------------------------------- domain
struct Domain {
  int Prnx, Prny, Prnz, Unx, Uny, Unz, Vnx, Vny, Vnz, Wnx, Wny, Wnz;
  int Btype[7], PrBtype[7];
  int gridtype;  // 0 uniform, 1 variable z
  double dxmin, dymin, dzmin;
  A1 xU, yV, zW, xPr, dxPr, yPr, dyPr, zPr, dzPr, dxU, dyV, dzW;
  double molecular_viscosity, C_Smagorinsky, filter_ratio;
  int sgstype, wallmodeltype;
  double z0s[7];
  int en_prgx, en_prgy;
  double prgx, prgy;
  double dt, time;
  int enable_CFL_check;
  double CFL;
  // variable time steps (t_s%variable_time_steps, CFL, dt_max, end_time)
  int variable_time_steps;
  double CFL_target, dt_max, end_time, dt0;
  A3 U, V, W, U2, V2, W2, Ustar, Vstar, Wstar, Pr, Viscosity, Phi, RHS;
  std::vector<WMPointUVW> wm[7][4];  // [direction][component]
  // Poisson
  FFTPlan px, py;
  int nxh;
  std::vector<double> lamx, lamy, Ab, At, dzc, dzf;  // tridiagonal data
  int zper;
  double max_div;
  // potential temperature (ScalarRK3, scalars.f90:88-381)
  int enable_buoyancy;
  int TempBtype[7];
  double sideTemp[7];
  double temperature_ref, grav_acc, molecular_diffusivity;
  // temperature_flux of the wall-model points of the bottom and top walls and
  // their ComputeAreaFactor (wallmodels.f90:173-203, 590-596, 650-656)
  double wm_tflux[7] = {0, 0, 0, 0, 0, 0, 0};
  double area_factor_z = 0;
  // Pr wall-model points of the bottom and top with a prescribed surface
  // temperature (TempBtype BC_DIRICHLET at a wall-model wall)
  std::vector<WMPointPr> wmpr[7];
  // solid bodies with passive scalars: Prtype > 0 as 1 (periodic images in
  // the x and y ghosts) and the Pr wall-model points of the scalars
  bool scal_solids = false;
  A3 Prsolid;
  // temperature_flux x area_factor of the heated Pr wall-model points at
  // solid faces (0 elsewhere)
  A3 HeatQ;
  // the wall points the deduplication keeps beside the bodies (1)
  A3 WallPt;
  std::vector<std::array<int, 3>> wmprs;
  A3 T, Tadv, T2, TDiff;
  // passive scalars (ScalarRK3's loop over num_of_scalars, scalars.f90:217-223)
  int num_scalars;
  int ScalBtype[7];
  double sideScal[7];
  A3 S[ELMM_MAX_SCALARS], Sadv[ELMM_MAX_SCALARS], S2[ELMM_MAX_SCALARS];
  // ScalFlVolumes from the point sources (pointsources.f90:24-39), in the
  // order they were added: scalar, cell, flux / volumePr
  struct FlVolume { int sc, i, j, k; double flux; };
  std::vector<FlVolume> flvolumes;
  // time-averaged slices of Scalar_avg (outputs.f90:1043-1045)
  int avg_k, avg_j;
  double avg_w;
  std::vector<double> acc_xy[ELMM_MAX_SCALARS], acc_xz[ELMM_MAX_SCALARS];
  // immersed solids: UIBPoints.. (index = component), ScalFlIBPoints, Unull..
  // (src/immersedboundary.f90:519-580, src/tsteps.f90:360-567)
  bool solids = false;
  std::vector<elmm_ib_point> ibp[4], scalfl;
  std::vector<std::array<int, 3>> nullp[4];
  A3 Q;        // IBMassSources, Q(0:Prnx+1,0:Prny+1,0:Prnz+1)
  // PuffSources (src/puffs.f90:15-23) and their ScalarFlVolumes
  struct Puff {
    double start_time, end_time, period, duration;
    bool clear;
    double last_start;
    bool restart;
    double dt_fraction;
  };
  std::vector<Puff> puffs;
  struct PuffVol { int puff, sc, i, j, k; double flux; };
  std::vector<PuffVol> puffvols;
  int called = 0;  // the "called" flag of TMarchRK3 (src/tsteps.f90:35)
};

// ------------------------------------------------- grid, initial.f90:4395-4480
static void init_grid(Domain &d, const elmm_config &c) {
  int nx = d.Prnx, ny = d.Prny, nz = d.Prnz;
  A1 xU2, yV2, zW2;
  xU2.init(-3, nx + 3);
  yV2.init(-3, ny + 3);
  zW2.init(-3, nz + 3);
  for (int i = -3; i <= nx + 3; i++) xU2(i) = i * d.dxmin + c.xmin;
  for (int j = -3; j <= ny + 3; j++) yV2(j) = j * d.dymin + c.ymin;
  if (c.zW) {
    for (int k = 0; k <= nz; k++) zW2(k) = c.zW[k];
    if (d.Btype[Bo] == BC_PERIODIC) {
      for (int j = -1; j >= -3; j--) zW2(j) = zW2(0) - (zW2(nz - 1) - zW2(nz - 1 + j));
    } else {
      for (int j = -1; j >= -3; j--) zW2(j) = zW2(0) - (zW2(-j) - zW2(0));
    }
    if (d.Btype[To] == BC_PERIODIC) {
      for (int j = nz + 1; j <= nz + 3; j++) zW2(j) = zW2(nz - 1) + (zW2(j - nz + 1) - zW2(0));
    } else {
      // initial.f90:4427-4430, kept as written (mirror about zW(nz-1))
      for (int j = nz + 1; j <= nz + 3; j++)
        zW2(j) = zW2(nz - 1) + (zW2(nz - 1) - zW2(nz - 1 - (j - nz + 1)));
    }
  } else {
    for (int k = -3; k <= nz + 3; k++) zW2(k) = k * d.dzmin + c.zmin;
  }
  d.xU = xU2; d.yV = yV2; d.zW = zW2;
  d.xPr.init(-2, nx + 3); d.dxPr.init(-2, nx + 3);
  d.yPr.init(-2, ny + 3); d.dyPr.init(-2, ny + 3);
  d.zPr.init(-2, nz + 3); d.dzPr.init(-2, nz + 3);
  d.dxU.init(-2, nx + 2); d.dyV.init(-2, ny + 2); d.dzW.init(-2, nz + 2);
  for (int i = -2; i <= nx + 3; i++) { d.xPr(i) = (d.xU(i - 1) + d.xU(i)) / 2.0; d.dxPr(i) = d.xU(i) - d.xU(i - 1); }
  for (int j = -2; j <= ny + 3; j++) { d.yPr(j) = (d.yV(j - 1) + d.yV(j)) / 2.0; d.dyPr(j) = d.yV(j) - d.yV(j - 1); }
  for (int k = -2; k <= nz + 3; k++) { d.zPr(k) = (d.zW(k - 1) + d.zW(k)) / 2.0; d.dzPr(k) = d.zW(k) - d.zW(k - 1); }
  for (int i = -2; i <= nx + 2; i++) d.dxU(i) = d.xPr(i + 1) - d.xPr(i);
  for (int j = -2; j <= ny + 2; j++) d.dyV(j) = d.yPr(j + 1) - d.yPr(j);
  for (int k = -2; k <= nz + 2; k++) d.dzW(k) = d.zPr(k + 1) - d.zPr(k);
  if (c.zW) {
    double m = d.dzPr(-2);
    for (int k = -2; k <= nz + 3; k++) m = std::min(m, d.dzPr(k));
    d.dzmin = m;
  }
}

// ------------------------------------ wall-model points, wallmodels.f90:690-909
static void add_wm_points(Domain &d) {
  for (int comp = 1; comp <= 3; comp++) {
    int nx = comp == 1 ? d.Unx : comp == 2 ? d.Vnx : d.Wnx;
    int ny = comp == 1 ? d.Uny : comp == 2 ? d.Vny : d.Wny;
    int nz = comp == 1 ? d.Unz : comp == 2 ? d.Vnz : d.Wnz;
    const A1 &x = comp == 1 ? d.xU : d.xPr;
    const A1 &y = comp == 2 ? d.yV : d.yPr;
    const A1 &z = comp == 3 ? d.zW : d.zPr;
    WMPointUVW p;
    if (d.Btype[We] == BC_NOSLIP)
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++) {
          p = WMPointUVW(); p.xi = 1; p.yj = j; p.zk = k;
          p.distx = d.xU(0) - x(1); p.z0 = d.z0s[We];
          d.wm[MINUSX][comp].push_back(p);
        }
    if (d.Btype[Ea] == BC_NOSLIP)
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++) {
          p = WMPointUVW(); p.xi = nx; p.yj = j; p.zk = k;
          p.distx = d.xU(d.Unx + 1) - x(nx); p.z0 = d.z0s[Ea];
          d.wm[PLUSX][comp].push_back(p);
        }
    if (d.Btype[So] == BC_NOSLIP)
      for (int k = 1; k <= nz; k++)
        for (int i = 1; i <= nx; i++) {
          p = WMPointUVW(); p.xi = i; p.yj = 1; p.zk = k;
          p.disty = d.yV(0) - y(1); p.z0 = d.z0s[So];
          d.wm[MINUSY][comp].push_back(p);
        }
    if (d.Btype[No] == BC_NOSLIP)
      for (int k = 1; k <= nz; k++)
        for (int i = 1; i <= nx; i++) {
          p = WMPointUVW(); p.xi = i; p.yj = ny; p.zk = k;
          p.disty = d.yV(d.Vny + 1) - y(ny); p.z0 = d.z0s[No];
          d.wm[PLUSY][comp].push_back(p);
        }
    if (d.Btype[Bo] == BC_NOSLIP)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          p = WMPointUVW(); p.xi = i; p.yj = j; p.zk = 1;
          p.distz = d.zW(0) - z(1); p.z0 = d.z0s[Bo];
          p.temperature_flux = d.wm_tflux[Bo];
          p.prescribed_temperature = !d.wmpr[Bo].empty(); p.temperature = d.sideTemp[Bo];
          d.wm[MINUSZ][comp].push_back(p);
        }
    if (d.Btype[To] == BC_NOSLIP)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          p = WMPointUVW(); p.xi = i; p.yj = j; p.zk = nz;
          p.distz = d.zW(d.Wnz + 1) - z(nz); p.z0 = d.z0s[To];
          p.temperature_flux = d.wm_tflux[To];
          p.prescribed_temperature = !d.wmpr[To].empty(); p.temperature = d.sideTemp[To];
          d.wm[PLUSZ][comp].push_back(p);
        }
  }
}

// ------------------------------------------ BoundUVW_do_BC, boundaries.f90:398-1791
// The x pass fills i-ghosts for interior j,k; the y pass all i; the z pass all
// i,j.  periodic_corners_edges (boundaries.f90:189-394) only writes cells that
// these three passes overwrite afterwards, so it does not change the result.
static void bound_x(Domain &d, A3 &X, int comp, int n, int ny, int nz) {
  bool normal = comp == 1;
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++) {
      switch (d.Btype[We]) {
        case BC_NOSLIP:
          if (normal) { X(0, j, k) = 0; X(-1, j, k) = -X(1, j, k); X(-2, j, k) = -X(2, j, k); }
          else { X(0, j, k) = -X(1, j, k); X(-1, j, k) = -X(2, j, k); X(-2, j, k) = -X(3, j, k); }
          break;
        case BC_NEUMANN:
          X(0, j, k) = X(1, j, k); X(-1, j, k) = X(1, j, k); X(-2, j, k) = X(1, j, k);
          break;
        case BC_FREESLIP:
          if (normal) { X(0, j, k) = 0; X(-1, j, k) = -X(1, j, k); X(-2, j, k) = -X(2, j, k); }
          else { X(0, j, k) = X(1, j, k); X(-1, j, k) = X(1, j, k); X(-2, j, k) = X(1, j, k); }
          break;
        case BC_PERIODIC:
          X(0, j, k) = X(n, j, k); X(-1, j, k) = X(n - 1, j, k); X(-2, j, k) = X(n - 2, j, k);
          break;
      }
    }
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++) {
      switch (d.Btype[Ea]) {
        case BC_NOSLIP:
          if (normal) { X(n + 1, j, k) = 0; X(n + 2, j, k) = -X(n, j, k); X(n + 3, j, k) = -X(n - 1, j, k); }
          else { X(n + 1, j, k) = -X(n, j, k); X(n + 2, j, k) = -X(n - 1, j, k); X(n + 3, j, k) = -X(n - 2, j, k); }
          break;
        case BC_NEUMANN:
          X(n + 1, j, k) = X(n, j, k); X(n + 2, j, k) = X(n, j, k); X(n + 3, j, k) = X(n, j, k);
          break;
        case BC_FREESLIP:
          if (normal) { X(n + 1, j, k) = 0; X(n + 2, j, k) = -X(n, j, k); X(n + 3, j, k) = -X(n - 1, j, k); }
          else { X(n + 1, j, k) = X(n, j, k); X(n + 2, j, k) = X(n, j, k); X(n + 3, j, k) = X(n, j, k); }
          break;
        case BC_PERIODIC:
          X(n + 1, j, k) = X(1, j, k); X(n + 2, j, k) = X(2, j, k); X(n + 3, j, k) = X(3, j, k);
          break;
      }
    }
}

static void bound_y(Domain &d, A3 &X, int comp, int nx, int n, int nz) {
  bool normal = comp == 2;
  for (int k = 1; k <= nz; k++)
    for (int i = -2; i <= nx + 3; i++) {
      switch (d.Btype[So]) {
        case BC_NOSLIP:
          if (normal) { X(i, 0, k) = 0; X(i, -1, k) = -X(i, 1, k); X(i, -2, k) = -X(i, 2, k); }
          else { X(i, 0, k) = -X(i, 1, k); X(i, -1, k) = -X(i, 2, k); X(i, -2, k) = -X(i, 3, k); }
          break;
        case BC_NEUMANN:
          X(i, 0, k) = X(i, 1, k); X(i, -1, k) = X(i, 1, k); X(i, -2, k) = X(i, 1, k);
          break;
        case BC_FREESLIP:
          if (normal) { X(i, 0, k) = 0; X(i, -1, k) = -X(i, 1, k); X(i, -2, k) = -X(i, 2, k); }
          else { X(i, 0, k) = X(i, 1, k); X(i, -1, k) = X(i, 1, k); X(i, -2, k) = X(i, 1, k); }
          break;
        case BC_PERIODIC:
          X(i, 0, k) = X(i, n, k); X(i, -1, k) = X(i, n - 1, k); X(i, -2, k) = X(i, n - 2, k);
          break;
      }
    }
  for (int k = 1; k <= nz; k++)
    for (int i = -2; i <= nx + 3; i++) {
      switch (d.Btype[No]) {
        case BC_NOSLIP:
          if (normal) { X(i, n + 1, k) = 0; X(i, n + 2, k) = -X(i, n, k); X(i, n + 3, k) = -X(i, n - 1, k); }
          else { X(i, n + 1, k) = -X(i, n, k); X(i, n + 2, k) = -X(i, n - 1, k); X(i, n + 3, k) = -X(i, n - 2, k); }
          break;
        case BC_NEUMANN:
          X(i, n + 1, k) = X(i, n, k); X(i, n + 2, k) = X(i, n, k); X(i, n + 3, k) = X(i, n, k);
          break;
        case BC_FREESLIP:
          if (normal) { X(i, n + 1, k) = 0; X(i, n + 2, k) = -X(i, n, k); X(i, n + 3, k) = -X(i, n - 1, k); }
          else { X(i, n + 1, k) = X(i, n, k); X(i, n + 2, k) = X(i, n, k); X(i, n + 3, k) = X(i, n, k); }
          break;
        case BC_PERIODIC:
          X(i, n + 1, k) = X(i, 1, k); X(i, n + 2, k) = X(i, 2, k); X(i, n + 3, k) = X(i, 3, k);
          break;
      }
    }
}

static void bound_z(Domain &d, A3 &X, int comp, int nx, int ny, int n) {
  bool normal = comp == 3;
  for (int j = -2; j <= ny + 3; j++)
    for (int i = -2; i <= nx + 3; i++) {
      switch (d.Btype[Bo]) {
        case BC_NOSLIP:
          if (normal) { X(i, j, 0) = 0; X(i, j, -1) = -X(i, j, 1); X(i, j, -2) = -X(i, j, 2); }
          else { X(i, j, 0) = -X(i, j, 1); X(i, j, -1) = -X(i, j, 2); X(i, j, -2) = -X(i, j, 3); }
          break;
        case BC_NEUMANN:
          X(i, j, 0) = X(i, j, 1); X(i, j, -1) = X(i, j, 1); X(i, j, -2) = X(i, j, 1);
          break;
        case BC_FREESLIP:
          if (normal) { X(i, j, 0) = 0; X(i, j, -1) = -X(i, j, 1); X(i, j, -2) = -X(i, j, 2); }
          else { X(i, j, 0) = X(i, j, 1); X(i, j, -1) = X(i, j, 1); X(i, j, -2) = X(i, j, 1); }
          break;
        case BC_PERIODIC:
          X(i, j, 0) = X(i, j, n); X(i, j, -1) = X(i, j, n - 1); X(i, j, -2) = X(i, j, n - 2);
          break;
      }
    }
  for (int j = -2; j <= ny + 3; j++)
    for (int i = -2; i <= nx + 3; i++) {
      switch (d.Btype[To]) {
        case BC_NOSLIP:
          if (normal) { X(i, j, n + 1) = 0; X(i, j, n + 2) = -X(i, j, n); X(i, j, n + 3) = -X(i, j, n - 1); }
          else { X(i, j, n + 1) = -X(i, j, n); X(i, j, n + 2) = -X(i, j, n - 1); X(i, j, n + 3) = -X(i, j, n - 2); }
          break;
        case BC_NEUMANN:
          X(i, j, n + 1) = X(i, j, n); X(i, j, n + 2) = X(i, j, n); X(i, j, n + 3) = X(i, j, n);
          break;
        case BC_FREESLIP:
          if (normal) { X(i, j, n + 1) = 0; X(i, j, n + 2) = -X(i, j, n); X(i, j, n + 3) = -X(i, j, n - 1); }
          else { X(i, j, n + 1) = X(i, j, n); X(i, j, n + 2) = X(i, j, n); X(i, j, n + 3) = X(i, j, n); }
          break;
        case BC_PERIODIC:
          X(i, j, n + 1) = X(i, j, 1); X(i, j, n + 2) = X(i, j, 2); X(i, j, n + 3) = X(i, j, 3);
          break;
      }
    }
}

static void BoundUVW(Domain &d, A3 &U, A3 &V, A3 &W) {
  bound_x(d, U, 1, d.Unx, d.Uny, d.Unz);
  bound_x(d, V, 2, d.Vnx, d.Vny, d.Vnz);
  bound_x(d, W, 3, d.Wnx, d.Wny, d.Wnz);
  bound_y(d, V, 2, d.Vnx, d.Vny, d.Vnz);
  bound_y(d, U, 1, d.Unx, d.Uny, d.Unz);
  bound_y(d, W, 3, d.Wnx, d.Wny, d.Wnz);
  bound_z(d, W, 3, d.Wnx, d.Wny, d.Wnz);
  bound_z(d, U, 1, d.Unx, d.Uny, d.Unz);
  bound_z(d, V, 2, d.Vnx, d.Vny, d.Vnz);
}

// --------------------------------- BoundViscosity, scalarboundaries.f90:326-431
static void BoundViscosity(Domain &d, A3 &Nu) {
  int nx = d.Prnx, ny = d.Prny, nz = d.Prnz;
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++) Nu(0, j, k) = d.Btype[We] == BC_PERIODIC ? Nu(nx, j, k) : Nu(1, j, k);
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++) Nu(nx + 1, j, k) = d.Btype[Ea] == BC_PERIODIC ? Nu(1, j, k) : Nu(nx, j, k);
  for (int k = 1; k <= nz; k++)
    for (int i = 0; i <= nx + 1; i++) Nu(i, 0, k) = d.Btype[So] == BC_PERIODIC ? Nu(i, ny, k) : Nu(i, 1, k);
  for (int k = 1; k <= nz; k++)
    for (int i = 0; i <= nx + 1; i++) Nu(i, ny + 1, k) = d.Btype[No] == BC_PERIODIC ? Nu(i, 1, k) : Nu(i, ny, k);
  for (int j = 0; j <= ny + 1; j++)
    for (int i = 0; i <= nx + 1; i++) Nu(i, j, 0) = d.Btype[Bo] == BC_PERIODIC ? Nu(i, j, nz) : Nu(i, j, 1);
  for (int j = 0; j <= ny + 1; j++)
    for (int i = 0; i <= nx + 1; i++) Nu(i, j, nz + 1) = d.Btype[To] == BC_PERIODIC ? Nu(i, j, 1) : Nu(i, j, nz);
}

// --------------------------------------------- Bound_Phi, boundaries.f90:1817-1948
static void Bound_Phi(Domain &d, A3 &Phi) {
  int nx = d.Prnx, ny = d.Prny, nz = d.Prnz;
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++) {
      if (d.PrBtype[We] == BC_PERIODIC) { Phi(-1, j, k) = Phi(nx - 1, j, k); Phi(0, j, k) = Phi(nx, j, k); }
      else { Phi(-1, j, k) = Phi(2, j, k); Phi(0, j, k) = Phi(1, j, k); }
      if (d.PrBtype[Ea] == BC_PERIODIC) { Phi(nx + 1, j, k) = Phi(1, j, k); Phi(nx + 2, j, k) = Phi(2, j, k); }
      else { Phi(nx + 1, j, k) = Phi(nx, j, k); Phi(nx + 2, j, k) = Phi(nx - 1, j, k); }
    }
  for (int k = 1; k <= nz; k++)
    for (int i = 1; i <= nx; i++) {
      if (d.PrBtype[So] == BC_PERIODIC) { Phi(i, -1, k) = Phi(i, ny - 1, k); Phi(i, 0, k) = Phi(i, ny, k); }
      else { Phi(i, -1, k) = Phi(i, 2, k); Phi(i, 0, k) = Phi(i, 1, k); }
      if (d.PrBtype[No] == BC_PERIODIC) { Phi(i, ny + 1, k) = Phi(i, 1, k); Phi(i, ny + 2, k) = Phi(i, 2, k); }
      else { Phi(i, ny + 1, k) = Phi(i, ny, k); Phi(i, ny + 2, k) = Phi(i, ny - 1, k); }
    }
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++) {
      if (d.PrBtype[Bo] == BC_PERIODIC) { Phi(i, j, -1) = Phi(i, j, nz - 1); Phi(i, j, 0) = Phi(i, j, nz); }
      else { Phi(i, j, -1) = Phi(i, j, 2); Phi(i, j, 0) = Phi(i, j, 1); }
      if (d.PrBtype[To] == BC_PERIODIC) { Phi(i, j, nz + 1) = Phi(i, j, 1); Phi(i, j, nz + 2) = Phi(i, j, 2); }
      else { Phi(i, j, nz + 1) = Phi(i, j, nz); Phi(i, j, nz + 2) = Phi(i, j, nz - 1); }
    }
}

// ---------------------------------------------- Bound_Pr, boundaries.f90:1951-2091
static void Bound_Pr(Domain &d, A3 &Pr) {
  int nx = d.Prnx, ny = d.Prny, nz = d.Prnz;
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++) {
      if (d.PrBtype[We] == BC_PERIODIC) { Pr(-1, j, k) = Pr(nx - 1, j, k); Pr(0, j, k) = Pr(nx, j, k); }
      else { Pr(0, j, k) = Pr(3, j, k) - 3 * (Pr(2, j, k) - Pr(1, j, k)); Pr(-1, j, k) = Pr(2, j, k); }
      if (d.PrBtype[Ea] == BC_PERIODIC) { Pr(nx + 1, j, k) = Pr(1, j, k); Pr(nx + 2, j, k) = Pr(2, j, k); }
      else { Pr(nx + 1, j, k) = Pr(nx - 2, j, k) - 3 * (Pr(nx - 1, j, k) - Pr(nx, j, k)); Pr(nx + 2, j, k) = Pr(nx - 1, j, k); }
    }
  for (int k = 1; k <= nz; k++)
    for (int i = 1; i <= nx; i++) {
      if (d.PrBtype[So] == BC_PERIODIC) { Pr(i, -1, k) = Pr(i, ny - 1, k); Pr(i, 0, k) = Pr(i, ny, k); }
      else { Pr(i, 0, k) = Pr(i, 3, k) - 3 * (Pr(i, 2, k) - Pr(i, 1, k)); Pr(i, -1, k) = Pr(i, 2, k); }
      if (d.PrBtype[No] == BC_PERIODIC) { Pr(i, ny + 1, k) = Pr(i, 1, k); Pr(i, ny + 2, k) = Pr(i, 2, k); }
      else { Pr(i, ny + 1, k) = Pr(i, ny - 2, k) - 3 * (Pr(i, ny - 1, k) - Pr(i, ny, k)); Pr(i, ny + 2, k) = Pr(i, ny - 1, k); }
    }
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++) {
      if (d.PrBtype[Bo] == BC_PERIODIC) { Pr(i, j, -1) = Pr(i, j, nz - 1); Pr(i, j, 0) = Pr(i, j, nz); }
      else { Pr(i, j, 0) = Pr(i, j, 3) - 3 * (Pr(i, j, 2) - Pr(i, j, 1)); Pr(i, j, -1) = Pr(i, j, 2); }
      if (d.PrBtype[To] == BC_PERIODIC) { Pr(i, j, nz + 1) = Pr(i, j, 1); Pr(i, j, nz + 2) = Pr(i, j, 2); }
      else { Pr(i, j, nz + 1) = Pr(i, j, nz - 2) - 3 * (Pr(i, j, nz - 1) - Pr(i, j, nz)); Pr(i, j, nz + 2) = Pr(i, j, nz - 1); }
    }
}

// --------------------------------------- SGS_Smag / NuSmag, subgrid.f90:30-67, :170-209
static inline double nusmag(const Domain &d, int i, int j, int k) {
  const A3 &U = d.U, &V = d.V, &W = d.W;
  double width = d.filter_ratio * std::pow(d.dxPr(i) * d.dyPr(j) * d.dzPr(k), 1.0 / 3.0);
  double D[3][3];
  D[0][0] = (U(i, j, k) - U(i - 1, j, k)) / d.dxmin;
  D[1][1] = (V(i, j, k) - V(i, j - 1, k)) / d.dymin;
  D[2][2] = (W(i, j, k) - W(i, j, k - 1)) / d.dzPr(k);
  D[0][1] = (U(i, j + 1, k) + U(i - 1, j + 1, k) - U(i, j - 1, k) - U(i - 1, j - 1, k)) / (4 * d.dymin);
  D[0][2] = (U(i, j, k + 1) + U(i - 1, j, k + 1) - U(i, j, k - 1) - U(i - 1, j, k - 1)) / (2 * (d.zPr(k + 1) - d.zPr(k - 1)));
  D[1][0] = (V(i + 1, j, k) + V(i + 1, j - 1, k) - V(i - 1, j, k) - V(i - 1, j - 1, k)) / (4 * d.dxmin);
  D[1][2] = (V(i, j, k + 1) + V(i, j - 1, k + 1) - V(i, j, k - 1) - V(i, j - 1, k - 1)) / (2 * (d.zPr(k + 1) - d.zPr(k - 1)));
  D[2][0] = (W(i + 1, j, k) + W(i + 1, j, k - 1) - W(i - 1, j, k) - W(i - 1, j, k - 1)) / (4 * d.dxmin);
  D[2][1] = (W(i, j + 1, k) + W(i, j + 1, k - 1) - W(i, j - 1, k) - W(i, j - 1, k - 1)) / (4 * d.dymin);
  double S = 0;
  for (int jj = 0; jj < 3; jj++)
    for (int ii = 0; ii < 3; ii++) {
      double s = (D[ii][jj] + D[jj][ii]) / 2;
      S = S + s * s;
    }
  double Sbar = std::sqrt(2.0 * S);
  double wc = width * d.C_Smagorinsky;
  return Sbar * (wc * wc);
}

static void SubgridModel(Domain &d) {
  if (d.sgstype == 1) {
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= d.Prnz; k++)
      for (int j = 1; j <= d.Prny; j++)
        for (int i = 1; i <= d.Prnx; i++) d.Viscosity(i, j, k) = nusmag(d, i, j, k);
    if (d.molecular_viscosity > 0)
      for (auto &x : d.Viscosity.v) x = x + d.molecular_viscosity;
  } else {
    d.Viscosity.fill(d.molecular_viscosity);
  }
}

// ----------------------------------------------- wall model, wallmodels.f90:1190-1400
// NORM2 evaluated with the scaled sum of squares used by gfortran.
static inline double norm2_3(const double *x) {
  double scale = 0, ssq = 1;
  for (int m = 0; m < 3; m++) {
    if (x[m] != 0) {
      double ax = std::fabs(x[m]);
      if (scale < ax) { double r = scale / ax; ssq = 1 + ssq * (r * r); scale = ax; }
      else { double r = ax / scale; ssq = ssq + r * r; }
    }
  }
  return scale * std::sqrt(ssq);
}

static void WMFlatUstar(const Domain &d, double &ustar, double vel, double dist) {
  const double nu = d.molecular_viscosity;
  const double eps = 1e-4, zpl_lam = 5.0, zpl_turb = 30.0;
  if (nu <= 0) { ustar = 0; return; }
  double ustar_lam = std::sqrt(nu * vel / dist);
  if ((dist * ustar_lam / nu) < zpl_lam) {
    ustar = ustar_lam;
  } else {
    int i = 0;
    for (;;) {
      i = i + 1;
      double ustar2 = ustar;
      double z_pl = dist * ustar2 / nu;
      if (z_pl <= zpl_lam) ustar = std::sqrt(nu * vel / dist);
      else if (z_pl < zpl_turb) ustar = vel / (5 * std::log(z_pl) - (double)3.05f);  // 3.05 is a default-real literal
      else ustar = vel / (std::log(z_pl) / 0.4 + 5.5);
      if (std::fabs(ustar - ustar2) / std::fabs(ustar) < eps) break;
      if (i >= 50) { ustar = 0; break; }
    }
  }
}

static void WMRoughUstar(const Domain &d, double &ustar, double vel, double dist, double z0) {
  const double nu = d.molecular_viscosity;
  const double yplcrit = 11.225;
  if (nu > 0) {
    ustar = std::sqrt(nu * vel / dist);
    if (dist * ustar / nu < yplcrit * 1.1) return;
  }
  if (dist <= z0 * 2) {
    if (nu > 0) WMFlatUstar(d, ustar, vel, dist);
    else ustar = 0;
  } else {
    ustar = vel * 0.41 / std::log(dist / z0);
  }
}

// PsiM_MO, wallmodels.f90:1546-1556
static double PsiM_MO(double zeta) {
  if (zeta < 0) {
    const double x = std::pow(1 - 15.0 * zeta, 1 / 4.0);
    const double h = (1 + x) / 2.0;
    return std::log(((1 + x * x) / 2.0) * (h * h)) - 2.0 * std::atan(x) + std::acos(-1.0) / 2;
  }
  return -4.8 * zeta;
}

// WM_MO_Flux_ustar, wallmodels.f90:1606-1660, with Obukhov_zL (:1598-1602);
// eps = 1e-3, 1E-4 and 1E-5 are default-real literals there
static void WM_MO_Flux_ustar(const Domain &d, double vel, double dist, double &ustar, double z0, double tflux) {
  const double nu = d.molecular_viscosity;
  const double eps = (double)1e-3f, yplcrit = 11.225;
  if (dist <= z0) {
    if (nu > 0) {
      if ((dist * ustar / nu) < yplcrit) ustar = std::sqrt(nu * vel / dist);
      else ustar = vel / (std::log(std::fabs(ustar * dist / nu)) / 0.4 + 5.2);
    } else {
      ustar = 0;
    }
    return;
  }
  int i = 0;
  double zL = 0, Psi = 0;
  for (;;) {
    i = i + 1;
    const double ustar2 = ustar;
    ustar = ustar + (std::max(vel * 0.4 / (std::log(std::max((dist / z0) - Psi, (double)1e-5f))), 0.0) - ustar) / 2;
    if (ustar < (double)1e-4f) {
      zL = -10000;
    } else {
      const double zL2 = dist * (0.4 * (d.grav_acc / d.temperature_ref) * tflux) / (-(ustar * ustar * ustar));
      zL = zL + (zL2 - zL) / 2;
    }
    Psi = PsiM_MO(zL);
    if (std::fabs(ustar - ustar2) / std::max(std::fabs(ustar), 1.e-3) < eps) break;
    if (i >= 50) { ustar = 0; break; }
  }
}

// PsiM_MO_mod / PsiH_MO_mod, wallmodels.f90:1572-1595
static double PsiM_MO_mod(double zeta, double k_U) {
  if (zeta < 0) {
    const double x = std::pow(1 - 6.0 * zeta * k_U, 1 / 4.0);
    const double h = (1 + x) / 2.0;
    return std::log(((1 + x * x) / 2.0) * (h * h)) - 2.0 * std::atan(x) + std::acos(-1.0) / 2;
  }
  return -(3 * std::pow(zeta * k_U, 5.0 / 6.0));
}

static double PsiH_MO_mod(double zeta, double k_U) {
  if (zeta < 0) {
    const double x = std::pow(1 - 6.0 * zeta * k_U, 1 / 4.0);
    return 2.0 * std::log((1 + x * x) / 2.0);
  }
  return -(2.5 * std::pow(zeta * k_U, 4.0 / 5.0));
}

// WM_MO_Dirichlet_ustar_tfl, wallmodels.f90:1664-1716 (its 1.1 is a
// default-real literal); tempdif = theta(point) - theta(surface)
static void WM_MO_Dirichlet_ustar_tfl(const Domain &d, double &ustar, double &tflux, double dist, double z0,
                                      double z0H, double vel, double tempdif) {
  const double eps = 1e-3, yplcrit = 11.225, k_U = 0.4, k_T = 0.47;
  const double nu = d.molecular_viscosity;
  WMRoughUstar(d, ustar, vel, dist, z0);
  double dist_plus;
  if (nu > 0) {
    const double ustar_lam = std::sqrt(nu * vel / dist);
    dist_plus = dist * ustar_lam / nu;
  } else {
    dist_plus = std::numeric_limits<double>::max();
  }
  if (dist <= z0 || dist_plus < (double)1.1f * yplcrit) {
    tflux = -d.molecular_diffusivity * tempdif / dist;
    return;
  }
  double zL = 0, zL0 = -10000.0;
  int i = 0;
  for (;;) {
    i = i + 1;
    zL = -dist * d.grav_acc * tflux / (k_U * d.temperature_ref * (ustar * ustar * ustar));
    const double psi_m = PsiM_MO_mod(zL, k_U), psi_h = PsiH_MO_mod(zL, k_U);
    ustar = vel * k_U / (std::log(dist / z0) - psi_m);
    tflux = -tempdif * ustar * k_T / (std::log(dist / z0H) - psi_h);
    if (i > 1 && std::fabs(zL - zL0) / std::max(std::fabs(zL), 1.e-4) < eps) break;
    if (i >= 50 || zL > 10000) break;
    zL0 = zL;
  }
  if (i >= 50 || zL > 10000) {
    ustar = std::sqrt(nu * vel / dist);
    tflux = -d.molecular_diffusivity * tempdif / dist;
  }
}

// ComputeViscsWM, wallmodels.f90:2050-2152, for the Pr points with a
// prescribed surface temperature (WM_MO_Dirichlet, :1858-1884): their u*
// and surface temperature flux.  The viscosity it forms is overwritten by
// SubgridModel in a stage (dynamics.f90:882-889) and is not kept.
static void ComputeViscsWM(Domain &d) {
  for (int side : {Bo, To})
    for (WMPointPr &p : d.wmpr[side]) {
      const int xi = p.xi, yj = p.yj, zk = p.zk;
      const double dv[3] = {0, 0, p.distz};
      const double uv[3] = {(d.U(xi, yj, zk) + d.U(xi - 1, yj, zk)) / 2.0,
                            (d.V(xi, yj, zk) + d.V(xi, yj - 1, zk)) / 2.0,
                            (d.W(xi, yj, zk) + d.W(xi, yj, zk - 1)) / 2.0};
      const double tdif = d.T(xi, yj, zk) - p.temperature;
      if (!(p.z0 > 0)) continue;
      // WM_MO_Dirichlet: sqrt(sum(...**2)) and the tangential part
      const double dist = std::sqrt((dv[0] * dv[0] + dv[1] * dv[1]) + dv[2] * dv[2]);
      const double dot = (uv[0] * dv[0] + uv[1] * dv[1]) + uv[2] * dv[2];
      double vect[3];
      for (int m = 0; m < 3; m++) vect[m] = uv[m] - dot * dv[m] / (dist * dist);
      const double vel = std::sqrt((vect[0] * vect[0] + vect[1] * vect[1]) + vect[2] * vect[2]);
      WM_MO_Dirichlet_ustar_tfl(d, p.ustar, p.temperature_flux, dist, p.z0, p.z0, vel, tdif);
      if (p.ustar < 0) p.ustar = 0;
    }
}

// local_value, wallmodels.f90:2340-2353
static double local_value(const A3 &C, int comp, int xi, int yj, int zk) {
  if (comp == 1) return (C(xi + 1, yj, zk) + C(xi, yj, zk)) / 2;
  if (comp == 2) return (C(xi, yj + 1, zk) + C(xi, yj, zk)) / 2;
  return (C(xi, yj, zk + 1) + C(xi, yj, zk)) / 2;
}

// local_velocity, wallmodels.f90:2354-2396
static void local_velocity(const Domain &d, int comp, int xi, int yj, int zk, double *vel) {
  const A3 &U = d.U, &V = d.V, &W = d.W;
  if (comp == 1) {
    vel[0] = U(xi, yj, zk);
    vel[1] = (V(xi + 1, yj, zk) + V(xi, yj, zk) + V(xi + 1, yj - 1, zk) + V(xi, yj - 1, zk)) / 4.0;
    vel[2] = (W(xi + 1, yj, zk) + W(xi, yj, zk) + W(xi + 1, yj, zk - 1) + W(xi, yj, zk - 1)) / 4.0;
  } else if (comp == 2) {
    vel[0] = (U(xi, yj + 1, zk) + U(xi, yj, zk) + U(xi - 1, yj + 1, zk) + U(xi - 1, yj, zk)) / 4.0;
    vel[1] = V(xi, yj, zk);
    vel[2] = (W(xi, yj + 1, zk) + W(xi, yj, zk) + W(xi, yj + 1, zk - 1) + W(xi, yj, zk - 1)) / 4.0;
  } else {
    vel[0] = (U(xi, yj, zk + 1) + U(xi, yj, zk) + U(xi - 1, yj, zk + 1) + U(xi - 1, yj, zk)) / 4.0;
    vel[1] = (V(xi, yj, zk + 1) + V(xi, yj, zk) + V(xi, yj - 1, zk + 1) + V(xi, yj - 1, zk)) / 4.0;
    vel[2] = W(xi, yj, zk);
  }
}

// ComputeUVWFluxesWM / fluxes, wallmodels.f90:2159-2338
static void ComputeUVWFluxesWM(Domain &d) {
  const double eps = std::sqrt(2.220446049250313e-16);
  double drec[7] = {0, 1 / d.dxmin, 1 / d.dxmin, 1 / d.dymin, 1 / d.dymin, 1 / d.dzmin, 1 / d.dzmin};
  for (int comp = 1; comp <= 3; comp++)
    for (int dir = 1; dir <= 6; dir++) {
      auto &pts = d.wm[dir][comp];
      for (size_t n = 0; n < pts.size(); n++) {
        WMPointUVW &p = pts[n];
        double dist[3] = {p.distx, p.disty, p.distz};
        double vel[3];
        local_velocity(d, comp, p.xi, p.yj, p.zk, vel);
        double wallvel[3] = {p.wallu, p.wallv, p.wallw};
        // WMRoughStress -> vel_and_dist (wallmodels.f90:1383-1389)
        double dd = norm2_3(dist);
        double t[3];
        for (int m = 0; m < 3; m++) t[m] = vel[m] - wallvel[m];
        double dot = t[0] * dist[0] + t[1] * dist[1] + t[2] * dist[2];
        for (int m = 0; m < 3; m++) t[m] = t[m] - dot * dist[m] / (dd * dd);
        double tv = norm2_3(t);
        // WM_MO_FluxStress for a rough wall with a temperature flux into the
        // flow, else WMRoughStress with a roughness length, WMFlatStress for a
        // smooth wall (wallmodels.f90:2255-2275; WM_MO_FluxStress, :1836-1854;
        // WMFlatStress, :1243-1265)
        if (p.z0 > 0 && d.enable_buoyancy && p.prescribed_temperature) {
          // WM_MO_DirichletStress (:1922-1938): sqrt(sum(tan_vect**2))
          const double vel2 = std::sqrt((t[0] * t[0] + t[1] * t[1]) + t[2] * t[2]);
          const double temp = local_value(d.T, comp, p.xi, p.yj, p.zk);
          WM_MO_Dirichlet_ustar_tfl(d, p.ustar, p.temperature_flux, dd, p.z0, p.z0, vel2, temp - p.temperature);
        } else if (p.z0 > 0 && d.enable_buoyancy && p.temperature_flux > 0) {
          if (tv != 0) WM_MO_Flux_ustar(d, tv, dd, p.ustar, p.z0, p.temperature_flux);
          else p.ustar = 0;
        } else if (tv != 0) {
          if (p.z0 > 0) WMRoughUstar(d, p.ustar, tv, dd, p.z0);
          else WMFlatUstar(d, p.ustar, tv, dd);
        }
        if (p.ustar < 0) p.ustar = 0;
        double mag = norm2_3(t);
        if (mag > eps) {
          if (d.gridtype == 1 && dir == MINUSZ) {
            p.fluxp = (t[comp - 1] / mag) * (p.ustar * p.ustar);
            p.fluxm = p.fluxp;
            if (comp == 1 || comp == 2) { p.fluxp = p.fluxp / d.dzPr(p.zk); p.fluxm = p.fluxm / d.dzPr(p.zk - 1); }
            else { p.fluxp = p.fluxp / d.dzW(p.zk); p.fluxm = p.fluxm / d.dzW(p.zk - 1); }
          } else if (d.gridtype == 1 && dir == PLUSZ) {
            p.fluxp = (t[comp - 1] / mag) * (p.ustar * p.ustar);
            p.fluxm = p.fluxp;
            if (comp == 1 || comp == 2) { p.fluxp = p.fluxp / d.dzPr(p.zk + 1); p.fluxm = p.fluxm / d.dzPr(p.zk); }
            else { p.fluxp = p.fluxp / d.dzW(p.zk + 1); p.fluxm = p.fluxm / d.dzW(p.zk); }
          } else {
            p.fluxp = (t[comp - 1] / mag) * (p.ustar * p.ustar) * drec[dir];
            p.fluxm = p.fluxp;
          }
          if (dir % 2 == 1) { p.fluxp = -p.fluxp; p.fluxm = -p.fluxm; }
        } else {
          p.fluxp = 0;
          p.fluxm = p.fluxp;
        }
      }
    }
}

// ComputeTDiff, scalar_diffusion.f90:983-1009 (constant Pr_sgs = 0.6,
// scalar_diffusion.f90:22)
static void ComputeTDiff(Domain &d) {
  const double Pr_sgs = 0.6;
  for (int k = 1; k <= d.Prnz; k++)
    for (int j = 1; j <= d.Prny; j++)
      for (int i = 1; i <= d.Prnx; i++) {
        if (d.molecular_viscosity > 0)
          d.TDiff(i, j, k) = (d.Viscosity(i, j, k) - d.molecular_viscosity) / Pr_sgs + d.molecular_diffusivity;
        else
          d.TDiff(i, j, k) = d.Viscosity(i, j, k) / Pr_sgs;
      }
}

// SubgridStresses, dynamics.f90:869-908 (ComputeViscsWM only sets Viscosity at
// wall cells, which SubgridModel then overwrites everywhere; it is omitted).
// TIBPoint_Interpolate, immersedboundary.f90:637-651
static double IBInterpolate(const elmm_ib_point &p, const A3 &F) {
  double v = 0;
  for (int n = 0; n < p.interp; n++) v = v + p.coef[n] * F(p.ii[n], p.jj[n], p.kk[n]);
  return v;
}

static void SubgridStresses(Domain &d) {
  if (d.wallmodeltype > 0) ComputeViscsWM(d);  // dynamics.f90:882-885
  SubgridModel(d);
  if (d.wallmodeltype > 0) ComputeUVWFluxesWM(d);
  BoundViscosity(d, d.Viscosity);
  // viscosity of the ScalFl IB points, in place in list order (dynamics.f90:899-902)
  for (auto &p : d.scalfl) d.Viscosity(p.xi, p.yj, p.zk) = IBInterpolate(p, d.Viscosity);
  if (d.enable_buoyancy) ComputeTDiff(d);  // dynamics.f90:904
  if (d.enable_buoyancy || d.num_scalars > 0) BoundViscosity(d, d.TDiff);  // dynamics.f90:906
}

// BuoyancyForce, FD2 branch of dynamics.f90:679-688
static void BuoyancyForce(Domain &d, A3 &Wst) {
  const double A = d.grav_acc / d.temperature_ref, A2 = A / 2.0;
  for (int k = 1; k <= d.Wnz; k++)
    for (int j = 1; j <= d.Wny; j++)
      for (int i = 1; i <= d.Wnx; i++)
        Wst(i, j, k) = Wst(i, j, k) + A2 * (d.T(i, j, k + 1) + d.T(i, j, k)) - A * d.temperature_ref;
}

// BoundTemperature -> CommonBase, scalarboundaries.f90:12-300: periodic and
// constant-flux x and y sides, and in z periodic, Dirichlet, Neumann,
// constant-flux and (TempBtype 0 after GetOutsideBoundariesWM_Pr) mirror
// sides (the x, y loops run over the ranges of the reference, corners
// included where it includes them)
static void CommonBase(Domain &d, A3 &a, const int *bt, const double *side) {
  const int nx = d.Prnx, ny = d.Prny, nz = d.Prnz;
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++) {
      if (bt[We] == BC_PERIODIC) {
        for (int g = -2; g <= 0; g++) a(g, j, k) = a(nx + g, j, k);
      } else {
        a(0, j, k) = a(1, j, k) + side[We] * d.dxU(0) / ((d.TDiff(1, j, k) + d.TDiff(0, j, k)) / 2.0);
        a(-1, j, k) = a(0, j, k) - (a(1, j, k) - a(0, j, k));
        a(-2, j, k) = a(0, j, k) - 2 * (a(1, j, k) - a(0, j, k));
      }
      if (bt[Ea] == BC_PERIODIC) {
        for (int g = 1; g <= 3; g++) a(nx + g, j, k) = a(g, j, k);
      } else {
        a(nx + 1, j, k) = a(nx, j, k) - side[Ea] * d.dxU(nx) / ((d.TDiff(nx, j, k) + d.TDiff(nx + 1, j, k)) / 2.0);
        a(nx + 2, j, k) = a(nx + 1, j, k) - (a(nx, j, k) - a(nx + 1, j, k));
        a(nx + 3, j, k) = a(nx + 1, j, k) - 2 * (a(nx, j, k) - a(nx + 1, j, k));
      }
    }
  for (int k = 1; k <= nz; k++)
    for (int i = -1; i <= nx + 2; i++) {
      if (bt[So] == BC_PERIODIC) {
        for (int g = -2; g <= 0; g++) a(i, g, k) = a(i, ny + g, k);
      } else {
        a(i, 0, k) = a(i, 1, k) + side[So] * d.dyV(0) / ((d.TDiff(i, 1, k) + d.TDiff(i, 0, k)) / 2.0);
        a(i, -1, k) = a(i, 0, k) - (a(i, 1, k) - a(i, 0, k));
        a(i, -2, k) = a(i, 0, k) - 2 * (a(i, 1, k) - a(i, 0, k));
      }
      if (bt[No] == BC_PERIODIC) {
        for (int g = 1; g <= 3; g++) a(i, ny + g, k) = a(i, g, k);
      } else {
        a(i, ny + 1, k) = a(i, ny + 1, k) - side[No] * d.dyV(ny) / ((d.TDiff(i, ny, k) + d.TDiff(i, ny + 1, k)) / 2.0);
        a(i, ny + 2, k) = a(i, ny + 1, k) - (a(i, ny, k) - a(i, ny + 1, k));
        a(i, ny + 3, k) = a(i, ny + 1, k) - 2 * (a(i, ny, k) - a(i, ny + 1, k));
      }
    }
  for (int j = -1; j <= ny + 2; j++)
    for (int i = -1; i <= nx + 2; i++) {
      if (bt[Bo] == BC_PERIODIC) {
        for (int g = -2; g <= 0; g++) a(i, j, g) = a(i, j, nz + g);
      } else if (bt[Bo] == 0) {  // mirror
        for (int g = -2; g <= 0; g++) a(i, j, g) = a(i, j, 1 - g);
      } else if (bt[Bo] == ELMM_BC_DIRICHLET) {
        for (int g = -2; g <= 0; g++) a(i, j, g) = side[Bo] - (a(i, j, 1 - g) - side[Bo]);
      } else if (bt[Bo] == BC_NEUMANN) {
        a(i, j, 0) = a(i, j, 1) - side[Bo] * d.dzW(0);
        a(i, j, -1) = a(i, j, 1) - side[Bo] * (d.zPr(1) - d.zPr(-1));
        a(i, j, -2) = a(i, j, 1) - side[Bo] * (d.zPr(1) - d.zPr(-2));
      } else {
        a(i, j, 0) = a(i, j, 1) + side[Bo] * d.dzW(0) / ((d.TDiff(i, j, 1) + d.TDiff(i, j, 0)) / 2.0);
        a(i, j, -1) = a(i, j, 0) - (a(i, j, 1) - a(i, j, 0));
        a(i, j, -2) = a(i, j, 0) - 2 * (a(i, j, 1) - a(i, j, 0));
      }
      if (bt[To] == BC_PERIODIC) {
        for (int g = 1; g <= 3; g++) a(i, j, nz + g) = a(i, j, g);
      } else if (bt[To] == 0) {  // mirror
        for (int g = 1; g <= 3; g++) a(i, j, nz + g) = a(i, j, nz + 1 - g);
      } else if (bt[To] == ELMM_BC_DIRICHLET) {
        for (int g = 1; g <= 3; g++) a(i, j, nz + g) = side[To] - (a(i, j, nz + 1 - g) - side[To]);
      } else if (bt[To] == BC_NEUMANN) {
        a(i, j, nz + 1) = a(i, j, nz) + side[To] * d.dzW(nz + 1);
        a(i, j, nz + 2) = a(i, j, nz) + side[To] * (d.zPr(nz + 2) - d.zPr(nz));
        a(i, j, nz + 3) = a(i, j, nz) + side[To] * (d.zPr(nz + 3) - d.zPr(nz));
      } else {
        a(i, j, nz + 1) = a(i, j, nz) - side[To] * d.dzW(nz) / ((d.TDiff(i, j, nz) + d.TDiff(i, j, nz + 1)) / 2.0);
        a(i, j, nz + 2) = a(i, j, nz + 1) - (a(i, j, nz) - a(i, j, nz + 1));
        a(i, j, nz + 3) = a(i, j, nz + 1) - 2 * (a(i, j, nz) - a(i, j, nz + 1));
      }
    }
}

static void BoundTemperature(Domain &d, A3 &a) { CommonBase(d, a, d.TempBtype, d.sideTemp); }
// BoundScalar, scalarboundaries.f90:284-289
static void BoundScalar(Domain &d, A3 &a) { CommonBase(d, a, d.ScalBtype, d.sideScal); }

// FluxLimiter of KappaScalar, scalar_advection.f90:262-270
static inline double kappa_limiter(double r) { return std::max(0.0, std::min(2 * r, std::min(2.0, (1 + 2 * r) / 3))); }
static inline double fsign(double a, double b) { return std::signbit(b) ? -std::fabs(a) : std::fabs(a); }

// KappaScalar, scalar_advection.f90:102-272 (no masked faces without solid
// bodies, wallmodels.f90:910-950): slopes and fluxes per face, accumulated in
// the reference's loop order (the z faces even before odd)
static void KappaScalar(Domain &d, A3 &S2, const A3 &S) {
  const int nx = d.Prnx, ny = d.Prny, nz = d.Prnz;
  const A3 &U = d.U, &V = d.V, &W = d.W;
  const double eps = 1e-8;
  const double Ax = 1 / d.dxmin, Ay = 1 / d.dymin, Az = 1 / d.dzmin;
  S2.fill(0);
  auto slope = [&](double sr, double sl) { return kappa_limiter((sr + eps * fsign(1.0, sl)) / (sl + eps * fsign(1.0, sl))); };
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        double sr, sl, flux;
        if (U(i, j, k) > 0) { sr = S(i + 1, j, k) - S(i, j, k); sl = S(i, j, k) - S(i - 1, j, k); }
        else { sr = S(i, j, k) - S(i + 1, j, k); sl = S(i + 1, j, k) - S(i + 2, j, k); }
        const double sp = slope(sr, sl);
        if (U(i, j, k) > 0) flux = U(i, j, k) * (S(i, j, k) + (S(i, j, k) - S(i - 1, j, k)) * sp / 2.0);
        else flux = U(i, j, k) * (S(i + 1, j, k) + (S(i + 1, j, k) - S(i + 2, j, k)) * sp / 2.0);
        S2(i, j, k) = S2(i, j, k) - Ax * flux;
        S2(i + 1, j, k) = S2(i + 1, j, k) + Ax * flux;
      }
  for (int k = 1; k <= nz; k++)
    for (int j = 0; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        double sr, sl, flux;
        if (V(i, j, k) > 0) { sr = S(i, j + 1, k) - S(i, j, k); sl = S(i, j, k) - S(i, j - 1, k); }
        else { sr = S(i, j, k) - S(i, j + 1, k); sl = S(i, j + 1, k) - S(i, j + 2, k); }
        const double sp = slope(sr, sl);
        if (V(i, j, k) > 0) flux = V(i, j, k) * (S(i, j, k) + (S(i, j, k) - S(i, j - 1, k)) * sp / 2.0);
        else flux = V(i, j, k) * (S(i, j + 1, k) + (S(i, j + 1, k) - S(i, j + 2, k)) * sp / 2.0);
        S2(i, j, k) = S2(i, j, k) - Ay * flux;
        S2(i, j + 1, k) = S2(i, j + 1, k) + Ay * flux;
      }
  for (int l = 0; l <= 1; l++)
    for (int k = l; k <= nz; k += 2)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          double sr, sl, flux;
          const double vel = W(i, j, k);
          if (vel > 0) { sr = S(i, j, k + 1) - S(i, j, k); sl = S(i, j, k) - S(i, j, k - 1); }
          else { sr = S(i, j, k) - S(i, j, k + 1); sl = S(i, j, k + 1) - S(i, j, k + 2); }
          const double sp = slope(sr, sl);
          if (vel > 0) flux = vel * (S(i, j, k) + (S(i, j, k) - S(i, j, k - 1)) * sp / 2.0);
          else flux = vel * (S(i, j, k + 1) + (S(i, j, k + 1) - S(i, j, k + 2)) * sp / 2.0);
          S2(i, j, k) = S2(i, j, k) - Az * flux;
          S2(i, j, k + 1) = S2(i, j, k + 1) + Az * flux;
        }
}

// ScalarDiffusion_nobranch, scalar_diffusion.f90:404-507 (no flux points
// without solid bodies)
static void ScalarDiffusion(Domain &d, A3 &S2, const A3 &S) {
  const A3 &K = d.TDiff;
  const double Ax = 1 / (2 * d.dxmin * d.dxmin), Ay = 1 / (2 * d.dymin * d.dymin), Az = 1 / (2 * d.dzmin * d.dzmin);
  for (int k = 1; k <= d.Prnz; k++)
    for (int j = 1; j <= d.Prny; j++)
      for (int i = 1; i <= d.Prnx; i++) {
        double a = S2(i, j, k);
        a = a + (K(i + 1, j, k) + K(i, j, k)) * (S(i + 1, j, k) - S(i, j, k)) * Ax;
        a = a - (K(i, j, k) + K(i - 1, j, k)) * (S(i, j, k) - S(i - 1, j, k)) * Ax;
        a = a + (K(i, j + 1, k) + K(i, j, k)) * (S(i, j + 1, k) - S(i, j, k)) * Ay;
        a = a - (K(i, j, k) + K(i, j - 1, k)) * (S(i, j, k) - S(i, j - 1, k)) * Ay;
        a = a + (K(i, j, k + 1) + K(i, j, k)) * (S(i, j, k + 1) - S(i, j, k)) * Az;
        a = a - (K(i, j, k) + K(i, j, k - 1)) * (S(i, j, k) - S(i, j, k - 1)) * Az;
        S2(i, j, k) = a;
      }
}

// stage() of ScalarRK3 (scalars.f90:233-299) for one field: the temperature
// (sc = 0) or passive scalar sc.  The scalar wall-model points are the cells
// next to a wall-model side (DivergenceWM, wallmodels.f90:1150-1166, with the
// velocity at the start of the stage); TemperatureExtra adds the surface
// flux (temperature_flux * area_factor) and div * T there
// (scalars.f90:301-334), ScalarExtra first the volume sources of the scalar
// (ScalarVolumeSources -> FluxKernel, volumesources.f90:741-771) and then
// div * S (scalars.f90:364-379).
static void ScalarStage(Domain &d, int stage, double dt, A3 &Arr, A3 &Arr2, A3 &Adv, int sc) {
  const int nx = d.Prnx, ny = d.Prny, nz = d.Prnz;
  auto bound = [&](A3 &a) { if (sc == 0) BoundTemperature(d, a); else BoundScalar(d, a); };
  std::vector<double> divb((size_t)nx * ny, 0.0), divt((size_t)nx * ny, 0.0);
  const bool wb = d.wallmodeltype > 0 && d.Btype[Bo] == BC_NOSLIP, wt = d.wallmodeltype > 0 && d.Btype[To] == BC_NOSLIP;
  auto wmdiv = [&](int i, int j, int k) {
    double div = 0;
    div = div + d.U(i, j, k) / d.dxmin;
    div = div - d.U(i - 1, j, k) / d.dxmin;
    div = div + d.V(i, j, k) / d.dymin;
    div = div - d.V(i, j - 1, k) / d.dymin;
    div = div + d.W(i, j, k) / d.dzPr(k);
    div = div - d.W(i, j, k - 1) / d.dzPr(k);
    return div;
  };
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++) {
      if (wb) divb[(size_t)(j - 1) * nx + i - 1] = wmdiv(i, j, 1);
      if (wt) divt[(size_t)(j - 1) * nx + i - 1] = wmdiv(i, j, nz);
    }
  bound(Arr);
  const double rdt = RK_rho[stage - 1] * dt, bdt = RK_beta[stage - 1] * dt;
  if (stage > 1) {
    for (size_t q = 0; q < Arr2.v.size(); q++) Arr2.v[q] = Adv.v[q] * rdt;
  } else {
    Arr2.fill(0);
  }
  KappaScalar(d, Adv, Arr);
  if (d.scal_solids)  // Array_adv = 0 at the solid cells (scalars.f90:259-268)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++)
          if (d.Prsolid(i, j, k) != 0) Adv(i, j, k) = 0;
  ScalarDiffusion(d, Adv, Arr);
  if (sc > 0)
    for (const auto &v : d.flvolumes)
      if (v.sc == sc) Adv(v.i, v.j, v.k) = Adv(v.i, v.j, v.k) + v.flux;
  // DoPuffs / DoPuff, puffs.f90:86-126 (ScalarExtra, scalars.f90:366-372)
  if (sc > 0)
    for (size_t q = 0; q < d.puffs.size(); q++)
      if (d.puffs[q].dt_fraction > 0)
        for (const auto &v : d.puffvols)
          if (v.puff == (int)q && v.sc == sc)
            Adv(v.i, v.j, v.k) = Adv(v.i, v.j, v.k) + d.puffs[q].dt_fraction * v.flux;
  // with solid bodies: DivergenceWM over the points of the list, without the
  // faces towards solid cells (wallmodels.f90:1150-1166)
  if (d.scal_solids)
    for (const auto &p : d.wmprs) {
      const int i = p[0], j = p[1], k = p[2];
      double div = 0;
      if (d.Prsolid(i + 1, j, k) == 0) div = div + d.U(i, j, k) / d.dxmin;
      if (d.Prsolid(i - 1, j, k) == 0) div = div - d.U(i - 1, j, k) / d.dxmin;
      if (d.Prsolid(i, j + 1, k) == 0) div = div + d.V(i, j, k) / d.dymin;
      if (d.Prsolid(i, j - 1, k) == 0) div = div - d.V(i, j - 1, k) / d.dymin;
      if (d.Prsolid(i, j, k + 1) == 0) div = div + d.W(i, j, k) / d.dzPr(k);
      if (d.Prsolid(i, j, k - 1) == 0) div = div - d.W(i, j, k - 1) / d.dzPr(k);
      if (sc == 0) {  // the kept point's temperature_flux * area_factor: the wall's, or the body's
        double q = d.HeatQ(i, j, k);
        if (d.WallPt(i, j, k) != 0) {
          const int side = k == 1 ? Bo : To;
          const size_t c = (size_t)(j - 1) * nx + i - 1;
          q = (d.wmpr[side].empty() ? d.wm_tflux[side] : d.wmpr[side][c].temperature_flux) * d.area_factor_z;
        }
        Adv(i, j, k) = Adv(i, j, k) + q;
      }
      Adv(i, j, k) = Adv(i, j, k) + div * Arr(i, j, k);
    }
  for (int j = 1; j <= ny && !d.scal_solids; j++)
    for (int i = 1; i <= nx; i++) {
      const size_t q = (size_t)(j - 1) * nx + i - 1;
      if (wb) {
        if (sc == 0 && !d.wmpr[Bo].empty()) Adv(i, j, 1) = Adv(i, j, 1) + d.wmpr[Bo][q].temperature_flux * d.area_factor_z;
        else if (sc == 0) Adv(i, j, 1) = Adv(i, j, 1) + d.wm_tflux[Bo] * d.area_factor_z;
        Adv(i, j, 1) = Adv(i, j, 1) + divb[(size_t)(j - 1) * nx + i - 1] * Arr(i, j, 1);
      }
      if (wt) {
        if (sc == 0 && !d.wmpr[To].empty()) Adv(i, j, nz) = Adv(i, j, nz) + d.wmpr[To][q].temperature_flux * d.area_factor_z;
        else if (sc == 0) Adv(i, j, nz) = Adv(i, j, nz) + d.wm_tflux[To] * d.area_factor_z;
        Adv(i, j, nz) = Adv(i, j, nz) + divt[(size_t)(j - 1) * nx + i - 1] * Arr(i, j, nz);
      }
    }
  for (size_t q = 0; q < Arr2.v.size(); q++) Arr2.v[q] = Arr2.v[q] + Adv.v[q] * bdt;
  for (size_t q = 0; q < Arr.v.size(); q++) Arr.v[q] = Arr.v[q] + Arr2.v[q];
  bound(Arr);
}

// PreparePuffs, puffs.f90:30-84 (RK_stages = 3), with its
// `time + dt - max(...) / dt` as written
static void PreparePuffs(Domain &d, int stage, double time, double dt) {
  for (size_t q = 0; q < d.puffs.size(); q++) {
    Domain::Puff &p = d.puffs[q];
    if (stage == 1) {
      p.restart = time + dt > p.last_start + p.period && time + dt >= p.start_time && time <= p.end_time;
      if (!p.restart && time <= p.last_start + p.duration && time >= p.start_time)
        p.dt_fraction = std::max(std::min(std::min(p.last_start + p.duration, time + dt), p.end_time) - time, 0.0) / dt;
      else if (p.restart)
        p.dt_fraction = time + dt - std::max(std::max(p.last_start + p.period, time), p.start_time) / dt;
      else
        p.dt_fraction = 0;
      if (p.clear && p.restart)
        for (const auto &v : d.puffvols)
          if (v.puff == (int)q && v.sc >= 1 && v.sc <= d.num_scalars) d.S[v.sc - 1].fill(0);
    }
    if (p.restart && stage == 3) p.last_start = p.last_start >= p.start_time ? p.last_start + p.period : p.start_time;
  }
}

// The fill of the solid cells after the temperature stage, scalars.f90:129-198,
// in its loop order: a solid cell with fluid neighbours (range -1..n+2)
// becomes their mean; for a cell without any the reference sums all six
// neighbours and assigns nothing, so it keeps its value
static void FillSolidTemperature(Domain &d) {
  const int nx = d.Prnx, ny = d.Prny, nz = d.Prnz;
  A3 &T = d.T;
  const A3 &P = d.Prsolid;
  for (int k = -1; k <= nz + 2; k++)
    for (int j = -1; j <= ny + 2; j++)
      for (int i = -1; i <= nx + 2; i++) {
        if (P(i, j, k) == 0) continue;
        double t = 0;
        int n = 0;
        if (i > -1 && P(i - 1, j, k) == 0) { t = t + T(i - 1, j, k); n = n + 1; }
        if (i < nx + 2 && P(i + 1, j, k) == 0) { t = t + T(i + 1, j, k); n = n + 1; }
        if (j > -1 && P(i, j - 1, k) == 0) { t = t + T(i, j - 1, k); n = n + 1; }
        if (j < ny + 2 && P(i, j + 1, k) == 0) { t = t + T(i, j + 1, k); n = n + 1; }
        if (k > -1 && P(i, j, k - 1) == 0) { t = t + T(i, j, k - 1); n = n + 1; }
        if (k < nz + 2 && P(i, j, k + 1) == 0) { t = t + T(i, j, k + 1); n = n + 1; }
        if (n > 0) T(i, j, k) = t / n;
      }
}

// ScalarRK3 (scalars.f90:88-381): the temperature, then each passive scalar
static void ScalarRK3(Domain &d, int stage, double dt) {
  if (d.enable_buoyancy) {
    ScalarStage(d, stage, dt, d.T, d.T2, d.Tadv, 0);
    if (d.scal_solids) FillSolidTemperature(d);
  }
  PreparePuffs(d, stage, d.time, dt);  // scalars.f90:217
  for (int sc = 1; sc <= d.num_scalars; sc++)
    ScalarStage(d, stage, dt, d.S[sc - 1], d.S2[sc - 1], d.Sadv[sc - 1], sc);
}

// Scalar_avg = Scalar_avg + Scalar * time_weight (outputs.f90:1043-1045) on
// the two slice planes
static void AccumulateScalarAverages(Domain &d) {
  const int nx = d.Prnx, ny = d.Prny, nz = d.Prnz;
  // time_weight is proportional to the step's length: avg_weight belongs to a
  // step of length dt, a variable step weighs its length / dt of it
  const double avg_w = d.variable_time_steps ? d.avg_w * (d.dt / d.dt0) : d.avg_w;
  for (int sc = 0; sc < d.num_scalars; sc++) {
    const A3 &S = d.S[sc];
    if (d.avg_k > 0)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          double &a = d.acc_xy[sc][(size_t)(j - 1) * nx + i - 1];
          a = a + S(i, j, d.avg_k) * avg_w;
        }
    if (d.avg_j > 0)
      for (int k = 1; k <= nz; k++)
        for (int i = 1; i <= nx; i++) {
          double &a = d.acc_xz[sc][(size_t)(k - 1) * nx + i - 1];
          a = a + S(i, d.avg_j, k) * avg_w;
        }
  }
}

// ---------------------------------------------- CDS2 advection, advection.f90:15-327
static void CDU(Domain &d, A3 &U2) {
  const A3 &U = d.U, &V = d.V, &W = d.W;
  U2.fill(0);
  if (d.gridtype == 0) {
    double Ax = 0.25 / d.dxmin, Ay = 0.25 / d.dymin, Az = 0.25 / d.dzmin;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= d.Unz; k++)
      for (int j = 1; j <= d.Uny; j++)
        for (int i = 1; i <= d.Unx; i++) {
          U2(i, j, k) = -((Ax * (U(i + 1, j, k) + U(i, j, k)) * (U(i + 1, j, k) + U(i, j, k))
                           - Ax * (U(i, j, k) + U(i - 1, j, k)) * (U(i, j, k) + U(i - 1, j, k)))
                          + (Ay * (U(i, j + 1, k) + U(i, j, k)) * (V(i + 1, j, k) + V(i, j, k))
                             - Ay * (U(i, j, k) + U(i, j - 1, k)) * (V(i + 1, j - 1, k) + V(i, j - 1, k)))
                          + (Az * (U(i, j, k + 1) + U(i, j, k)) * (W(i + 1, j, k) + W(i, j, k))
                             - Az * (U(i, j, k) + U(i, j, k - 1)) * (W(i + 1, j, k - 1) + W(i, j, k - 1))));
        }
    Ax = 0.5 / d.dxmin; Ay = 0.125 / d.dymin; Az = 0.125 / d.dzmin;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= d.Unz; k++)
      for (int j = 1; j <= d.Uny; j++)
        for (int i = 1; i <= d.Unx; i++) {
          double Vadv = (V(i, j, k) + V(i + 1, j, k) + V(i, j - 1, k) + V(i + 1, j - 1, k));
          double Wadv = (W(i, j, k) + W(i + 1, j, k) + W(i, j, k - 1) + W(i + 1, j, k - 1));
          U2(i, j, k) = U2(i, j, k) - (Ax * (U(i + 1, j, k) - U(i - 1, j, k)) * U(i, j, k)
                                       + Ay * (U(i, j + 1, k) - U(i, j - 1, k)) * Vadv
                                       + Az * (U(i, j, k + 1) - U(i, j, k - 1)) * Wadv);
        }
  } else {  // advection_variable_z.f90:15-46, :151-181
    double Ax = 0.25 / d.dxmin, Ay = 0.25 / d.dymin;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= d.Unz; k++)
      for (int j = 1; j <= d.Uny; j++)
        for (int i = 1; i <= d.Unx; i++) {
          U2(i, j, k) = -((Ax * (U(i + 1, j, k) + U(i, j, k)) * (U(i + 1, j, k) + U(i, j, k))
                           - Ax * (U(i, j, k) + U(i - 1, j, k)) * (U(i, j, k) + U(i - 1, j, k)))
                          + (Ay * (U(i, j + 1, k) + U(i, j, k)) * (V(i + 1, j, k) + V(i, j, k))
                             - Ay * (U(i, j, k) + U(i, j - 1, k)) * (V(i + 1, j - 1, k) + V(i, j - 1, k)))
                          + ((U(i, j, k + 1) + U(i, j, k)) * (W(i + 1, j, k) + W(i, j, k))
                             - (U(i, j, k) + U(i, j, k - 1)) * (W(i + 1, j, k - 1) + W(i, j, k - 1))) / d.dzPr(k) / 4);
        }
    Ax = 0.5 / d.dxmin; Ay = 0.125 / d.dymin;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= d.Unz; k++)
      for (int j = 1; j <= d.Uny; j++)
        for (int i = 1; i <= d.Unx; i++) {
          double Vadv = (V(i, j, k) + V(i + 1, j, k) + V(i, j - 1, k) + V(i + 1, j - 1, k));
          double Wadv = (W(i, j, k) + W(i + 1, j, k) + W(i, j, k - 1) + W(i + 1, j, k - 1)) / 4;
          U2(i, j, k) = U2(i, j, k) - (Ax * (U(i + 1, j, k) - U(i - 1, j, k)) * U(i, j, k)
                                       + Ay * (U(i, j + 1, k) - U(i, j - 1, k)) * Vadv
                                       + (U(i, j, k + 1) - U(i, j, k - 1)) / (d.zPr(k + 1) - d.zPr(k - 1)) * Wadv);
        }
  }
  for (auto &x : U2.v) x = x * 0.5;
}

static void CDV(Domain &d, A3 &V2) {
  const A3 &U = d.U, &V = d.V, &W = d.W;
  V2.fill(0);
  if (d.gridtype == 0) {
    double Ax = 0.25 / d.dxmin, Ay = 0.25 / d.dymin, Az = 0.25 / d.dzmin;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= d.Vnz; k++)
      for (int j = 1; j <= d.Vny; j++)
        for (int i = 1; i <= d.Vnx; i++) {
          V2(i, j, k) = -((Ay * (V(i, j + 1, k) + V(i, j, k)) * (V(i, j + 1, k) + V(i, j, k))
                           - Ay * (V(i, j, k) + V(i, j - 1, k)) * (V(i, j, k) + V(i, j - 1, k)))
                          + (Ax * (V(i + 1, j, k) + V(i, j, k)) * (U(i, j + 1, k) + U(i, j, k))
                             - Ax * (V(i, j, k) + V(i - 1, j, k)) * (U(i - 1, j + 1, k) + U(i - 1, j, k)))
                          + (Az * (V(i, j, k + 1) + V(i, j, k)) * (W(i, j + 1, k) + W(i, j, k))
                             - Az * (V(i, j, k) + V(i, j, k - 1)) * (W(i, j + 1, k - 1) + W(i, j, k - 1))));
        }
    Ax = 0.125 / d.dxmin; Ay = 0.5 / d.dymin; Az = 0.125 / d.dzmin;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= d.Vnz; k++)
      for (int j = 1; j <= d.Vny; j++)
        for (int i = 1; i <= d.Vnx; i++) {
          double Uadv = (U(i, j, k) + U(i, j + 1, k) + U(i - 1, j, k) + U(i - 1, j + 1, k));
          double Wadv = (W(i, j, k) + W(i, j + 1, k) + W(i, j, k - 1) + W(i, j + 1, k - 1));
          V2(i, j, k) = V2(i, j, k) - (Ax * (V(i + 1, j, k) - V(i - 1, j, k)) * Uadv
                                       + Ay * (V(i, j + 1, k) - V(i, j - 1, k)) * V(i, j, k)
                                       + Az * (V(i, j, k + 1) - V(i, j, k - 1)) * Wadv);
        }
  } else {  // advection_variable_z.f90:54-84, :184-214
    double Ax = 0.25 / d.dxmin, Ay = 0.25 / d.dymin;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= d.Vnz; k++)
      for (int j = 1; j <= d.Vny; j++)
        for (int i = 1; i <= d.Vnx; i++) {
          V2(i, j, k) = -((Ay * (V(i, j + 1, k) + V(i, j, k)) * (V(i, j + 1, k) + V(i, j, k))
                           - Ay * (V(i, j, k) + V(i, j - 1, k)) * (V(i, j, k) + V(i, j - 1, k)))
                          + (Ax * (V(i + 1, j, k) + V(i, j, k)) * (U(i, j + 1, k) + U(i, j, k))
                             - Ax * (V(i, j, k) + V(i - 1, j, k)) * (U(i - 1, j + 1, k) + U(i - 1, j, k)))
                          + ((V(i, j, k + 1) + V(i, j, k)) * (W(i, j + 1, k) + W(i, j, k))
                             - (V(i, j, k) + V(i, j, k - 1)) * (W(i, j + 1, k - 1) + W(i, j, k - 1))) / d.dzPr(k) / 4);
        }
    Ax = 0.125 / d.dxmin; Ay = 0.5 / d.dymin;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= d.Vnz; k++)
      for (int j = 1; j <= d.Vny; j++)
        for (int i = 1; i <= d.Vnx; i++) {
          double Uadv = (U(i, j, k) + U(i, j + 1, k) + U(i - 1, j, k) + U(i - 1, j + 1, k));
          double Wadv = (W(i, j, k) + W(i, j + 1, k) + W(i, j, k - 1) + W(i, j + 1, k - 1)) / 4;
          V2(i, j, k) = V2(i, j, k) - (Ax * (V(i + 1, j, k) - V(i - 1, j, k)) * Uadv
                                       + Ay * (V(i, j + 1, k) - V(i, j - 1, k)) * V(i, j, k)
                                       + (V(i, j, k + 1) - V(i, j, k - 1)) / (d.zPr(k + 1) - d.zPr(k - 1)) * Wadv);
        }
  }
  for (auto &x : V2.v) x = x * 0.5;
}

static void CDW(Domain &d, A3 &W2) {
  const A3 &U = d.U, &V = d.V, &W = d.W;
  W2.fill(0);
  if (d.gridtype == 0) {
    double Ax = 0.25 / d.dxmin, Ay = 0.25 / d.dymin, Az = 0.25 / d.dzmin;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= d.Wnz; k++)
      for (int j = 1; j <= d.Wny; j++)
        for (int i = 1; i <= d.Wnx; i++) {
          W2(i, j, k) = -((Az * (W(i, j, k + 1) + W(i, j, k)) * (W(i, j, k + 1) + W(i, j, k))
                           - Az * (W(i, j, k) + W(i, j, k - 1)) * (W(i, j, k) + W(i, j, k - 1)))
                          + (Ay * (W(i, j + 1, k) + W(i, j, k)) * (V(i, j, k + 1) + V(i, j, k))
                             - Ay * (W(i, j, k) + W(i, j - 1, k)) * (V(i, j - 1, k) + V(i, j - 1, k + 1)))
                          + (Ax * (W(i + 1, j, k) + W(i, j, k)) * (U(i, j, k + 1) + U(i, j, k))
                             - Ax * (W(i, j, k) + W(i - 1, j, k)) * (U(i - 1, j, k + 1) + U(i - 1, j, k))));
        }
    Ax = 0.125 / d.dxmin; Ay = 0.125 / d.dymin; Az = 0.5 / d.dzmin;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= d.Wnz; k++)
      for (int j = 1; j <= d.Wny; j++)
        for (int i = 1; i <= d.Wnx; i++) {
          double Uadv = (U(i, j, k) + U(i, j, k + 1) + U(i - 1, j, k) + U(i - 1, j, k + 1));
          double Vadv = (V(i, j, k) + V(i, j, k + 1) + V(i, j - 1, k) + V(i, j - 1, k + 1));
          W2(i, j, k) = W2(i, j, k) - (Ax * (W(i + 1, j, k) - W(i - 1, j, k)) * Uadv
                                       + Ay * (W(i, j + 1, k) - W(i, j - 1, k)) * Vadv
                                       + Az * (W(i, j, k + 1) - W(i, j, k - 1)) * W(i, j, k));
        }
  } else {  // advection_variable_z.f90:92-122, :217-247
    double Ax = 0.25 / d.dxmin, Ay = 0.25 / d.dymin;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= d.Wnz; k++)
      for (int j = 1; j <= d.Wny; j++)
        for (int i = 1; i <= d.Wnx; i++) {
          W2(i, j, k) = -(((W(i, j, k + 1) + W(i, j, k)) * (W(i, j, k + 1) + W(i, j, k))
                           - (W(i, j, k) + W(i, j, k - 1)) * (W(i, j, k) + W(i, j, k - 1))) / d.dzW(k) / 4
                          + (Ay * (W(i, j + 1, k) + W(i, j, k)) * (V(i, j, k + 1) + V(i, j, k))
                             - Ay * (W(i, j, k) + W(i, j - 1, k)) * (V(i, j - 1, k + 1) + V(i, j - 1, k)))
                          + (Ax * (W(i + 1, j, k) + W(i, j, k)) * (U(i, j, k + 1) + U(i, j, k))
                             - Ax * (W(i, j, k) + W(i - 1, j, k)) * (U(i - 1, j, k + 1) + U(i - 1, j, k))));
        }
    Ax = 0.125 / d.dxmin; Ay = 0.125 / d.dymin;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= d.Wnz; k++)
      for (int j = 1; j <= d.Wny; j++)
        for (int i = 1; i <= d.Wnx; i++) {
          double Uadv = (U(i, j, k) + U(i, j, k + 1) + U(i - 1, j, k) + U(i - 1, j, k + 1));
          double Vadv = (V(i, j, k) + V(i, j, k + 1) + V(i, j - 1, k) + V(i, j - 1, k + 1));
          W2(i, j, k) = W2(i, j, k) - (Ax * (W(i + 1, j, k) - W(i - 1, j, k)) * Uadv
                                       + Ay * (W(i, j + 1, k) - W(i, j - 1, k)) * Vadv
                                       + (W(i, j, k + 1) - W(i, j, k - 1)) / (d.zW(k + 1) - d.zW(k - 1)) * W(i, j, k));
        }
  }
  for (auto &x : W2.v) x = x * 0.5;
}

// ------------------------ MomentumDiffusion_nobranch_2ord, momentum_diffusion.f90:169-420
// followed by the wall-flux includes wmfluxes-[variable_z-]nobranch-{U,V,W}-inc.f90.
static void MomentumDiffusion(Domain &d, A3 &U2, A3 &V2, A3 &W2) {
  const A3 &U = d.U, &V = d.V, &W = d.W, &nu = d.Viscosity;
  const double rx = 1.0 / (d.dxmin * d.dxmin), ry = 1.0 / (d.dymin * d.dymin), rz = 1.0 / (d.dzmin * d.dzmin);
  const bool vz = d.gridtype == 1;
  const A1 &dzW = d.dzW, &dzPr = d.dzPr;
  // U
#pragma omp parallel for collapse(2)
  for (int k = 1; k <= d.Unz; k++)
    for (int j = 1; j <= d.Uny; j++)
      for (int i = 1; i <= d.Unx; i++) {
        double a = U2(i, j, k);
        a = a + nu(i + 1, j, k) * (U(i + 1, j, k) - U(i, j, k)) * rx;
        a = a - nu(i, j, k) * (U(i, j, k) - U(i - 1, j, k)) * rx;
        a = a + 0.25 * (nu(i + 1, j + 1, k) + nu(i + 1, j, k) + nu(i, j + 1, k) + nu(i, j, k)) * (U(i, j + 1, k) - U(i, j, k)) * ry;
        a = a - 0.25 * (nu(i + 1, j, k) + nu(i + 1, j - 1, k) + nu(i, j, k) + nu(i, j - 1, k)) * (U(i, j, k) - U(i, j - 1, k)) * ry;
        if (!vz) {
          a = a + 0.25 * (nu(i + 1, j, k + 1) + nu(i + 1, j, k) + nu(i, j, k + 1) + nu(i, j, k)) * (U(i, j, k + 1) - U(i, j, k)) * rz;
          a = a - 0.25 * (nu(i + 1, j, k) + nu(i + 1, j, k - 1) + nu(i, j, k) + nu(i, j, k - 1)) * (U(i, j, k) - U(i, j, k - 1)) * rz;
        } else {
          double t = 0.25 * (nu(i + 1, j, k + 1) + nu(i + 1, j, k) + nu(i, j, k + 1) + nu(i, j, k)) * (U(i, j, k + 1) - U(i, j, k)) / dzW(k);
          t = t - 0.25 * (nu(i + 1, j, k) + nu(i + 1, j, k - 1) + nu(i, j, k) + nu(i, j, k - 1)) * (U(i, j, k) - U(i, j, k - 1)) / dzW(k - 1);
          t = t / dzPr(k);
          a = a + t;
        }
        U2(i, j, k) = a;
      }
  // wmfluxes-nobranch-U-inc.f90 / wmfluxes-variable_z-nobranch-U-inc.f90
  for (auto &p : d.wm[MINUSX][1]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = nu((x - 1) + 1, y, z) * (U((x - 1) + 1, y, z) - U(x - 1, y, z)) * rx;
    U2(x, y, z) = U2(x, y, z) + f; U2(x, y, z) = U2(x, y, z) + p.fluxp;
  }
  for (auto &p : d.wm[MINUSX][1]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = nu((x - 1) + 1, y, z) * (U((x - 1) + 1, y, z) - U(x - 1, y, z)) * rx;
    if (vz) f = f / dzPr(z - 1);
    U2(x - 1, y, z) = U2(x - 1, y, z) - f; U2(x - 1, y, z) = U2(x - 1, y, z) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[PLUSX][1]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = nu(x + 1, y, z) * (U(x + 1, y, z) - U(x, y, z)) * rx;
    U2(x + 1, y, z) = U2(x + 1, y, z) + f; U2(x + 1, y, z) = U2(x + 1, y, z) + p.fluxp;
  }
  for (auto &p : d.wm[PLUSX][1]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = nu(x + 1, y, z) * (U(x + 1, y, z) - U(x, y, z)) * rx;
    U2(x, y, z) = U2(x, y, z) - f; U2(x, y, z) = U2(x, y, z) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[MINUSY][1]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x + 1, y, z) + nu(x + 1, y - 1, z) + nu(x, y, z) + nu(x, y - 1, z)) * (U(x, y, z) - U(x, y - 1, z)) * ry / 4;
    U2(x, y, z) = U2(x, y, z) + f; U2(x, y, z) = U2(x, y, z) + p.fluxp;
  }
  for (auto &p : d.wm[MINUSY][1]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x + 1, y, z) + nu(x + 1, y - 1, z) + nu(x, y, z) + nu(x, y - 1, z)) * (U(x, y, z) - U(x, y - 1, z)) * ry / 4;
    U2(x, y - 1, z) = U2(x, y - 1, z) - f; U2(x, y - 1, z) = U2(x, y - 1, z) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[PLUSY][1]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x + 1, y + 1, z) + nu(x + 1, y, z) + nu(x, y + 1, z) + nu(x, y, z)) * (U(x, y + 1, z) - U(x, y, z)) * ry / 4;
    U2(x, y + 1, z) = U2(x, y + 1, z) + f; U2(x, y + 1, z) = U2(x, y + 1, z) + p.fluxp;
  }
  for (auto &p : d.wm[PLUSY][1]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x + 1, y + 1, z) + nu(x + 1, y, z) + nu(x, y + 1, z) + nu(x, y, z)) * (U(x, y + 1, z) - U(x, y, z)) * ry / 4;
    U2(x, y, z) = U2(x, y, z) - f; U2(x, y, z) = U2(x, y, z) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[MINUSZ][1]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double s = nu(x + 1, y, z) + nu(x + 1, y, z - 1) + nu(x, y, z) + nu(x, y, z - 1);
    double f = vz ? s * (U(x, y, z) - U(x, y, z - 1)) / dzW(z - 1) / 4 / dzPr(z) : s * (U(x, y, z) - U(x, y, z - 1)) * rz / 4;
    U2(x, y, z) = U2(x, y, z) + f; U2(x, y, z) = U2(x, y, z) + p.fluxp;
  }
  for (auto &p : d.wm[MINUSZ][1]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double s = nu(x + 1, y, z) + nu(x + 1, y, z - 1) + nu(x, y, z) + nu(x, y, z - 1);
    double f = vz ? s * (U(x, y, z) - U(x, y, z - 1)) / dzW(z - 1) / 4 / dzPr(z - 1) : s * (U(x, y, z) - U(x, y, z - 1)) * rz / 4;
    U2(x, y, z - 1) = U2(x, y, z - 1) - f; U2(x, y, z - 1) = U2(x, y, z - 1) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[PLUSZ][1]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double s = nu(x + 1, y, z + 1) + nu(x + 1, y, z) + nu(x, y, z + 1) + nu(x, y, z);
    double f = vz ? s * (U(x, y, z + 1) - U(x, y, z)) / dzW(z) / 4 / dzPr(z + 1) : s * (U(x, y, z + 1) - U(x, y, z)) * rz / 4;
    U2(x, y, z + 1) = U2(x, y, z + 1) + f; U2(x, y, z + 1) = U2(x, y, z + 1) + p.fluxp;
  }
  for (auto &p : d.wm[PLUSZ][1]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double s = nu(x + 1, y, z + 1) + nu(x + 1, y, z) + nu(x, y, z + 1) + nu(x, y, z);
    double f = vz ? s * (U(x, y, z + 1) - U(x, y, z)) / dzW(z) / 4 / dzPr(z) : s * (U(x, y, z + 1) - U(x, y, z)) * rz / 4;
    U2(x, y, z) = U2(x, y, z) - f; U2(x, y, z) = U2(x, y, z) - (vz ? p.fluxm : p.fluxp);
  }

  // V
#pragma omp parallel for collapse(2)
  for (int k = 1; k <= d.Vnz; k++)
    for (int j = 1; j <= d.Vny; j++)
      for (int i = 1; i <= d.Vnx; i++) {
        double a = V2(i, j, k);
        a = a + 0.25 * (nu(i + 1, j + 1, k) + nu(i + 1, j, k) + nu(i, j + 1, k) + nu(i, j, k)) * (V(i + 1, j, k) - V(i, j, k)) * rx;
        a = a - 0.25 * (nu(i, j + 1, k) + nu(i, j, k) + nu(i - 1, j + 1, k) + nu(i - 1, j, k)) * (V(i, j, k) - V(i - 1, j, k)) * rx;
        a = a + nu(i, j + 1, k) * (V(i, j + 1, k) - V(i, j, k)) * ry;
        a = a - nu(i, j, k) * (V(i, j, k) - V(i, j - 1, k)) * ry;
        if (!vz) {
          a = a + 0.25 * (nu(i, j + 1, k + 1) + nu(i, j + 1, k) + nu(i, j, k + 1) + nu(i, j, k)) * (V(i, j, k + 1) - V(i, j, k)) * rz;
          a = a - 0.25 * (nu(i, j + 1, k) + nu(i, j + 1, k - 1) + nu(i, j, k) + nu(i, j, k - 1)) * (V(i, j, k) - V(i, j, k - 1)) * rz;
        } else {
          double t = 0.25 * (nu(i, j + 1, k + 1) + nu(i, j + 1, k) + nu(i, j, k + 1) + nu(i, j, k)) * (V(i, j, k + 1) - V(i, j, k)) / dzW(k);
          t = t - 0.25 * (nu(i, j + 1, k) + nu(i, j + 1, k - 1) + nu(i, j, k) + nu(i, j, k - 1)) * (V(i, j, k) - V(i, j, k - 1)) / dzW(k - 1);
          t = t / dzPr(k);
          a = a + t;
        }
        V2(i, j, k) = a;
      }
  for (auto &p : d.wm[MINUSX][2]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x, y + 1, z) + nu(x, y, z) + nu(x - 1, y + 1, z) + nu(x - 1, y, z)) * (V(x, y, z) - V(x - 1, y, z)) * rx / 4;
    V2(x, y, z) = V2(x, y, z) + f; V2(x, y, z) = V2(x, y, z) + p.fluxp;
  }
  for (auto &p : d.wm[MINUSX][2]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x, y + 1, z) + nu(x, y, z) + nu(x - 1, y + 1, z) + nu(x - 1, y, z)) * (V(x, y, z) - V(x - 1, y, z)) * rx / 4;
    if (vz) f = f / dzPr(z - 1);
    V2(x - 1, y, z) = V2(x - 1, y, z) - f; V2(x - 1, y, z) = V2(x - 1, y, z) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[PLUSX][2]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x + 1, y + 1, z) + nu(x + 1, y, z) + nu(x, y + 1, z) + nu(x, y, z)) * (V(x + 1, y, z) - V(x, y, z)) * rx / 4;
    V2(x + 1, y, z) = V2(x + 1, y, z) + f; V2(x + 1, y, z) = V2(x + 1, y, z) + p.fluxp;
  }
  for (auto &p : d.wm[PLUSX][2]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x + 1, y + 1, z) + nu(x + 1, y, z) + nu(x, y + 1, z) + nu(x, y, z)) * (V(x + 1, y, z) - V(x, y, z)) * rx / 4;
    V2(x, y, z) = V2(x, y, z) - f; V2(x, y, z) = V2(x, y, z) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[MINUSY][2]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = nu(x, y, z) * (V(x, y, z) - V(x, y - 1, z)) * ry;
    V2(x, y, z) = V2(x, y, z) + f; V2(x, y, z) = V2(x, y, z) + p.fluxp;
  }
  for (auto &p : d.wm[MINUSY][2]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = nu(x, y, z) * (V(x, y, z) - V(x, y - 1, z)) * ry;
    V2(x, y - 1, z) = V2(x, y - 1, z) - f; V2(x, y - 1, z) = V2(x, y - 1, z) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[PLUSY][2]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = nu(x, y + 1, z) * (V(x, y + 1, z) - V(x, y, z)) * ry;
    V2(x, y + 1, z) = V2(x, y + 1, z) + f; V2(x, y + 1, z) = V2(x, y + 1, z) + p.fluxp;
  }
  for (auto &p : d.wm[PLUSY][2]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = nu(x, y + 1, z) * (V(x, y + 1, z) - V(x, y, z)) * ry;
    V2(x, y, z) = V2(x, y, z) - f; V2(x, y, z) = V2(x, y, z) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[MINUSZ][2]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double s = nu(x, y + 1, z) + nu(x, y + 1, z - 1) + nu(x, y, z) + nu(x, y, z - 1);
    double f = vz ? s * (V(x, y, z) - V(x, y, z - 1)) / dzW(z - 1) / 4 / dzPr(z) : s * (V(x, y, z) - V(x, y, z - 1)) * rz / 4;
    V2(x, y, z) = V2(x, y, z) + f; V2(x, y, z) = V2(x, y, z) + p.fluxp;
  }
  for (auto &p : d.wm[MINUSZ][2]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double s = nu(x, y + 1, z) + nu(x, y + 1, z - 1) + nu(x, y, z) + nu(x, y, z - 1);
    double f = vz ? s * (V(x, y, z) - V(x, y, z - 1)) / dzW(z - 1) / 4 / dzPr(z - 1) : s * (V(x, y, z) - V(x, y, z - 1)) * rz / 4;
    V2(x, y, z - 1) = V2(x, y, z - 1) - f; V2(x, y, z - 1) = V2(x, y, z - 1) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[PLUSZ][2]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double s = nu(x, y + 1, z + 1) + nu(x, y + 1, z) + nu(x, y, z + 1) + nu(x, y, z);
    double f = vz ? s * (V(x, y, z + 1) - V(x, y, z)) / dzW(z) / 4 / dzPr(z + 1) : s * (V(x, y, z + 1) - V(x, y, z)) * rz / 4;
    V2(x, y, z + 1) = V2(x, y, z + 1) + f; V2(x, y, z + 1) = V2(x, y, z + 1) + p.fluxp;
  }
  for (auto &p : d.wm[PLUSZ][2]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double s = nu(x, y + 1, z + 1) + nu(x, y + 1, z) + nu(x, y, z + 1) + nu(x, y, z);
    double f = vz ? s * (V(x, y, z + 1) - V(x, y, z)) / dzW(z) / 4 / dzPr(z) : s * (V(x, y, z + 1) - V(x, y, z)) * rz / 4;
    V2(x, y, z) = V2(x, y, z) - f; V2(x, y, z) = V2(x, y, z) - (vz ? p.fluxm : p.fluxp);
  }

  // W
#pragma omp parallel for collapse(2)
  for (int k = 1; k <= d.Wnz; k++)
    for (int j = 1; j <= d.Wny; j++)
      for (int i = 1; i <= d.Wnx; i++) {
        double a = W2(i, j, k);
        a = a + 0.25 * (nu(i + 1, j, k + 1) + nu(i + 1, j, k) + nu(i, j, k + 1) + nu(i, j, k)) * (W(i + 1, j, k) - W(i, j, k)) * rx;
        a = a - 0.25 * (nu(i, j, k + 1) + nu(i, j, k) + nu(i - 1, j, k + 1) + nu(i - 1, j, k)) * (W(i, j, k) - W(i - 1, j, k)) * rx;
        a = a + 0.25 * (nu(i, j + 1, k + 1) + nu(i, j, k + 1) + nu(i, j + 1, k) + nu(i, j, k)) * (W(i, j + 1, k) - W(i, j, k)) * ry;
        a = a - 0.25 * (nu(i, j, k + 1) + nu(i, j - 1, k + 1) + nu(i, j, k) + nu(i, j - 1, k)) * (W(i, j, k) - W(i, j - 1, k)) * ry;
        if (!vz) {
          a = a + nu(i, j, k + 1) * (W(i, j, k + 1) - W(i, j, k)) * rz;
          a = a - nu(i, j, k) * (W(i, j, k) - W(i, j, k - 1)) * rz;
        } else {
          double t = nu(i, j, k + 1) * (W(i, j, k + 1) - W(i, j, k)) / dzPr(k + 1);
          t = t - nu(i, j, k) * (W(i, j, k) - W(i, j, k - 1)) / dzPr(k);
          t = t / dzW(k);
          a = a + t;
        }
        W2(i, j, k) = a;
      }
  for (auto &p : d.wm[MINUSX][3]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x, y, z + 1) + nu(x, y, z) + nu(x - 1, y, z + 1) + nu(x - 1, y, z)) * (W(x, y, z) - W(x - 1, y, z)) * rx / 4;
    W2(x, y, z) = W2(x, y, z) + f; W2(x, y, z) = W2(x, y, z) + p.fluxp;
  }
  for (auto &p : d.wm[MINUSX][3]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x, y, z + 1) + nu(x, y, z) + nu(x - 1, y, z + 1) + nu(x - 1, y, z)) * (W(x, y, z) - W(x - 1, y, z)) * rx / 4;
    if (vz) f = f / dzW(z - 1);
    W2(x - 1, y, z) = W2(x - 1, y, z) - f; W2(x - 1, y, z) = W2(x - 1, y, z) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[PLUSX][3]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x + 1, y, z + 1) + nu(x + 1, y, z) + nu(x, y, z + 1) + nu(x, y, z)) * (W(x + 1, y, z) - W(x, y, z)) * rx / 4;
    W2(x + 1, y, z) = W2(x + 1, y, z) + f; W2(x + 1, y, z) = W2(x + 1, y, z) + p.fluxp;
  }
  for (auto &p : d.wm[PLUSX][3]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x + 1, y, z + 1) + nu(x + 1, y, z) + nu(x, y, z + 1) + nu(x, y, z)) * (W(x + 1, y, z) - W(x, y, z)) * rx / 4;
    W2(x, y, z) = W2(x, y, z) - f; W2(x, y, z) = W2(x, y, z) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[MINUSY][3]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x, y, z + 1) + nu(x, y - 1, z + 1) + nu(x, y, z) + nu(x, y - 1, z)) * (W(x, y, z) - W(x, y - 1, z)) * ry / 4;
    W2(x, y, z) = W2(x, y, z) + f; W2(x, y, z) = W2(x, y, z) + p.fluxp;
  }
  for (auto &p : d.wm[MINUSY][3]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x, y, z + 1) + nu(x, y - 1, z + 1) + nu(x, y, z) + nu(x, y - 1, z)) * (W(x, y, z) - W(x, y - 1, z)) * ry / 4;
    W2(x, y - 1, z) = W2(x, y - 1, z) - f; W2(x, y - 1, z) = W2(x, y - 1, z) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[PLUSY][3]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x, y + 1, z + 1) + nu(x, y, z + 1) + nu(x, y + 1, z) + nu(x, y, z)) * (W(x, y + 1, z) - W(x, y, z)) * ry / 4;
    W2(x, y + 1, z) = W2(x, y + 1, z) + f; W2(x, y + 1, z) = W2(x, y + 1, z) + p.fluxp;
  }
  for (auto &p : d.wm[PLUSY][3]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = (nu(x, y + 1, z + 1) + nu(x, y, z + 1) + nu(x, y + 1, z) + nu(x, y, z)) * (W(x, y + 1, z) - W(x, y, z)) * ry / 4;
    W2(x, y, z) = W2(x, y, z) - f; W2(x, y, z) = W2(x, y, z) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[MINUSZ][3]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = vz ? nu(x, y, z) * (W(x, y, z) - W(x, y, z - 1)) / dzPr(z) / dzW(z) : nu(x, y, z) * (W(x, y, z) - W(x, y, z - 1)) * rz;
    W2(x, y, z) = W2(x, y, z) + f; W2(x, y, z) = W2(x, y, z) + p.fluxp;
  }
  for (auto &p : d.wm[MINUSZ][3]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = vz ? nu(x, y, z) * (W(x, y, z) - W(x, y, z - 1)) / dzPr(z) / dzW(z - 1) : nu(x, y, z) * (W(x, y, z) - W(x, y, z - 1)) * rz;
    W2(x, y, z - 1) = W2(x, y, z - 1) - f; W2(x, y, z - 1) = W2(x, y, z - 1) - (vz ? p.fluxm : p.fluxp);
  }
  for (auto &p : d.wm[PLUSZ][3]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = vz ? nu(x, y, z + 1) * (W(x, y, z + 1) - W(x, y, z)) / dzPr(z + 1) / dzW(z + 1) : nu(x, y, z + 1) * (W(x, y, z + 1) - W(x, y, z)) * rz;
    W2(x, y, z + 1) = W2(x, y, z + 1) + f; W2(x, y, z + 1) = W2(x, y, z + 1) + p.fluxp;
  }
  for (auto &p : d.wm[PLUSZ][3]) {
    int x = p.xi, y = p.yj, z = p.zk;
    double f = vz ? nu(x, y, z + 1) * (W(x, y, z + 1) - W(x, y, z)) / dzPr(z + 1) / dzW(z) : nu(x, y, z + 1) * (W(x, y, z + 1) - W(x, y, z)) * rz;
    W2(x, y, z) = W2(x, y, z) - f; W2(x, y, z) = W2(x, y, z) - (vz ? p.fluxm : p.fluxp);
  }
}

// ------------------------------------------------- Convection, dynamics.f90:230-499
static void Convection(Domain &d, int stage, double dt) {
  const double rho = RK_rho[stage - 1], beta = RK_beta[stage - 1];
  if (stage > 1) {
    for (int k = 1; k <= d.Unz; k++) for (int j = 1; j <= d.Uny; j++) for (int i = 1; i <= d.Unx; i++) d.U2(i, j, k) = d.Ustar(i, j, k) * rho * dt;
    for (int k = 1; k <= d.Vnz; k++) for (int j = 1; j <= d.Vny; j++) for (int i = 1; i <= d.Vnx; i++) d.V2(i, j, k) = d.Vstar(i, j, k) * rho * dt;
    for (int k = 1; k <= d.Wnz; k++) for (int j = 1; j <= d.Wny; j++) for (int i = 1; i <= d.Wnx; i++) d.W2(i, j, k) = d.Wstar(i, j, k) * rho * dt;
  } else {
    for (int k = 1; k <= d.Unz; k++) for (int j = 1; j <= d.Uny; j++) for (int i = 1; i <= d.Unx; i++) { d.Ustar(i, j, k) = 0; d.U2(i, j, k) = 0; }
    for (int k = 1; k <= d.Vnz; k++) for (int j = 1; j <= d.Vny; j++) for (int i = 1; i <= d.Vnx; i++) { d.Vstar(i, j, k) = 0; d.V2(i, j, k) = 0; }
    for (int k = 1; k <= d.Wnz; k++) for (int j = 1; j <= d.Wny; j++) for (int i = 1; i <= d.Wnx; i++) { d.Wstar(i, j, k) = 0; d.W2(i, j, k) = 0; }
  }
  // advection_method == 2: CDU/CDV/CDW (dynamics.f90:359-368)
  CDU(d, d.Ustar);
  CDV(d, d.Vstar);
  CDW(d, d.Wstar);
  if (d.enable_buoyancy) BuoyancyForce(d, d.Wstar);  // dynamics.f90:423
  MomentumDiffusion(d, d.Ustar, d.Vstar, d.Wstar);
  for (int k = 1; k <= d.Unz; k++) for (int j = 1; j <= d.Uny; j++) for (int i = 1; i <= d.Unx; i++) d.U2(i, j, k) = d.U2(i, j, k) + d.Ustar(i, j, k) * beta * dt;
  for (int k = 1; k <= d.Vnz; k++) for (int j = 1; j <= d.Vny; j++) for (int i = 1; i <= d.Vnx; i++) d.V2(i, j, k) = d.V2(i, j, k) + d.Vstar(i, j, k) * beta * dt;
  for (int k = 1; k <= d.Wnz; k++) for (int j = 1; j <= d.Wny; j++) for (int i = 1; i <= d.Wnx; i++) d.W2(i, j, k) = d.W2(i, j, k) + d.Wstar(i, j, k) * beta * dt;
}

// ------------------------ OtherTerms, tsteps.f90:263-358; PressureGrad, dynamics.f90:58-199
static void OtherTerms(Domain &d, double coef) {
  const double A = -coef, Ax = -coef / d.dxmin, Ay = -coef / d.dymin, Az = -coef / d.dzmin;
  A3 &Pr = d.Pr;
  if (d.en_prgx)
    for (int k = 1; k <= d.Unz; k++) for (int j = 1; j <= d.Uny; j++) for (int i = 1; i <= d.Unx; i++) d.U2(i, j, k) = d.U2(i, j, k) + A * d.prgx;
  if (d.en_prgy)
    for (int k = 1; k <= d.Vnz; k++) for (int j = 1; j <= d.Vny; j++) for (int i = 1; i <= d.Vnx; i++) d.V2(i, j, k) = d.V2(i, j, k) + A * d.prgy;
  for (int k = 1; k <= d.Unz; k++) for (int j = 1; j <= d.Uny; j++) for (int i = 1; i <= d.Unx; i++) d.U2(i, j, k) = d.U2(i, j, k) + Ax * (Pr(i + 1, j, k) - Pr(i, j, k));
  for (int k = 1; k <= d.Vnz; k++) for (int j = 1; j <= d.Vny; j++) for (int i = 1; i <= d.Vnx; i++) d.V2(i, j, k) = d.V2(i, j, k) + Ay * (Pr(i, j + 1, k) - Pr(i, j, k));
  if (d.gridtype == 1) {
    for (int k = 1; k <= d.Wnz; k++) for (int j = 1; j <= d.Wny; j++) for (int i = 1; i <= d.Wnx; i++) d.W2(i, j, k) = d.W2(i, j, k) - coef * (Pr(i, j, k + 1) - Pr(i, j, k)) / d.dzW(k);
  } else {
    for (int k = 1; k <= d.Wnz; k++) for (int j = 1; j <= d.Wny; j++) for (int i = 1; i <= d.Wnx; i++) d.W2(i, j, k) = d.W2(i, j, k) + Az * (Pr(i, j, k + 1) - Pr(i, j, k));
  }
  // explicit_diffusion: add(U2, U) over the whole arrays (tsteps.f90:352-354)
  for (size_t n = 0; n < d.U2.v.size(); n++) d.U2.v[n] = d.U2.v[n] + d.U.v[n];
  for (size_t n = 0; n < d.V2.v.size(); n++) d.V2.v[n] = d.V2.v[n] + d.V.v[n];
  for (size_t n = 0; n < d.W2.v.size(); n++) d.W2.v[n] = d.W2.v[n] + d.W.v[n];
}

// ---------------------------------------------------------------- Poisson
// Exact FP64 solve of the operator of Residue_variable_z (poisson.f90:23-60):
// FFT in x and y, then for each (kx,ky) a tridiagonal system in z.
static bool init_poisson(Domain &d) {
  int nx = d.Prnx, ny = d.Prny, nz = d.Prnz;
  if (d.PrBtype[We] != BC_PERIODIC || d.PrBtype[So] != BC_PERIODIC) return false;
  if (!d.px.init(nx) || !d.py.init(ny)) return false;
  d.nxh = nx / 2 + 1;
  double rx = 1 / (d.dxmin * d.dxmin), ry = 1 / (d.dymin * d.dymin);
  d.lamx.resize(nx); d.lamy.resize(ny);
  for (int m = 0; m < nx; m++) { double s = std::sin(M_PI * m / nx); d.lamx[m] = -4.0 * s * s * rx; }
  for (int m = 0; m < ny; m++) { double s = std::sin(M_PI * m / ny); d.lamy[m] = -4.0 * s * s * ry; }
  d.zper = d.PrBtype[Bo] == BC_PERIODIC;
  d.Ab.assign(nz + 2, 0.0); d.At.assign(nz + 2, 0.0); d.dzc.assign(nz + 2, 0.0); d.dzf.assign(nz + 2, 0.0);
  for (int k = 1; k <= nz; k++) {
    d.Ab[k] = 1 / ((d.zPr(k) - d.zPr(k - 1)) * (d.zW(k) - d.zW(k - 1)));
    d.At[k] = 1 / ((d.zPr(k + 1) - d.zPr(k)) * (d.zW(k) - d.zW(k - 1)));
    d.dzc[k] = d.zW(k) - d.zW(k - 1);      // cell height
    d.dzf[k] = d.zPr(k + 1) - d.zPr(k);    // distance of centres k, k+1
  }
  if (!d.zper) { d.Ab[1] = 0; d.At[nz] = 0; }
  return true;
}

// Solves (Lz + lam) x = r for one column; lam == 0 with Neumann z is the
// singular mode, solved by two prefix sums and pinned to zero mean.
static void tridiag(const Domain &d, double lam, bool zero_mode, const cd *r, cd *x, std::vector<cd> &cp_) {
  int nz = d.Prnz;
  const std::vector<double> &Ab = d.Ab, &At = d.At;
  if (zero_mode && !d.zper) {
    cd F = 0;
    x[0] = 0;
    for (int k = 1; k <= nz - 1; k++) {
      F = F + r[k - 1] * d.dzc[k];
      x[k] = x[k - 1] + F * d.dzf[k];
    }
    cd s = 0;
    for (int k = 0; k < nz; k++) s += x[k];
    s = s / (double)nz;
    for (int k = 0; k < nz; k++) x[k] -= s;
    return;
  }
  if (zero_mode && d.zper) {
    // periodic singular mode: fluxes F(k) = F(0) + sum dzc r, with F(0) chosen
    // so that sum_k dzf(k) F(k) = 0 (periodicity of x).
    std::vector<cd> F(nz + 1);
    F[0] = 0;
    for (int k = 1; k <= nz; k++) F[k] = F[k - 1] + r[k - 1] * d.dzc[k];
    cd sw = 0; double sd = 0;
    for (int k = 1; k <= nz; k++) { sw += F[k] * d.dzf[k]; sd += d.dzf[k]; }
    cd F0 = -sw / sd;
    x[0] = 0;
    for (int k = 1; k <= nz - 1; k++) x[k] = x[k - 1] + (F[k] + F0) * d.dzf[k];
    cd s = 0;
    for (int k = 0; k < nz; k++) s += x[k];
    s = s / (double)nz;
    for (int k = 0; k < nz; k++) x[k] -= s;
    return;
  }
  std::vector<double> cp(nz);
  if (!d.zper) {
    // Thomas algorithm, rows k=1..nz: Ab(k) x(k-1) + (-(Ab+At)+lam) x(k) + At(k) x(k+1)
    double b = -(Ab[1] + At[1]) + lam;
    cp[0] = At[1] / b;
    x[0] = r[0] / b;
    for (int k = 2; k <= nz; k++) {
      double den = (-(Ab[k] + At[k]) + lam) - Ab[k] * cp[k - 2];
      cp[k - 1] = At[k] / den;
      x[k - 1] = (r[k - 1] - Ab[k] * x[k - 2]) / den;
    }
    for (int k = nz - 1; k >= 1; k--) x[k - 1] = x[k - 1] - cp[k - 1] * x[k];
  } else {
    // cyclic system by Sherman-Morrison
    std::vector<double> a(nz), b(nz), c(nz);
    for (int k = 1; k <= nz; k++) { a[k - 1] = Ab[k]; c[k - 1] = At[k]; b[k - 1] = -(Ab[k] + At[k]) + lam; }
    double alpha = c[nz - 1], beta = a[0];
    double gamma = -b[0];
    std::vector<double> bb(b);
    bb[0] = b[0] - gamma;
    bb[nz - 1] = b[nz - 1] - alpha * beta / gamma;
    std::vector<cd> y(nz);
    std::vector<double> u(nz, 0.0), z(nz);
    u[0] = gamma; u[nz - 1] = alpha;
    // solve bb-system for r -> y and for u -> z
    std::vector<double> c2(nz);
    double den = bb[0];
    c2[0] = c[0] / den; y[0] = r[0] / den; z[0] = u[0] / den;
    for (int k = 1; k < nz; k++) {
      den = bb[k] - a[k] * c2[k - 1];
      c2[k] = c[k] / den;
      y[k] = (r[k] - a[k] * y[k - 1]) / den;
      z[k] = (u[k] - a[k] * z[k - 1]) / den;
    }
    for (int k = nz - 2; k >= 0; k--) { y[k] = y[k] - c2[k] * y[k + 1]; z[k] = z[k] - c2[k] * z[k + 1]; }
    cd fac = (y[0] + beta * y[nz - 1] / gamma) / (1.0 + z[0] + beta * z[nz - 1] / gamma);
    for (int k = 0; k < nz; k++) x[k] = y[k] - fac * z[k];
  }
  (void)cp_;
}

static void poisson_solve(Domain &d) {
  int nx = d.Prnx, ny = d.Prny, nz = d.Prnz, nxh = d.nxh;
  // S[k][ky][kx]
  std::vector<cd> S((size_t)nz * ny * nxh);
  const double norm = 1.0 / ((double)nx * ny);
#pragma omp parallel
  {
    std::vector<cd> a(nx), b(nx), t(std::max(nx, std::max(ny, nz))), c(ny), e(ny), rz(nz), xz(nz);
    std::vector<cd> cp;
#pragma omp for collapse(2)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++) {
        for (int i = 1; i <= nx; i++) a[i - 1] = d.RHS(i, j, k);
        d.px.forward(a.data(), b.data());
        for (int m = 0; m < nxh; m++) S[((size_t)(k - 1) * ny + (j - 1)) * nxh + m] = b[m];
      }
#pragma omp for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int m = 0; m < nxh; m++) {
        for (int j = 0; j < ny; j++) c[j] = S[((size_t)k * ny + j) * nxh + m];
        d.py.forward(c.data(), e.data());
        for (int j = 0; j < ny; j++) S[((size_t)k * ny + j) * nxh + m] = e[j];
      }
#pragma omp for collapse(2)
    for (int j = 0; j < ny; j++)
      for (int m = 0; m < nxh; m++) {
        for (int k = 0; k < nz; k++) rz[k] = S[((size_t)k * ny + j) * nxh + m] * norm;
        double lam = d.lamx[m] + d.lamy[j];
        tridiag(d, lam, m == 0 && j == 0, rz.data(), xz.data(), cp);
        for (int k = 0; k < nz; k++) S[((size_t)k * ny + j) * nxh + m] = xz[k];
      }
#pragma omp for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int m = 0; m < nxh; m++) {
        for (int j = 0; j < ny; j++) c[j] = S[((size_t)k * ny + j) * nxh + m];
        d.py.inverse(c.data(), e.data(), t);
        for (int j = 0; j < ny; j++) S[((size_t)k * ny + j) * nxh + m] = e[j];
      }
#pragma omp for collapse(2)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++) {
        const cd *row = &S[((size_t)(k - 1) * ny + (j - 1)) * nxh];
        for (int m = 0; m < nxh; m++) a[m] = row[m];
        for (int m = nxh; m < nx; m++) a[m] = std::conj(row[nx - m]);
        d.px.inverse(a.data(), b.data(), t);
        for (int i = 1; i <= nx; i++) d.Phi(i, j, k) = b[i - 1].real();
      }
  }
}

// ------------------------------------------ PressureCorrection, pressure.f90:169-266
// ------------------------------------------- immersed solids, tsteps.f90:360-567
// IBMomentum: every value interpolated first, then all assigned (:360-409)
static void IBMomentum(Domain &d, A3 &U, A3 &V, A3 &W) {
  A3 *F[4] = {nullptr, &U, &V, &W};
  for (int c = 1; c <= 3; c++) {
    std::vector<double> wm(d.ibp[c].size());
    for (size_t i = 0; i < wm.size(); i++) wm[i] = IBInterpolate(d.ibp[c][i], *F[c]);
    for (size_t i = 0; i < wm.size(); i++) (*F[c])(d.ibp[c][i].xi, d.ibp[c][i].yj, d.ibp[c][i].zk) = wm[i];
  }
}

// IBMassSources, second-order branch (:415-533); Bound_Q fills ghosts that
// the right-hand side does not read
static void IBMassSources(Domain &d, const A3 &U, const A3 &V, const A3 &W) {
  d.Q.fill(0);
  for (auto &p : d.ibp[1]) {
    d.Q(p.xi, p.yj, p.zk) = d.Q(p.xi, p.yj, p.zk) + U(p.xi, p.yj, p.zk) / d.dxPr(p.xi);
    d.Q(p.xi + 1, p.yj, p.zk) = d.Q(p.xi + 1, p.yj, p.zk) - U(p.xi, p.yj, p.zk) / d.dxPr(p.xi + 1);
  }
  for (auto &p : d.ibp[2]) {
    d.Q(p.xi, p.yj, p.zk) = d.Q(p.xi, p.yj, p.zk) + V(p.xi, p.yj, p.zk) / d.dyPr(p.yj);
    d.Q(p.xi, p.yj + 1, p.zk) = d.Q(p.xi, p.yj + 1, p.zk) - V(p.xi, p.yj, p.zk) / d.dyPr(p.yj + 1);
  }
  for (auto &p : d.ibp[3]) {
    d.Q(p.xi, p.yj, p.zk) = d.Q(p.xi, p.yj, p.zk) + W(p.xi, p.yj, p.zk) / d.dzPr(p.zk);
    d.Q(p.xi, p.yj, p.zk + 1) = d.Q(p.xi, p.yj, p.zk + 1) - W(p.xi, p.yj, p.zk) / d.dzPr(p.zk + 1);
  }
}

// NullInterior (:540-567)
static void NullInterior(Domain &d, A3 &U, A3 &V, A3 &W) {
  A3 *F[4] = {nullptr, &U, &V, &W};
  for (int c = 1; c <= 3; c++)
    for (auto &q : d.nullp[c]) (*F[c])(q[0], q[1], q[2]) = 0;
}

static void PressureCorrection(Domain &d, double coef, bool check_div, bool with_q = false) {
  A3 &U = d.U2, &V = d.V2, &W = d.W2;
  const double dt2 = coef;
  // PrePoisson (pressure.f90:272-723): ghosts, then RHS = (div U - Q) / dt2;
  // Q is the IB mass source inside TMarchRK3 and absent in the initial
  // projection (a local, unallocated Q in InitialConditions, initial.f90:3829)
  BoundUVW(d, U, V, W);
  const double dt2_rec = 1.0 / dt2;
#pragma omp parallel for collapse(2)
  for (int k = 1; k <= d.Prnz; k++)
    for (int j = 1; j <= d.Prny; j++)
      for (int i = 1; i <= d.Prnx; i++) {
        double r;
        if (d.gridtype == 1)
          r = (U(i, j, k) - U(i - 1, j, k)) / d.dxmin + (V(i, j, k) - V(i, j - 1, k)) / d.dymin + (W(i, j, k) - W(i, j, k - 1)) / d.dzPr(k) - (with_q ? d.Q(i, j, k) : 0.0);
        else
          r = (U(i, j, k) - U(i - 1, j, k)) / d.dxmin + (V(i, j, k) - V(i, j - 1, k)) / d.dymin + (W(i, j, k) - W(i, j, k - 1)) / d.dzmin - (with_q ? d.Q(i, j, k) : 0.0);
        d.RHS(i, j, k) = r * dt2_rec;
      }
  poisson_solve(d);
  Bound_Phi(d, d.Phi);
  // PostPoisson (pressure.f90:728-991)
  const double Au = dt2 / d.dxmin, Av = dt2 / d.dymin, Aw = dt2 / d.dzmin;
  A3 &Phi = d.Phi;
  for (int k = 1; k <= d.Unz; k++) for (int j = 1; j <= d.Uny; j++) for (int i = 1; i <= d.Unx; i++) U(i, j, k) = U(i, j, k) - Au * (Phi(i + 1, j, k) - Phi(i, j, k));
  for (int k = 1; k <= d.Vnz; k++) for (int j = 1; j <= d.Vny; j++) for (int i = 1; i <= d.Vnx; i++) V(i, j, k) = V(i, j, k) - Av * (Phi(i, j + 1, k) - Phi(i, j, k));
  if (d.gridtype == 1) {
    for (int k = 1; k <= d.Wnz; k++) for (int j = 1; j <= d.Wny; j++) for (int i = 1; i <= d.Wnx; i++) W(i, j, k) = W(i, j, k) - dt2 * (Phi(i, j, k + 1) - Phi(i, j, k)) / d.dzW(k);
  } else {
    for (int k = 1; k <= d.Wnz; k++) for (int j = 1; j <= d.Wny; j++) for (int i = 1; i <= d.Wnx; i++) W(i, j, k) = W(i, j, k) - Aw * (Phi(i, j, k + 1) - Phi(i, j, k));
  }
  A3 &Pr = d.Pr;
  for (int k = 1; k <= d.Prnz; k++) for (int j = 1; j <= d.Prny; j++) for (int i = 1; i <= d.Prnx; i++) Pr(i, j, k) = Pr(i, j, k) + Phi(i, j, k);
  // FixPressureToReference, PRESSURE_REFERENCE_BOUNDARY at To (pressure.f90:1160-1220)
  double Phi_ref = 0;
  for (int j = 1; j <= d.Prny; j++) for (int i = 1; i <= d.Prnx; i++) Phi_ref = Phi_ref + Pr(i, j, d.Prnz);
  Phi_ref = Phi_ref / (d.Prnx * d.Prny);
  if (Phi_ref != 0)
    for (int k = 1; k <= d.Prnz; k++) for (int j = 1; j <= d.Prny; j++) for (int i = 1; i <= d.Prnx; i++) Pr(i, j, k) = Pr(i, j, k) - Phi_ref;
  Bound_Pr(d, Pr);
  if (check_div) {  // pressure.f90:884-989, after BoundUVW
    BoundUVW(d, U, V, W);
    double S = 0;
    for (int k = 1; k <= d.Prnz; k++)
      for (int j = 1; j <= d.Prny; j++)
        for (int i = 1; i <= d.Prnx; i++) {
          double dzk = d.gridtype == 1 ? d.dzPr(k) : d.dzmin;
          double p = (U(i, j, k) - U(i - 1, j, k)) / d.dxmin + (V(i, j, k) - V(i, j - 1, k)) / d.dymin + (W(i, j, k) - W(i, j, k - 1)) / dzk - (with_q ? d.Q(i, j, k) : 0.0);
          S = std::max(S, std::fabs(p));
        }
    d.max_div = S;
  }
}

// ---------------------------------------------- TimeStepLength, dynamics.f90:511-600
static void TimeStepLength(Domain &d) {
  if (!d.enable_CFL_check && !d.variable_time_steps) { d.CFL = 0; return; }
  double U_dx_max = 0;
  bool nan = false;
  for (int k = 1; k <= d.Prnz; k++)
    for (int j = 1; j <= d.Prny; j++)
      for (int i = 1; i <= d.Prnx; i++) {
        double dx = d.gridtype == 1 ? d.dxPr(i) : d.dxmin;
        double dy = d.gridtype == 1 ? d.dyPr(j) : d.dymin;
        double dz = d.gridtype == 1 ? d.dzPr(k) : d.dzmin;
        double p = std::max(std::fabs(d.U(i, j, k)), std::fabs(d.U(i - 1, j, k))) / dx;
        p = p + std::max(std::fabs(d.V(i, j, k)), std::fabs(d.V(i, j - 1, k))) / dy;
        p = p + std::max(std::fabs(d.W(i, j, k)), std::fabs(d.W(i, j, k - 1))) / dz;
        U_dx_max = std::max(U_dx_max, p);
        if (p != p) nan = true;
      }
  if (d.variable_time_steps) {  // dynamics.f90:517-529
    if (nan) d.dt = std::numeric_limits<double>::min();
    else if (U_dx_max > 0) d.dt = std::min(d.CFL_target / U_dx_max, d.dt_max);
    else d.dt = d.dt_max;
    // the step that would pass end_time ends there (dynamics.f90:547-548)
    if (d.end_time > 0 && d.end_time - d.time > 1e-12 * d.end_time && d.dt + d.time > d.end_time)
      d.dt = d.end_time - d.time;
    d.CFL = U_dx_max * d.dt;
    return;
  }
  d.CFL = U_dx_max * d.dt;
}

// one RK3 stage of TMarchRK3 (tsteps.f90:111-241) up to a stop point
static void run_stage(Domain &d, int stage, int stop) {
  const double dt = d.dt;
  SubgridStresses(d);
  if (stop == 1) return;
  Convection(d, stage, dt);
  if (d.enable_buoyancy || d.num_scalars > 0) ScalarRK3(d, stage, dt);  // tsteps.f90:132-135
  OtherTerms(d, 2 * RK_alpha[stage - 1] * dt);
  BoundUVW(d, d.U2, d.V2, d.W2);
  if (d.solids) {  // tsteps.f90:146-152
    IBMomentum(d, d.U2, d.V2, d.W2);
    BoundUVW(d, d.U2, d.V2, d.W2);
    IBMassSources(d, d.U2, d.V2, d.W2);
  }
  if (stop == 2) return;
  PressureCorrection(d, 2 * RK_alpha[stage - 1] * dt, true, d.solids);
  std::swap(d.U.v, d.U2.v);
  std::swap(d.V.v, d.V2.v);
  std::swap(d.W.v, d.W2.v);
  if (d.solids) {  // tsteps.f90:201-206
    NullInterior(d, d.U, d.V, d.W);
    BoundUVW(d, d.U, d.V, d.W);
    IBMomentum(d, d.U, d.V, d.W);
  }
  BoundUVW(d, d.U, d.V, d.W);
}

static void TMarchRK3(Domain &d) {
  BoundUVW(d, d.U, d.V, d.W);
  // first call: IBMomentum after the ghosts, which keep their values until
  // the end of the first stage (tsteps.f90:31-54)
  if (d.called == 0 && d.solids) IBMomentum(d, d.U, d.V, d.W);
  d.called = 1;
  TimeStepLength(d);
  for (int s = 1; s <= 3; s++) run_stage(d, s, 3);
  d.time += d.dt;
  AccumulateScalarAverages(d);
}

// InDomain (boundaries.f90:163-168) and GridCoords_scalar
// (boundaries.f90:54-97): the cell of a point; nint rounds half away from 0
static bool GridCoords(const Domain &d, const double *r, int *ip) {
  const int nx = d.Prnx, ny = d.Prny, nz = d.Prnz;
  if (!((r[0] >= d.xU(0) && r[0] <= d.xU(nx)) && (r[1] >= d.yV(0) && r[1] <= d.yV(ny)) &&
        (r[2] >= d.zW(0) && r[2] <= d.zW(nz))))
    return false;
  if (d.gridtype == 0) {
    ip[0] = std::min(std::max((int)std::lround((r[0] - d.xU(0)) / d.dxmin + 0.5), 1), nx);
    ip[1] = std::min(std::max((int)std::lround((r[1] - d.yV(0)) / d.dymin + 0.5), 1), ny);
    ip[2] = std::min(std::max((int)std::lround((r[2] - d.zW(0)) / d.dzmin + 0.5), 1), nz);
  } else {
    ip[0] = nx; ip[1] = ny; ip[2] = nz;
    for (int i = 1; i <= nx; i++) if (d.xU(i) >= r[0]) { ip[0] = i; break; }
    for (int j = 1; j <= ny; j++) if (d.yV(j) >= r[1]) { ip[1] = j; break; }
    for (int k = 1; k <= nz; k++) if (d.zW(k) >= r[2]) { ip[2] = k; break; }
  }
  return true;
}

// the end of InitialConditions after the projection (initial.f90:4290-4320):
// eddy viscosity, its ghosts and, with any scalar, the diffusivity
static void InitialDiffusivity(Domain &d) {
  SubgridModel(d);
  BoundViscosity(d, d.Viscosity);
  if (d.enable_buoyancy || d.num_scalars > 0) {
    const double Pr_sgs = 0.6;  // constPr_sgs, scalar_diffusion.f90:22
    for (int k = 1; k <= d.Prnz; k++)
      for (int j = 1; j <= d.Prny; j++)
        for (int i = 1; i <= d.Prnx; i++)
          d.TDiff(i, j, k) = (d.Viscosity(i, j, k) - d.molecular_viscosity) / Pr_sgs + d.molecular_diffusivity;
    BoundViscosity(d, d.TDiff);
  }
  if (d.enable_buoyancy) BoundTemperature(d, d.T);
  // the wall model once on the initial fields (initial.f90:4331-4336): the
  // points' u* and surface fluxes, from which the first stage starts
  if (d.wallmodeltype > 0) {
    ComputeViscsWM(d);
    ComputeUVWFluxesWM(d);
  }
}

}  // namespace orc

// ================================================================ C API
using namespace orc;

extern "C" {

struct orc_domain;

static int sides_ok(const int *b) {
  for (int s = 0; s < 6; s++)
    if (b[s] != BC_NOSLIP && b[s] != BC_FREESLIP && b[s] != BC_PERIODIC && b[s] != BC_NEUMANN) return 0;
  for (int a = 0; a < 3; a++)
    if ((b[2 * a] == BC_PERIODIC) != (b[2 * a + 1] == BC_PERIODIC)) return 0;
  return 1;
}

void *orc_create(const elmm_config *c) {
  if (!c || c->Prnx < 4 || c->Prny < 4 || c->Prnz < 4 || !sides_ok(c->Btype)) return nullptr;
  Domain *d = new Domain();
  d->Prnx = c->Prnx; d->Prny = c->Prny; d->Prnz = c->Prnz;
  for (int s = 0; s < 6; s++) d->Btype[s + 1] = c->Btype[s];
  // PrBtype from Btype, initial.f90:817-826
  for (int s = 1; s <= 6; s++) d->PrBtype[s] = d->Btype[s] == BC_PERIODIC ? BC_PERIODIC : BC_NEUMANN;
  d->Unx = d->Btype[Ea] == BC_PERIODIC ? d->Prnx : d->Prnx - 1; d->Uny = d->Prny; d->Unz = d->Prnz;
  d->Vnx = d->Prnx; d->Vny = d->Btype[No] == BC_PERIODIC ? d->Prny : d->Prny - 1; d->Vnz = d->Prnz;
  d->Wnx = d->Prnx; d->Wny = d->Prny; d->Wnz = d->Btype[To] == BC_PERIODIC ? d->Prnz : d->Prnz - 1;
  d->gridtype = c->zW ? 1 : 0;
  d->dxmin = c->dxmin; d->dymin = c->dymin; d->dzmin = c->dzmin;
  d->molecular_viscosity = c->molecular_viscosity;
  d->C_Smagorinsky = c->C_Smagorinsky;
  d->filter_ratio = c->filter_ratio;
  d->sgstype = c->sgstype;
  d->wallmodeltype = c->wallmodeltype;
  for (int s = 0; s < 6; s++) d->z0s[s + 1] = c->z0[s];
  d->en_prgx = c->enable_pr_gradient_x_uniform; d->en_prgy = c->enable_pr_gradient_y_uniform;
  d->prgx = c->pr_gradient_x; d->prgy = c->pr_gradient_y;
  d->dt = c->dt; d->time = 0;
  d->enable_CFL_check = c->enable_CFL_check; d->CFL = 0; d->max_div = 0;
  d->variable_time_steps = c->variable_time_steps;
  d->CFL_target = c->CFL; d->dt_max = c->dt_max; d->end_time = c->end_time; d->dt0 = c->dt;
  init_grid(*d, *c);
  int nx = d->Prnx, ny = d->Prny, nz = d->Prnz;
  for (A3 *a : {&d->U, &d->U2, &d->Ustar}) a->init(-2, d->Unx + 3, -2, d->Uny + 3, -2, d->Unz + 3);
  for (A3 *a : {&d->V, &d->V2, &d->Vstar}) a->init(-2, d->Vnx + 3, -2, d->Vny + 3, -2, d->Vnz + 3);
  for (A3 *a : {&d->W, &d->W2, &d->Wstar}) a->init(-2, d->Wnx + 3, -2, d->Wny + 3, -2, d->Wnz + 3);
  for (A3 *a : {&d->Pr, &d->Viscosity, &d->Phi}) a->init(-1, nx + 2, -1, ny + 2, -1, nz + 2);
  d->RHS.init(0, nx + 1, 0, ny + 1, 0, nz + 1);
  d->Viscosity.fill(d->molecular_viscosity);
  d->enable_buoyancy = c->enable_buoyancy;
  for (int s = 0; s < 6; s++) { d->TempBtype[s + 1] = c->TempBtype[s]; d->sideTemp[s + 1] = c->sideTemp[s]; }
  d->temperature_ref = c->temperature_ref;
  d->grav_acc = c->grav_acc;
  d->molecular_diffusivity = c->molecular_diffusivity;
  if (c->num_scalars < 0 || c->num_scalars > ELMM_MAX_SCALARS) { delete d; return nullptr; }
  d->num_scalars = c->num_scalars;
  for (int s = 0; s < 6; s++) { d->ScalBtype[s + 1] = c->ScalBtype[s]; d->sideScal[s + 1] = c->sideScal[s]; }
  if (d->enable_buoyancy) {
    for (A3 *a : {&d->T, &d->Tadv, &d->T2}) a->init(-2, nx + 3, -2, ny + 3, -2, nz + 3);
  }
  for (int sc = 0; sc < d->num_scalars; sc++)
    for (A3 *a : {&d->S[sc], &d->Sadv[sc], &d->S2[sc]}) a->init(-2, nx + 3, -2, ny + 3, -2, nz + 3);
  if (d->enable_buoyancy || d->num_scalars > 0) {
    d->TDiff.init(-1, nx + 2, -1, ny + 2, -1, nz + 2);
    if (d->molecular_viscosity > 0) d->TDiff.fill(d->molecular_diffusivity);  // initial.f90:4262-4268
  }
  // point sources -> single-cell volume sources (pointsources.f90:24-39,
  // InitPointSources :41-60)
  if (c->num_point_sources < 0 || c->num_point_sources > ELMM_MAX_POINT_SOURCES) { delete d; return nullptr; }
  for (int q = 0; q < c->num_point_sources; q++) {
    const elmm_point_source &ps = c->point_sources[q];
    if (ps.scalar_number < 1 || ps.scalar_number > d->num_scalars) { delete d; return nullptr; }
    int ip[3];
    if (!GridCoords(*d, ps.position, ip)) continue;
    const double vol = d->dxPr(ip[0]) * d->dyPr(ip[1]) * d->dzPr(ip[2]);
    d->flvolumes.push_back({ps.scalar_number, ip[0], ip[1], ip[2], ps.flux / vol});
  }
  d->avg_k = c->avg_slice_k;
  d->avg_j = c->avg_slice_j;
  d->avg_w = c->avg_weight;
  if (d->avg_k < 0 || d->avg_k > nz || d->avg_j < 0 || d->avg_j > ny) { delete d; return nullptr; }
  for (int sc = 0; sc < d->num_scalars; sc++) {
    d->acc_xy[sc].assign((size_t)nx * ny, 0.0);
    d->acc_xz[sc].assign((size_t)nx * nz, 0.0);
  }
  if (d->wallmodeltype > 0) {
    // GetOutsideBoundariesWM_UVW / _Pr (wallmodels.f90:570-627, 819-827):
    // a constant temperature flux at a wall becomes the flux of its
    // wall-model points, and the side's TempBtype becomes 0 (the mirror
    // ghosts of CommonBase's last branch)
    for (int side : {Bo, To}) {
      if (d->Btype[side] != BC_NOSLIP) continue;
      if (d->TempBtype[side] == ELMM_BC_CONSTFLUX) {
        d->wm_tflux[side] = side == Bo ? d->sideTemp[side] : -d->sideTemp[side];
        d->TempBtype[side] = 0;
      } else if (d->TempBtype[side] == ELMM_BC_DIRICHLET) {
        const int k = side == Bo ? 1 : nz;
        for (int j = 1; j <= ny; j++)
          for (int i = 1; i <= nx; i++) {
            WMPointPr p;
            p.xi = i; p.yj = j; p.zk = k;
            p.distz = side == Bo ? d->zW(0) - d->zPr(1) : d->zW(d->Wnz + 1) - d->zPr(nz);
            p.z0 = d->z0s[side];
            p.temperature = d->sideTemp[side];
            d->wmpr[side].push_back(p);
          }
        d->TempBtype[side] = 0;
      }
    }
    // ComputeAreaFactor of a point below or above its cell: out_norm = e_z
    const double dq = std::sqrt(d->dxmin * d->dymin), l = dq / 1.0;
    d->area_factor_z = dq * l / (d->dxmin * d->dymin * d->dzmin);
    add_wm_points(*d);
  }
  if (!init_poisson(*d)) { delete d; return nullptr; }
  return d;
}

void orc_destroy(void *h) { delete (Domain *)h; }

// Puff sources in the layout of elmm_set_puffs; PuffSource%last_start starts
// at -huge (puffs.f90:16)
int orc_set_puffs(void *h, const elmm_puff *pf, int np, const elmm_puff_volume *vol, int nv) {
  Domain &d = *(Domain *)h;
  d.puffs.clear();
  d.puffvols.clear();
  for (int q = 0; q < np; q++)
    d.puffs.push_back({pf[q].start_time, pf[q].end_time, pf[q].period, pf[q].duration, pf[q].clear != 0,
                       -std::numeric_limits<double>::max(), false, 0.0});
  for (int q = 0; q < nv; q++) {
    if (vol[q].puff < 0 || vol[q].puff >= np) return 1;
    d.puffvols.push_back({vol[q].puff, vol[q].scalar_number, vol[q].xi, vol[q].yj, vol[q].zk, vol[q].flux});
  }
  return 0;
}

// The solid bodies of GetSolidBodiesBC / SetNullifiedPoints as lists (the
// layout of elmm_solids): IB points, nullified points, ScalFl points, the
// solid-face wall-model points appended to the lists of
// GetOutsideBoundariesWM_UVW, and the bottom-wall points that list leaves
// out next to and under the bodies (wallmodels.f90:700-820).
int orc_set_solids(void *h, const elmm_solids *s) {
  Domain &d = *(Domain *)h;
  for (int c = 1; c <= 3; c++) { d.ibp[c].clear(); d.nullp[c].clear(); }
  d.scalfl.clear();
  d.solids = false;
  d.called = 0;
  d.scal_solids = false;
  d.wmprs.clear();
  if (!s) return 0;
  if (d.num_scalars > 0 || d.enable_buoyancy) {
    const int nx = d.Prnx, ny = d.Prny, nz = d.Prnz;
    d.Prsolid.init(-1, nx + 2, -1, ny + 2, -1, nz + 2);
    for (int64_t q = 0; q < s->n_solid_pr; q++) {
      const int32_t *t = s->solid_pr_ijk + 3 * q;
      for (int oi : {-nx, 0, nx})
        for (int oj : {-ny, 0, ny}) {
          const int i = t[0] + oi, j = t[1] + oj;
          if (i >= -1 && i <= nx + 2 && j >= -1 && j <= ny + 2) d.Prsolid(i, j, t[2]) = 1;
        }
    }
    for (int64_t q = 0; q < s->n_wm_pr; q++) {
      const int32_t *t = s->wm_pr_ijk + 3 * q;
      d.wmprs.push_back({t[0], t[1], t[2]});
    }
    d.HeatQ.init(1, nx, 1, ny, 1, nz);
    d.WallPt.init(1, nx, 1, ny, 1, nz);
    for (int64_t q = 0; q < s->n_wall_pr; q++) {
      const int32_t *t = s->wall_pr_ijk + 3 * q;
      d.WallPt(t[0], t[1], t[2]) = 1;
    }
    for (int64_t q = 0; q < s->n_heat_pr; q++) {
      const int32_t *t = s->heat_pr_ijk + 3 * q;
      d.HeatQ(t[0], t[1], t[2]) = s->heat_pr_q[q];
    }
    d.scal_solids = true;
  }
  for (int c = 1; c <= 3; c++) {
    if (s->n_ib[c - 1] > 0) d.ibp[c].assign(s->ib[c - 1], s->ib[c - 1] + s->n_ib[c - 1]);
    for (int64_t q = 0; q < s->n_null[c - 1]; q++) {
      const int32_t *t = s->null_ijk[c - 1] + 3 * q;
      d.nullp[c].push_back({t[0], t[1], t[2]});
    }
    if (s->n_bottom_skip[c - 1] > 0) {
      std::vector<char> skip;
      const int nx = c == 1 ? d.Unx : c == 2 ? d.Vnx : d.Wnx, ny = c == 1 ? d.Uny : c == 2 ? d.Vny : d.Wny;
      skip.assign((size_t)(nx + 2) * (ny + 2), 0);
      for (int64_t q = 0; q < s->n_bottom_skip[c - 1]; q++) {
        const int32_t *t = s->bottom_skip_ij[c - 1] + 2 * q;
        skip[(size_t)t[0] + (size_t)(nx + 2) * t[1]] = 1;
      }
      auto &pts = d.wm[MINUSZ][c];
      std::vector<WMPointUVW> keep;
      for (auto &p : pts)
        if (!(p.zk == 1 && skip[(size_t)p.xi + (size_t)(nx + 2) * p.yj])) keep.push_back(p);
      pts.swap(keep);
    }
  }
  if (s->n_scalfl > 0) d.scalfl.assign(s->scalfl, s->scalfl + s->n_scalfl);
  for (int64_t q = 0; q < s->n_wm; q++) {
    const elmm_wm_point &w = s->wm[q];
    if (w.component < 1 || w.component > 3 || w.direction < 1 || w.direction > 6) return 1;
    WMPointUVW p;
    p.xi = w.xi; p.yj = w.yj; p.zk = w.zk;
    p.distx = w.dist[0]; p.disty = w.dist[1]; p.distz = w.dist[2];
    p.z0 = w.z0;
    p.temperature_flux = w.temperature_flux;
    d.wm[w.direction][w.component].push_back(p);
  }
  d.Q.init(0, d.Prnx + 1, 0, d.Prny + 1, 0, d.Prnz + 1);
  d.solids = true;
  return 0;
}

int orc_sizes(void *h, int32_t *out12) {
  Domain *d = (Domain *)h;
  int v[12] = {d->Prnx, d->Prny, d->Prnz, d->Unx, d->Uny, d->Unz, d->Vnx, d->Vny, d->Vnz, d->Wnx, d->Wny, d->Wnz};
  for (int i = 0; i < 12; i++) out12[i] = v[i];
  return 0;
}

static A3 *field_of(Domain *d, int f) {
  switch (f) {
    case ELMM_FIELD_U: return &d->U;
    case ELMM_FIELD_V: return &d->V;
    case ELMM_FIELD_W: return &d->W;
    case ELMM_FIELD_PR: return &d->Pr;
    case ELMM_FIELD_VISCOSITY: return &d->Viscosity;
    case ELMM_FIELD_U2: return &d->U2;
    case ELMM_FIELD_V2: return &d->V2;
    case ELMM_FIELD_W2: return &d->W2;
    case ELMM_FIELD_USTAR: return &d->Ustar;
    case ELMM_FIELD_VSTAR: return &d->Vstar;
    case ELMM_FIELD_WSTAR: return &d->Wstar;
    case ELMM_FIELD_PHI: return &d->Phi;
    case ELMM_FIELD_TEMPERATURE: return d->enable_buoyancy ? &d->T : nullptr;
    case ELMM_FIELD_TDIFF: return d->enable_buoyancy || d->num_scalars > 0 ? &d->TDiff : nullptr;
    case ELMM_FIELD_TEMPERATURE_ADV: return d->enable_buoyancy ? &d->Tadv : nullptr;
  }
  if (f >= ELMM_FIELD_SCALAR && f < ELMM_FIELD_SCALAR + d->num_scalars) return &d->S[f - ELMM_FIELD_SCALAR];
  if (f >= ELMM_FIELD_SCALAR_ADV && f < ELMM_FIELD_SCALAR_ADV + d->num_scalars) return &d->Sadv[f - ELMM_FIELD_SCALAR_ADV];
  return nullptr;
}

// the time-averaged slices of scalar sc (1-based): xy (ny, nx), xz (nz, nx)
int orc_scalar_slices(void *h, int sc, double *xy, double *xz) {
  Domain *d = (Domain *)h;
  if (sc < 1 || sc > d->num_scalars) return ELMM_ERR_INVALID_ARG;
  if (xy) std::memcpy(xy, d->acc_xy[sc - 1].data(), d->acc_xy[sc - 1].size() * sizeof(double));
  if (xz) std::memcpy(xz, d->acc_xz[sc - 1].data(), d->acc_xz[sc - 1].size() * sizeof(double));
  return 0;
}

int orc_set_field(void *h, int f, const double *src) {
  A3 *a = field_of((Domain *)h, f);
  if (!a) return ELMM_ERR_INVALID_ARG;
  std::memcpy(a->v.data(), src, a->v.size() * sizeof(double));
  return 0;
}

int orc_get_field(void *h, int f, double *dst) {
  A3 *a = field_of((Domain *)h, f);
  if (!a) return ELMM_ERR_INVALID_ARG;
  std::memcpy(dst, a->v.data(), a->v.size() * sizeof(double));
  return 0;
}

int orc_project(void *h, double coef, double *max_div) {
  Domain *d = (Domain *)h;
  std::swap(d->U.v, d->U2.v); std::swap(d->V.v, d->V2.v); std::swap(d->W.v, d->W2.v);
  PressureCorrection(*d, coef, true);
  std::swap(d->U.v, d->U2.v); std::swap(d->V.v, d->V2.v); std::swap(d->W.v, d->W2.v);
  BoundUVW(*d, d->U, d->V, d->W);
  InitialDiffusivity(*d);
  if (max_div) *max_div = d->max_div;
  return 0;
}

int orc_step(void *h, int nsteps, double *max_div, double *cfl) {
  Domain *d = (Domain *)h;
  for (int s = 0; s < nsteps; s++) TMarchRK3(*d);
  if (max_div) *max_div = d->max_div;
  if (cfl) *cfl = d->CFL;
  return 0;
}

// the time and the length of the last step
int orc_clock(void *h, double *out2) {
  Domain *d = (Domain *)h;
  out2[0] = d->time;
  out2[1] = d->dt;
  return 0;
}

int orc_run_stage(void *h, int stage, int stop) {
  Domain *d = (Domain *)h;
  if (stage < 1 || stage > 3 || stop < 1 || stop > 3) return ELMM_ERR_INVALID_ARG;
  if (stage == 1) BoundUVW(*d, d->U, d->V, d->W);
  run_stage(*d, stage, stop);
  return 0;
}

// Poisson operator alone: RHS(0:n+1)^3 in, Phi(-1:n+2)^3 out (interior).
int orc_poisson(void *h, const double *RHS, double *Phi) {
  Domain *d = (Domain *)h;
  std::memcpy(d->RHS.v.data(), RHS, d->RHS.v.size() * sizeof(double));
  poisson_solve(*d);
  std::memcpy(Phi, d->Phi.v.data(), d->Phi.v.size() * sizeof(double));
  return 0;
}

// BoundUVW on the resident U, V, W (for ghost-cell parity checks)
int orc_bound_uvw(void *h) {
  Domain *d = (Domain *)h;
  BoundUVW(*d, d->U, d->V, d->W);
  Bound_Pr(*d, d->Pr);
  return 0;
}

int orc_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

}  // extern "C"
