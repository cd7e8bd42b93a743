// elmm_momentum.cuh -- Convection + OtherTerms of one RK3 stage in one pass:
// CDS2 skew-symmetric advection (advection.f90:15-327,
// advection_variable_z.f90:15-324), explicit diffusion with the wall-flux
// corrections (momentum_diffusion.f90:169-420 and the wmfluxes-*-inc.f90
// includes), the RK combine (dynamics.f90:266-354, :450-478), the
// old-pressure gradient (dynamics.f90:58-199) and U2 += U (tsteps.f90:352-354).
//
// A block owns an MX x MY column of cells and marches up a chunk of MKC
// planes.  U, V, W, Viscosity and Pr of each plane (with a one-cell halo in
// x and y) and the old Ustar (tile only) arrive by tensor-map TMA in a ring
// of kRingSlots plane slots in shared memory, requested several planes ahead
// of their use.  Every input cell is thus read from HBM once per chunk
// instead of once per stencil use.  The SGS kernel, k_sgs, streams U, V, W
// the same way.
#pragma once

#include <type_traits>

#include "elmm_common.cuh"
#include "elmm_packed.cuh"
#include "elmm_stream.cuh"

namespace elmm {

struct StageCoef {
  double rho, beta, alpha2;  // RK_rho, RK_beta, 2*RK_alpha of the stage
  int stage;
};

#ifndef ELMM_MOM_CHUNK
#define ELMM_MOM_CHUNK 16
#endif
constexpr int MX = 32, MY = 8, MKC = ELMM_MOM_CHUNK;
// per-tile context in shared memory: everything the stencil code reads
// besides the fields, so that no descriptor load sits on its critical path
template <typename T>
struct MomCtx {
  T cA[3], cB[3][3], rec2[3];
  int wallmask;  // bit s: wall-model fluxes on side s
  int vz;
  int ext[3][3];
  const double *dzPr, *dzW, *zPr, *zW;
  const T *fluxp[kFaces], *fluxm[kFaces];
  const unsigned char *bskip[3];
};

template <typename T>
__device__ __forceinline__ void fill_ctx(MomCtx<T> &m, const Dom<T> &d) {
  // called by one thread
  for (int a = 0; a < 3; a++) {
    m.cA[a] = (T)d.cA[a];
    m.rec2[a] = (T)d.rec2[a];
    for (int c = 0; c < 3; c++) { m.cB[c][a] = (T)d.cB[c][a]; m.ext[c][a] = d.ext[c][a]; }
  }
  int wm = 0;
  for (int f = 0; f < 6; f++) wm |= d.wall[f] ? (1 << f) : 0;
  m.wallmask = wm;
  m.vz = d.vz;
  m.dzPr = d.dzPr; m.dzW = d.dzW; m.zPr = d.zPr; m.zW = d.zW;
  for (int f = 0; f < kFaces; f++) { m.fluxp[f] = d.wm_fluxp[f]; m.fluxm[f] = d.wm_fluxm[f]; }
  for (int c = 0; c < 3; c++) m.bskip[c] = d.bskip[c];
}

// one velocity component's tendency at (i,j,k): advection + diffusion +
// wall corrections, in the reference's order of operations
// bt, bsub: the buoyancy of W, (a + bt) - bsub after the advection
// (BuoyancyForce, src/dynamics.f90:679-688; zero without a temperature field)
template <typename T, int C, typename RT>
__device__ __forceinline__ T tendency(const MomCtx<T> &m, const RT &R, int i, int j, int k, int wallhere,
                                      T bt = (T)0, T bsub = (T)0) {
  // X(dx,dy,dz) with the component's own axis first: along = C, a1, a2 the others
#define FU(dx, dy, dz) R.g(0, dx, dy, dz)
#define FV(dx, dy, dz) R.g(1, dx, dy, dz)
#define FW(dx, dy, dz) R.g(2, dx, dy, dz)
#define FN(dx, dy, dz) R.g(3, dx, dy, dz)
  T a;
  const T rx = m.rec2[0], ry = m.rec2[1], rz = m.rec2[2];
  if (C == 0) {
    const T u = FU(0, 0, 0), ue = FU(1, 0, 0), uw = FU(-1, 0, 0), un = FU(0, 1, 0), us = FU(0, -1, 0);
    const T ut = FU(0, 0, 1), ub = FU(0, 0, -1);
    const T v = FV(0, 0, 0), ve = FV(1, 0, 0), vs = FV(0, -1, 0), vse = FV(1, -1, 0);
    const T w = FW(0, 0, 0), we = FW(1, 0, 0), wb = FW(0, 0, -1), wbe = FW(1, 0, -1);
    const T Ax = m.cA[0], Ay = m.cA[1];
    const T Bx = m.cB[0][0], By = m.cB[0][1];
    if (!m.vz) {
      const T Az = m.cA[2], Bz = m.cB[0][2];
      a = -((Ax * (ue + u) * (ue + u) - Ax * (u + uw) * (u + uw)) + (Ay * (un + u) * (ve + v) - Ay * (u + us) * (vse + vs)) +
            (Az * (ut + u) * (we + w) - Az * (u + ub) * (wbe + wb)));
      T Vadv = (v + ve + vs + vse);
      T Wadv = (w + we + wb + wbe);
      a = a - (Bx * (ue - uw) * u + By * (un - us) * Vadv + Bz * (ut - ub) * Wadv);
    } else {
      const T dzp = (T)m.dzPr[k + 2];
      a = -((Ax * (ue + u) * (ue + u) - Ax * (u + uw) * (u + uw)) + (Ay * (un + u) * (ve + v) - Ay * (u + us) * (vse + vs)) +
            ((ut + u) * (we + w) - (u + ub) * (wbe + wb)) / dzp / 4);
      T Vadv = (v + ve + vs + vse);
      T Wadv = (w + we + wb + wbe) / 4;
      a = a - (Bx * (ue - uw) * u + By * (un - us) * Vadv + (ut - ub) / (T)(m.zPr[k + 1 + 2] - m.zPr[k - 1 + 2]) * Wadv);
    }
    a = a * (T)0.5;
    const T n0 = FN(0, 0, 0), ne = FN(1, 0, 0), nn = FN(0, 1, 0), nne = FN(1, 1, 0), ns = FN(0, -1, 0), nse = FN(1, -1, 0);
    const T nt = FN(0, 0, 1), nte = FN(1, 0, 1), nb = FN(0, 0, -1), nbe = FN(1, 0, -1);
    a = a + ne * (ue - u) * rx;
    a = a - n0 * (u - uw) * rx;
    a = a + (T)0.25 * (nne + ne + nn + n0) * (un - u) * ry;
    a = a - (T)0.25 * (ne + nse + n0 + ns) * (u - us) * ry;
    if (!m.vz) {
      a = a + (T)0.25 * (nte + ne + nt + n0) * (ut - u) * rz;
      a = a - (T)0.25 * (ne + nbe + n0 + nb) * (u - ub) * rz;
    } else {
      T tz = (T)0.25 * (nte + ne + nt + n0) * (ut - u) / (T)m.dzW[k + 2];
      tz = tz - (T)0.25 * (ne + nbe + n0 + nb) * (u - ub) / (T)m.dzW[k - 1 + 2];
      tz = tz / (T)m.dzPr[k + 2];
      a = a + tz;
    }
    if (wallhere) {
      const int *e = m.ext[0];
      if ((m.wallmask & (1 << SIDE_WE)) && i == 1) {
        long long p = (long long)(j - 1) + (long long)e[1] * (k - 1);
        a = a + n0 * (u - uw) * rx;
        a = a + m.fluxp[0 * 6 + SIDE_WE][p];
      }
      if ((m.wallmask & (1 << SIDE_EA)) && i == e[0]) {
        long long p = (long long)(j - 1) + (long long)e[1] * (k - 1);
        a = a - ne * (ue - u) * rx;
        a = a - m.fluxm[0 * 6 + SIDE_EA][p];
      }
      if ((m.wallmask & (1 << SIDE_SO)) && j == 1) {
        long long p = (long long)(i - 1) + (long long)e[0] * (k - 1);
        a = a + (ne + nse + n0 + ns) * (u - us) * ry / 4;
        a = a + m.fluxp[0 * 6 + SIDE_SO][p];
      }
      if ((m.wallmask & (1 << SIDE_NO)) && j == e[1]) {
        long long p = (long long)(i - 1) + (long long)e[0] * (k - 1);
        a = a - (nne + ne + nn + n0) * (un - u) * ry / 4;
        a = a - m.fluxm[0 * 6 + SIDE_NO][p];
      }
      if ((m.wallmask & (1 << SIDE_BO)) && k == 1 &&
          !(m.bskip[0] && m.bskip[0][(long long)(i - 1) + (long long)e[0] * (j - 1)])) {
        long long p = (long long)(i - 1) + (long long)e[0] * (j - 1);
        T s = ne + nbe + n0 + nb;
        if (m.vz) a = a + s * (u - ub) / (T)m.dzW[k - 1 + 2] / 4 / (T)m.dzPr[k + 2];
        else a = a + s * (u - ub) * rz / 4;
        a = a + m.fluxp[0 * 6 + SIDE_BO][p];
      }
      if ((m.wallmask & (1 << SIDE_TO)) && k == e[2]) {
        long long p = (long long)(i - 1) + (long long)e[0] * (j - 1);
        T s = nte + ne + nt + n0;
        if (m.vz) a = a - s * (ut - u) / (T)m.dzW[k + 2] / 4 / (T)m.dzPr[k + 2];
        else a = a - s * (ut - u) * rz / 4;
        a = a - m.fluxm[0 * 6 + SIDE_TO][p];
      }
    }
  } else if (C == 1) {
    const T v = FV(0, 0, 0), ve = FV(1, 0, 0), vw = FV(-1, 0, 0), vn = FV(0, 1, 0), vs = FV(0, -1, 0);
    const T vt = FV(0, 0, 1), vb = FV(0, 0, -1);
    const T u = FU(0, 0, 0), un = FU(0, 1, 0), uw = FU(-1, 0, 0), unw = FU(-1, 1, 0);
    const T w = FW(0, 0, 0), wn = FW(0, 1, 0), wb = FW(0, 0, -1), wbn = FW(0, 1, -1);
    const T Ax = m.cA[0], Ay = m.cA[1];
    const T Bx = m.cB[1][0], By = m.cB[1][1];
    if (!m.vz) {
      const T Az = m.cA[2], Bz = m.cB[1][2];
      a = -((Ay * (vn + v) * (vn + v) - Ay * (v + vs) * (v + vs)) + (Ax * (ve + v) * (un + u) - Ax * (v + vw) * (unw + uw)) +
            (Az * (vt + v) * (wn + w) - Az * (v + vb) * (wbn + wb)));
      T Uadv = (u + un + uw + unw);
      T Wadv = (w + wn + wb + wbn);
      a = a - (Bx * (ve - vw) * Uadv + By * (vn - vs) * v + Bz * (vt - vb) * Wadv);
    } else {
      const T dzp = (T)m.dzPr[k + 2];
      a = -((Ay * (vn + v) * (vn + v) - Ay * (v + vs) * (v + vs)) + (Ax * (ve + v) * (un + u) - Ax * (v + vw) * (unw + uw)) +
            ((vt + v) * (wn + w) - (v + vb) * (wbn + wb)) / dzp / 4);
      T Uadv = (u + un + uw + unw);
      T Wadv = (w + wn + wb + wbn) / 4;
      a = a - (Bx * (ve - vw) * Uadv + By * (vn - vs) * v + (vt - vb) / (T)(m.zPr[k + 1 + 2] - m.zPr[k - 1 + 2]) * Wadv);
    }
    a = a * (T)0.5;
    const T n0 = FN(0, 0, 0), ne = FN(1, 0, 0), nn = FN(0, 1, 0), nne = FN(1, 1, 0), nw = FN(-1, 0, 0), nnw = FN(-1, 1, 0);
    const T nt = FN(0, 0, 1), nnt = FN(0, 1, 1), nb = FN(0, 0, -1), nnb = FN(0, 1, -1);
    a = a + (T)0.25 * (nne + ne + nn + n0) * (ve - v) * rx;
    a = a - (T)0.25 * (nn + n0 + nnw + nw) * (v - vw) * rx;
    a = a + nn * (vn - v) * ry;
    a = a - n0 * (v - vs) * ry;
    if (!m.vz) {
      a = a + (T)0.25 * (nnt + nn + nt + n0) * (vt - v) * rz;
      a = a - (T)0.25 * (nn + nnb + n0 + nb) * (v - vb) * rz;
    } else {
      T tz = (T)0.25 * (nnt + nn + nt + n0) * (vt - v) / (T)m.dzW[k + 2];
      tz = tz - (T)0.25 * (nn + nnb + n0 + nb) * (v - vb) / (T)m.dzW[k - 1 + 2];
      tz = tz / (T)m.dzPr[k + 2];
      a = a + tz;
    }
    if (wallhere) {
      const int *e = m.ext[1];
      if ((m.wallmask & (1 << SIDE_WE)) && i == 1) {
        long long p = (long long)(j - 1) + (long long)e[1] * (k - 1);
        a = a + (nn + n0 + nnw + nw) * (v - vw) * rx / 4;
        a = a + m.fluxp[1 * 6 + SIDE_WE][p];
      }
      if ((m.wallmask & (1 << SIDE_EA)) && i == e[0]) {
        long long p = (long long)(j - 1) + (long long)e[1] * (k - 1);
        a = a - (nne + ne + nn + n0) * (ve - v) * rx / 4;
        a = a - m.fluxm[1 * 6 + SIDE_EA][p];
      }
      if ((m.wallmask & (1 << SIDE_SO)) && j == 1) {
        long long p = (long long)(i - 1) + (long long)e[0] * (k - 1);
        a = a + n0 * (v - vs) * ry;
        a = a + m.fluxp[1 * 6 + SIDE_SO][p];
      }
      if ((m.wallmask & (1 << SIDE_NO)) && j == e[1]) {
        long long p = (long long)(i - 1) + (long long)e[0] * (k - 1);
        a = a - nn * (vn - v) * ry;
        a = a - m.fluxm[1 * 6 + SIDE_NO][p];
      }
      if ((m.wallmask & (1 << SIDE_BO)) && k == 1 &&
          !(m.bskip[1] && m.bskip[1][(long long)(i - 1) + (long long)e[0] * (j - 1)])) {
        long long p = (long long)(i - 1) + (long long)e[0] * (j - 1);
        T s = nn + nnb + n0 + nb;
        if (m.vz) a = a + s * (v - vb) / (T)m.dzW[k - 1 + 2] / 4 / (T)m.dzPr[k + 2];
        else a = a + s * (v - vb) * rz / 4;
        a = a + m.fluxp[1 * 6 + SIDE_BO][p];
      }
      if ((m.wallmask & (1 << SIDE_TO)) && k == e[2]) {
        long long p = (long long)(i - 1) + (long long)e[0] * (j - 1);
        T s = nnt + nn + nt + n0;
        if (m.vz) a = a - s * (vt - v) / (T)m.dzW[k + 2] / 4 / (T)m.dzPr[k + 2];
        else a = a - s * (vt - v) * rz / 4;
        a = a - m.fluxm[1 * 6 + SIDE_TO][p];
      }
    }
  } else {
    const T w = FW(0, 0, 0), we = FW(1, 0, 0), ww = FW(-1, 0, 0), wn = FW(0, 1, 0), ws = FW(0, -1, 0);
    const T wt = FW(0, 0, 1), wb = FW(0, 0, -1);
    const T u = FU(0, 0, 0), ut = FU(0, 0, 1), uw = FU(-1, 0, 0), utw = FU(-1, 0, 1);
    const T v = FV(0, 0, 0), vt = FV(0, 0, 1), vs = FV(0, -1, 0), vts = FV(0, -1, 1);
    const T Ax = m.cA[0], Ay = m.cA[1];
    const T Bx = m.cB[2][0], By = m.cB[2][1];
    if (!m.vz) {
      const T Az = m.cA[2], Bz = m.cB[2][2];
      a = -((Az * (wt + w) * (wt + w) - Az * (w + wb) * (w + wb)) + (Ay * (wn + w) * (vt + v) - Ay * (w + ws) * (vs + vts)) +
            (Ax * (we + w) * (ut + u) - Ax * (w + ww) * (utw + uw)));
      T Uadv = (u + ut + uw + utw);
      T Vadv = (v + vt + vs + vts);
      a = a - (Bx * (we - ww) * Uadv + By * (wn - ws) * Vadv + Bz * (wt - wb) * w);
    } else {
      const T dzw = (T)m.dzW[k + 2];
      a = -(((wt + w) * (wt + w) - (w + wb) * (w + wb)) / dzw / 4 + (Ay * (wn + w) * (vt + v) - Ay * (w + ws) * (vts + vs)) +
            (Ax * (we + w) * (ut + u) - Ax * (w + ww) * (utw + uw)));
      T Uadv = (u + ut + uw + utw);
      T Vadv = (v + vt + vs + vts);
      a = a - (Bx * (we - ww) * Uadv + By * (wn - ws) * Vadv + (wt - wb) / (T)(m.zW[k + 1 + 2] - m.zW[k - 1 + 2]) * w);
    }
    a = a * (T)0.5;
    a = (a + bt) - bsub;
    const T n0 = FN(0, 0, 0), ne = FN(1, 0, 0), nt = FN(0, 0, 1), nte = FN(1, 0, 1), nw = FN(-1, 0, 0), ntw = FN(-1, 0, 1);
    const T nn = FN(0, 1, 0), ntn = FN(0, 1, 1), ns = FN(0, -1, 0), nts = FN(0, -1, 1);
    a = a + (T)0.25 * (nte + ne + nt + n0) * (we - w) * rx;
    a = a - (T)0.25 * (nt + n0 + ntw + nw) * (w - ww) * rx;
    a = a + (T)0.25 * (ntn + nt + nn + n0) * (wn - w) * ry;
    a = a - (T)0.25 * (nt + nts + n0 + ns) * (w - ws) * ry;
    if (!m.vz) {
      a = a + nt * (wt - w) * rz;
      a = a - n0 * (w - wb) * rz;
    } else {
      T tz = nt * (wt - w) / (T)m.dzPr[k + 1 + 2];
      tz = tz - n0 * (w - wb) / (T)m.dzPr[k + 2];
      tz = tz / (T)m.dzW[k + 2];
      a = a + tz;
    }
    if (wallhere) {
      const int *e = m.ext[2];
      if ((m.wallmask & (1 << SIDE_WE)) && i == 1) {
        long long p = (long long)(j - 1) + (long long)e[1] * (k - 1);
        a = a + (nt + n0 + ntw + nw) * (w - ww) * rx / 4;
        a = a + m.fluxp[2 * 6 + SIDE_WE][p];
      }
      if ((m.wallmask & (1 << SIDE_EA)) && i == e[0]) {
        long long p = (long long)(j - 1) + (long long)e[1] * (k - 1);
        a = a - (nte + ne + nt + n0) * (we - w) * rx / 4;
        a = a - m.fluxm[2 * 6 + SIDE_EA][p];
      }
      if ((m.wallmask & (1 << SIDE_SO)) && j == 1) {
        long long p = (long long)(i - 1) + (long long)e[0] * (k - 1);
        a = a + (nt + nts + n0 + ns) * (w - ws) * ry / 4;
        a = a + m.fluxp[2 * 6 + SIDE_SO][p];
      }
      if ((m.wallmask & (1 << SIDE_NO)) && j == e[1]) {
        long long p = (long long)(i - 1) + (long long)e[0] * (k - 1);
        a = a - (ntn + nt + nn + n0) * (wn - w) * ry / 4;
        a = a - m.fluxm[2 * 6 + SIDE_NO][p];
      }
      if ((m.wallmask & (1 << SIDE_BO)) && k == 1 &&
          !(m.bskip[2] && m.bskip[2][(long long)(i - 1) + (long long)e[0] * (j - 1)])) {
        long long p = (long long)(i - 1) + (long long)e[0] * (j - 1);
        if (m.vz) a = a + n0 * (w - wb) / (T)m.dzPr[k + 2] / (T)m.dzW[k + 2];
        else a = a + n0 * (w - wb) * rz;
        a = a + m.fluxp[2 * 6 + SIDE_BO][p];
      }
      if ((m.wallmask & (1 << SIDE_TO)) && k == e[2]) {
        long long p = (long long)(i - 1) + (long long)e[0] * (j - 1);
        if (m.vz) a = a - nt * (wt - w) / (T)m.dzPr[k + 1 + 2] / (T)m.dzW[k + 2];
        else a = a - nt * (wt - w) * rz;
        a = a - m.fluxm[2 * 6 + SIDE_TO][p];
      }
    }
  }
#undef FU
#undef FV
#undef FW
#undef FN
  return a;
}

// The wall-model corrections of one cell on the mixed path (the wall blocks
// of tendency<T, C>: the diffusive flux through the face towards a wall-model
// side taken back, the wall-model flux added; the wmfluxes-*-inc.f90
// includes), on stored deviations: a difference across levels is the stored
// difference plus the difference of the offsets (O, see tendency_dev).
template <int C, typename RT>
__device__ __forceinline__ float wall_dev(const MomCtx<float> &m, const RT &R, const VelOffN<float> &O, int i, int j,
                                          int k) {
#define FN(dx, dy, dz) R.g(3, dx, dy, dz)
  const float rx = m.rec2[0], ry = m.rec2[1], rz = m.rec2[2];
  const int *e = m.ext[C];
  float a = 0.f;
  const long long pyz = (long long)(j - 1) + (long long)e[1] * (k - 1), pxz = (long long)(i - 1) + (long long)e[0] * (k - 1);
  const long long pxy = (long long)(i - 1) + (long long)e[0] * (j - 1);
  const bool bo = (m.wallmask & (1 << SIDE_BO)) && k == 1 && !(m.bskip[C] && m.bskip[C][pxy]);
  const bool to = (m.wallmask & (1 << SIDE_TO)) && k == e[2];
  if (C < 2) {
    // U (C = 0) or V (C = 1): the component F and its offsets
    const float f = R.g(C, 0, 0, 0), fe = R.g(C, 1, 0, 0), fw = R.g(C, -1, 0, 0), fn = R.g(C, 0, 1, 0);
    const float fs = R.g(C, 0, -1, 0), ft = R.g(C, 0, 0, 1), fb = R.g(C, 0, 0, -1);
    const float *o = C == 0 ? O.o : O.p;
    const float n0 = FN(0, 0, 0), ne = FN(1, 0, 0), nn = FN(0, 1, 0), nne = FN(1, 1, 0);
    // the viscosities of the x- and y-faces of the point
    const float nW = C == 0 ? n0 : 0.25f * (((nn + n0) + FN(-1, 1, 0)) + FN(-1, 0, 0));
    const float nE = C == 0 ? ne : 0.25f * (((nne + ne) + nn) + n0);
    const float nS = C == 0 ? 0.25f * (((ne + FN(1, -1, 0)) + n0) + FN(0, -1, 0)) : n0;
    const float nN = C == 0 ? 0.25f * (((nne + ne) + nn) + n0) : nn;
    if ((m.wallmask & (1 << SIDE_WE)) && i == 1) { a = a + nW * (f - fw) * rx; a = a + m.fluxp[C * 6 + SIDE_WE][pyz]; }
    if ((m.wallmask & (1 << SIDE_EA)) && i == e[0]) { a = a - nE * (fe - f) * rx; a = a - m.fluxm[C * 6 + SIDE_EA][pyz]; }
    if ((m.wallmask & (1 << SIDE_SO)) && j == 1) { a = a + nS * (f - fs) * ry; a = a + m.fluxp[C * 6 + SIDE_SO][pxz]; }
    if ((m.wallmask & (1 << SIDE_NO)) && j == e[1]) { a = a - nN * (fn - f) * ry; a = a - m.fluxm[C * 6 + SIDE_NO][pxz]; }
    if (bo) {
      const float s = C == 0 ? ((ne + FN(1, 0, -1)) + n0) + FN(0, 0, -1) : ((nn + FN(0, 1, -1)) + n0) + FN(0, 0, -1);
      const float db = (f - fb) + (o[1] - o[0]);
      if (m.vz) a = a + s * db / (float)m.dzW[k - 1 + 2] / 4 / (float)m.dzPr[k + 2];
      else a = a + s * db * rz / 4;
      a = a + m.fluxp[C * 6 + SIDE_BO][pxy];
    }
    if (to) {
      const float s = C == 0 ? ((FN(1, 0, 1) + ne) + FN(0, 0, 1)) + n0 : ((FN(0, 1, 1) + nn) + FN(0, 0, 1)) + n0;
      const float dt = (ft - f) + (o[2] - o[1]);
      if (m.vz) a = a - s * dt / (float)m.dzW[k + 2] / 4 / (float)m.dzPr[k + 2];
      else a = a - s * dt * rz / 4;
      a = a - m.fluxm[C * 6 + SIDE_TO][pxy];
    }
  } else {
    const float w = R.g(2, 0, 0, 0), we = R.g(2, 1, 0, 0), ww = R.g(2, -1, 0, 0), wn = R.g(2, 0, 1, 0);
    const float ws = R.g(2, 0, -1, 0), wt = R.g(2, 0, 0, 1), wb = R.g(2, 0, 0, -1);
    const float n0 = FN(0, 0, 0), ne = FN(1, 0, 0), nt = FN(0, 0, 1), nte = FN(1, 0, 1), nw = FN(-1, 0, 0);
    const float ntw = FN(-1, 0, 1), nn = FN(0, 1, 0), ntn = FN(0, 1, 1), ns = FN(0, -1, 0), nts = FN(0, -1, 1);
    if ((m.wallmask & (1 << SIDE_WE)) && i == 1) {
      a = a + (((nt + n0) + ntw) + nw) * (w - ww) * rx / 4;
      a = a + m.fluxp[2 * 6 + SIDE_WE][pyz];
    }
    if ((m.wallmask & (1 << SIDE_EA)) && i == e[0]) {
      a = a - (((nte + ne) + nt) + n0) * (we - w) * rx / 4;
      a = a - m.fluxm[2 * 6 + SIDE_EA][pyz];
    }
    if ((m.wallmask & (1 << SIDE_SO)) && j == 1) {
      a = a + (((nt + nts) + n0) + ns) * (w - ws) * ry / 4;
      a = a + m.fluxp[2 * 6 + SIDE_SO][pxz];
    }
    if ((m.wallmask & (1 << SIDE_NO)) && j == e[1]) {
      a = a - (((ntn + nt) + nn) + n0) * (wn - w) * ry / 4;
      a = a - m.fluxm[2 * 6 + SIDE_NO][pxz];
    }
    if (bo) {
      if (m.vz) a = a + n0 * (w - wb) / (float)m.dzPr[k + 2] / (float)m.dzW[k + 2];
      else a = a + n0 * (w - wb) * rz;
      a = a + m.fluxp[2 * 6 + SIDE_BO][pxy];
    }
    if (to) {
      if (m.vz) a = a - nt * (wt - w) / (float)m.dzPr[k + 1 + 2] / (float)m.dzW[k + 2];
      else a = a - nt * (wt - w) * rz;
      a = a - m.fluxm[2 * 6 + SIDE_TO][pxy];
    }
  }
#undef FN
  return a;
}

// Layout of one ring slot (one plane k of the tile): NWF "wide" fields with
// the x/y halo (rows j0-1..j0+MY, columns i0-XO..i0+MX+XO-1) and NNF
// "narrow" fields of the tile's own cells (rows j0..j0+MY-1, columns
// i0..i0+MX-1).  XO = 16 bytes of halo on each side keeps every copied row
// segment 16-byte aligned in global and shared memory.
template <typename T, int NWF, int NNF>
struct SlotLayout {
  static constexpr int XO = 16 / (int)sizeof(T);
  static constexpr int SPW = MX + 2 * XO;  // wide row
  static constexpr int WROWS = MY + 2;
  static constexpr int WB = ((WROWS * SPW * (int)sizeof(T) + 127) / 128) * 128 / (int)sizeof(T);  // wide block
  static constexpr int NB = ((MY * MX * (int)sizeof(T) + 127) / 128) * 128 / (int)sizeof(T);      // narrow block
  static constexpr int WIDE = NWF * WB;
  static constexpr int SIZE = WIDE + NNF * NB;  // elements per slot (a multiple of 128 bytes)
  static constexpr int BYTES = SIZE * (int)sizeof(T);
  static constexpr uint32_t WBOX = WROWS * SPW * sizeof(T);  // bytes one wide box delivers
  static constexpr uint32_t NBOX = MY * MX * sizeof(T);
};

// ring accessor: field f (wide), offsets (dx,dy) of the thread's cell and
// plane k+dz
template <typename T, int NWF, int NNF>
struct WideRing {
  typedef SlotLayout<T, NWF, NNF> Lay;
  const T *__restrict__ p[3];
  int o;
  __device__ __forceinline__ T g(int f, int dx, int dy, int dz) const {
    return p[dz + 1][f * Lay::WB + o + dy * Lay::SPW + dx];
  }
};

// Issues the tensor-map loads of plane kk of the tile into one slot: one
// box per field (thread 0 only).
template <typename T, int NWF, int NNF>
__device__ __forceinline__ void issue_plane(T *slot, uint64_t *bar, const CUtensorMap *maps, const int *wide,
                                            const int *narrow, bool with_narrow, int aln, int i0, int j0, int kk) {
  typedef SlotLayout<T, NWF, NNF> Lay;
  const uint32_t bytes = NWF * Lay::WBOX + (with_narrow ? NNF * Lay::NBOX : 0u);
  mbar_expect_tx(bar, bytes);
  const int xw = aln - 1 + i0 - Lay::XO, xn = aln - 1 + i0;
#pragma unroll
  for (int f = 0; f < NWF; f++) tma_load_3d(slot + f * Lay::WB, maps + BOX_WIDE * F_COUNT + wide[f], xw, j0 - 1, kk, bar);
  if (with_narrow) {
#pragma unroll
    for (int f = 0; f < NNF; f++)
      tma_load_3d(slot + Lay::WIDE + f * Lay::NB, maps + BOX_NARROW * F_COUNT + narrow[f], xn, j0, kk, bar);
  }
}

// The momentum kernel's planes: U, V, W, Viscosity, P wide; the old Ustar,
// Vstar, Wstar narrow (stages 2 and 3), and on the FP32 path also the
// potential temperature of the stage as a fourth narrow field (buoyancy),
// from its own tensor maps (tmapT: one per value buffer).
template <typename T, int NNF>
__device__ __forceinline__ void issue_mom_plane(T *slot, uint64_t *bar, const CUtensorMap *maps,
                                                const CUtensorMap *tmapT, bool with_star, int aln, int i0, int j0,
                                                int kk) {
  typedef SlotLayout<T, 5, NNF> Lay;
  const uint32_t bytes = 5 * Lay::WBOX + (with_star ? 3 * Lay::NBOX : 0u) + (tmapT ? Lay::NBOX : 0u);
  mbar_expect_tx(bar, bytes);
  const int xw = aln - 1 + i0 - Lay::XO, xn = aln - 1 + i0;
  const int wide[5] = {F_U, F_V, F_W, F_NU, F_P};
#pragma unroll
  for (int f = 0; f < 5; f++) tma_load_3d(slot + f * Lay::WB, maps + BOX_WIDE * F_COUNT + wide[f], xw, j0 - 1, kk, bar);
  if (with_star) {
#pragma unroll
    for (int f = 0; f < 3; f++)
      tma_load_3d(slot + Lay::WIDE + f * Lay::NB, maps + BOX_NARROW * F_COUNT + F_US + f, xn, j0, kk, bar);
  }
  if (NNF == 4 && tmapT) tma_load_3d(slot + Lay::WIDE + 3 * Lay::NB, tmapT, xn, j0, kk, bar);
}

constexpr int kRingSlots = 5;

// Cells per thread along x and ring slots of the momentum kernel: FP32
// threads compute two x-adjacent cells with packed FP32x2 arithmetic
// (elmm_packed.cuh); a four-slot ring leaves room for four 128-thread blocks
// per SM.  FP64 keeps one cell per thread and five slots.
// nnf: narrow fields per slot (FP32 adds the temperature; the FP64 slots
// would not leave room for two blocks per SM and read it from global memory).
template <typename T>
struct MomShape {
  static constexpr int cpt = 1, slots = 5, threads = MX * MY, min_blocks = 2, nnf = 3;
};
template <>
struct MomShape<float> {
  static constexpr int cpt = 2, slots = 4, threads = MX * MY / 2, min_blocks = 4, nnf = 4;
};

// KC: planes of a tile's column (a tuning choice: every cell's arithmetic is
// the same for any KC)
template <typename T, int KC = MKC>
__global__ void __launch_bounds__(MomShape<T>::threads, MomShape<T>::min_blocks)
    k_momentum(const Dom<T> *__restrict__ doms, Launch L, StageCoef sc) {
  constexpr int NNF = MomShape<T>::nnf;
  typedef SlotLayout<T, 5, NNF> Lay;
  constexpr int CPT = MomShape<T>::cpt, NSL = MomShape<T>::slots, TXN = MX / CPT;
  extern __shared__ __align__(128) unsigned char dyn_smem[];
  T *ring = reinterpret_cast<T *>(dyn_smem);
  __shared__ __align__(8) uint64_t bars[NSL];
  __shared__ MomCtx<T> ctx;
  // mixed path: offsets of U and V on planes k0-1 .. k0+KC of the tile (see Dom::voff)
  __shared__ float soff[2][KC + 2];
  __shared__ int abort_flag;
  const int tx = threadIdx.x % TXN, ty = threadIdx.x / TXN;
  // tensor copies need 128-byte aligned destinations
  if (smem_addr(ring) & 127u) {
    if (threadIdx.x == 0) doms[0].flags[1] = 1;
    return;
  }
  if (threadIdx.x == 0) {
    for (int s2 = 0; s2 < NSL; s2++) mbar_init(&bars[s2], 1);
    abort_flag = 0;
    fence_async_shared();
  }
  __syncthreads();
  uint32_t phase = 0;  // bit s: parity of the next wait on slot s
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    int lt = t - __ldg(L.starts + di);
    const int ntx = (d.nx + MX - 1) / MX, nty = (d.ny + MY - 1) / MY;
    const int bx = lt % ntx; lt /= ntx;
    const int by = lt % nty;
    const int bk = lt / nty;
    const int i0 = bx * MX + 1, j0 = by * MY + 1, k0 = bk * KC + 1;
    const int k1 = min(k0 + KC - 1, d.nz);
    const int i = i0 + CPT * tx, j = j0 + ty;  // the thread's first cell
    const int nx = d.nx, ny = d.ny;
    const long long plane = d.plane;
    const bool stage1 = sc.stage == 1;
    const CUtensorMap *maps = reinterpret_cast<const CUtensorMap *>(d.tmaps);
    // the temperature of the stage start through the ring (FP32 with buoyancy)
    const CUtensorMap *tmapT = (NNF == 4 && d.buoy && d.tmapT)
                                   ? reinterpret_cast<const CUtensorMap *>(d.tmapT) + (sc.stage - 1) % 3
                                   : nullptr;
    __syncthreads();  // every slot and the context of the previous tile are free
    if (threadIdx.x == 0) fill_ctx(ctx, d);
    if constexpr (sizeof(T) == 4) {
      if (threadIdx.x < 2 * (KC + 2)) {
        const int c = threadIdx.x / (KC + 2), kk = k0 - 1 + threadIdx.x % (KC + 2);
        soff[c][kk - k0 + 1] = kk <= d.nz + 1 ? __ldg(d.voff + c * (d.nz + 2) + kk) : 0.f;
      }
    }
    if (threadIdx.x == 0) {
      fence_async_shared();
      for (int kk = k0 - 1; kk <= min(k0 - 1 + NSL - 1, k1 + 1); kk++)
        if (kk != d.skip_plane)
          issue_mom_plane<T, NNF>(ring + (kk % NSL) * Lay::SIZE, &bars[kk % NSL], maps, tmapT, !stage1, d.aln, i0, j0,
                                  kk);
    }
    __syncthreads();  // the context is written
    const T dt = (T)d.dt, rdt = (T)sc.rho, bdt = (T)sc.beta;
    const double coefd = sc.alpha2 * d.dt;
    const T coef = (T)coefd;
    const T gx = (T)(-coefd / d.dx), gy = (T)(-coefd / d.dy), gz = (T)(-coefd / d.dz);
    const T m = (T)(*d.prm);
    const int kU = d.ext[0][2], kV = d.ext[1][2], kW = d.ext[2][2];
    const bool vz = d.vz != 0;
    const bool prgx_on = d.prgx_on != 0, prgy_on = d.prgy_on != 0;
    const T fx = prgx_on ? (-coef) * (T)d.prgx : (T)0, fy = prgy_on ? (-coef) * (T)d.prgy : (T)0;
    const double *dzW = d.dzW;
    T *__restrict__ U2o = d.U2;
    T *__restrict__ V2o = d.V2;
    T *__restrict__ W2o = d.W2;
    T *__restrict__ Us = d.Us;
    T *__restrict__ Vs = d.Vs;
    T *__restrict__ Ws = d.Ws;
    const int o = (ty + 1) * Lay::SPW + (CPT * tx + Lay::XO);
    const bool inside0 = i <= nx && j <= ny;
    long long c = bidx(d, inside0 ? i : 1, inside0 ? j : 1, k0);
    const int nz = d.nz;
    // block-uniform: only tiles on a side of the box and the planes next to
    // the bottom and top have wall-model corrections; a component's last
    // index is n or n-1 (src/initial.f90:871-896)
    const bool xlo = i0 == 1, xhi = i0 + MX - 1 >= nx - 1, ylo = j0 == 1, yhi = j0 + MY - 1 >= ny - 1;
    int wmask = 0;
    for (int f = 0; f < 6; f++) wmask |= d.wall[f] ? (1 << f) : 0;
    const int wtile = wmask & ((xlo ? 1 : 0) | (xhi ? 2 : 0) | (ylo ? 4 : 0) | (yhi ? 8 : 0));
    // both cells of the thread's pair have all three components (the pairs of
    // a partial tile past the last cell take the per-cell path)
    const bool pair_full = i + CPT - 1 <= min(d.ext[0][0], min(d.ext[1][0], d.ext[2][0])) &&
                           j <= min(d.ext[0][1], min(d.ext[1][1], d.ext[2][1]));
    // buoyancy of W (BuoyancyForce, src/dynamics.f90:679-688): A = g / T_ref;
    // with theta stored as theta - T_ref the constant term cancels exactly
    const bool buoy = d.buoy != 0;
    const T bA2 = (T)(d.grav / d.tref / 2.0);
    const T bsub = buoy && d.toff == 0 ? (T)(d.grav / d.tref * d.tref) : (T)0;
    const T *__restrict__ Tm = buoy ? d.slot[0].buf[(sc.stage - 1) % 3] : nullptr;  // theta at the stage start
    MomK2 K2;
    if constexpr (CPT == 2) {
      K2.Ax = bc2((float)ctx.cA[0]); K2.Ay = bc2((float)ctx.cA[1]); K2.Az = bc2((float)ctx.cA[2]);
      K2.rx = bc2((float)ctx.rec2[0]); K2.ry = bc2((float)ctx.rec2[1]); K2.rz = bc2((float)ctx.rec2[2]);
      K2.q = bc2(0.25f);
      for (int cc = 0; cc < 3; cc++)
        for (int a2 = 0; a2 < 3; a2++) K2.B[cc][a2] = bc2((float)ctx.cB[cc][a2]);
    }
    for (int k = k0; k <= k1; k++) {
      // planes k-1, k, k+1 must have landed
      bool ok = true;
      for (int kk = (k == k0 ? k0 - 1 : k + 1); kk <= k + 1; kk++) {
        const int s2 = kk % NSL;
        bool w = mbar_wait(&bars[s2], (phase >> s2) & 1u, d.wait_limit);
        // a plane whose copies were issued always lands before the block
        // moves on or gives up (so no copy into this block's shared memory
        // outlives it): a lowered limit only cuts the wait on a skipped one
        if (!w && kk != d.skip_plane) w = mbar_wait(&bars[s2], (phase >> s2) & 1u);
        ok &= w;
        phase ^= 1u << s2;
      }
      if (!ok) { abort_flag = 1; d.flags[1] = 1; }
      const int wallhere = wtile | (wmask & ((k == 1 ? 16 : 0) | (k >= nz - 1 ? 32 : 0)));
      const T *p0s = ring + ((k - 1) % NSL) * Lay::SIZE, *p1s = ring + (k % NSL) * Lay::SIZE,
              *p2s = ring + ((k + 1) % NSL) * Lay::SIZE;
      bool packed = false;
      if constexpr (CPT == 2)
        packed = (!vz || d.kz2) && !wallhere && pair_full && k <= min(kU, min(kV, kW));
      if (packed && ok) {
        if constexpr (CPT == 2) {
          // two cells per thread, every operation on a pair
          Ring2<Lay::WB, Lay::SPW> R2;
          R2.p[0] = p0s; R2.p[1] = p1s; R2.p[2] = p2s;
          R2.o = o;
          // the stencils take the offsets of U and V separately
          // (tendency_dev); the RK combine below works on the stored
          // deviations (U2 is stored the same way)
          VelOffN<F2> O;
#pragma unroll
          for (int q = 0; q < 3; q++) { O.o[q] = bc2(soff[0][k - k0 + q]); O.p[q] = bc2(soff[1][k - k0 + q]); }
          const float *nar = p1s + Lay::WIDE + ty * MX + CPT * tx;
          const F2 mm = bc2(m);
          const F2 p0 = R2.g(4, 0, 0, 0) - mm;
          F2 btp = bc2(0.f);
          if (buoy) {
            const int ot = Lay::WIDE + 3 * Lay::NB + ty * MX + CPT * tx;  // the temperature, narrow field 3
            btp = bc2(bA2) * (F2{*reinterpret_cast<const float2 *>(p2s + ot)} +
                              F2{*reinterpret_cast<const float2 *>(p1s + ot)});
          }
          F2 tu, tv, tw;
          F2 gz2 = bc2(gz);
          if (!vz) {
            tu = tendency_dev<0, false>(K2, R2, O, bc2(0.f), (const KZ2 *)nullptr);
            tv = tendency_dev<1, false>(K2, R2, O, bc2(0.f), (const KZ2 *)nullptr);
            tw = tendency_dev<2, false>(K2, R2, O, btp, (const KZ2 *)nullptr);
          } else {
            const int nzp = nz + 2;
            const float *kz = d.kz2 + k;
            KZ2 Z;
            Z.auv = bc2(__ldg(kz + KZ_AUV * nzp)); Z.buv = bc2(__ldg(kz + KZ_BUV * nzp));
            Z.d1uv = bc2(__ldg(kz + KZ_D1UV * nzp)); Z.d2uv = bc2(__ldg(kz + KZ_D2UV * nzp));
            Z.aw = bc2(__ldg(kz + KZ_AW * nzp)); Z.bw = bc2(__ldg(kz + KZ_BW * nzp));
            Z.d1w = bc2(__ldg(kz + KZ_D1W * nzp)); Z.d2w = bc2(__ldg(kz + KZ_D2W * nzp));
            gz2 = bc2((-coef) * __ldg(kz + KZ_RDZW * nzp));
            tu = tendency_dev<0, true>(K2, R2, O, bc2(0.f), &Z);
            tv = tendency_dev<1, true>(K2, R2, O, bc2(0.f), &Z);
            tw = tendency_dev<2, true>(K2, R2, O, btp, &Z);
          }
          const F2 rd = bc2(rdt), dd = bc2(dt), bd = bc2(bdt);
          const F2 zero = bc2(0.f);
          F2 u2 = stage1 ? zero : F2{*reinterpret_cast<const float2 *>(nar)} * rd * dd;
          F2 v2 = stage1 ? zero : F2{*reinterpret_cast<const float2 *>(nar + Lay::NB)} * rd * dd;
          F2 w2 = stage1 ? zero : F2{*reinterpret_cast<const float2 *>(nar + 2 * Lay::NB)} * rd * dd;
          u2 = u2 + tu * bd * dd;
          if (prgx_on) u2 = u2 + bc2(fx);
          u2 = u2 + bc2(gx) * ((R2.g(4, 1, 0, 0) - mm) - p0);
          u2 = u2 + R2.g(0, 0, 0, 0);
          v2 = v2 + tv * bd * dd;
          if (prgy_on) v2 = v2 + bc2(fy);
          v2 = v2 + bc2(gy) * ((R2.g(4, 0, 1, 0) - mm) - p0);
          v2 = v2 + R2.g(1, 0, 0, 0);
          w2 = w2 + tw * bd * dd;
          w2 = w2 + gz2 * ((R2.g(4, 0, 0, 1) - mm) - p0);
          w2 = w2 + R2.g(2, 0, 0, 0);
          *reinterpret_cast<float2 *>(Us + c) = tu.v;
          *reinterpret_cast<float2 *>(U2o + c) = u2.v;
          *reinterpret_cast<float2 *>(Vs + c) = tv.v;
          *reinterpret_cast<float2 *>(V2o + c) = v2.v;
          *reinterpret_cast<float2 *>(Ws + c) = tw.v;
          *reinterpret_cast<float2 *>(W2o + c) = w2.v;
        }
      } else if (ok) {
#pragma unroll
        for (int q = 0; q < CPT; q++) {
          const int iq = i + q;
          if (!(iq <= nx && j <= ny)) continue;
          WideRing<T, 5, 3> R;
          R.p[0] = p0s; R.p[1] = p1s; R.p[2] = p2s;
          R.o = o + q;
          const T *nar = p1s + Lay::WIDE + ty * MX + CPT * tx + q;  // narrow blocks are NB apart
          const long long cq = c + q;
          const T p0 = R.g(4, 0, 0, 0) - m;
          // all shared-memory reads first, then the stores: a global store in
          // between would make the compiler reload every shared value it may
          // alias
          const bool doU = iq <= d.ext[0][0] && j <= d.ext[0][1] && k <= kU;
          const bool doV = iq <= d.ext[1][0] && j <= d.ext[1][1] && k <= kV;
          const bool doW = iq <= d.ext[2][0] && j <= d.ext[2][1] && k <= kW;
          T bt = (T)0;
          if (buoy && doW) {
            if constexpr (NNF == 4) {  // the temperature of planes k+1 and k from the ring
              const int ot = Lay::WIDE + 3 * Lay::NB + ty * MX + CPT * tx + q;
              bt = bA2 * (p2s[ot] + p1s[ot]);
            } else {
              bt = bA2 * (ld(Tm, cq + plane) + ld(Tm, cq));
            }
          }
          T tu, tv, tw;
          if constexpr (sizeof(T) == 4) {
            // mixed path: the deviation forms of tendency_dev plus the wall
            // corrections of wall_dev (U and V are stored as deviations)
            VelOffN<float> O;
#pragma unroll
            for (int q3 = 0; q3 < 3; q3++) { O.o[q3] = soff[0][k - k0 + q3]; O.p[q3] = soff[1][k - k0 + q3]; }
            MomKN<float> K1;
            K1.Ax = ctx.cA[0]; K1.Ay = ctx.cA[1]; K1.Az = ctx.cA[2];
            K1.rx = ctx.rec2[0]; K1.ry = ctx.rec2[1]; K1.rz = ctx.rec2[2];
            K1.q = 0.25f;
            for (int c3 = 0; c3 < 3; c3++)
              for (int a3 = 0; a3 < 3; a3++) K1.B[c3][a3] = ctx.cB[c3][a3];
            KZN<float> Z1;
            if (vz) {
              const int nzp = nz + 2;
              const float *kz = d.kz2 + k;
              Z1.auv = __ldg(kz + KZ_AUV * nzp); Z1.buv = __ldg(kz + KZ_BUV * nzp);
              Z1.d1uv = __ldg(kz + KZ_D1UV * nzp); Z1.d2uv = __ldg(kz + KZ_D2UV * nzp);
              Z1.aw = __ldg(kz + KZ_AW * nzp); Z1.bw = __ldg(kz + KZ_BW * nzp);
              Z1.d1w = __ldg(kz + KZ_D1W * nzp); Z1.d2w = __ldg(kz + KZ_D2W * nzp);
            }
            auto td = [&](auto cc) -> float {
              constexpr int CC = decltype(cc)::value;
              const float b3 = CC == 2 ? bt : 0.f;
              float a3 = vz ? tendency_dev<CC, true>(K1, R, O, b3, &Z1) : tendency_dev<CC, false>(K1, R, O, b3, &Z1);
              if (wallhere) a3 = a3 + wall_dev<CC>(ctx, R, O, iq, j, k);
              return a3;
            };
            tu = doU ? td(std::integral_constant<int, 0>{}) : 0.f;
            tv = doV ? td(std::integral_constant<int, 1>{}) : 0.f;
            tw = doW ? td(std::integral_constant<int, 2>{}) : 0.f;
          } else {
            tu = doU ? tendency<T, 0>(ctx, R, iq, j, k, wallhere) : (T)0;
            tv = doV ? tendency<T, 1>(ctx, R, iq, j, k, wallhere) : (T)0;
            tw = doW ? tendency<T, 2>(ctx, R, iq, j, k, wallhere, bt, bsub) : (T)0;
          }
          T u2 = stage1 ? (T)0 : nar[0] * rdt * dt;
          T v2 = stage1 ? (T)0 : nar[Lay::NB] * rdt * dt;
          T w2 = stage1 ? (T)0 : nar[2 * Lay::NB] * rdt * dt;
          u2 = u2 + tu * bdt * dt;
          if (prgx_on) u2 = u2 + fx;
          u2 = u2 + gx * ((R.g(4, 1, 0, 0) - m) - p0);
          u2 = u2 + R.g(0, 0, 0, 0);
          v2 = v2 + tv * bdt * dt;
          if (prgy_on) v2 = v2 + fy;
          v2 = v2 + gy * ((R.g(4, 0, 1, 0) - m) - p0);
          v2 = v2 + R.g(1, 0, 0, 0);
          w2 = w2 + tw * bdt * dt;
          const T dpz = (R.g(4, 0, 0, 1) - m) - p0;
          if (vz) w2 = w2 - coef * dpz / (T)dzW[k + 2];
          else w2 = w2 + gz * dpz;
          w2 = w2 + R.g(2, 0, 0, 0);
          if (doU) { Us[cq] = tu; U2o[cq] = u2; }
          if (doV) { Vs[cq] = tv; V2o[cq] = v2; }
          if (doW) { Ws[cq] = tw; W2o[cq] = w2; }
        }
      }
      __syncthreads();  // plane k-1 is no longer read
      if (abort_flag) {
        // a plane did not arrive: wait (bounded) for the copies still in
        // flight into this block's shared memory, then give up
        if (threadIdx.x == 0)
          for (int kk = k + 2; kk <= min(k - 1 + NSL - 1, k1 + 1); kk++) {
            const int s2 = kk % NSL;
            if (kk != d.skip_plane) mbar_wait(&bars[s2], (phase >> s2) & 1u);  // issued copies land: the full limit
            phase ^= 1u << s2;
          }
        return;
      }
      const int kn = k - 1 + NSL;
      if (threadIdx.x == 0 && kn <= k1 + 1 && kn != d.skip_plane) {
        fence_async_shared();
        issue_mom_plane<T, NNF>(ring + (kn % NSL) * Lay::SIZE, &bars[kn % NSL], maps, tmapT, !stage1, d.aln, i0, j0,
                                kn);
      }
      c += plane;
    }
  }
}

// ---------------------------------------------------------------- k_sgs
// SubgridStresses (src/dynamics.f90:869-908): Smagorinsky viscosity
// (SGS_Smag / NuSmag / StrainIJ, src/subgrid.f90:30-67, :170-209) from a
// ring of U, V, W planes (the ghosts of BoundViscosity,
// src/scalarboundaries.f90:326-431, are filled afterwards by k_ghosts).
// Cells next to a wall-model side compute the wall fluxes of the velocity
// points there.
template <typename T>
struct SgsK {  // factors of NuSmag at one level k
  T rdx, rdy, r4dx, r4dy, rdz, r2zz, wc2;
  // mixed path: the part of the z differences of U and V (D02, D12) that
  // comes from their per-level offsets, 2 (off(k+1) - off(k-1)) r2zz, in
  // shared memory per plane of the tile (the ring holds the stored
  // deviations; every other difference is taken within one level, where the
  // offset cancels)
  const float *du, *dv;
};

// The divisions by the (uniform) spacings of StrainIJ are multiplications by
// reciprocals computed once, which changes the result by at most one
// rounding; the sum of squares keeps the order of Strainu.
template <typename T, typename RT>
__device__ __forceinline__ T nusmag_ring(const SgsK<T> &q, const RT &R) {
#define GU(dx, dy, dz) R.g(0, dx, dy, dz)
#define GV(dx, dy, dz) R.g(1, dx, dy, dz)
#define GW(dx, dy, dz) R.g(2, dx, dy, dz)
  T D00 = (GU(0, 0, 0) - GU(-1, 0, 0)) * q.rdx;
  T D11 = (GV(0, 0, 0) - GV(0, -1, 0)) * q.rdy;
  T D22 = (GW(0, 0, 0) - GW(0, 0, -1)) * q.rdz;
  T D01 = (GU(0, 1, 0) + GU(-1, 1, 0) - GU(0, -1, 0) - GU(-1, -1, 0)) * q.r4dy;
  T D02 = (GU(0, 0, 1) + GU(-1, 0, 1) - GU(0, 0, -1) - GU(-1, 0, -1)) * q.r2zz;
  T D10 = (GV(1, 0, 0) + GV(1, -1, 0) - GV(-1, 0, 0) - GV(-1, -1, 0)) * q.r4dx;
  T D12 = (GV(0, 0, 1) + GV(0, -1, 1) - GV(0, 0, -1) - GV(0, -1, -1)) * q.r2zz;
  if constexpr (sizeof(T) == 4) {
    D02 = D02 + *q.du;
    D12 = D12 + *q.dv;
  }
  T D20 = (GW(1, 0, 0) + GW(1, 0, -1) - GW(-1, 0, 0) - GW(-1, 0, -1)) * q.r4dx;
  T D21 = (GW(0, 1, 0) + GW(0, 1, -1) - GW(0, -1, 0) - GW(0, -1, -1)) * q.r4dy;
#undef GU
#undef GV
#undef GW
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
  return Sbar * q.wc2;
}

// nusmag_ring for a pair of x-adjacent cells with packed FP32x2 arithmetic;
// the square root is taken per cell
template <typename RT>
__device__ __forceinline__ F2 nusmag2(const SgsK<float> &q, const RT &R) {
#define GU(dx, dy, dz) R.g(0, dx, dy, dz)
#define GV(dx, dy, dz) R.g(1, dx, dy, dz)
#define GW(dx, dy, dz) R.g(2, dx, dy, dz)
  const F2 rdx = bc2(q.rdx), rdy = bc2(q.rdy), rdz = bc2(q.rdz), r4dx = bc2(q.r4dx), r4dy = bc2(q.r4dy),
           r2zz = bc2(q.r2zz), half = bc2(0.5f);
  const F2 D00 = (GU(0, 0, 0) - GU(-1, 0, 0)) * rdx;
  const F2 D11 = (GV(0, 0, 0) - GV(0, -1, 0)) * rdy;
  const F2 D22 = (GW(0, 0, 0) - GW(0, 0, -1)) * rdz;
  const F2 D01 = (((GU(0, 1, 0) + GU(-1, 1, 0)) - GU(0, -1, 0)) - GU(-1, -1, 0)) * r4dy;
  const F2 D02 = (((GU(0, 0, 1) + GU(-1, 0, 1)) - GU(0, 0, -1)) - GU(-1, 0, -1)) * r2zz + bc2(*q.du);
  const F2 D10 = (((GV(1, 0, 0) + GV(1, -1, 0)) - GV(-1, 0, 0)) - GV(-1, -1, 0)) * r4dx;
  const F2 D12 = (((GV(0, 0, 1) + GV(0, -1, 1)) - GV(0, 0, -1)) - GV(0, -1, -1)) * r2zz + bc2(*q.dv);
  const F2 D20 = (((GW(1, 0, 0) + GW(1, 0, -1)) - GW(-1, 0, 0)) - GW(-1, 0, -1)) * r4dx;
  const F2 D21 = (((GW(0, 1, 0) + GW(0, 1, -1)) - GW(0, -1, 0)) - GW(0, -1, -1)) * r4dy;
#undef GU
#undef GV
#undef GW
  F2 s, S = bc2(0.f);
  s = (D00 + D00) * half; S = S + s * s;
  s = (D10 + D01) * half; S = S + s * s;
  s = (D20 + D02) * half; S = S + s * s;
  s = (D01 + D10) * half; S = S + s * s;
  s = (D11 + D11) * half; S = S + s * s;
  s = (D21 + D12) * half; S = S + s * s;
  s = (D02 + D20) * half; S = S + s * s;
  s = (D12 + D21) * half; S = S + s * s;
  s = (D22 + D22) * half; S = S + s * s;
  const F2 Sbar{make_float2(sqrtf(2.f * S.v.x), sqrtf(2.f * S.v.y))};
  return Sbar * bc2(q.wc2);
}


// ComputeTDiff (src/scalar_diffusion.f90:983-1009): the temperature
// diffusivity from the viscosity, constant Pr_sgs = 0.6
// (src/scalar_diffusion.f90:22)
template <typename T>
__device__ __forceinline__ T tdiff_of(T nu, T nu_mol, T kappa_mol) {
  return nu_mol > 0 ? (nu - nu_mol) / (T)0.6 + kappa_mol : nu / (T)0.6;
}

// Cells per thread of k_sgs: two for FP32 (packed arithmetic), one for FP64.
template <typename T>
struct SgsShape {
  static constexpr int cpt = 1, threads = MX * MY, min_blocks = 3;
};
template <>
struct SgsShape<float> {
  static constexpr int cpt = 2, threads = MX * MY / 2, min_blocks = 7;
};

// init: 0 a stage (viscosity and diffusivity), 1 the initial viscosity and
// diffusivity after the projection, 2 the autotuner's timing launches (a
// stage's arithmetic; its outputs the real stage overwrites).  The
// wall-model points are k_wm_points'.
template <typename T, int KC = MKC>
__global__ void __launch_bounds__(SgsShape<T>::threads, SgsShape<T>::min_blocks)
    k_sgs(const Dom<T> *__restrict__ doms, Launch L, int init) {
  // planes of U, V, W (tile plus one-cell halo) arrive by tensor-map TMA in
  // a ring of kRingSlots slots, as in k_momentum
  typedef SlotLayout<T, 3, 0> Lay;
  constexpr int CPT = SgsShape<T>::cpt, TXN = MX / CPT;
  extern __shared__ __align__(128) unsigned char dyn_smem[];
  T *ring = reinterpret_cast<T *>(dyn_smem);
  __shared__ __align__(8) uint64_t bars[kRingSlots];
  __shared__ int abort_flag;
  // mixed path: the z-difference parts du, dv of the tile's planes (SgsK)
  __shared__ float sdz[2][KC];
  const int tx = threadIdx.x % TXN, ty = threadIdx.x / TXN;
  if (smem_addr(ring) & 127u) {  // tensor copies need 128-byte aligned destinations
    if (threadIdx.x == 0) doms[0].flags[1] = 1;
    return;
  }
  if (threadIdx.x == 0) {
    for (int s2 = 0; s2 < kRingSlots; s2++) mbar_init(&bars[s2], 1);
    abort_flag = 0;
    fence_async_shared();
  }
  __syncthreads();
  uint32_t phase = 0;  // bit s: parity of the next wait on slot s
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    int lt = t - __ldg(L.starts + di);
    const int ntx = (d.nx + MX - 1) / MX, nty = (d.ny + MY - 1) / MY;
    const int bx = lt % ntx; lt /= ntx;
    const int by = lt % nty;
    const int bk = lt / nty;
    const int i0 = bx * MX + 1, j0 = by * MY + 1, k0 = bk * KC + 1;
    const int k1 = min(k0 + KC - 1, d.nz);
    const int i = i0 + CPT * tx, j = j0 + ty;  // the thread's first cell
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const int wide[3] = {F_U, F_V, F_W};
    const int none[1] = {0};
    const CUtensorMap *maps = reinterpret_cast<const CUtensorMap *>(d.tmaps);
    __syncthreads();  // every slot and the z-difference parts of the previous tile are free
    if constexpr (sizeof(T) == 4) {
      if (threadIdx.x < 2 * KC) {
        const int c = threadIdx.x / KC, kk = k0 + threadIdx.x % KC;
        if (kk <= k1) {
          const float *o = d.voff + c * (d.nz + 2);
          sdz[c][kk - k0] = 2.f * (__ldg(o + kk + 1) - __ldg(o + kk - 1)) * (float)d.sgs_r2zz[kk];
        }
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      fence_async_shared();
      for (int kk = k0 - 1; kk <= min(k0 - 1 + kRingSlots - 1, k1 + 1); kk++)
        if (kk != d.skip_plane)
          issue_plane<T, 3, 0>(ring + (kk % kRingSlots) * Lay::SIZE, &bars[kk % kRingSlots], maps, wide, none, false,
                               d.aln, i0, j0, kk);
    }
    const T num = (T)d.nu_mol;
    const bool sgs = d.sgs != 0, addmol = d.nu_mol > 0;
    // the scalar diffusivity too: every stage with buoyancy (ComputeTDiff,
    // src/dynamics.f90:904), and once after the initial projection whenever
    // a scalar is transported (src/initial.f90:4296-4313, which uses the
    // first formula of ComputeTDiff for any molecular viscosity)
    const bool buoy = d.tdiff_live != 0 || (init == 1 && d.nslot > 0);
    const T kap = (T)d.kappa_mol;
    SgsK<T> q;
    q.rdx = (T)(1.0 / d.dx); q.rdy = (T)(1.0 / d.dy);
    q.r4dx = (T)(1.0 / (4 * d.dx)); q.r4dy = (T)(1.0 / (4 * d.dy));
    const double *tr = d.sgs_rdz, *t2 = d.sgs_r2zz, *tw = d.sgs_wc2;
    T *__restrict__ nu = d.nu;
    const int o = (ty + 1) * Lay::SPW + (CPT * tx + Lay::XO);
    const bool inside0 = i <= nx && j <= ny;
    const bool pair_inside = i + CPT - 1 <= nx && j <= ny;
    long long c = bidx(d, inside0 ? i : 1, inside0 ? j : 1, k0);
    const long long plane = d.plane;
    for (int k = k0; k <= k1; k++) {
      q.rdz = (T)tr[k]; q.r2zz = (T)t2[k]; q.wc2 = (T)tw[k];
      q.du = &sdz[0][k - k0];
      q.dv = &sdz[1][k - k0];
      // planes k-1, k, k+1 must have landed
      bool ok = true;
      for (int kk = (k == k0 ? k0 - 1 : k + 1); kk <= k + 1; kk++) {
        const int s2 = kk % kRingSlots;
        bool w = mbar_wait(&bars[s2], (phase >> s2) & 1u, d.wait_limit);
        // a plane whose copies were issued always lands before the block
        // moves on or gives up (so no copy into this block's shared memory
        // outlives it): a lowered limit only cuts the wait on a skipped one
        if (!w && kk != d.skip_plane) w = mbar_wait(&bars[s2], (phase >> s2) & 1u);
        ok &= w;
        phase ^= 1u << s2;
      }
      if (!ok) { abort_flag = 1; d.flags[1] = 1; }
      const T *p0s = ring + ((k - 1) % kRingSlots) * Lay::SIZE, *p1s = ring + (k % kRingSlots) * Lay::SIZE,
              *p2s = ring + ((k + 1) % kRingSlots) * Lay::SIZE;
      if (ok && CPT == 2 && sgs && pair_inside) {
        if constexpr (CPT == 2) {
          Ring2<Lay::WB, Lay::SPW> R2;
          R2.p[0] = p0s; R2.p[1] = p1s; R2.p[2] = p2s;
          R2.o = o;
          F2 v = nusmag2(q, R2);
          if (addmol) v = v + bc2(num);
          *reinterpret_cast<float2 *>(nu + c) = v.v;
          // the periodic x ghosts of the row's end cells (the ghost pass covers y and z)
          if (i == 1) nu[c + nx] = v.v.x;
          if (i + 1 == nx) nu[c + 1 - nx] = v.v.y;
          if (buoy) {
            const float2 td = init == 1 ? make_float2((v.v.x - num) / 0.6f + kap, (v.v.y - num) / 0.6f + kap)
                                   : make_float2(tdiff_of(v.v.x, num, kap), tdiff_of(v.v.y, num, kap));
            *reinterpret_cast<float2 *>(d.TDiff + c) = td;
          }
        }
      } else if (ok) {
#pragma unroll
        for (int qc = 0; qc < CPT; qc++) {
          if (!(i + qc <= nx && j <= ny)) continue;
          WideRing<T, 3, 0> R;
          R.p[0] = p0s; R.p[1] = p1s; R.p[2] = p2s;
          R.o = o + qc;
          T v = num;
          if (sgs) {
            v = nusmag_ring(q, R);
            if (addmol) v = v + num;
          }
          nu[c + qc] = v;
          if (i + qc == 1) nu[c + qc + nx] = v;  // periodic x ghosts (the ghost pass covers y and z)
          if (i + qc == nx) nu[c + qc - nx] = v;
          if (buoy) d.TDiff[c + qc] = init == 1 ? (v - num) / (T)0.6 + kap : tdiff_of(v, num, kap);
        }
      }
      __syncthreads();  // plane k-1 is no longer read
      if (abort_flag) {
        // a plane did not arrive: wait (bounded) for the copies still in
        // flight into this block's shared memory, then give up
        if (threadIdx.x == 0)
          for (int kk = k + 2; kk <= min(k - 1 + kRingSlots - 1, k1 + 1); kk++) {
            const int s2 = kk % kRingSlots;
            if (kk != d.skip_plane) mbar_wait(&bars[s2], (phase >> s2) & 1u);  // issued copies land: the full limit
            phase ^= 1u << s2;
          }
        return;
      }
      const int kn = k - 1 + kRingSlots;
      if (threadIdx.x == 0 && kn <= k1 + 1 && kn != d.skip_plane) {
        fence_async_shared();
        issue_plane<T, 3, 0>(ring + (kn % kRingSlots) * Lay::SIZE, &bars[kn % kRingSlots], maps, wide, none, false,
                             d.aln, i0, j0, kn);
      }
      c += plane;
    }
  }
}

}  // namespace elmm
