// elmm_packed.cuh -- packed FP32x2 arithmetic (sm_100 FFMA2 / FADD2 / FMUL2)
// for the mixed-precision momentum kernel: one thread computes two
// x-adjacent cells with one instruction per operation pair.
//
// tendency2<C> is the wall-free form of tendency<float, C> (elmm_momentum.cuh)
// with the same operations in the same order on a uniform grid; on a
// stretched z grid (VZ) the z terms use per-level factors (below).  Tiles
// with wall-model corrections use the scalar code.
#pragma once

#include <cuda_runtime.h>

namespace elmm {

struct F2 {
  float2 v;
};

__device__ __forceinline__ F2 bc2(float a) { return F2{make_float2(a, a)}; }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2{__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2{__fmul2_rn(a.v, b.v)}; }
// a - b: the product b * (-1) is exact, so this is one rounding of a - b
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2{__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)}; }
__device__ __forceinline__ F2 neg2(F2 a) { return F2{__fmul2_rn(a.v, make_float2(-1.f, -1.f))}; }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return F2{__ffma2_rn(a.v, b.v, c.v)}; }

// Pair accessor over the momentum plane ring: the thread's two cells sit at
// o and o + 1 of a slot (o even, so pairs at even offsets are 8-byte
// aligned); a pair at an odd x offset is assembled from its two aligned
// neighbours.
template <int WB, int SPW>
struct Ring2 {
  const float *__restrict__ p[3];  // planes k-1, k, k+1
  int o;
  __device__ __forceinline__ float2 ld(const float *q) const { return *reinterpret_cast<const float2 *>(q); }
  __device__ __forceinline__ F2 g(int f, int dx, int dy, int dz) const {
    const float *b = p[dz + 1] + f * WB + o + dy * SPW;
    if ((dx & 1) == 0) return F2{ld(b + dx)};
    const float2 lo = ld(b + dx - 1), hi = ld(b + dx + 1);
    return F2{make_float2(lo.y, hi.x)};
  }
};

// per-tile constants of the packed path, broadcast to pairs
struct MomK2 {
  F2 Ax, Ay, Az, rx, ry, rz, q;  // cA, rec2, 0.25
  F2 B[3][3];                    // cB
};

// Stretched z (CDU/CDV/CDW_variable_z, src/advection_variable_z.f90:15-324,
// and MomentumDiffusion_variable_z_nobranch_2ord, src/momentum_diffusion.f90:
// 298-420): the divisions by dzPr(k), dzW(k) and the centred differences of
// zPr, zW become multiplications by per-level factors computed once in FP64
// and rounded to FP32 (one rounding where the reference's form has two).
// Table rows of Dom::kz2:
enum {
  KZ_AUV = 0,   // 1 / (4 dzPr(k))                    U, V advection through z faces
  KZ_BUV = 1,   // 1 / (4 (zPr(k+1) - zPr(k-1)))       U, V advective form, W averaged over 4
  KZ_D1UV = 2,  // 1 / (dzW(k) dzPr(k))                U, V diffusion through the top face
  KZ_D2UV = 3,  // 1 / (dzW(k-1) dzPr(k))              ... the bottom face
  KZ_AW = 4,    // 1 / (4 dzW(k))                      W advection
  KZ_BW = 5,    // 1 / (zW(k+1) - zW(k-1))             W advective form
  KZ_D1W = 6,   // 1 / (dzPr(k+1) dzW(k))              W diffusion, top
  KZ_D2W = 7,   // 1 / (dzPr(k) dzW(k))                W diffusion, bottom
  KZ_RDZW = 8,  // 1 / dzW(k)                          pressure gradient of W
  kZ2 = 9
};
struct KZ2 {
  F2 auv, buv, d1uv, d2uv, aw, bw, d1w, d2w;
};

template <int C, bool VZ = false, typename RT>
__device__ __forceinline__ F2 tendency2(const MomK2 &K, const RT &R, F2 bt = F2{make_float2(0.f, 0.f)},
                                        const KZ2 *Z = nullptr) {
#define FU(dx, dy, dz) R.g(0, dx, dy, dz)
#define FV(dx, dy, dz) R.g(1, dx, dy, dz)
#define FW(dx, dy, dz) R.g(2, dx, dy, dz)
#define FN(dx, dy, dz) R.g(3, dx, dy, dz)
  F2 a;
  if (C == 0) {
    const F2 u = FU(0, 0, 0), ue = FU(1, 0, 0), uw = FU(-1, 0, 0), un = FU(0, 1, 0), us = FU(0, -1, 0);
    const F2 ut = FU(0, 0, 1), ub = FU(0, 0, -1);
    const F2 v = FV(0, 0, 0), ve = FV(1, 0, 0), vs = FV(0, -1, 0), vse = FV(1, -1, 0);
    const F2 w = FW(0, 0, 0), we = FW(1, 0, 0), wb = FW(0, 0, -1), wbe = FW(1, 0, -1);
    const F2 Bx = K.B[0][0], By = K.B[0][1], Bz = K.B[0][2];
    if (!VZ) {
      a = neg2(((K.Ax * (ue + u) * (ue + u) - K.Ax * (u + uw) * (u + uw)) +
                (K.Ay * (un + u) * (ve + v) - K.Ay * (u + us) * (vse + vs))) +
               (K.Az * (ut + u) * (we + w) - K.Az * (u + ub) * (wbe + wb)));
    } else {
      a = neg2(((K.Ax * (ue + u) * (ue + u) - K.Ax * (u + uw) * (u + uw)) +
                (K.Ay * (un + u) * (ve + v) - K.Ay * (u + us) * (vse + vs))) +
               ((ut + u) * (we + w) - (u + ub) * (wbe + wb)) * Z->auv);
    }
    const F2 Vadv = ((v + ve) + vs) + vse;
    const F2 Wadv = ((w + we) + wb) + wbe;
    if (!VZ) a = a - ((Bx * (ue - uw) * u + By * (un - us) * Vadv) + Bz * (ut - ub) * Wadv);
    else a = a - ((Bx * (ue - uw) * u + By * (un - us) * Vadv) + (ut - ub) * Z->buv * Wadv);
    a = a * bc2(0.5f);
    const F2 n0 = FN(0, 0, 0), ne = FN(1, 0, 0), nn = FN(0, 1, 0), nne = FN(1, 1, 0), ns = FN(0, -1, 0);
    const F2 nse = FN(1, -1, 0), nt = FN(0, 0, 1), nte = FN(1, 0, 1), nb = FN(0, 0, -1), nbe = FN(1, 0, -1);
    a = a + ne * (ue - u) * K.rx;
    a = a - n0 * (u - uw) * K.rx;
    a = a + K.q * (((nne + ne) + nn) + n0) * (un - u) * K.ry;
    a = a - K.q * (((ne + nse) + n0) + ns) * (u - us) * K.ry;
    if (!VZ) {
      a = a + K.q * (((nte + ne) + nt) + n0) * (ut - u) * K.rz;
      a = a - K.q * (((ne + nbe) + n0) + nb) * (u - ub) * K.rz;
    } else {
      a = a + K.q * (((nte + ne) + nt) + n0) * (ut - u) * Z->d1uv;
      a = a - K.q * (((ne + nbe) + n0) + nb) * (u - ub) * Z->d2uv;
    }
  } else if (C == 1) {
    const F2 v = FV(0, 0, 0), ve = FV(1, 0, 0), vw = FV(-1, 0, 0), vn = FV(0, 1, 0), vs = FV(0, -1, 0);
    const F2 vt = FV(0, 0, 1), vb = FV(0, 0, -1);
    const F2 u = FU(0, 0, 0), un = FU(0, 1, 0), uw = FU(-1, 0, 0), unw = FU(-1, 1, 0);
    const F2 w = FW(0, 0, 0), wn = FW(0, 1, 0), wb = FW(0, 0, -1), wbn = FW(0, 1, -1);
    const F2 Bx = K.B[1][0], By = K.B[1][1], Bz = K.B[1][2];
    if (!VZ) {
      a = neg2(((K.Ay * (vn + v) * (vn + v) - K.Ay * (v + vs) * (v + vs)) +
                (K.Ax * (ve + v) * (un + u) - K.Ax * (v + vw) * (unw + uw))) +
               (K.Az * (vt + v) * (wn + w) - K.Az * (v + vb) * (wbn + wb)));
    } else {
      a = neg2(((K.Ay * (vn + v) * (vn + v) - K.Ay * (v + vs) * (v + vs)) +
                (K.Ax * (ve + v) * (un + u) - K.Ax * (v + vw) * (unw + uw))) +
               ((vt + v) * (wn + w) - (v + vb) * (wbn + wb)) * Z->auv);
    }
    const F2 Uadv = ((u + un) + uw) + unw;
    const F2 Wadv = ((w + wn) + wb) + wbn;
    if (!VZ) a = a - ((Bx * (ve - vw) * Uadv + By * (vn - vs) * v) + Bz * (vt - vb) * Wadv);
    else a = a - ((Bx * (ve - vw) * Uadv + By * (vn - vs) * v) + (vt - vb) * Z->buv * Wadv);
    a = a * bc2(0.5f);
    const F2 n0 = FN(0, 0, 0), ne = FN(1, 0, 0), nn = FN(0, 1, 0), nne = FN(1, 1, 0), nw = FN(-1, 0, 0);
    const F2 nnw = FN(-1, 1, 0), nt = FN(0, 0, 1), nnt = FN(0, 1, 1), nb = FN(0, 0, -1), nnb = FN(0, 1, -1);
    a = a + K.q * (((nne + ne) + nn) + n0) * (ve - v) * K.rx;
    a = a - K.q * (((nn + n0) + nnw) + nw) * (v - vw) * K.rx;
    a = a + nn * (vn - v) * K.ry;
    a = a - n0 * (v - vs) * K.ry;
    if (!VZ) {
      a = a + K.q * (((nnt + nn) + nt) + n0) * (vt - v) * K.rz;
      a = a - K.q * (((nn + nnb) + n0) + nb) * (v - vb) * K.rz;
    } else {
      a = a + K.q * (((nnt + nn) + nt) + n0) * (vt - v) * Z->d1uv;
      a = a - K.q * (((nn + nnb) + n0) + nb) * (v - vb) * Z->d2uv;
    }
  } else {
    const F2 w = FW(0, 0, 0), we = FW(1, 0, 0), ww = FW(-1, 0, 0), wn = FW(0, 1, 0), ws = FW(0, -1, 0);
    const F2 wt = FW(0, 0, 1), wb = FW(0, 0, -1);
    const F2 u = FU(0, 0, 0), ut = FU(0, 0, 1), uw = FU(-1, 0, 0), utw = FU(-1, 0, 1);
    const F2 v = FV(0, 0, 0), vt = FV(0, 0, 1), vs = FV(0, -1, 0), vts = FV(0, -1, 1);
    const F2 Bx = K.B[2][0], By = K.B[2][1], Bz = K.B[2][2];
    if (!VZ) {
      a = neg2(((K.Az * (wt + w) * (wt + w) - K.Az * (w + wb) * (w + wb)) +
                (K.Ay * (wn + w) * (vt + v) - K.Ay * (w + ws) * (vs + vts))) +
               (K.Ax * (we + w) * (ut + u) - K.Ax * (w + ww) * (utw + uw)));
    } else {
      a = neg2((((wt + w) * (wt + w) - (w + wb) * (w + wb)) * Z->aw +
                (K.Ay * (wn + w) * (vt + v) - K.Ay * (w + ws) * (vts + vs))) +
               (K.Ax * (we + w) * (ut + u) - K.Ax * (w + ww) * (utw + uw)));
    }
    const F2 Uadv = ((u + ut) + uw) + utw;
    const F2 Vadv = ((v + vt) + vs) + vts;
    if (!VZ) a = a - ((Bx * (we - ww) * Uadv + By * (wn - ws) * Vadv) + Bz * (wt - wb) * w);
    else a = a - ((Bx * (we - ww) * Uadv + By * (wn - ws) * Vadv) + (wt - wb) * Z->bw * w);
    a = a * bc2(0.5f);
    a = a + bt;  // buoyancy (the mixed path stores theta - temperature_ref)
    const F2 n0 = FN(0, 0, 0), ne = FN(1, 0, 0), nt = FN(0, 0, 1), nte = FN(1, 0, 1), nw = FN(-1, 0, 0);
    const F2 ntw = FN(-1, 0, 1), nn = FN(0, 1, 0), ntn = FN(0, 1, 1), ns = FN(0, -1, 0), nts = FN(0, -1, 1);
    a = a + K.q * (((nte + ne) + nt) + n0) * (we - w) * K.rx;
    a = a - K.q * (((nt + n0) + ntw) + nw) * (w - ww) * K.rx;
    a = a + K.q * (((ntn + nt) + nn) + n0) * (wn - w) * K.ry;
    a = a - K.q * (((nt + nts) + n0) + ns) * (w - ws) * K.ry;
    if (!VZ) {
      a = a + nt * (wt - w) * K.rz;
      a = a - n0 * (w - wb) * K.rz;
    } else {
      a = a + nt * (wt - w) * Z->d1w;
      a = a - n0 * (w - wb) * Z->d2w;
    }
  }
#undef FU
#undef FV
#undef FW
#undef FN
  return a;
}

}  // namespace elmm
