// elmm_packed.cuh -- packed FP32x2 arithmetic (sm_100 FFMA2 / FADD2 / FMUL2)
// for the mixed-precision momentum kernel: one thread computes two
// x-adjacent cells with one instruction per operation pair.
//
// tendency_dev<C> is the wall-free tendency of the mixed path, for one cell
// (float) or a pair (F2); on a stretched z grid (VZ) the z terms use
// per-level factors (below).  Tiles with wall-model corrections use the
// per-cell code.
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

// Arithmetic on one value (float) or on a pair (F2) in the same source.
__device__ __forceinline__ float cst(float a, float) { return a; }
__device__ __forceinline__ F2 cst(float a, F2) { return bc2(a); }

// per-tile constants of the FP32 tendencies (float for one cell, F2 broadcast
// to a pair)
template <typename N>
struct MomKN {
  N Ax, Ay, Az, rx, ry, rz, q;  // cA, rec2, 0.25
  N B[3][3];                    // cB
};
typedef MomKN<F2> MomK2;

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
template <typename N>
struct KZN {
  N auv, buv, d1uv, d2uv, aw, bw, d1w, d2w;
};
typedef KZN<F2> KZ2;

// The per-level offsets of U (o) and V (p) on planes k-1, k, k+1 (the mixed
// path stores U and V as deviations from them; see Dom::voff).
template <typename N>
struct VelOffN {
  N o[3], p[3];
};

// One velocity component's tendency on the mixed path without wall
// corrections: the skew-symmetric CDS2 advection (advection.f90:15-327,
// advection_variable_z.f90:15-324 with VZ) and the explicit diffusion
// (momentum_diffusion.f90:169-420) of the FP32 state, whose U and V hold
// deviations from per-level offsets.  R.g() returns stored values; the
// offsets enter only where the full value is needed, through algebraic
// identities that keep every difference of neighbouring values a difference
// of stored deviations:
//   (ue + u)^2 - (u + uw)^2 = (ue - uw)(ue + 2u + uw)                 (same level)
//   (A + 2o)(B + 2p) - (C + 2o)(D + 2p) = (AB - CD) + 2p (A - C) + 2o (B - D)
//   a value at level k+1 minus one at level k-1 = stored difference + (o1 - om)
// The forms are equal to the reference's term by term in exact arithmetic;
// in FP32 they avoid differences of rounded products of the full ~several m/s
// velocity, whose rounding noise the projection would otherwise turn into
// pressure.  bt: the buoyancy of W (theta stored as theta - T_ref).
template <int C, bool VZ, typename N, typename RT>
__device__ __forceinline__ N tendency_dev(const MomKN<N> &K, const RT &R, const VelOffN<N> &O, N bt,
                                          const KZN<N> *Z) {
#define FU(dx, dy, dz) R.g(0, dx, dy, dz)
#define FV(dx, dy, dz) R.g(1, dx, dy, dz)
#define FW(dx, dy, dz) R.g(2, dx, dy, dz)
#define FN(dx, dy, dz) R.g(3, dx, dy, dz)
  const N two = cst(2.f, N{}), four = cst(4.f, N{});
  N a;
  if (C == 0) {
    const N u = FU(0, 0, 0), ue = FU(1, 0, 0), uw = FU(-1, 0, 0), un = FU(0, 1, 0), us = FU(0, -1, 0);
    const N ut = FU(0, 0, 1), ub = FU(0, 0, -1);
    const N v = FV(0, 0, 0), ve = FV(1, 0, 0), vs = FV(0, -1, 0), vse = FV(1, -1, 0);
    const N w = FW(0, 0, 0), we = FW(1, 0, 0), wb = FW(0, 0, -1), wbe = FW(1, 0, -1);
    const N om = O.o[0], o0 = O.o[1], o1 = O.o[2], p0 = O.p[1];
    const N Bx = K.B[0][0], By = K.B[0][1], Bz = K.B[0][2];
    const N X1 = K.Ax * (ue - uw) * (((ue + u) + (u + uw)) + four * o0);
    const N A = un + u, B = ve + v, Cc = u + us, D = vse + vs;
    const N Y1 = K.Ay * (((A * B - Cc * D) + two * p0 * (un - us)) + two * o0 * (B - D));
    const N Z1v = ((ut + u) * (we + w) - (u + ub) * (wbe + wb)) + ((o1 + o0) * (we + w) - (o0 + om) * (wbe + wb));
    const N Z1 = VZ ? Z1v * Z->auv : K.Az * Z1v;
    a = cst(0.f, N{}) - ((X1 + Y1) + Z1);
    const N Vadv = (((v + ve) + vs) + vse) + four * p0;
    const N Wadv = ((w + we) + wb) + wbe;
    const N dzu = (ut - ub) + (o1 - om);
    a = a - ((Bx * (ue - uw) * (u + o0) + By * (un - us) * Vadv) + (VZ ? dzu * Z->buv * Wadv : Bz * dzu * Wadv));
    a = a * cst(0.5f, N{});
    const N n0 = FN(0, 0, 0), ne = FN(1, 0, 0), nn = FN(0, 1, 0), nne = FN(1, 1, 0), ns = FN(0, -1, 0);
    const N nse = FN(1, -1, 0), nt = FN(0, 0, 1), nte = FN(1, 0, 1), nb = FN(0, 0, -1), nbe = FN(1, 0, -1);
    a = a + ne * (ue - u) * K.rx;
    a = a - n0 * (u - uw) * K.rx;
    a = a + K.q * (((nne + ne) + nn) + n0) * (un - u) * K.ry;
    a = a - K.q * (((ne + nse) + n0) + ns) * (u - us) * K.ry;
    const N dt = (ut - u) + (o1 - o0), db = (u - ub) + (o0 - om);
    a = a + K.q * (((nte + ne) + nt) + n0) * dt * (VZ ? Z->d1uv : K.rz);
    a = a - K.q * (((ne + nbe) + n0) + nb) * db * (VZ ? Z->d2uv : K.rz);
  } else if (C == 1) {
    const N v = FV(0, 0, 0), ve = FV(1, 0, 0), vw = FV(-1, 0, 0), vn = FV(0, 1, 0), vs = FV(0, -1, 0);
    const N vt = FV(0, 0, 1), vb = FV(0, 0, -1);
    const N u = FU(0, 0, 0), un = FU(0, 1, 0), uw = FU(-1, 0, 0), unw = FU(-1, 1, 0);
    const N w = FW(0, 0, 0), wn = FW(0, 1, 0), wb = FW(0, 0, -1), wbn = FW(0, 1, -1);
    const N o0 = O.o[1], pm = O.p[0], p0 = O.p[1], p1 = O.p[2];
    const N Bx = K.B[1][0], By = K.B[1][1], Bz = K.B[1][2];
    const N Y1 = K.Ay * (vn - vs) * (((vn + v) + (v + vs)) + four * p0);
    const N A = ve + v, B = un + u, Cc = v + vw, D = unw + uw;
    const N X1 = K.Ax * (((A * B - Cc * D) + two * o0 * (ve - vw)) + two * p0 * (B - D));
    const N Z1v = ((vt + v) * (wn + w) - (v + vb) * (wbn + wb)) + ((p1 + p0) * (wn + w) - (p0 + pm) * (wbn + wb));
    const N Z1 = VZ ? Z1v * Z->auv : K.Az * Z1v;
    a = cst(0.f, N{}) - ((Y1 + X1) + Z1);
    const N Uadv = (((u + un) + uw) + unw) + four * o0;
    const N Wadv = ((w + wn) + wb) + wbn;
    const N dzv = (vt - vb) + (p1 - pm);
    a = a - ((Bx * (ve - vw) * Uadv + By * (vn - vs) * (v + p0)) + (VZ ? dzv * Z->buv * Wadv : Bz * dzv * Wadv));
    a = a * cst(0.5f, N{});
    const N n0 = FN(0, 0, 0), ne = FN(1, 0, 0), nn = FN(0, 1, 0), nne = FN(1, 1, 0), nw = FN(-1, 0, 0);
    const N nnw = FN(-1, 1, 0), nt = FN(0, 0, 1), nnt = FN(0, 1, 1), nb = FN(0, 0, -1), nnb = FN(0, 1, -1);
    a = a + K.q * (((nne + ne) + nn) + n0) * (ve - v) * K.rx;
    a = a - K.q * (((nn + n0) + nnw) + nw) * (v - vw) * K.rx;
    a = a + nn * (vn - v) * K.ry;
    a = a - n0 * (v - vs) * K.ry;
    const N dt = (vt - v) + (p1 - p0), db = (v - vb) + (p0 - pm);
    a = a + K.q * (((nnt + nn) + nt) + n0) * dt * (VZ ? Z->d1uv : K.rz);
    a = a - K.q * (((nn + nnb) + n0) + nb) * db * (VZ ? Z->d2uv : K.rz);
  } else {
    const N w = FW(0, 0, 0), we = FW(1, 0, 0), ww = FW(-1, 0, 0), wn = FW(0, 1, 0), ws = FW(0, -1, 0);
    const N wt = FW(0, 0, 1), wb = FW(0, 0, -1);
    const N u = FU(0, 0, 0), ut = FU(0, 0, 1), uw = FU(-1, 0, 0), utw = FU(-1, 0, 1);
    const N v = FV(0, 0, 0), vt = FV(0, 0, 1), vs = FV(0, -1, 0), vts = FV(0, -1, 1);
    const N o01 = O.o[1] + O.o[2], p01 = O.p[1] + O.p[2];
    const N Bx = K.B[2][0], By = K.B[2][1], Bz = K.B[2][2];
    const N Z1v = (wt + w) * (wt + w) - (w + wb) * (w + wb);
    const N Z1 = VZ ? Z1v * Z->aw : K.Az * Z1v;
    const N Y1 = K.Ay * (((wn + w) * (vt + v) - (w + ws) * (vs + vts)) + p01 * (wn - ws));
    const N X1 = K.Ax * (((we + w) * (ut + u) - (w + ww) * (utw + uw)) + o01 * (we - ww));
    a = cst(0.f, N{}) - ((Z1 + Y1) + X1);
    const N Uadv = (((u + ut) + uw) + utw) + two * o01;
    const N Vadv = (((v + vt) + vs) + vts) + two * p01;
    a = a - ((Bx * (we - ww) * Uadv + By * (wn - ws) * Vadv) + (VZ ? (wt - wb) * Z->bw * w : Bz * (wt - wb) * w));
    a = a * cst(0.5f, N{});
    a = a + bt;  // buoyancy (the mixed path stores theta - temperature_ref)
    const N n0 = FN(0, 0, 0), ne = FN(1, 0, 0), nt = FN(0, 0, 1), nte = FN(1, 0, 1), nw = FN(-1, 0, 0);
    const N ntw = FN(-1, 0, 1), nn = FN(0, 1, 0), ntn = FN(0, 1, 1), ns = FN(0, -1, 0), nts = FN(0, -1, 1);
    a = a + K.q * (((nte + ne) + nt) + n0) * (we - w) * K.rx;
    a = a - K.q * (((nt + n0) + ntw) + nw) * (w - ww) * K.rx;
    a = a + K.q * (((ntn + nt) + nn) + n0) * (wn - w) * K.ry;
    a = a - K.q * (((nt + nts) + n0) + ns) * (w - ws) * K.ry;
    a = a + nt * (wt - w) * (VZ ? Z->d1w : K.rz);
    a = a - n0 * (w - wb) * (VZ ? Z->d2w : K.rz);
  }
#undef FU
#undef FV
#undef FW
#undef FN
  return a;
}

}  // namespace elmm
