// elmm_fftreg.cuh -- register-resident FFTs for lengths known at compile
// time (the x and y transforms of the Poisson solve, src/poisson.f90:76-210).
//
// A length-N sequence is spread over P threads, E = N / P elements each
// (four-step / Stockham form, n = n1 + P n2, k = k2 + E k1):
//   pass 1: thread n1 holds x[n1 + P n2] and takes the E-point DFT over n2
//           in registers, then multiplies by W_N^(n1 k2);
//   exchange through shared memory;
//   pass 2: P-point DFTs over n1 for each k2, in ceil(E / P) rounds.
// The in-register DFTs are built recursively from radix 2, 3, 4 and 5 with
// compile-time twiddles; only W_N^(n1 k2) comes from the per-length table.
// The result is the unnormalised DFT, as the generic shared-memory FFT of
// elmm_fft.cuh computes it.
#pragma once

#include <type_traits>

#include "elmm_fft.cuh"

namespace elmm {

// ---------------------------------------------- compile-time twiddle values
// cos and sin of 2 pi n / D, reduced exactly (integer arithmetic) to an
// angle in [0, pi/4] and evaluated there by Taylor series.
struct CosSin {
  double c, s;
};

constexpr double kTwoPi = 6.283185307179586476925286766559;

constexpr double taylor_sin(double x) {
  double t = x, s = x;
  for (int n = 1; n < 16; n++) {
    t *= -x * x / ((2.0 * n) * (2.0 * n + 1));
    s += t;
  }
  return s;
}

constexpr double taylor_cos(double x) {
  double t = 1, s = 1;
  for (int n = 1; n < 16; n++) {
    t *= -x * x / ((2.0 * n - 1) * (2.0 * n));
    s += t;
  }
  return s;
}

constexpr CosSin cis(long long n, long long D) {
  n %= D;
  if (n < 0) n += D;
  double sc = 1, ss = 1;  // signs of cos and sin
  bool swap = false;
  if (2 * n > D) { n = D - n; ss = -ss; }                   // theta -> 2 pi - theta
  if (4 * n > D) { n = D - 2 * n; D = 2 * D; sc = -sc; }    // theta -> pi - theta
  if (8 * n > D) { n = D - 4 * n; D = 4 * D; swap = true; } // theta -> pi/2 - theta
  const double x = kTwoPi * (double)n / (double)D;
  const double c = taylor_cos(x), s = taylor_sin(x);
  return swap ? CosSin{sc * s, ss * c} : CosSin{sc * c, ss * s};
}

// x * exp(-+ 2 pi i M / R): forward uses the minus sign, inverse the plus
template <typename T, typename T2, int R, int M, bool INV>
__device__ __forceinline__ T2 twc(T2 x) {
  constexpr int m = ((M % R) + R) % R;
  if constexpr (m == 0) {
    return x;
  } else if constexpr ((4 * m) % R == 0) {  // a quarter turn: exact
    constexpr int q = 4 * m / R;               // 1, 2, 3 quarter turns
    T2 r;
    if constexpr (q == 2) { r.x = -x.x; r.y = -x.y; }
    else if constexpr ((q == 1) != INV) { r.x = x.y; r.y = -x.x; }  // * -i
    else { r.x = -x.y; r.y = x.x; }                                 // * +i
    return r;
  } else {
    constexpr CosSin w = cis(m, R);
    const T c = (T)w.c, s = INV ? (T)w.s : (T)(-w.s);
    T2 r;
    r.x = x.x * c - x.y * s;
    r.y = x.x * s + x.y * c;
    return r;
  }
}

// calls f(std::integral_constant<int, I>) for I = B .. E-1
template <int B, int E, typename F>
__device__ __forceinline__ void static_for(F &&f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    static_for<B + 1, E>(f);
  }
}

// In-place R-point DFT of v[0..R-1] (natural order in and out).
template <typename T, typename T2, int R, bool INV>
__device__ __forceinline__ void dft_reg(T2 *v) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2 || R == 3 || R == 4 || R == 5) {
    dft_small<T, T2>(v, R, INV);
  } else {
    constexpr int A = (R % 4 == 0) ? 4 : (R % 3 == 0) ? 3 : (R % 2 == 0) ? 2 : 5;
    constexpr int B = R / A;
    static_assert(A * B == R, "radix");
    T2 s[A][B];
#pragma unroll
    for (int a = 0; a < A; a++)
#pragma unroll
      for (int b = 0; b < B; b++) s[a][b] = v[a + A * b];
#pragma unroll
    for (int a = 0; a < A; a++) dft_reg<T, T2, B, INV>(s[a]);
    // X[k1 + B k2] = sum_a W_A^(a k2) W_R^(a k1) Y_a[k1]
    static_for<0, B>([&](auto k1c) {
      constexpr int k1 = decltype(k1c)::value;
      T2 u[A];
      static_for<0, A>([&](auto ac) {
        constexpr int a = decltype(ac)::value;
        u[a] = twc<T, T2, R, a * k1, INV>(s[a][k1]);
      });
      dft_small<T, T2>(u, A, INV);
#pragma unroll
      for (int k2 = 0; k2 < A; k2++) v[k1 + B * k2] = u[k2];
    });
  }
}

// ------------------------------------------------------------------- plans
// P: the largest power of two with P * P <= N that divides N.
__host__ __device__ constexpr int fplan_P(int N) {
  int P = 1;
  while ((2 * P) * (2 * P) <= N && N % (2 * P) == 0) P *= 2;
  return P;
}

template <int N>
struct FPlan {
  static constexpr int P = fplan_P(N);
  static constexpr int E = N / P;
  static constexpr int YS = P + 1;         // row stride of the pass-1 exchange
  static constexpr int SEQ = N + E + 1;    // shared-memory elements per sequence (odd)
  static constexpr int RR = (E + P - 1) / P;
  static_assert(P >= 2 && E >= P, "plan");
};

// Lengths with a register FFT; the generic transform handles the others.
#define ELMM_FFT_SIZES(X) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384)

__host__ __device__ constexpr bool fft_reg_supported(int n) {
#define ELMM_FFT_CASE(n_) (n) == (n_) ||
  return ELMM_FFT_SIZES(ELMM_FFT_CASE) false;
#undef ELMM_FFT_CASE
}

__host__ __device__ constexpr int fft_reg_seq(int n) { return n + n / fplan_P(n) + 1; }

// Length-N DFT of the sequence whose lane t in [0, P) holds v[e] = x[t + P e].
// On return the DFT X[0..N-1] is in sh[0..N-1] (natural order).  tw is the
// per-length table W_N^m.  Contains block-wide barriers: every thread of the
// block calls it the same number of times.
template <typename T, typename T2, int N, bool INV>
__device__ __forceinline__ void fft_reg(T2 (&v)[FPlan<N>::E], T2 *sh, int t, const T2 *__restrict__ tw) {
  typedef FPlan<N> Pl;
  constexpr int P = Pl::P, E = Pl::E, YS = Pl::YS, RR = Pl::RR;
  dft_reg<T, T2, E, INV>(v);
#pragma unroll
  for (int k2 = 1; k2 < E; k2++) {
    T2 w = __ldg(tw + t * k2);
    if (INV) w.y = -w.y;
    v[k2] = cmul(v[k2], w);
  }
#pragma unroll
  for (int k2 = 0; k2 < E; k2++) sh[k2 * YS + t] = v[k2];
  __syncthreads();
  T2 u[RR][P];
#pragma unroll
  for (int r = 0; r < RR; r++) {
    const int k2 = r * P + t;
    if (k2 < E) {
#pragma unroll
      for (int n1 = 0; n1 < P; n1++) u[r][n1] = sh[k2 * YS + n1];
      dft_reg<T, T2, P, INV>(u[r]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RR; r++) {
    const int k2 = r * P + t;
    if (k2 < E) {
#pragma unroll
      for (int k1 = 0; k1 < P; k1++) sh[k2 + E * k1] = u[r][k1];
    }
  }
  __syncthreads();
}

}  // namespace elmm
