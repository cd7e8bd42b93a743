// elmm_fft.cuh -- in-shared-memory mixed-radix FFT (Stockham autosort).
//
// Used by the Poisson solve that replaces the PoisFFT call of
// src/poisson.f90:76-210: real-to-complex transforms along x, complex
// transforms along y.  A block transforms `ntr` sequences of length N held
// contiguously in shared memory; each pass applies radix-R butterflies with
// twiddles from a per-length table tw[m] = exp(-2 pi i m / N) and writes the
// result in natural order into the other buffer (no bit reversal).
#pragma once

#include "elmm_common.cuh"

namespace elmm {

constexpr int kMaxFac = 12;

struct FFTFactors {
  int n;
  int nfac;
  int fac[kMaxFac];
};

template <typename T2>
__device__ __forceinline__ T2 cmul(T2 a, T2 b) {
  T2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}

template <typename T2>
__device__ __forceinline__ T2 cadd(T2 a, T2 b) { T2 r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename T2>
__device__ __forceinline__ T2 csub(T2 a, T2 b) { T2 r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
// multiply by -i (forward) or +i (inverse)
template <typename T2>
__device__ __forceinline__ T2 mul_mi(T2 a, bool inv) {
  T2 r;
  if (!inv) { r.x = a.y; r.y = -a.x; } else { r.x = -a.y; r.y = a.x; }
  return r;
}

// radix-R DFT of v in registers, sign of the exponent: forward -1, inverse +1
template <typename T, typename T2>
__device__ __forceinline__ void dft_small(T2 *v, int R, bool inv) {
  if (R == 2) {
    T2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (R == 4) {
    T2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    T2 s13 = cadd(v[1], v[3]), d13 = mul_mi(csub(v[1], v[3]), inv);
    v[0] = cadd(s02, s13);
    v[2] = csub(s02, s13);
    v[1] = cadd(d02, d13);
    v[3] = csub(d02, d13);
  } else if (R == 3) {
    const T s3 = (T)0.86602540378443864676;  // sin(2 pi / 3)
    T2 t1 = cadd(v[1], v[2]);
    T2 t2 = csub(v[1], v[2]);
    T2 m;
    m.x = v[0].x - (T)0.5 * t1.x;
    m.y = v[0].y - (T)0.5 * t1.y;
    // -i s3 t2 (forward), +i s3 t2 (inverse)
    T2 q = mul_mi(t2, inv);
    q.x *= s3; q.y *= s3;
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m, q);
    v[2] = csub(m, q);
  } else {  // R == 5
    const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;
    const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;
    T2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    T2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    T2 m1, m2;
    m1.x = v[0].x + c1 * a1.x + c2 * a2.x; m1.y = v[0].y + c1 * a1.y + c2 * a2.y;
    m2.x = v[0].x + c2 * a1.x + c1 * a2.x; m2.y = v[0].y + c2 * a1.y + c1 * a2.y;
    T2 n1, n2;  // -i (s1 b1 + s2 b2), -i (s2 b1 - s1 b2) for forward
    n1.x = s1 * b1.x + s2 * b2.x; n1.y = s1 * b1.y + s2 * b2.y;
    n2.x = s2 * b1.x - s1 * b2.x; n2.y = s2 * b1.y - s1 * b2.y;
    n1 = mul_mi(n1, inv);
    n2 = mul_mi(n2, inv);
    T2 x0 = cadd(cadd(v[0], a1), a2);
    v[0] = x0;
    v[1] = cadd(m1, n1);
    v[4] = csub(m1, n1);
    v[2] = cadd(m2, n2);
    v[3] = csub(m2, n2);
  }
}

// Transforms ntr sequences of length f.n stored back to back in buf0;
// returns the buffer (buf0 or buf1) that holds the result.  All threads of
// the block must call it; it ends with __syncthreads().
template <typename T, typename T2>
__device__ T2 *fft_block(T2 *buf0, T2 *buf1, int ntr, const FFTFactors &f, const T2 *__restrict__ tw,
                         bool inv) {
  const int N = f.n;
  T2 *src = buf0, *dst = buf1;
  int Ns = 1;
  for (int p = 0; p < f.nfac; p++) {
    const int R = f.fac[p];
    const int nb = N / R;
    const int tstep = N / (Ns * R);
    for (int w = threadIdx.x; w < nb * ntr; w += blockDim.x) {
      int tr = w / nb;
      int j = w - tr * nb;
      const T2 *s = src + tr * N;
      T2 *o = dst + tr * N;
      int jm = j % Ns;
      T2 v[5];
#pragma unroll
      for (int r = 0; r < 5; r++) {
        if (r < R) {
          T2 x = s[j + r * nb];
          if (r > 0 && jm > 0) {
            T2 t = __ldg(&tw[r * jm * tstep]);
            if (inv) t.y = -t.y;
            x = cmul(x, t);
          }
          v[r] = x;
        }
      }
      dft_small<T, T2>(v, R, inv);
      int od = (j - jm) * R + jm;
#pragma unroll
      for (int r = 0; r < 5; r++)
        if (r < R) o[od + r * Ns] = v[r];
    }
    __syncthreads();
    T2 *t = src; src = dst; dst = t;
    Ns *= R;
  }
  return src;
}

}  // namespace elmm
