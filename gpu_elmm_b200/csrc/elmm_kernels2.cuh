// elmm_kernels2.cuh -- inverse transform, projection, reductions and the
// host-layout pack / unpack kernels.
#pragma once

#include <cfloat>

#include "elmm_kernels.cuh"

namespace elmm {

// inverse real FFT along x of kRowsX rows -> interior of Phi (its ghosts are
// filled afterwards by k_ghosts)
template <typename T>
__global__ void __launch_bounds__(kFFTThreads) k_fftx_inv(const Dom<T> *__restrict__ doms, Launch L,
                                                  const PoisPlan *__restrict__ plans, int gate) {
  typedef typename Vec2<T>::type T2;
  extern __shared__ unsigned char smem_raw[];
  T2 *buf0 = reinterpret_cast<T2 *>(smem_raw);
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    if (gate && !*d.refine_flag) continue;
    const PoisPlan &pl = plans[di];
    const int N = d.nx, nxh = d.nxh;
    const int ntr = kRowsX / 2;
    T2 *buf1 = buf0 + ntr * N;
    const int lt = t - __ldg(L.starts + di);
    const int row0 = lt * kRowsX;
    const int nrows = d.ny * d.nz;
    // Z_m = A_m + i B_m with the Hermitian completion A_{N-m} = conj(A_m);
    // A_0 and A_{N/2} are real for a real row.
#pragma unroll 4
    for (int w = threadIdx.x; w < ntr * N; w += blockDim.x) {
      const int p = w / N, m = w - p * N;
      const int ra = row0 + 2 * p, rb = ra + 1;
      const int mm = m < nxh ? m : N - m;
      const bool cj = m >= nxh;
      T2 A, B;
      A.x = 0; A.y = 0; B.x = 0; B.y = 0;
      if (ra < nrows) A = d.S[((long long)(ra / d.ny) * d.ny + ra % d.ny) * d.spitch + mm];
      if (rb < nrows) B = d.S[((long long)(rb / d.ny) * d.ny + rb % d.ny) * d.spitch + mm];
      if (mm == 0 || 2 * mm == N) { A.y = 0; B.y = 0; }
      if (cj) { A.y = -A.y; B.y = -B.y; }
      T2 z;
      z.x = A.x - B.y;
      z.y = A.y + B.x;
      buf0[p * N + m] = z;
    }
    __syncthreads();
    T2 *res = fft_block<T, T2>(buf0, buf1, ntr, pl.fx, d.twx, true);
#pragma unroll 4
    for (int w = threadIdx.x; w < kRowsX * N; w += blockDim.x) {
      const int r = w / N, i = w - r * N + 1;
      const int row = row0 + r;
      if (row >= nrows) continue;
      const int j = row % d.ny + 1, k = row / d.ny + 1;
      const T2 z = res[(r >> 1) * N + i - 1];
      d.Phi[bidx(d, i, j, k)] = (r & 1) ? z.y : z.x;
    }
    __syncthreads();
  }
}

// PostPoisson (src/pressure.f90:728-870): velocity correction, Pr += Phi and
// the partial sums of the top layer for FixPressureToReference.  A block
// marches up an MX x MY column of MKC planes; the inputs of plane k+1 are in
// flight while plane k is written, and Phi(k+1) of plane k is Phi of k+1.
// HZ: the domains are slabs whose top face is shared (BC_HALO); a
// compile-time choice, since a run-time test of the face here cost the
// kernel a fifth of its speed.
template <typename T, bool HZ = false>
__global__ void __launch_bounds__(MX *MY) k_project(const Dom<T> *__restrict__ doms, Launch L, double coef_alpha2,
                                                    int use_dt, int in_place, int gate) {
  __shared__ double red[MX * MY / 32];
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    if (gate && !*d.refine_flag) continue;
    int lt = t - __ldg(L.starts + di);
    const int ntx = (d.nx + MX - 1) / MX, nty = (d.ny + MY - 1) / MY;
    const int bx = lt % ntx; lt /= ntx;
    const int by = lt % nty;
    const int bk = lt / nty;
    const int k0 = bk * MKC + 1, k1 = min(k0 + MKC - 1, d.nz);
    const int i = bx * MX + (threadIdx.x % MX) + 1;
    const int j = by * MY + (threadIdx.x / MX) + 1;
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const bool inside = i <= nx && j <= ny;
    const double coef = use_dt ? coef_alpha2 * d.dt : coef_alpha2;
    const T dt2 = (T)coef;
    const T Au = (T)(coef / d.dx), Av = (T)(coef / d.dy), Aw = (T)(coef / d.dz);
    const T *__restrict__ Usrc = in_place ? d.U : d.U2;
    const T *__restrict__ Vsrc = in_place ? d.V : d.V2;
    const T *__restrict__ Wsrc = in_place ? d.W : d.W2;
    const T *__restrict__ Phi = d.Phi;
    T *__restrict__ P = d.P;
    const long long pitch = d.pitch, plane = d.plane;
    const bool hu = inside && i <= d.ext[0][0] && j <= d.ext[0][1];
    const bool hv = inside && i <= d.ext[1][0] && j <= d.ext[1][1];
    const bool hw = inside && i <= d.ext[2][0] && j <= d.ext[2][1];
    const T m = (T)(*d.prm);
    long long c = bidx(d, inside ? i : 1, inside ? j : 1, k0);
    // Phi at i+1, j+1, k+1: past the last cell the neighbour folds onto the
    // interior as Bound_Phi fills it (periodic copy, else the cell itself)
    const bool px = d.bt[SIDE_WE] == BC_PERIODIC, py = d.bt[SIDE_SO] == BC_PERIODIC, pz = d.bt[SIDE_BO] == BC_PERIODIC;
    const long long oe = i < nx ? 1 : (px ? 1 - nx : 0);
    const long long on = j < ny ? pitch : (py ? pitch - (long long)ny * pitch : 0);
    // past the top: the periodic image, the cell itself, or (HZ: a slab's
    // top face) the exchanged ghost plane
    auto ot = [&](int kk) -> long long {
      return kk < nz || HZ ? plane : (pz ? plane - (long long)nz * plane : 0);
    };
    T phi = 0, pe = 0, pn = 0, pt = 0, u0 = 0, v0 = 0, w0 = 0, p0 = 0;
    if (inside) {
      phi = __ldg(Phi + c); pe = __ldg(Phi + c + oe); pn = __ldg(Phi + c + on); pt = __ldg(Phi + c + ot(k0));
      if (hu) u0 = __ldg(Usrc + c);
      if (hv) v0 = __ldg(Vsrc + c);
      if (hw) w0 = __ldg(Wsrc + c);
      p0 = P[c];
    }
    for (int k = k0; k <= k1; k++) {
      const bool more = k + 1 <= k1;
      T npe = 0, npn = 0, npt = 0, nu0 = 0, nv0 = 0, nw0 = 0, np0 = 0;
      if (more && inside) {
        const long long cn = c + plane;
        npe = __ldg(Phi + cn + oe); npn = __ldg(Phi + cn + on); npt = __ldg(Phi + cn + ot(k + 1));
        if (hu) nu0 = __ldg(Usrc + cn);
        if (hv) nv0 = __ldg(Vsrc + cn);
        if (hw) nw0 = __ldg(Wsrc + cn);
        np0 = P[cn];
      }
      double top = 0;
      if (inside) {
        // x is periodic: the end cells of a row also write their ghost
        // images (the ghost pass covers y and z)
        const bool g1 = i == 1, gn = i == nx;
        auto ghost = [&](T *F, T v) {
          if (g1) F[c + nx] = v;
          if (gn) F[c - nx] = v;
        };
        if (hu && k <= d.ext[0][2]) {
          T u = u0 - Au * (pe - phi);
          d.U[c] = u;
          ghost(d.U, u);
        }
        if (hv && k <= d.ext[1][2]) {
          T v = v0 - Av * (pn - phi);
          d.V[c] = v;
          ghost(d.V, v);
        }
        if (hw && k <= d.ext[2][2]) {
          T w;
          if (d.vz) w = w0 - dt2 * (pt - phi) / (T)d.dzW[k + 2];
          else w = w0 - Aw * (pt - phi);
          d.W[c] = w;
          ghost(d.W, w);
        }
        T p = (p0 - m) + phi;
        P[c] = p;
        ghost(P, p);
        top = (double)p;
      }
      if (k == nz) {  // block-uniform: the top layer's partial sum of this column
        for (int o = 16; o > 0; o >>= 1) top += __shfl_down_sync(0xffffffffu, top, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = top;
        __syncthreads();
        if (threadIdx.x == 0) {
          double sum = 0;
          for (int w = 0; w < MX * MY / 32; w++) sum += red[w];
          d.prpart[by * ntx + bx] = sum;
        }
        __syncthreads();
      }
      phi = pt; pe = npe; pn = npn; pt = npt; u0 = nu0; v0 = nv0; w0 = nw0; p0 = np0;
      c += plane;
    }
  }
}

// k_project for FP32 domains with an even Prnx (x is periodic for every
// domain): two x-adjacent cells per thread, float2 loads and stores, the
// same tiles (MX x MY x MKC) and partial sums per tile column.  Slabs of a
// split domain take k_project<float, true> instead.
__global__ void __launch_bounds__(MX *MY / 2) k_project_pair(const Dom<float> *__restrict__ doms, Launch L,
                                                          double coef_alpha2, int use_dt, int in_place, int gate) {
  typedef float T;
  __shared__ double red[MX * MY / 64];
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    if (gate && !*d.refine_flag) continue;
    int lt = t - __ldg(L.starts + di);
    const int ntx = (d.nx + MX - 1) / MX, nty = (d.ny + MY - 1) / MY;
    const int bx = lt % ntx; lt /= ntx;
    const int by = lt % nty;
    const int bk = lt / nty;
    const int k0 = bk * MKC + 1, k1 = min(k0 + MKC - 1, d.nz);
    const int i = bx * MX + 2 * (threadIdx.x % (MX / 2)) + 1;  // odd: the pair is 8-byte aligned
    const int j = by * MY + (threadIdx.x / (MX / 2)) + 1;
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const bool inside = i <= nx && j <= ny;  // nx even: i + 1 <= nx too
    const double coef = use_dt ? coef_alpha2 * d.dt : coef_alpha2;
    const T dt2 = (T)coef;
    const T Au = (T)(coef / d.dx), Av = (T)(coef / d.dy), Aw = (T)(coef / d.dz);
    const T *__restrict__ Usrc = in_place ? d.U : d.U2;
    const T *__restrict__ Vsrc = in_place ? d.V : d.V2;
    const T *__restrict__ Wsrc = in_place ? d.W : d.W2;
    const T *__restrict__ Phi = d.Phi;
    T *__restrict__ P = d.P;
    const long long pitch = d.pitch, plane = d.plane;
    const bool hu = inside && j <= d.ext[0][1], hv = inside && j <= d.ext[1][1], hw = inside && j <= d.ext[2][1];
    const T m = (T)(*d.prm);
    long long c = bidx(d, inside ? i : 1, inside ? j : 1, k0);
    // Phi at i+2 (the second cell's x neighbour), j+1, k+1, folded as Bound_Phi fills the ghosts
    const bool px = d.bt[SIDE_WE] == BC_PERIODIC, py = d.bt[SIDE_SO] == BC_PERIODIC, pz = d.bt[SIDE_BO] == BC_PERIODIC;
    const bool last = i + 1 >= nx;
    const long long oe = !last ? 2 : (px ? 1 - i : 0);  // the neighbour pair; for a wall, the cell itself
    const long long on = j < ny ? pitch : (py ? pitch - (long long)ny * pitch : 0);
    auto ot = [&](int kk) -> long long { return kk < nz ? plane : (pz ? plane - (long long)nz * plane : 0); };
    auto ld2 = [](const T *p, long long o) { return __ldg(reinterpret_cast<const float2 *>(p + o)); };
    float2 phi = {0, 0}, pe = {0, 0}, pn = {0, 0}, pt = {0, 0}, u0 = {0, 0}, v0 = {0, 0}, w0 = {0, 0}, p0 = {0, 0};
    auto east = [&](const float2 &own, long long cc) {
      const float2 nb = ld2(Phi, cc + oe);
      return make_float2(own.y, (last && !px) ? own.y : nb.x);
    };
    if (inside) {
      phi = ld2(Phi, c);
      pe = east(phi, c);
      pn = ld2(Phi, c + on);
      pt = ld2(Phi, c + ot(k0));
      if (hu) u0 = ld2(Usrc, c);
      if (hv) v0 = ld2(Vsrc, c);
      if (hw) w0 = ld2(Wsrc, c);
      p0 = *reinterpret_cast<const float2 *>(P + c);
    }
    for (int k = k0; k <= k1; k++) {
      const bool more = k + 1 <= k1;
      float2 npe = {0, 0}, npn = {0, 0}, npt = {0, 0}, nu0 = {0, 0}, nv0 = {0, 0}, nw0 = {0, 0}, np0 = {0, 0};
      if (more && inside) {
        const long long cn = c + plane;
        npe = east(pt, cn);
        npn = ld2(Phi, cn + on);
        npt = ld2(Phi, cn + ot(k + 1));
        if (hu) nu0 = ld2(Usrc, cn);
        if (hv) nv0 = ld2(Vsrc, cn);
        if (hw) nw0 = ld2(Wsrc, cn);
        np0 = *reinterpret_cast<const float2 *>(P + cn);
      }
      double top = 0;
      if (inside) {
        // periodic x ghost images of the row's end cells (the ghost pass
        // covers y and z): cell 1 -> column nx + 1, cell nx -> column 0
        const bool g1 = i == 1, gn = i + 1 == nx;
        auto ghost = [&](T *F, const float2 &v) {
          if (g1) F[c + nx] = v.x;
          if (gn) F[c + 1 - nx] = v.y;
        };
        if (hu && k <= d.ext[0][2]) {
          const float2 u = make_float2(u0.x - Au * (pe.x - phi.x), u0.y - Au * (pe.y - phi.y));
          *reinterpret_cast<float2 *>(d.U + c) = u;
          ghost(d.U, u);
        }
        if (hv && k <= d.ext[1][2]) {
          const float2 v = make_float2(v0.x - Av * (pn.x - phi.x), v0.y - Av * (pn.y - phi.y));
          *reinterpret_cast<float2 *>(d.V + c) = v;
          ghost(d.V, v);
        }
        if (hw && k <= d.ext[2][2]) {
          float2 w;
          if (d.vz) {
            const T dzw = (T)d.dzW[k + 2];
            w = make_float2(w0.x - dt2 * (pt.x - phi.x) / dzw, w0.y - dt2 * (pt.y - phi.y) / dzw);
          } else {
            w = make_float2(w0.x - Aw * (pt.x - phi.x), w0.y - Aw * (pt.y - phi.y));
          }
          *reinterpret_cast<float2 *>(d.W + c) = w;
          ghost(d.W, w);
        }
        const float2 p = make_float2((p0.x - m) + phi.x, (p0.y - m) + phi.y);
        *reinterpret_cast<float2 *>(P + c) = p;
        ghost(P, p);
        top = (double)p.x + (double)p.y;
      }
      if (k == nz) {  // block-uniform: the top layer's partial sum of this column
        for (int o = 16; o > 0; o >>= 1) top += __shfl_down_sync(0xffffffffu, top, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = top;
        __syncthreads();
        if (threadIdx.x == 0) {
          double sum = 0;
          for (int w = 0; w < MX * MY / 64; w++) sum += red[w];
          d.prpart[by * ntx + bx] = sum;
        }
        __syncthreads();
      }
      phi = pt; pe = npe; pn = npn; pt = npt; u0 = nu0; v0 = nv0; w0 = nw0; p0 = np0;
      c += plane;
    }
  }
}

// FixPressureToReference, reference at side To (src/pressure.f90:1160-1229):
// the new reference is the mean of the top layer; it is applied lazily,
// every reader of P subtracts it.
template <typename T>
__device__ __forceinline__ void prref_reduce(const Dom<T> *__restrict__ doms, int nd, int gate, int b0, int nb,
                                             double *red) {
  for (int di = b0; di < nd; di += nb) {
    const Dom<T> &d = doms[di];
    if (gate && !*d.refine_flag) continue;
    double s = 0;
    for (int p = threadIdx.x; p < d.nprpart; p += blockDim.x) s += d.prpart[p];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double tot = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += red[w];
      *d.prm = tot / ((double)d.nx * (double)d.ny);
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void k_prref(const Dom<T> *__restrict__ doms, int nd, int gate) {
  __shared__ double red[32];
  prref_reduce(doms, nd, gate, blockIdx.x, gridDim.x, red);
}

// Ghost shell of up to four box fields, pulled from the interior after the
// kernel that wrote it: every one-deep ghost cell of the y and z faces takes
// the value of the interior cell it folds onto (the periodic x images are
// written by the producers: k_sgs, k_project, k_project_pair).  Velocities follow BoundUVW
// (src/boundaries.f90:398-1791; the sequential x, y, z passes there make the
// fold a product of per-dimension folds), viscosity and Phi a periodic or
// adjacent-cell copy (src/scalarboundaries.f90:326-431,
// src/boundaries.f90:1817-1948), and the pressure only its periodic copies
// (its other ghosts are never read before the next Bound_Pr).
// fields: up to four field ids (F_*), one per byte; the grid covers
// L.total shell tiles of kShellThreads x PER cells per field; each thread
// takes PER cells, all their sources read before any ghost is written (PER
// 4 for batches, whose many small shells leave the launch latency-bound; 1
// for a single domain).
constexpr int kShellThreads = 256;

template <typename T>
__host__ __device__ __forceinline__ T *box_field(const Dom<T> &d, int f) {
  switch (f) {
    case F_U: return d.U;
    case F_V: return d.V;
    case F_W: return d.W;
    case F_U2: return d.U2;
    case F_V2: return d.V2;
    case F_W2: return d.W2;
    case F_P: return d.P;
    case F_NU: return d.nu;
    default: return d.Phi;
  }
}

// cells of the one-deep shell around an ex x ey x ez interior, without the
// x faces (j in 1..ey, k in 1..ez): x is periodic for every domain and the
// producers of the fields with a ghost pass write those images themselves
__host__ __device__ __forceinline__ long long shell_cells(int ex, int ey, int ez) {
  return 2LL * (ex + 2) * (ey + 2) + 2LL * (ex + 2) * ez;
}

template <typename T, int PER = 1>
__global__ void __launch_bounds__(kShellThreads) k_ghosts(const Dom<T> *__restrict__ doms, Launch L, unsigned fields,
                                                          int nf, int gate, int prref = 0) {
  const int nblk = L.total * nf;  // shell tiles times fields (a few million at most)
  for (int b = blockIdx.x; b < nblk; b += gridDim.x) {
    const int f = b / L.total, t = b - f * L.total;
    const int di = find_dom(L.starts, L.nd, t);
    const Dom<T> &d = doms[di];
    if (gate && !*d.refine_flag) continue;
    const int fid = (fields >> (8 * f)) & 0xff;
    const bool vel = fid <= F_W2;
    const int comp = fid % 3;
    const int ex = vel ? d.ext[comp][0] : d.nx, ey = vel ? d.ext[comp][1] : d.ny, ez = vel ? d.ext[comp][2] : d.nz;
    const int ncell = (int)shell_cells(ex, ey, ez);
    const int base = (t - __ldg(L.starts + di)) * kShellThreads * PER + threadIdx.x;
    T *F = box_field(d, fid);
    const bool per[3] = {d.bt[SIDE_WE] == BC_PERIODIC, d.bt[SIDE_SO] == BC_PERIODIC, d.bt[SIDE_BO] == BC_PERIODIC};
    const int rx = ex + 2, zf = rx * (ey + 2), yf = rx * ez;
    // the thread's PER cells: every source read first, then the ghosts written
    T val[PER];
    long long dst[PER];
    bool ok[PER];
#pragma unroll
    for (int r = 0; r < PER; r++) {
      ok[r] = false;
      int w = base + r * kShellThreads;
      if (w >= ncell) continue;
      // z faces (full planes), then y faces (k in 1..ez)
      int i, j, k;
      if (w < 2 * zf) {
        const int side = w >= zf;
        w -= side * zf;
        j = w / rx; i = w - j * rx; k = side ? ez + 1 : 0;
      } else {
        w -= 2 * zf;
        const int side = w >= yf;
        w -= side * yf;
        k = w / rx; i = w - k * rx; k += 1; j = side ? ey + 1 : 0;
      }
      if (halo_plane(k, ez, d.bt)) continue;  // the slab exchange fills it
      T v;
      if (vel) {
        const Fold fx = fold_vel(i, ex, d.bt[0], d.bt[1], comp == 0);
        const Fold fy = fold_vel(j, ey, d.bt[2], d.bt[3], comp == 1);
        const Fold fz = fold_vel(k, ez, d.bt[4], d.bt[5], comp == 2);
        if (fx.zero | fy.zero | fz.zero) {
          v = (T)0;
        } else {
          v = F[bidx(d, fx.src, fy.src, fz.src)];
          if (fx.sign * fy.sign * fz.sign < 0) v = -v;
        }
      } else if (fid == F_P) {
        const bool gx = i < 1 || i > ex, gy = j < 1 || j > ey, gz = k < 1 || k > ez;
        if ((gx && !per[0]) || (gy && !per[1]) || (gz && !per[2])) continue;
        v = F[bidx(d, fold_rep(i, ex, true), fold_rep(j, ey, true), fold_rep(k, ez, true))];
      } else {
        v = F[bidx(d, fold_rep(i, ex, per[0]), fold_rep(j, ey, per[1]), fold_rep(k, ez, per[2]))];
      }
      val[r] = v;
      dst[r] = bidx(d, i, j, k);
      ok[r] = true;
    }
#pragma unroll
    for (int r = 0; r < PER; r++)
      if (ok[r]) F[dst[r]] = val[r];
  }
  // prref: the last blocks (one per domain, as many as there are) also reduce
  // the top-layer partial sums of the projection into the pressure reference
  // (k_prref without a launch of its own)
  const int nb = min(L.nd, (int)gridDim.x), b0 = (int)gridDim.x - 1 - (int)blockIdx.x;
  if (prref && b0 < nb) {
    __shared__ double red[32];
    prref_reduce(doms, L.nd, gate, b0, nb, red);
  }
}

// planes per column chunk of k_divmax
constexpr int kDivChunk = 16;

// Order-preserving bits of a non-negative double; NaN maps above every
// finite value, so an integer maximum propagates it.
__device__ __forceinline__ unsigned long long max_bits(double v) {
  return v >= 0 ? (unsigned long long)__double_as_longlong(v) : 0x7ff8000000000000ULL;
}

// Block-wide maximum of per-thread bits b, merged into *dst with one atomic.
// Every thread of the block calls it.
template <int NT>
__device__ __forceinline__ void block_max_flush(unsigned long long *dst, unsigned long long b,
                                                unsigned long long *red) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long x = __shfl_down_sync(0xffffffffu, b, o);
    b = x > b ? x : b;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long m = 0;
    for (int w = 0; w < NT / 32; w++) m = red[w] > m ? red[w] : m;
    if (m) atomicMax(dst, m);
  }
  __syncthreads();
}

// max |div u| in FP64 (the check of src/pressure.f90:884-989)
template <typename T>
__global__ void __launch_bounds__(TX *TY) k_divmax(const Dom<T> *__restrict__ doms, Launch L) {
  // a TX x TY column of cells marches up a chunk of kDivChunk planes; W at
  // k-1 rides along in a register.  One block reduction and one atomic per
  // domain the block visits.
  __shared__ unsigned long long red[TX * TY / 32];
  unsigned long long run = 0;
  int cur = -1;
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    if (di != cur) {  // block-uniform
      if (cur >= 0) block_max_flush<TX * TY>(doms[cur].maxdiv_bits, run, red);
      run = 0;
      cur = di;
    }
    const Dom<T> &d = doms[di];
    int lt = t - __ldg(L.starts + di);
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const int ntx = (nx + TX - 1) / TX, nty = (ny + TY - 1) / TY;
    const int tx = lt % ntx; lt /= ntx;
    const int ty = lt % nty;
    const int k0 = (lt / nty) * kDivChunk + 1, k1 = min(k0 + kDivChunk - 1, nz);
    const int i = tx * TX + (threadIdx.x % TX) + 1;
    const int j = ty * TY + (threadIdx.x / TX) + 1;
    if (i > nx || j > ny) continue;
    const T *__restrict__ U = d.U;
    const T *__restrict__ V = d.V;
    const T *__restrict__ W = d.W;
    const long long pitch = d.pitch, plane = d.plane;
    // reciprocal spacings: a multiplication instead of an FP64 division per
    // term (the check is a diagnostic; it moves by at most an ulp)
    const double rdx = 1.0 / d.dx, rdy = 1.0 / d.dy, rdz = 1.0 / d.dz;
    const bool vz = d.vz != 0;
    const double *rdzk_tab = d.sgs_rdz;  // 1 / dzPr(k), index k
    long long c = bidx(d, i, j, k0);
    double wb = (double)ld(W, c - plane);
    for (int k = k0; k <= k1; k++) {
      const double rdzk = vz ? rdzk_tab[k] : rdz;
      const double wt = (double)ld(W, c);
      const double a = fabs(((double)ld(U, c) - (double)ld(U, c - 1)) * rdx +
                            ((double)ld(V, c) - (double)ld(V, c - pitch)) * rdy + (wt - wb) * rdzk);
      const unsigned long long bits = max_bits(a);
      run = bits > run ? bits : run;
      wb = wt;
      c += plane;
    }
  }
  if (cur >= 0) block_max_flush<TX * TY>(doms[cur].maxdiv_bits, run, red);
}


// k_divmax for FP32 domains with an even Prnx: two x-adjacent cells per
// thread with float2 loads, a tile of 2 * TX x TY cells; the same FP64
// arithmetic per cell.
__global__ void __launch_bounds__(TX *TY) k_divmax_pair(const Dom<float> *__restrict__ doms, Launch L) {
  __shared__ unsigned long long red[TX * TY / 32];
  unsigned long long run = 0;
  int cur = -1;
  auto ld2 = [](const float *p, long long o) { return __ldg(reinterpret_cast<const float2 *>(p + o)); };
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    if (di != cur) {  // block-uniform
      if (cur >= 0) block_max_flush<TX * TY>(doms[cur].maxdiv_bits, run, red);
      run = 0;
      cur = di;
    }
    const Dom<float> &d = doms[di];
    int lt = t - __ldg(L.starts + di);
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const int ntx = (nx + 2 * TX - 1) / (2 * TX), nty = (ny + TY - 1) / TY;
    const int tx = lt % ntx; lt /= ntx;
    const int ty = lt % nty;
    const int k0 = (lt / nty) * kDivChunk + 1, k1 = min(k0 + kDivChunk - 1, nz);
    const int i = tx * 2 * TX + 2 * (threadIdx.x % TX) + 1;  // odd: the pair is 8-byte aligned
    const int j = ty * TY + (threadIdx.x / TX) + 1;
    if (i > nx || j > ny) continue;
    const float *__restrict__ U = d.U;
    const float *__restrict__ V = d.V;
    const float *__restrict__ W = d.W;
    const long long pitch = d.pitch, plane = d.plane;
    const double rdx = 1.0 / d.dx, rdy = 1.0 / d.dy, rdz = 1.0 / d.dz;
    const bool vz = d.vz != 0;
    const double *rdzk_tab = d.sgs_rdz;
    long long c = bidx(d, i, j, k0);
    float2 wb = ld2(W, c - plane);
    for (int k = k0; k <= k1; k++) {
      const double rdzk = vz ? rdzk_tab[k] : rdz;
      const float2 wt = ld2(W, c), u = ld2(U, c), um = ld2(U, c - 2), v = ld2(V, c), vs = ld2(V, c - pitch);
      const double a0 = fabs(((double)u.x - (double)um.y) * rdx + ((double)v.x - (double)vs.x) * rdy +
                             ((double)wt.x - (double)wb.x) * rdzk);
      const double a1 = fabs(((double)u.y - (double)u.x) * rdx + ((double)v.y - (double)vs.y) * rdy +
                             ((double)wt.y - (double)wb.y) * rdzk);
      const unsigned long long b0 = max_bits(a0), b1 = max_bits(a1);
      run = b0 > run ? b0 : run;
      run = b1 > run ? b1 : run;
      wb = wt;
      c += plane;
    }
  }
  if (cur >= 0) block_max_flush<TX * TY>(doms[cur].maxdiv_bits, run, red);
}

// Defect correction of the mixed path: the divergence residual of the
// FP32 velocity field evaluated in FP64 (the discrete divergence of
// src/pressure.f90:688-717), stored as the right-hand side of a correction
// solve, and its maximum.  gate: run only for domains whose flag is set.
template <typename T>
__global__ void __launch_bounds__(TX *TY) k_divres(const Dom<T> *__restrict__ doms, Launch L, int gate) {
  // a running maximum per thread over the block's tiles; one block
  // reduction and one atomic per domain the block visits
  __shared__ unsigned long long red[TX * TY / 32];
  unsigned long long run = 0;
  int cur = -1;
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    if (di != cur) {  // block-uniform
      if (cur >= 0) block_max_flush<TX * TY>(doms[cur].maxdiv_bits, run, red);
      run = 0;
      cur = di;
    }
    const Dom<T> &d = doms[di];
    if (gate && !*d.refine_flag) continue;
    int lt = t - __ldg(L.starts + di);
    const int ntx = (d.nx + TX - 1) / TX, nty = (d.ny + TY - 1) / TY;
    const int tx = lt % ntx; lt /= ntx;
    const int ty = lt % nty;
    const int k = lt / nty + 1;
    const int i = tx * TX + (threadIdx.x % TX) + 1;
    const int j = ty * TY + (threadIdx.x / TX) + 1;
    if (i <= d.nx && j <= d.ny) {
      const long long c = bidx(d, i, j, k);
      const double dzk = d.vz ? d.dzPr[k + 2] : d.dz;
      const double p = ((double)ld(d.U, c) - (double)ld(d.U, c - 1)) / d.dx +
                       ((double)ld(d.V, c) - (double)ld(d.V, c - d.pitch)) / d.dy +
                       ((double)ld(d.W, c) - (double)ld(d.W, c - d.plane)) / dzk;
      d.Phi[c] = (T)p;
      const double a = fabs(p);
      const unsigned long long b = max_bits(a);
      run = b > run ? b : run;
    }
  }
  if (cur >= 0) block_max_flush<TX * TY>(doms[cur].maxdiv_bits, run, red);
}

// Whether another correction sweep runs: max |div u| above the tolerance
// and fewer than max_refine sweeps in this stage.  first: a new stage.
template <typename T>
__global__ void k_refine_decide(const Dom<T> *__restrict__ doms, int nd, int first) {
  for (int di = blockIdx.x * blockDim.x + threadIdx.x; di < nd; di += gridDim.x * blockDim.x) {
    const Dom<T> &d = doms[di];
    if (first) *d.refine_flag = 1;  // the residual of the first decision is always current
    if (!*d.refine_flag) continue;
    unsigned long long b = *d.maxdiv_bits;
    double md = __longlong_as_double((long long)b);
    int sweeps = first ? 0 : d.refine_count[1];
    int go = (md > d.refine_tol) && sweeps < d.max_refine;
    *d.refine_flag = go;
    if (go) {
      d.refine_count[0] += 1;      // total sweeps since the host reset the counter
      d.refine_count[1] = sweeps + 1;
      *d.maxdiv_bits = 0ULL;       // the sweep ends with a new residual
    } else if (first) {
      d.refine_count[1] = 0;
    }
  }
}

// CFL of TimeStepLength (src/dynamics.f90:553-595)
template <typename T>
__global__ void __launch_bounds__(TX *TY) k_cfl(const Dom<T> *__restrict__ doms, Launch L) {
  // a running maximum per thread over the block's tiles; one block
  // reduction and one atomic per domain the block visits
  __shared__ unsigned long long red[TX * TY / 32];
  unsigned long long run = 0;
  int cur = -1;
  for (int t = blockIdx.x; t < L.total; t += gridDim.x) {
    const int di = find_dom(L.starts, L.nd, t);
    if (di != cur) {  // block-uniform
      if (cur >= 0) block_max_flush<TX * TY>(doms[cur].cfl_bits, run, red);
      run = 0;
      cur = di;
    }
    const Dom<T> &d = doms[di];
    int lt = t - __ldg(L.starts + di);
    const int ntx = (d.nx + TX - 1) / TX, nty = (d.ny + TY - 1) / TY;
    const int tx = lt % ntx; lt /= ntx;
    const int ty = lt % nty;
    const int k = lt / nty + 1;
    const int i = tx * TX + (threadIdx.x % TX) + 1;
    const int j = ty * TY + (threadIdx.x / TX) + 1;
    if (i <= d.nx && j <= d.ny) {
      const long long c = bidx(d, i, j, k);
      const double dzk = d.vz ? d.dzPr[k + 2] : d.dz;
      // NaN-propagating maximum of |u| over the two faces (fmax would drop a NaN)
      auto fm = [](double x, double y) { return (x != x || x > y) ? x : y; };
      // full velocities (the per-level offsets of the mixed path; none in FP64)
      double uc = (double)ld(d.U, c), uw = (double)ld(d.U, c - 1);
      double vc = (double)ld(d.V, c), vs = (double)ld(d.V, c - d.pitch);
      if constexpr (sizeof(T) == 4) {
        const double uo = vel_off(d, 0, k), vo = vel_off(d, 1, k);
        uc += uo; uw += uo; vc += vo; vs += vo;
      }
      double a = fm(fabs(uc), fabs(uw)) / d.dx;
      a = a + fm(fabs(vc), fabs(vs)) / d.dy;
      a = a + fm(fabs((double)ld(d.W, c)), fabs((double)ld(d.W, c - d.plane))) / dzk;
      const unsigned long long b = max_bits(a);
      run = b > run ? b : run;
    }
  }
  if (cur >= 0) block_max_flush<TX * TY>(doms[cur].cfl_bits, run, red);
}

// TimeStepLength with variable time steps (src/dynamics.f90:517-529,
// :547-548), one thread per domain after k_cfl: the step's length from the
// largest U_dx_max of the state at its start, written into the descriptor
// that every kernel of the step reads, and the domain's clock.
template <typename T>
__global__ void k_dt(Dom<T> *doms, int nd) {
  const int di = blockIdx.x * blockDim.x + threadIdx.x;
  if (di >= nd) return;
  Dom<T> &d = doms[di];
  if (!d.vdt) return;
  const double u = __longlong_as_double((long long)*d.cfl_bits);  // a NaN in the field reads as NaN here
  double dt;
  if (u != u) dt = DBL_MIN;                                      // tiny(dt)
  else if (u > 0) dt = fmin(d.cfl_target / u, d.dt_max);
  else dt = d.dt_max;
  const double time = d.tstate[0];
  if (d.end_time > 0) {
    if (d.end_time - time <= 1e-12 * d.end_time) d.flags[2] = 1;  // the run is over: the host should not step
    else if (dt + time > d.end_time) dt = d.end_time - time;
  }
  d.dt = dt;
  d.tstate[0] = time + dt;
  d.tstate[1] = dt;
}

// ------------------------------------------------------ host layout copies
// Host arrays: Fortran layout, lower bound lo, extents n + 2*(1-lo) per dim.
struct HostBox {
  int lo;
  int n0, n1, n2;  // full extents of the host array
};

__device__ __forceinline__ long long hidx(const HostBox &h, int i, int j, int k) {
  return (long long)(i - h.lo) + (long long)h.n0 * ((long long)(j - h.lo) + (long long)h.n1 * (k - h.lo));
}

// interior of a host array (double) -> device box (T); counts non-finite
// values.  off: per-level offsets subtracted before the rounding to T (the
// U and V of the mixed path), or null.
template <typename T>
__global__ void k_unpack(const Dom<T> *__restrict__ dom, T *dst, const double *__restrict__ src, HostBox h, int nx,
                         int ny, int nz, int *bad, const float *off = nullptr) {
  const Dom<T> &d = *dom;
  long long total = (long long)nx * ny * nz;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total; w += (long long)gridDim.x * blockDim.x) {
    int i = (int)(w % nx) + 1;
    long long r = w / nx;
    int j = (int)(r % ny) + 1, k = (int)(r / ny) + 1;
    double v = src[hidx(h, i, j, k)];
    if (!isfinite(v)) atomicAdd(bad, 1);
    if (off) v -= (double)off[k];
    dst[bidx(d, i, j, k)] = (T)v;
  }
}

// The per-level offsets of velocity component c (0: U, 1: V) of the mixed
// path from a host-layout array (double, interior read): block g handles
// level g in [0, nz + 1] and writes the mean over the level that the
// BoundUVW fold of g points to, with the fold's sign (so the ghost levels
// fold as the velocity does), rounded to FP32.  Any fixed value would do;
// the mean keeps the stored deviations small.  A non-finite mean (the
// upload reports non-finite input anyway) is written as 0.
template <typename T>
__global__ void __launch_bounds__(256) k_level_offsets(const Dom<T> *__restrict__ dom, const double *__restrict__ src,
                                                       HostBox h, int c, float *off) {
  const Dom<T> &d = *dom;
  const int *e = d.ext[c];
  const int g = blockIdx.x;  // level, 0..nz+1 (the offset table's range)
  if (g > d.nz + 1) return;
  const Fold fz = fold_vel(g, e[2], d.bt[4], d.bt[5], false);  // U and V are tangential in z
  __shared__ double red[8];
  double s = 0;
  if (!fz.zero) {
    const long long n = (long long)e[0] * e[1];
    for (long long w = threadIdx.x; w < n; w += blockDim.x) {
      const int i = (int)(w % e[0]) + 1, j = (int)(w / e[0]) + 1;
      s += src[hidx(h, i, j, fz.src)];
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += red[q];
    double m = fz.zero ? 0.0 : t / ((double)e[0] * (double)e[1]);
    if (!isfinite(m)) m = 0.0;
    const float f = (float)m;
    off[c * (d.nz + 2) + g] = fz.sign < 0 ? -f : f;
  }
}

// Host arrays of a single-precision host (the reference's default prec=sp
// build): widened to double in a staging buffer on the way in, narrowed
// (round to nearest) on the way out, so every pack and unpack kernel keeps
// its double host layout.
__global__ void k_widen(double *dst, const float *__restrict__ src, long long n) {
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n; w += (long long)gridDim.x * blockDim.x)
    dst[w] = (double)src[w];
}
__global__ void k_narrow(float *dst, const double *__restrict__ src, long long n) {
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n; w += (long long)gridDim.x * blockDim.x)
    dst[w] = (float)src[w];
}

// ghost shell of a velocity component from its interior (BoundUVW rules)
template <typename T>
__global__ void k_halo_vel(const Dom<T> *__restrict__ dom, int comp) {
  const Dom<T> &d = *dom;
  T *F = comp == 0 ? d.U : comp == 1 ? d.V : d.W;
  const int *e = d.ext[comp];
  const int bx = d.nx + 2, by = d.ny + 2, bz = d.nz + 2;
  long long total = (long long)bx * by * bz;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total; w += (long long)gridDim.x * blockDim.x) {
    int i = (int)(w % bx);
    long long r = w / bx;
    int j = (int)(r % by), k = (int)(r / by);
    if (i > e[0] + 1 || j > e[1] + 1 || k > e[2] + 1) continue;
    bool gi = i < 1 || i > e[0], gj = j < 1 || j > e[1], gk = k < 1 || k > e[2];
    if (!(gi || gj || gk) || halo_plane(k, e[2], d.bt)) continue;
    Fold fx = fold_vel(i, e[0], d.bt[0], d.bt[1], comp == 0);
    Fold fy = fold_vel(j, e[1], d.bt[2], d.bt[3], comp == 1);
    Fold fz = fold_vel(k, e[2], d.bt[4], d.bt[5], comp == 2);
    T v = 0;
    if (!(fx.zero | fy.zero | fz.zero)) {
      v = F[bidx(d, fx.src, fy.src, fz.src)];
      if (fx.sign * fy.sign * fz.sign < 0) v = -v;
    }
    F[bidx(d, i, j, k)] = v;
  }
}

// periodic ghosts of P from its interior
template <typename T>
__global__ void k_halo_p(const Dom<T> *__restrict__ dom) {
  const Dom<T> &d = *dom;
  const int bx = d.nx + 2, by = d.ny + 2, bz = d.nz + 2;
  const bool px = d.bt[SIDE_WE] == BC_PERIODIC, py = d.bt[SIDE_SO] == BC_PERIODIC, pz = d.bt[SIDE_BO] == BC_PERIODIC;
  long long total = (long long)bx * by * bz;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total; w += (long long)gridDim.x * blockDim.x) {
    int i = (int)(w % bx);
    long long r = w / bx;
    int j = (int)(r % by), k = (int)(r / by);
    bool gi = i < 1 || i > d.nx, gj = j < 1 || j > d.ny, gk = k < 1 || k > d.nz;
    if (!(gi || gj || gk)) continue;
    if ((gi && !px) || (gj && !py) || (gk && !pz)) continue;
    d.P[bidx(d, i, j, k)] = d.P[bidx(d, fold_rep(i, d.nx, px), fold_rep(j, d.ny, py), fold_rep(k, d.nz, pz))];
  }
}

// device box -> host layout with the reference's three-deep ghosts
// (BoundUVW).  off: per-level offsets added to the stored values (the U and
// V of the mixed path, and their U2, V2), or null.
template <typename T>
__global__ void k_pack_vel(const Dom<T> *__restrict__ dom, const T *F, int comp, double *dst, HostBox h,
                           const float *off = nullptr) {
  const Dom<T> &d = *dom;
  const int *e = d.ext[comp];
  long long total = (long long)h.n0 * h.n1 * h.n2;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total; w += (long long)gridDim.x * blockDim.x) {
    int i = (int)(w % h.n0) + h.lo;
    long long r = w / h.n0;
    int j = (int)(r % h.n1) + h.lo, k = (int)(r / h.n1) + h.lo;
    Fold fx = fold_vel(i, e[0], d.bt[0], d.bt[1], comp == 0);
    Fold fy = fold_vel(j, e[1], d.bt[2], d.bt[3], comp == 1);
    Fold fz = fold_vel(k, e[2], d.bt[4], d.bt[5], comp == 2);
    double v = 0;
    if (!(fx.zero | fy.zero | fz.zero)) {
      v = (double)F[bidx(d, fx.src, fy.src, fz.src)];
      if (off) v += (double)off[fz.src];
      if (fx.sign * fy.sign * fz.sign < 0) v = -v;
    }
    dst[w] = v;
  }
}

// Mixed path, before solid bodies are installed: the stored deviations of
// U and V (every box cell, ghosts included) become full values, since the
// immersed-boundary kernels work on full values; the host then zeroes the
// offsets.
template <typename T>
__global__ void k_drop_offsets(const Dom<T> *__restrict__ dom) {
  const Dom<T> &d = *dom;
  if constexpr (sizeof(T) == 4) {
    const long long n = d.plane * (d.nz + 2);
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n; w += (long long)gridDim.x * blockDim.x) {
      const int k = (int)(w / d.plane);
      d.U[w] = d.U[w] + d.voff[k];
      d.V[w] = d.V[w] + d.voff[d.nz + 2 + k];
    }
  }
}

// interior of a box field -> host (double), optional subtraction of the
// pressure reference; mode 1: Bound_Pr faces, mode 2: Bound_Phi faces,
// mode 3: the one-cell shell as stored (Viscosity); other cells untouched.
// mode 0: interior only.  (nx, ny, nz): interior extents of the field.
template <typename T>
__global__ void k_pack_scalar(const Dom<T> *__restrict__ dom, const T *F, double *dst, HostBox h, int mode,
                              int sub_prm, int nx, int ny, int nz) {
  const Dom<T> &d = *dom;
  const double m = sub_prm ? *d.prm : 0.0;
  long long total = (long long)h.n0 * h.n1 * h.n2;
  const bool per[3] = {d.bt[SIDE_WE] == BC_PERIODIC, d.bt[SIDE_SO] == BC_PERIODIC, d.bt[SIDE_BO] == BC_PERIODIC};
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total; w += (long long)gridDim.x * blockDim.x) {
    int i = (int)(w % h.n0) + h.lo;
    long long r = w / h.n0;
    int j = (int)(r % h.n1) + h.lo, k = (int)(r / h.n1) + h.lo;
    bool gi = i < 1 || i > nx, gj = j < 1 || j > ny, gk = k < 1 || k > nz;
    int ng = (int)gi + (int)gj + (int)gk;
    auto val = [&](int a, int b, int c) { return (double)F[bidx(d, a, b, c)] - m; };
    if (ng == 0) { dst[w] = val(i, j, k); continue; }
    if (mode == 0) continue;
    if (mode == 3) {
      if (i >= 0 && i <= nx + 1 && j >= 0 && j <= ny + 1 && k >= 0 && k <= nz + 1) dst[w] = (double)F[bidx(d, i, j, k)];
      continue;
    }
    if (ng != 1) continue;  // edges and corners are not written by Bound_Pr / Bound_Phi
    int dim = gi ? 0 : gj ? 1 : 2;
    int g = dim == 0 ? i : dim == 1 ? j : k;
    int n = dim == 0 ? nx : dim == 1 ? ny : nz;
    auto at = [&](int q) {
      return dim == 0 ? val(q, j, k) : dim == 1 ? val(i, q, k) : val(i, j, q);
    };
    double v;
    if (per[dim]) {
      v = at(g < 1 ? n + g : g - n);
    } else if (mode == 1) {  // Neumann extrapolation of Bound_Pr (boundaries.f90:1976-1981)
      if (g == 0) v = at(3) - 3 * (at(2) - at(1));
      else if (g == -1) v = at(2);
      else if (g == n + 1) v = at(n - 2) - 3 * (at(n - 1) - at(n));
      else v = at(n - 1);
    } else {  // even reflection of Bound_Phi
      v = g < 1 ? at(1 - g) : at(2 * n + 1 - g);
    }
    dst[w] = v;
  }
}

}  // namespace elmm
