// elmm_solids.cuh -- immersed solid bodies on the device: the per-stage work of
// IBMomentum, NullInterior and IBMassSources (src/tsteps.f90:360-567) and the
// wall-model corrections at solid faces (ComputeUVWFluxesWM,
// src/wallmodels.f90:2159-2338, applied as the wmfluxes-*-nobranch-*-inc.f90
// corrections of src/momentum_diffusion.f90:169-420).
//
// The host turns the reference's point lists into box indices once
// (elmm_set_solids); the kernels below walk those lists.
#pragma once

namespace elmm {

// One target of a gather: F[tgt] = sum_m coef[m] * F[src[m]] (TIBPoint_Interpolate,
// src/immersedboundary.f90:637-651).  comp: 0..2 velocity component, 3 the
// viscosity.  n = 0: an IB point without interpolation points (its value
// becomes 0).  Nullified points are a separate list of box indices.  Interpolation
// points in the ghost layer are folded onto the interior cell (and sign) that
// the ghost rule copies, so a gather reads interior cells only.
struct IBGather {
  long long tgt;
  int comp, n;
  long long src[6];
  double coef[6];
};

// A wall-model point at a solid face (WMPointUVW): the free point (box index
// c, z index k) of component comp whose neighbour in direction dir (1..6 =
// -x, +x, -y, +y, -z, +z) is solid.
struct WMSolid {
  long long c;
  int comp, dir, k, pad;
  double dist[3];
  double z0;
  double tflux;  // the body's heat flux (with a temperature)
};

// mode 0: the gathers (after the projection, and the first IBMomentum of a
// run; or the viscosity of the ScalFl points), and after the n gathers the
// nullified points: box indices null[0 .. nnull[0]) of U, then of V, then of W;
// mode 1: U2, V2, W2 at the IB points set to zero before the divergence.
// IBMassSources adds U2(p)/dx at the cell behind an IB point p and takes it
// off the cell in front (src/tsteps.f90:490-533), and the right-hand side
// is div U2 - Q (src/pressure.f90:658-670): together they remove the face
// velocity of p from both divergences, which is the divergence of U2 with
// U2(p) = 0.  The value at p itself is replaced after the projection.
struct NullCounts {
  int n[3];  // nullified points of U, V, W
};

template <typename T>
__global__ void __launch_bounds__(256) k_ib_gather(const Dom<T> *__restrict__ doms, int di,
                                                   const IBGather *__restrict__ pts, int n, int mode,
                                                   const long long *__restrict__ null = nullptr,
                                                   NullCounts nn = NullCounts{{0, 0, 0}}) {
  const Dom<T> &d = doms[di];
  const int ntot = n + nn.n[0] + nn.n[1] + nn.n[2];
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ntot; q += gridDim.x * blockDim.x) {
    if (q >= n) {  // NullInterior (src/tsteps.f90:540-567)
      const int r = q - n;
      T *F = r < nn.n[0] ? d.U : r < nn.n[0] + nn.n[1] ? d.V : d.W;
      F[null[r]] = (T)0;
      continue;
    }
    const IBGather &p = pts[q];
    if (mode == 1) {
      T *F = p.comp == 0 ? d.U2 : p.comp == 1 ? d.V2 : d.W2;
      F[p.tgt] = (T)0;
      continue;
    }
    T *F = p.comp == 0 ? d.U : p.comp == 1 ? d.V : p.comp == 2 ? d.W : d.nu;
    double v = 0;
    for (int m = 0; m < p.n; m++) v = v + p.coef[m] * (double)F[p.src[m]];
    F[p.tgt] = (T)v;
    // with buoyancy the temperature diffusivity follows the viscosity the
    // ScalFl point now has (ComputeTDiff after the interpolation,
    // src/dynamics.f90:899-904)
    if (p.comp == 3 && d.tdiff_live) d.TDiff[p.tgt] = tdiff_of((T)v, (T)d.nu_mol, (T)d.kappa_mol);
  }
}

// One solid-face wall-model point per thread: u* and the flux from the
// velocity at the start of the stage (local_velocity, WMRoughStress), then
// the correction of the free point's tendency: the diffusive flux through
// the face towards the solid, which the stencil added, is taken back and
// the wall-model flux put in its place.  The tendency (Ustar) and U2
// (+ beta dt of it, the RK combine of src/dynamics.f90:450-478) are updated
// by atomics, as a free point can border two solid points.  ustar_only:
// the u* update alone (the wall model on the initial fields).
template <typename T>
__global__ void __launch_bounds__(128) k_ib_wm(const Dom<T> *__restrict__ doms, int di,
                                               const WMSolid *__restrict__ pts, double *__restrict__ ustar_state,
                                               int n, double beta, int ustar_only) {
  const Dom<T> &d = doms[di];
  const double beta_dt = beta * d.dt;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const WMSolid &p = pts[q];
    const T *U = d.U, *V = d.V, *W = d.W, *nu = d.nu;
    const long long c = p.c, sx = 1, sy = d.pitch, sz = d.plane;
    const int comp = p.comp, dir = p.dir, k = p.k;
    double vel[3];
    if (comp == 0) {
      vel[0] = (double)U[c];
      vel[1] = ((double)V[c + sx] + (double)V[c] + (double)V[c + sx - sy] + (double)V[c - sy]) / 4.0;
      vel[2] = ((double)W[c + sx] + (double)W[c] + (double)W[c + sx - sz] + (double)W[c - sz]) / 4.0;
    } else if (comp == 1) {
      vel[0] = ((double)U[c + sy] + (double)U[c] + (double)U[c - sx + sy] + (double)U[c - sx]) / 4.0;
      vel[1] = (double)V[c];
      vel[2] = ((double)W[c + sy] + (double)W[c] + (double)W[c + sy - sz] + (double)W[c - sz]) / 4.0;
    } else {
      vel[0] = ((double)U[c + sz] + (double)U[c] + (double)U[c - sx + sz] + (double)U[c - sx]) / 4.0;
      vel[1] = ((double)V[c + sz] + (double)V[c] + (double)V[c - sy + sz] + (double)V[c - sy]) / 4.0;
      vel[2] = (double)W[c];
    }
    const double dist[3] = {p.dist[0], p.dist[1], p.dist[2]};
    const double dd = norm2_3(dist);
    double t[3] = {vel[0], vel[1], vel[2]};
    const double dot = t[0] * dist[0] + t[1] * dist[1] + t[2] * dist[2];
#pragma unroll
    for (int m = 0; m < 3; m++) t[m] = t[m] - dot * dist[m] / (dd * dd);
    const double tv = norm2_3(t);
    double us = ustar_state[q];
    if (p.z0 > 0 && d.buoy && p.tflux > 0)  // WM_MO_FluxStress (src/wallmodels.f90:1836-1854, 2255-2259)
      us = tv != 0 ? wm_mo_flux_ustar(us, tv, dd, p.z0, p.tflux, d.tref, d.grav, d.nu_mol) : 0.0;
    else if (tv != 0)
      us = wm_ustar(us, tv, dd, p.z0, d.nu_mol);
    if (us < 0) us = 0;
    ustar_state[q] = us;
    if (ustar_only) continue;
    double fp = 0, fm = 0;
    if (tv > 1.4901161193847656e-08) {
      const double base = (t[comp] / tv) * (us * us);
      if (d.vz && dir == 5) {
        fp = comp < 2 ? base / d.dzPr[k + 2] : base / d.dzW[k + 2];
        fm = comp < 2 ? base / d.dzPr[k - 1 + 2] : base / d.dzW[k - 1 + 2];
      } else if (d.vz && dir == 6) {
        fp = comp < 2 ? base / d.dzPr[k + 1 + 2] : base / d.dzW[k + 1 + 2];
        fm = comp < 2 ? base / d.dzPr[k + 2] : base / d.dzW[k + 2];
      } else {
        const double drec = dir <= 2 ? 1 / d.dx : dir <= 4 ? 1 / d.dy : 1 / d.dz;
        fp = base * drec;
        fm = fp;
      }
      if (dir % 2 == 1) { fp = -fp; fm = -fm; }
    }
    const double rx = d.rec2[0], ry = d.rec2[1], rz = d.rec2[2];
    const bool vz = d.vz != 0;
    const T *F = comp == 0 ? U : comp == 1 ? V : W;
    auto N = [&](long long o) { return (double)nu[c + o]; };
    auto G = [&](long long o) { return (double)F[c + o]; };
    double f = 0;
    // the free-point lines of the includes: +(f + fluxp) on a minus side,
    // -(f + fluxp, or fluxm on a stretched grid) on a plus side
    if (comp == 0) {
      switch (dir) {
        case 1: f = N(0) * (G(0) - G(-sx)) * rx; break;
        case 2: f = N(sx) * (G(sx) - G(0)) * rx; break;
        case 3: f = (N(sx) + N(sx - sy) + N(0) + N(-sy)) * (G(0) - G(-sy)) * ry / 4; break;
        case 4: f = (N(sx + sy) + N(sx) + N(sy) + N(0)) * (G(sy) - G(0)) * ry / 4; break;
        case 5: {
          const double s = N(sx) + N(sx - sz) + N(0) + N(-sz);
          f = vz ? s * (G(0) - G(-sz)) / d.dzW[k - 1 + 2] / 4 / d.dzPr[k + 2] : s * (G(0) - G(-sz)) * rz / 4;
          break;
        }
        default: {
          const double s = N(sx + sz) + N(sx) + N(sz) + N(0);
          f = vz ? s * (G(sz) - G(0)) / d.dzW[k + 2] / 4 / d.dzPr[k + 2] : s * (G(sz) - G(0)) * rz / 4;
        }
      }
    } else if (comp == 1) {
      switch (dir) {
        case 1: f = (N(sy) + N(0) + N(sy - sx) + N(-sx)) * (G(0) - G(-sx)) * rx / 4; break;
        case 2: f = (N(sx + sy) + N(sx) + N(sy) + N(0)) * (G(sx) - G(0)) * rx / 4; break;
        case 3: f = N(0) * (G(0) - G(-sy)) * ry; break;
        case 4: f = N(sy) * (G(sy) - G(0)) * ry; break;
        case 5: {
          const double s = N(sy) + N(sy - sz) + N(0) + N(-sz);
          f = vz ? s * (G(0) - G(-sz)) / d.dzW[k - 1 + 2] / 4 / d.dzPr[k + 2] : s * (G(0) - G(-sz)) * rz / 4;
          break;
        }
        default: {
          const double s = N(sy + sz) + N(sy) + N(sz) + N(0);
          f = vz ? s * (G(sz) - G(0)) / d.dzW[k + 2] / 4 / d.dzPr[k + 2] : s * (G(sz) - G(0)) * rz / 4;
        }
      }
    } else {
      switch (dir) {
        case 1: f = (N(sz) + N(0) + N(sz - sx) + N(-sx)) * (G(0) - G(-sx)) * rx / 4; break;
        case 2: f = (N(sx + sz) + N(sx) + N(sz) + N(0)) * (G(sx) - G(0)) * rx / 4; break;
        case 3: f = (N(sz) + N(sz - sy) + N(0) + N(-sy)) * (G(0) - G(-sy)) * ry / 4; break;
        case 4: f = (N(sy + sz) + N(sz) + N(sy) + N(0)) * (G(sy) - G(0)) * ry / 4; break;
        case 5: f = vz ? N(0) * (G(0) - G(-sz)) / d.dzPr[k + 2] / d.dzW[k + 2] : N(0) * (G(0) - G(-sz)) * rz; break;
        default:
          f = vz ? N(sz) * (G(sz) - G(0)) / d.dzPr[k + 1 + 2] / d.dzW[k + 2] : N(sz) * (G(sz) - G(0)) * rz;
      }
    }
    const double delta = dir % 2 == 1 ? f + fp : -(f + (vz ? fm : fp));
    T *S = comp == 0 ? d.Us : comp == 1 ? d.Vs : d.Ws;
    T *S2 = comp == 0 ? d.U2 : comp == 1 ? d.V2 : d.W2;
    atomicAdd(S + c, (T)delta);
    atomicAdd(S2 + c, (T)(beta_dt * delta));
  }
}

// The heat flux of the Pr wall-model points at solid faces
// (TemperatureExtra, src/scalars.f90:323-327) after a temperature stage: q
// = temperature_flux x area_factor joins the stage tendency of its cell, and
// beta dt of it the new value (the RK combine is linear in the tendency).
struct HeatPoint {
  long long c;
  double q;
};
template <typename T>
__global__ void k_heat_add(const Dom<T> *__restrict__ doms, int di, const HeatPoint *__restrict__ pts, int n,
                           int stage, double beta) {
  const Dom<T> &d = doms[di];
  T *A = d.slot[0].adv, *S = d.slot[0].buf[stage % 3];
  const double bdt = beta * d.dt;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const HeatPoint p = pts[q];
    A[p.c] = (T)((double)A[p.c] + p.q);
    S[p.c] = (T)((double)S[p.c] + bdt * p.q);
  }
}

// The temperature's fill of the solid cells after each stage
// (src/scalars.f90:129-198): a solid Pr cell with fluid 6-neighbours (in
// range -1..n+2) becomes the mean of those, in the order i-1, i+1, j-1,
// j+1, k-1, k+1.  A cell deep inside a body keeps its value: the
// reference's branch for it sums all neighbours but assigns nothing.  The
// fill reads fluid cells only, which it never writes, so its order does not
// matter; a cell of a z ghost layer is filled for nothing (the next
// BoundTemperature replaces it before anything reads it) and is left out.
struct FillCell {
  long long box;     // the cell
  long long ref[6];  // its fluid neighbours' cells (the ghost rule's source for a ghost cell)
  int n;             // how many
  int pad;
};

template <typename T>
__global__ void __launch_bounds__(256) k_theta_fill(const Dom<T> *__restrict__ doms, int di,
                                                    const FillCell *__restrict__ cells, int n, int tb) {
  const Dom<T> &d = doms[di];
  T *S = d.slot[0].buf[tb];
  const double off = d.slot[0].off;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const FillCell &c = cells[q];
    double t = 0;
    for (int m = 0; m < c.n; m++) t = t + ((double)S[c.ref[m]] + off);
    S[c.box] = (T)(t / c.n - off);
  }
}

}  // namespace elmm
