// elmm_slabs.inl -- one domain split into z-slabs over the GPUs of a node
// (included by elmm_api.cu after BatchT).
//
// The reference splits a domain over MPI ranks (src/custom_mpi.f90:331-344)
// and exchanges ghost layers between neighbours (src/exchange_mpi.f90:84-503),
// with PFFT transposes in the Poisson solve (src/poisson.f90:107-114).  Here
// one process drives every slab: slab s is a single-domain BatchT on device
// devices[s] (a device may hold several slabs) with levels k0+1 .. k0+nzl of
// the whole domain and BC_HALO on the faces it shares.  Each stage runs the
// single-domain kernels on every slab and, where a kernel reads a plane the
// slab below or above owns, copies that plane (peer copy over NVLink between
// GPUs, a device copy on one GPU) into the one-deep ghost plane:
//
//   after the SGS kernel      nu          both ways
//   after the momentum kernel W2          upwards (the divergence reads W2(k-1))
//   z solve                   the maps of the forward and backward sweeps
//                             (3 numbers per column and slab) and the (0,0)
//                             column (elmm_slabs.cuh)
//   after the inverse FFTs    Phi         downwards (the projection reads Phi(k+1))
//   after the projection      U V W P     both ways, and the pressure
//                             reference of the top slab to every slab
//
// An exchange orders itself with events: each destination records that its
// earlier work is done, each source copies on its own stream after that and
// records the end of its copies, and each destination waits for those.  So
// no copy overwrites a plane still being read, no source changes a plane
// before it is copied, and nothing reads a ghost plane before it lands.  No
// kernel waits on another slab's kernel.
#pragma once

template <typename T>
struct SlabsT {
  int ns = 0, nzg = 0;
  elmm_config gcfg{};
  HostGrid ggrid;
  std::vector<int> k0, nzl, dev;
  std::vector<std::unique_ptr<BatchT<T>>> sl;
  // per slab: pivots of its levels, the sweep maps of every slab, the (0,0) column
  struct Tri {
    double *iv = nullptr, *fmaps = nullptr, *bmaps = nullptr, *zcol = nullptr;
    const double *dzc = nullptr, *dzf = nullptr;
  };
  std::vector<Tri> tri;
  // slabs of at most kTriTileMaxNz levels take the tiled sweep kernels
  static constexpr int kSlabCols = 16;
  typedef SlabTile<T, kSlabCols> Tile;
  bool tiled = false;
  size_t smem_tile = 0;
  std::vector<cudaEvent_t> pre, post;
  cudaEvent_t t0 = nullptr, t1 = nullptr, ev_fork = nullptr;
  double time = 0;
  int kernels = 0;  // launches of the last call
  // every slab on one device: one step captured once into a CUDA graph over
  // the slabs' streams and replayed (slabs on several devices launch eagerly)
  cudaGraphExec_t step_exec = nullptr;
  bool step_has_cfl = false;
  int step_kernels = 0;

  ~SlabsT() {
    if (step_exec) cudaGraphExecDestroy(step_exec);
    if (ev_fork) cudaEventDestroy(ev_fork);
    for (auto e : pre) if (e) cudaEventDestroy(e);
    for (auto e : post) if (e) cudaEventDestroy(e);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
  }

  int init(const elmm_config &c, int n, const int *devices, const int *nz_slab) {
    int r = check_config(c);
    if (r) return r;
    if (n < 1 || n > ELMM_MAX_SLABS) return fail(ELMM_ERR_INVALID_ARG, "nslabs in 1.." + std::to_string(ELMM_MAX_SLABS));
    if (c.Btype[ELMM_BO] == ELMM_BC_PERIODIC) return fail(ELMM_ERR_INVALID_CONFIG, "split domains need walls in z (periodic z is not built)");
    if (c.variable_time_steps) return fail(ELMM_ERR_INVALID_CONFIG, "split domains take constant time steps");
    if (c.max_refine_sweeps > 0) return fail(ELMM_ERR_INVALID_CONFIG, "split domains take no defect-correction sweeps");
    ns = n;
    nzg = c.Prnz;
    gcfg = c;
    k0.resize(n);
    nzl.resize(n);
    dev.resize(n);
    int acc = 0;
    for (int s = 0; s < n; s++) {
      nzl[s] = nz_slab ? nz_slab[s] : nzg / n + (s < nzg % n ? 1 : 0);
      dev[s] = devices ? devices[s] : c.device;
      if (nzl[s] < 4) return fail(ELMM_ERR_INVALID_ARG, "every slab needs at least 4 levels");
      k0[s] = acc;
      acc += nzl[s];
    }
    if (acc != nzg) return fail(ELMM_ERR_INVALID_ARG, "the slab levels must add up to Prnz");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess) return fail(ELMM_ERR_CUDA, "no CUDA device");
    for (int s = 0; s < n; s++)
      if (dev[s] < 0 || dev[s] >= ndev) return fail(ELMM_ERR_INVALID_ARG, "no CUDA device " + std::to_string(dev[s]));
    make_grid(c, ggrid);
    // the whole column's coefficients of the z solve and the (0,0) mode's
    // spacings (as init_domain forms them for one domain)
    std::vector<double> Ab(nzg + 2, 0.0), At(nzg + 2, 0.0), dzc(nzg + 2, 0.0), dzf(nzg + 2, 0.0);
    {
      auto zP = [&](int k) { return ggrid.zPr[k + 2]; };
      auto zWf = [&](int k) { return ggrid.zW[k + 2]; };
      for (int k = 1; k <= nzg; k++) {
        Ab[k] = 1 / ((zP(k) - zP(k - 1)) * (zWf(k) - zWf(k - 1)));
        At[k] = 1 / ((zP(k + 1) - zP(k)) * (zWf(k) - zWf(k - 1)));
        dzc[k] = zWf(k) - zWf(k - 1);
        dzf[k] = zP(k + 1) - zP(k);
      }
      Ab[1] = 0;
      At[nzg] = 0;
    }
    sl.resize(n);
    tri.resize(n);
    for (int s = 0; s < n; s++) {
      elmm_config cs = c;
      cs.Prnz = nzl[s];
      cs.device = dev[s];
      if (s > 0) cs.Btype[ELMM_BO] = cs.TempBtype[ELMM_BO] = cs.ScalBtype[ELMM_BO] = BC_HALO;
      if (s < n - 1) cs.Btype[ELMM_TO] = cs.TempBtype[ELMM_TO] = cs.ScalBtype[ELMM_TO] = BC_HALO;
      cs.zW = c.zW ? c.zW + k0[s] : nullptr;
      cs.zmin = c.zmin + k0[s] * c.dzmin;
      // the xy slice in the slab holding its level (the xz slice in every slab)
      cs.avg_slice_k = c.avg_slice_k > k0[s] && c.avg_slice_k <= k0[s] + nzl[s] ? c.avg_slice_k - k0[s] : 0;
      // the point sources whose cell of the whole domain lies in this slab
      cs.num_point_sources = 0;
      for (int q = 0; q < c.num_point_sources; q++) {
        int ip[3];
        if (point_cell(c, c.point_sources[q].position, ip) && ip[2] > k0[s] && ip[2] <= k0[s] + nzl[s])
          cs.point_sources[cs.num_point_sources++] = c.point_sources[q];
      }
      sl[s].reset(new BatchT<T>());
      BatchT<T> &B = *sl[s];
      B.slab_mode = true;
      B.zparent = &ggrid;
      B.zk0 = k0[s];
      if ((r = B.init(&cs, 1))) return r;
      B.tuned = true;  // the default shapes (the autotuner times the single-domain z solve)
      const Dom<T> &h = B.hdom[0];
      const int ncol = h.ny * h.spitch;
      Tri &x = tri[s];
      const double *Abg, *Atg;
      if ((r = B.upload_table(&Abg, Ab)) || (r = B.upload_table(&Atg, At)) || (r = B.upload_table(&x.dzc, dzc)) ||
          (r = B.upload_table(&x.dzf, dzf)))
        return r;
      if ((r = B.dalloc((void **)&x.iv, sizeof(double) * (size_t)nzl[s] * ncol)) ||
          (r = B.dalloc((void **)&x.fmaps, sizeof(double) * 3 * (size_t)ncol * n)) ||
          (r = B.dalloc((void **)&x.bmaps, sizeof(double) * 3 * (size_t)ncol * n)) ||
          (r = B.dalloc((void **)&x.zcol, sizeof(double) * 2 * (size_t)nzg)))
        return r;
      k_slab_tri_pivots<<<(ncol + 127) / 128, 128, 0, B.stream>>>(x.iv, h.lamx, h.lamy, Abg, Atg, h.nxh, h.spitch, h.ny,
                                                                  k0[s], nzl[s]);
      CU(cudaStreamSynchronize(B.stream));
      CU(cudaGetLastError());
    }
    // peer access between the GPUs of neighbouring slabs (the exchanges
    // also work without it, staged by the driver)
    for (int s = 0; s + 1 < n; s++)
      if (dev[s] != dev[s + 1])
        for (int a = 0; a < 2; a++) {
          const int from = a ? dev[s + 1] : dev[s], to = a ? dev[s] : dev[s + 1];
          int can = 0;
          cudaDeviceCanAccessPeer(&can, from, to);
          if (can) {
            CU(cudaSetDevice(from));
            cudaError_t e = cudaDeviceEnablePeerAccess(to, 0);
            if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled)
              return fail(ELMM_ERR_CUDA, std::string("cudaDeviceEnablePeerAccess: ") + cudaGetErrorString(e));
            cudaGetLastError();
          }
        }
    int maxnz = 0;
    for (int s = 0; s < n; s++) maxnz = std::max(maxnz, nzl[s]);
    tiled = maxnz <= kTriTileMaxNz;
    smem_tile = Tile::smem(maxnz);
    if (tiled)
      for (int s = 0; s < n; s++) {
        CU(cudaSetDevice(dev[s]));
        int optin = 0;
        CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev[s]));
        CU(cudaFuncSetAttribute(k_slab_tri_fmap_tile<T, kSlabCols>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        CU(cudaFuncSetAttribute(k_slab_tri_fwd_tile<T, kSlabCols>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        CU(cudaFuncSetAttribute(k_slab_tri_bwd_tile<T, kSlabCols>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
      }
    pre.assign(n, nullptr);
    post.assign(n, nullptr);
    for (int s = 0; s < n; s++) {
      CU(cudaSetDevice(dev[s]));
      CU(cudaEventCreateWithFlags(&pre[s], cudaEventDisableTiming));
      CU(cudaEventCreateWithFlags(&post[s], cudaEventDisableTiming));
    }
    CU(cudaSetDevice(dev[0]));
    CU(cudaEventCreate(&t0));
    CU(cudaEventCreate(&t1));
    CU(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    return ELMM_OK;
  }
  bool one_device() const {
    for (int s = 1; s < ns; s++)
      if (dev[s] != dev[0]) return false;
    return true;
  }

  // ------------------------------------------------------------ exchanges
  struct Copy {
    int src, dst;
    void *to;
    const void *from;
    size_t bytes;
  };
  int exchange(const std::vector<Copy> &cps) {
    std::vector<char> isdst(ns, 0), issrc(ns, 0), waited((size_t)ns * ns, 0), joined((size_t)ns * ns, 0);
    for (const Copy &c : cps) { isdst[c.dst] = 1; issrc[c.src] = 1; }
    for (int t = 0; t < ns; t++)
      if (isdst[t]) {
        CU(cudaSetDevice(dev[t]));
        CU(cudaEventRecord(pre[t], sl[t]->stream));
      }
    for (const Copy &c : cps) {
      BatchT<T> &S = *sl[c.src];
      CU(cudaSetDevice(dev[c.src]));
      if (!waited[(size_t)c.src * ns + c.dst]) {
        CU(cudaStreamWaitEvent(S.stream, pre[c.dst], 0));
        waited[(size_t)c.src * ns + c.dst] = 1;
      }
      if (dev[c.src] == dev[c.dst]) CU(cudaMemcpyAsync(c.to, c.from, c.bytes, cudaMemcpyDeviceToDevice, S.stream));
      else CU(cudaMemcpyPeerAsync(c.to, dev[c.dst], c.from, dev[c.src], c.bytes, S.stream));
    }
    for (int s = 0; s < ns; s++)
      if (issrc[s]) {
        CU(cudaSetDevice(dev[s]));
        CU(cudaEventRecord(post[s], sl[s]->stream));
      }
    for (const Copy &c : cps)
      if (!joined[(size_t)c.dst * ns + c.src]) {
        joined[(size_t)c.dst * ns + c.src] = 1;
        CU(cudaSetDevice(dev[c.dst]));
        CU(cudaStreamWaitEvent(sl[c.dst]->stream, post[c.src], 0));
      }
    return ELMM_OK;
  }
  // plane k of box field f of slab s
  T *plane_of(int s, int f, int k) const {
    const Dom<T> &h = sl[s]->hdom[0];
    return box_field(h, f) + (size_t)k * h.plane;
  }
  size_t plane_bytes(int s) const { return (size_t)sl[s]->hdom[0].plane * sizeof(T); }
  // the ghost planes of fields fs: up (slab s's top plane to the bottom
  // ghost of s + 1) and / or down (the first plane of s + 1 to the top ghost of s)
  void halo_copies(std::vector<Copy> &cps, std::initializer_list<int> fs, bool up, bool down) const {
    for (int f : fs)
      for (int s = 0; s + 1 < ns; s++) {
        if (up) cps.push_back(Copy{s, s + 1, plane_of(s + 1, f, 0), plane_of(s, f, nzl[s]), plane_bytes(s)});
        if (down) cps.push_back(Copy{s + 1, s, plane_of(s, f, nzl[s] + 1), plane_of(s + 1, f, 1), plane_bytes(s)});
      }
  }
  int exchange_halos(std::initializer_list<int> fs, bool up, bool down) {
    std::vector<Copy> cps;
    halo_copies(cps, fs, up, down);
    return exchange(cps);
  }
  // plane k of scalar slot q's buffer b of slab s, or of its diffusivity (q < 0)
  T *splane(int s, int q, int b, int k) const {
    const Dom<T> &h = sl[s]->hdom[0];
    return (q < 0 ? h.TDiff : h.slot[q].buf[b]) + (size_t)k * h.plane;
  }
  int nslots() const { return sl[0]->hdom[0].nslot; }
  // the halos of the scalar slots' buffer b: the top plane and the one below
  // it up into the next slab's ghost plane and second halo plane, the first
  // two planes down likewise (KappaScalar reads two levels either side)
  void scalar_copies(std::vector<Copy> &cps, int b) const {
    for (int q = 0; q < nslots(); q++)
      for (int s = 0; s + 1 < ns; s++) {
        const size_t pb = plane_bytes(s);
        cps.push_back(Copy{s, s + 1, splane(s + 1, q, b, 0), splane(s, q, b, nzl[s]), pb});
        cps.push_back(Copy{s, s + 1, sl[s + 1]->hdom[0].slot[q].h2[0], splane(s, q, b, nzl[s] - 1), pb});
        cps.push_back(Copy{s + 1, s, splane(s, q, b, nzl[s] + 1), splane(s + 1, q, b, 1), pb});
        cps.push_back(Copy{s + 1, s, sl[s]->hdom[0].slot[q].h2[1], splane(s + 1, q, b, 2), pb});
      }
  }
  // the diffusivity's ghost planes at the shared faces, both ways
  void tdiff_copies(std::vector<Copy> &cps) const {
    if (!sl[0]->hdom[0].TDiff) return;
    for (int s = 0; s + 1 < ns; s++) {
      cps.push_back(Copy{s, s + 1, splane(s + 1, -1, 0, 0), splane(s, -1, 0, nzl[s]), plane_bytes(s)});
      cps.push_back(Copy{s + 1, s, splane(s, -1, 0, nzl[s] + 1), splane(s + 1, -1, 0, 1), plane_bytes(s)});
    }
  }
  // after a projection: U V W P both ways, the top slab's pressure reference to all
  int exchange_state() {
    std::vector<Copy> cps;
    halo_copies(cps, {F_U, F_V, F_W, F_P}, true, true);
    for (int s = 0; s + 1 < ns; s++)
      cps.push_back(Copy{ns - 1, s, sl[s]->hdom[0].prm, sl[ns - 1]->hdom[0].prm, sizeof(double)});
    return exchange(cps);
  }

  // -------------------------------------------------------------- stages
  template <typename F>
  void each(F f) {
    for (int s = 0; s < ns; s++) {
      cudaSetDevice(dev[s]);  // a failure shows in the synchronisation that ends the call
      f(s, *sl[s]);
    }
  }
  // the Poisson solve and PostPoisson of every slab (coef_alpha2: 2 alpha
  // of the stage, times dt with use_dt); U2 -> U, as launch_projection
  int projection(double coef_alpha2, int use_dt) {
    int r;
    each([&](int, BatchT<T> &B) {
      B.launch_fftx_fwd(coef_alpha2, use_dt, 0, 0);
      B.launch_ffty(0, 0);
    });
    std::vector<Copy> cps;
    each([&](int s, BatchT<T> &B) {
      const int ncol = B.hdom[0].ny * B.hdom[0].spitch;
      const int ntile = (ncol + kSlabCols - 1) / kSlabCols;
      if (tiled)
        k_slab_tri_fmap_tile<T, kSlabCols><<<ntile, Tile::THREADS, smem_tile, B.stream>>>(
            B.ddom, tri[s].iv, tri[s].fmaps + 3LL * ncol * s, tri[s].zcol, k0[s], nzg);
      else
        k_slab_tri_fmap<T><<<(2 * ncol + 127) / 128, 128, 0, B.stream>>>(B.ddom, tri[s].iv, tri[s].fmaps + 3LL * ncol * s,
                                                                         tri[s].zcol, k0[s], nzg);
      B.nlaunch++;
      for (int t = 0; t < ns; t++) {
        if (t == s) continue;
        if (t > s) cps.push_back(Copy{s, t, tri[t].fmaps + 3LL * ncol * s, tri[s].fmaps + 3LL * ncol * s,
                                      sizeof(double) * 3 * ncol});
        for (int part = 0; part < 2; part++)
          cps.push_back(Copy{s, t, tri[t].zcol + (size_t)part * nzg + k0[s], tri[s].zcol + (size_t)part * nzg + k0[s],
                             sizeof(double) * nzl[s]});
      }
    });
    if ((r = exchange(cps))) return r;
    cps.clear();
    each([&](int s, BatchT<T> &B) {
      const int ncol = B.hdom[0].ny * B.hdom[0].spitch;
      const int ntile = (ncol + kSlabCols - 1) / kSlabCols;
      if (tiled)
        k_slab_tri_fwd_tile<T, kSlabCols><<<ntile, Tile::THREADS, smem_tile, B.stream>>>(
            B.ddom, tri[s].iv, tri[s].fmaps, tri[s].bmaps + 3LL * ncol * s, tri[s].zcol, tri[s].dzc, tri[s].dzf, k0[s],
            nzg, s);
      else
        k_slab_tri_fwd<T><<<(2 * ncol + 127) / 128, 128, 0, B.stream>>>(B.ddom, tri[s].iv, tri[s].fmaps,
                                                                        tri[s].bmaps + 3LL * ncol * s, tri[s].zcol,
                                                                        tri[s].dzc, tri[s].dzf, k0[s], nzg, s);
      B.nlaunch++;
      for (int t = 0; t < s; t++)
        cps.push_back(Copy{s, t, tri[t].bmaps + 3LL * ncol * s, tri[s].bmaps + 3LL * ncol * s, sizeof(double) * 3 * ncol});
    });
    if ((r = exchange(cps))) return r;
    each([&](int s, BatchT<T> &B) {
      const int ncol = B.hdom[0].ny * B.hdom[0].spitch;
      const int ntile = (ncol + kSlabCols - 1) / kSlabCols;
      if (tiled)
        k_slab_tri_bwd_tile<T, kSlabCols><<<ntile, Tile::THREADS, smem_tile, B.stream>>>(B.ddom, tri[s].iv, tri[s].bmaps,
                                                                                         s, ns);
      else
        k_slab_tri_bwd<T><<<(2 * ncol + 127) / 128, 128, 0, B.stream>>>(B.ddom, tri[s].iv, tri[s].bmaps, s, ns);
      B.nlaunch++;
      B.launch_ffty(1, 0);
      B.launch_fftx_inv(0);
    });
    if ((r = exchange_halos({F_PHI}, false, true))) return r;
    each([&](int, BatchT<T> &B) { B.launch_project(coef_alpha2, use_dt, 0, 0); });
    return exchange_state();
  }
  int stage(int st) {
    int r;
    std::vector<Copy> cps;
    each([&](int, BatchT<T> &B) { B.launch_sgs(st); });
    halo_copies(cps, {F_NU}, true, true);
    tdiff_copies(cps);
    if ((r = exchange(cps))) return r;
    // ScalarRK3 between Convection and the projection (src/tsteps.f90:132-135)
    each([&](int, BatchT<T> &B) {
      B.launch_momentum(st);
      B.launch_scalars(st, st == 3);
    });
    cps.clear();
    halo_copies(cps, {F_W2}, true, false);
    scalar_copies(cps, st % 3);
    if ((r = exchange(cps))) return r;
    return projection(2 * kAlpha[st - 1], 1);
  }
  // one step of every slab for the captured graph: fork the slabs' streams
  // from slab 0's, the step (the divergence check included, as in the
  // single-domain graph), join them back
  int enqueue_step(bool cfl) {
    CU(cudaEventRecord(ev_fork, sl[0]->stream));
    for (int s = 1; s < ns; s++) CU(cudaStreamWaitEvent(sl[s]->stream, ev_fork, 0));
    if (cfl) each([&](int, BatchT<T> &B) { B.launch_cfl(); });
    each([&](int, BatchT<T> &B) { B.launch_puff_prep(); });
    int r = ELMM_OK;
    for (int st = 1; st <= 3 && !r; st++) r = stage(st);
    if (r) return r;
    each([&](int, BatchT<T> &B) { B.launch_divmax(); });
    for (int s = 1; s < ns; s++) {
      CU(cudaEventRecord(post[s], sl[s]->stream));
      CU(cudaStreamWaitEvent(sl[0]->stream, post[s], 0));
    }
    return ELMM_OK;
  }
  int step_graph(int nsteps, bool cfl) {
    CU(cudaSetDevice(dev[0]));
    cudaStream_t s0 = sl[0]->stream;
    if (!step_exec || step_has_cfl != cfl) {
      if (step_exec) { cudaGraphExecDestroy(step_exec); step_exec = nullptr; }
      for (int s = 0; s < ns; s++) sl[s]->nlaunch = 0;
      CU(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
      const int r = enqueue_step(cfl);
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(s0, &g);  // ends the capture whatever happened
      if (r) {
        if (g) cudaGraphDestroy(g);
        return r;
      }
      if (e != cudaSuccess) return fail(ELMM_ERR_CUDA, std::string("slab step capture: ") + cudaGetErrorString(e));
      const cudaError_t ei = cudaGraphInstantiate(&step_exec, g, 0);
      cudaGraphDestroy(g);
      if (ei != cudaSuccess) return fail(ELMM_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ei));
      step_has_cfl = cfl;
      step_kernels = 0;
      for (int s = 0; s < ns; s++) step_kernels += sl[s]->nlaunch;
    }
    CU(cudaEventRecord(t0, s0));
    for (int n = 0; n < nsteps; n++) CU(cudaGraphLaunch(step_exec, s0));
    CU(cudaEventRecord(t1, s0));
    CU(cudaStreamSynchronize(s0));
    CU(cudaGetLastError());
    kernels = nsteps * step_kernels;
    return ELMM_OK;
  }
  int step(int nsteps, elmm_stats *stats) {
    if (nsteps < 0) return fail(ELMM_ERR_INVALID_ARG, "nsteps must be non-negative");
    const bool cfl = gcfg.enable_CFL_check != 0;
    if (one_device() && nsteps > 0) {
      int r = step_graph(nsteps, cfl);
      if (r) return r;
      time += nsteps * gcfg.dt;
      return stats_of(stats, nsteps);
    }
    int r = begin();
    if (r) return r;
    for (int n = 0; n < nsteps; n++) {
      if (cfl) each([&](int, BatchT<T> &B) { B.launch_cfl(); });
      each([&](int, BatchT<T> &B) { B.launch_puff_prep(); });
      for (int st = 1; st <= 3 && !r; st++) r = stage(st);
      if (r) return r;
      if (n == nsteps - 1) each([&](int, BatchT<T> &B) { B.launch_divmax(); });
    }
    if ((r = finish())) return r;
    time += nsteps * gcfg.dt;
    return stats_of(stats, nsteps);
  }
  // the initial projection (PressureCorrection on the state, then the eddy
  // viscosity of the projected field), as BatchT::project
  int project(double coef, elmm_stats *stats) {
    int r = begin();
    if (r) return r;
    each([&](int, BatchT<T> &B) {
      const Dom<T> &h = B.hdom[0];
      const size_t box = (size_t)h.plane * (h.nz + 2) * sizeof(T);
      cudaMemcpyAsync(h.U2, h.U, box, cudaMemcpyDeviceToDevice, B.stream);
      cudaMemcpyAsync(h.V2, h.V, box, cudaMemcpyDeviceToDevice, B.stream);
      cudaMemcpyAsync(h.W2, h.W, box, cudaMemcpyDeviceToDevice, B.stream);
    });
    if ((r = projection(coef, 0))) return r;
    each([&](int, BatchT<T> &B) {
      B.launch_divmax();
      B.sgs_kernel(1);
      B.wm_kernel(1, B.stream);
      B.launch_ghosts({F_NU}, 0);
    });
    {
      std::vector<Copy> cps;
      halo_copies(cps, {F_NU}, true, true);
      tdiff_copies(cps);
      if ((r = exchange(cps))) return r;
    }
    if ((r = finish())) return r;
    return stats_of(stats, 0);
  }
  int begin() {
    for (int s = 0; s < ns; s++) sl[s]->nlaunch = 0;
    CU(cudaSetDevice(dev[0]));
    CU(cudaEventRecord(t0, sl[0]->stream));
    // every slab starts after the call's start on slab 0
    for (int s = 1; s < ns; s++) {
      CU(cudaSetDevice(dev[s]));
      CU(cudaStreamWaitEvent(sl[s]->stream, t0, 0));
    }
    return ELMM_OK;
  }
  int finish() {
    for (int s = 1; s < ns; s++) {
      CU(cudaSetDevice(dev[s]));
      CU(cudaEventRecord(post[s], sl[s]->stream));
      CU(cudaSetDevice(dev[0]));
      CU(cudaStreamWaitEvent(sl[0]->stream, post[s], 0));
    }
    CU(cudaSetDevice(dev[0]));
    CU(cudaEventRecord(t1, sl[0]->stream));
    for (int s = 0; s < ns; s++) {
      CU(cudaSetDevice(dev[s]));
      CU(cudaStreamSynchronize(sl[s]->stream));
      CU(cudaGetLastError());
    }
    kernels = 0;
    for (int s = 0; s < ns; s++) kernels += sl[s]->nlaunch;
    return ELMM_OK;
  }
  int stats_of(elmm_stats *st, int nsteps) {
    double md = 0, cf = 0;
    int gave_up = 0;
    for (int s = 0; s < ns; s++) {
      const Dom<T> &h = sl[s]->hdom[0];
      CU(cudaSetDevice(dev[s]));
      int fl[2] = {0, 0};
      CU(cudaMemcpy(fl, h.flags, sizeof(fl), cudaMemcpyDeviceToHost));
      if (fl[1]) {
        gave_up = 1;
        CU(cudaMemset(h.flags + 1, 0, sizeof(int)));
      }
      unsigned long long b1 = 0, b2 = 0;
      CU(cudaMemcpy(&b1, h.maxdiv_bits, sizeof(b1), cudaMemcpyDeviceToHost));
      CU(cudaMemcpy(&b2, h.cfl_bits, sizeof(b2), cudaMemcpyDeviceToHost));
      double a, c2;
      memcpy(&a, &b1, 8);
      memcpy(&c2, &b2, 8);
      if (!(a <= md)) md = a;
      c2 *= gcfg.dt;
      if (!(c2 <= cf)) cf = c2;
    }
    float ms = 0;
    CU(cudaSetDevice(dev[0]));
    cudaEventElapsedTime(&ms, t0, t1);
    if (st) {
      memset(st, 0, sizeof(*st));
      st->steps_done = nsteps;
      st->time = time;
      st->dt = gcfg.dt;
      st->cfl = cf;
      st->max_div = md;
      st->nan_detected = !std::isfinite(md) || !std::isfinite(cf);
      st->elapsed_ms = ms;
      st->kernels = kernels;
    }
    if (gave_up) return fail(ELMM_ERR_TIMEOUT, "a bounded device-side wait gave up (TMA copy did not arrive)");
    if (!std::isfinite(md) || !std::isfinite(cf)) return fail(ELMM_ERR_NAN, "non-finite values in the state");
    return ELMM_OK;
  }

  // ---------------------------------------------------------- host arrays
  // The whole domain's Fortran arrays; slab s reads the planes of its
  // levels and their ghosts (a view starting k0 planes in) and writes only
  // the planes it owns: its interior, and the outer ghost planes for the
  // first and last slab.
  static size_t plane_elems(const HostBox &hb) { return (size_t)hb.n0 * hb.n1; }
  // H: double, or float for the real32 arrays of a prec=sp host (widened
  // and narrowed on the device, as the single-domain *_float calls)
  template <typename H>
  int upload(const H *U, const H *V, const H *W, const H *Pr) {
    if (!U || !V || !W) return fail(ELMM_ERR_INVALID_ARG, "NULL velocity array");
    for (int s = 0; s < ns; s++) {
      BatchT<T> &B = *sl[s];
      const size_t pv[3] = {plane_elems(B.hbox_vel(0, 0)), plane_elems(B.hbox_vel(0, 1)), plane_elems(B.hbox_vel(0, 2))};
      const size_t pp = plane_elems(B.hbox_p(0));
      B.hostf = sizeof(H) == 4;
      int r = B.upload(0, U + pv[0] * k0[s], V + pv[1] * k0[s], W + pv[2] * k0[s], Pr ? Pr + pp * k0[s] : nullptr);
      B.hostf = 0;
      if (r) return r;
    }
    int r = exchange_state();
    if (r) return r;
    for (int s = 0; s < ns; s++) {
      CU(cudaSetDevice(dev[s]));
      CU(cudaStreamSynchronize(sl[s]->stream));
    }
    return ELMM_OK;
  }
  template <typename H>
  int download(H *U, H *V, H *W, H *Pr) {
    H *dst[4] = {U, V, W, Pr};
    for (int s = 0; s < ns; s++) {
      BatchT<T> &B = *sl[s];
      CU(cudaSetDevice(dev[s]));
      if (sizeof(H) == 4) {
        int r = B.ensure_fstage();
        if (r) return r;
      }
      for (int f = 0; f < 4; f++) {
        if (!dst[f]) continue;
        const HostBox hb = f < 3 ? B.hbox_vel(0, f) : B.hbox_p(0);
        const int top = f < 3 ? B.hdom[0].ext[f][2] : B.hdom[0].nz;
        const int kw0 = s == 0 ? hb.lo : 1, kw1 = s == ns - 1 ? hb.lo + hb.n2 - 1 : top;
        const size_t pe = plane_elems(hb), skip = (size_t)(kw0 - hb.lo) * pe, cnt = pe * (kw1 - kw0 + 1);
        const size_t n = B.pack(0, f, B.dstage, B.stream);
        const void *src = B.dstage + skip;
        if (sizeof(H) == 4) {
          k_narrow<<<kPackBlocks, 256, 0, B.stream>>>(B.fstage, B.dstage, (long long)n);
          src = B.fstage + skip;
        }
        CU(cudaMemcpyAsync(dst[f] + pe * k0[s] + skip, src, sizeof(H) * cnt, cudaMemcpyDeviceToHost, B.stream));
        CU(cudaStreamSynchronize(B.stream));
      }
      CU(cudaGetLastError());
    }
    return ELMM_OK;
  }
  // TMarchRK3 on the whole domain's host arrays: upload, nsteps steps, download
  template <typename H>
  int march_host(H *U, H *V, H *W, H *Pr, int nsteps, elmm_stats *st) {
    int r = upload<H>(U, V, W, Pr);
    if (!r) r = step(nsteps, st);
    if (!r) r = download<H>(U, V, W, Pr);
    return r;
  }
  // the temperature (sc = 0) or passive scalar sc from the whole domain's
  // host array F(-2:nx+3, -2:ny+3, -2:nz+3): slab s takes the planes from its
  // k0 on, then the slabs exchange their halos
  int upload_scalar(int sc, const double *F) {
    if (!F) return fail(ELMM_ERR_INVALID_ARG, "NULL array");
    const Dom<T> &h0 = sl[0]->hdom[0];
    if (sc == 0 ? !h0.buoy : (sc < 1 || sc > gcfg.num_scalars))
      return fail(ELMM_ERR_INVALID_ARG, sc == 0 ? "no temperature field (enable_buoyancy is 0)"
                                                : "scalar number outside 1..num_scalars");
    const size_t ph = (size_t)(h0.nx + 6) * (h0.ny + 6);
    for (int s = 0; s < ns; s++) {
      BatchT<T> &B = *sl[s];
      int r = sc == 0 ? B.upload_temperature(0, F + ph * k0[s]) : B.upload_scalar(0, sc, F + ph * k0[s]);
      if (r) return r;
    }
    std::vector<Copy> cps;
    scalar_copies(cps, 0);
    int r = exchange(cps);
    if (r) return r;
    for (int s = 0; s < ns; s++) {
      CU(cudaSetDevice(dev[s]));
      CU(cudaStreamSynchronize(sl[s]->stream));
    }
    return ELMM_OK;
  }
  // puff sources (elmm_set_puffs): every slab runs every puff's windows, and
  // takes the volumes in its levels
  int set_puffs(const elmm_puff *pf, int np, const elmm_puff_volume *vol, int nv) {
    if (nv < 0 || nv > kMaxPuffVols || (nv > 0 && !vol)) return fail(ELMM_ERR_INVALID_ARG, "puff volumes");
    if (step_exec) { cudaGraphExecDestroy(step_exec); step_exec = nullptr; }
    for (int s = 0; s < ns; s++) {
      std::vector<elmm_puff_volume> mine;
      for (int q = 0; q < nv; q++)
        if (vol[q].zk > k0[s] && vol[q].zk <= k0[s] + nzl[s]) {
          elmm_puff_volume v = vol[q];
          v.zk -= k0[s];
          mine.push_back(v);
        }
      int r = sl[s]->set_puffs(0, pf, np, mine.data(), (int)mine.size(), vol, nv);  // a restart clears every slab
      if (r) return r;
    }
    return ELMM_OK;
  }
  // the time-averaged slices of scalar sc: xy from the slab holding its
  // level, xz(1:Prnx, 1:Prnz) row blocks from every slab
  int download_scalar_slices(int sc, double *xy, double *xz) {
    for (int s = 0; s < ns; s++) {
      const bool has_xy = sl[s]->cfg[0].avg_slice_k > 0;
      int r = sl[s]->download_scalar_slices(0, sc, has_xy ? xy : nullptr,
                                           xz ? xz + (size_t)sl[s]->hdom[0].nx * k0[s] : nullptr);
      if (r) return r;
    }
    if (xy && gcfg.avg_slice_k <= 0) return fail(ELMM_ERR_INVALID_ARG, "no such slice (avg_slice_k is 0)");
    return ELMM_OK;
  }
  // ELMM_FIELD_TEMPERATURE or ELMM_FIELD_SCALAR + sc - 1 into the whole
  // domain's host array, every element the single-domain download writes
  int download_field(int field, double *host) {
    if (!host) return fail(ELMM_ERR_INVALID_ARG, "NULL array");
    const Dom<T> &h0 = sl[0]->hdom[0];
    const bool ok = (field == ELMM_FIELD_TEMPERATURE && h0.buoy) ||
                    (field >= ELMM_FIELD_SCALAR && field < ELMM_FIELD_SCALAR + gcfg.num_scalars);
    if (!ok) return fail(ELMM_ERR_INVALID_ARG, "split domains download the temperature and the passive scalars");
    const size_t ph = (size_t)(h0.nx + 6) * (h0.ny + 6);
    for (int s = 0; s < ns; s++) {
      BatchT<T> &B = *sl[s];
      CU(cudaSetDevice(dev[s]));
      const int kw0 = s == 0 ? -2 : 1, kw1 = s == ns - 1 ? nzl[s] + 3 : nzl[s];
      const size_t skip = (size_t)(kw0 + 2) * ph;
      B.pack(0, field, B.dstage, B.stream);
      CU(cudaMemcpyAsync(host + ph * k0[s] + skip, B.dstage + skip, sizeof(double) * ph * (kw1 - kw0 + 1),
                         cudaMemcpyDeviceToHost, B.stream));
      CU(cudaStreamSynchronize(B.stream));
      CU(cudaGetLastError());
    }
    return ELMM_OK;
  }
};

struct elmm_slabs {
  int precision = 0;
  std::unique_ptr<SlabsT<double>> s64;
  std::unique_ptr<SlabsT<float>> s32;
};
#define SLAB_DISPATCH(H, EXPR) ((H)->precision == ELMM_PREC_MIXED ? (H)->s32->EXPR : (H)->s64->EXPR)

extern "C" int elmm_slabs_create(const elmm_config *cfg, int32_t nslabs, const int32_t *devices, const int32_t *nz_slab,
                                 elmm_slabs **out) {
  if (!cfg || !out) return fail(ELMM_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  std::unique_ptr<elmm_slabs> h(new elmm_slabs());
  h->precision = cfg->precision;
  int r;
  if (h->precision == ELMM_PREC_MIXED) {
    h->s32.reset(new SlabsT<float>());
    r = h->s32->init(*cfg, nslabs, devices, nz_slab);
  } else {
    h->s64.reset(new SlabsT<double>());
    r = h->s64->init(*cfg, nslabs, devices, nz_slab);
  }
  if (r) return r;
  *out = h.release();
  return ELMM_OK;
}

extern "C" int elmm_slabs_destroy(elmm_slabs *h) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  delete h;
  return ELMM_OK;
}

extern "C" int elmm_slabs_upload_state(elmm_slabs *h, const double *U, const double *V, const double *W,
                                       const double *Pr) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return SLAB_DISPATCH(h, upload(U, V, W, Pr));
}

extern "C" int elmm_slabs_download_state(elmm_slabs *h, double *U, double *V, double *W, double *Pr) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return SLAB_DISPATCH(h, download(U, V, W, Pr));
}

extern "C" int elmm_slabs_upload_state_float(elmm_slabs *h, const float *U, const float *V, const float *W,
                                             const float *Pr) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return SLAB_DISPATCH(h, upload(U, V, W, Pr));
}

extern "C" int elmm_slabs_download_state_float(elmm_slabs *h, float *U, float *V, float *W, float *Pr) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return SLAB_DISPATCH(h, download(U, V, W, Pr));
}

extern "C" int elmm_slabs_march_host(elmm_slabs *h, double *U, double *V, double *W, double *Pr, int32_t nsteps,
                                     elmm_stats *stats) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  if (nsteps < 0) return fail(ELMM_ERR_INVALID_ARG, "nsteps < 0");
  return SLAB_DISPATCH(h, march_host(U, V, W, Pr, nsteps, stats));
}

extern "C" int elmm_slabs_march_host_float(elmm_slabs *h, float *U, float *V, float *W, float *Pr, int32_t nsteps,
                                           elmm_stats *stats) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  if (nsteps < 0) return fail(ELMM_ERR_INVALID_ARG, "nsteps < 0");
  return SLAB_DISPATCH(h, march_host(U, V, W, Pr, nsteps, stats));
}

extern "C" int elmm_slabs_upload_temperature(elmm_slabs *h, const double *T) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return SLAB_DISPATCH(h, upload_scalar(0, T));
}

extern "C" int elmm_slabs_upload_scalar(elmm_slabs *h, int32_t sc, const double *S) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  if (sc < 1) return fail(ELMM_ERR_INVALID_ARG, "scalar number outside 1..num_scalars");
  return SLAB_DISPATCH(h, upload_scalar(sc, S));
}

extern "C" int elmm_slabs_download_field(elmm_slabs *h, int32_t field, double *host) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return SLAB_DISPATCH(h, download_field(field, host));
}

extern "C" int elmm_slabs_set_puffs(elmm_slabs *h, const elmm_puff *puffs, int32_t npuffs,
                                    const elmm_puff_volume *volumes, int32_t nvolumes) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return SLAB_DISPATCH(h, set_puffs(puffs, npuffs, volumes, nvolumes));
}

extern "C" int elmm_slabs_download_scalar_slices(elmm_slabs *h, int32_t sc, double *xy, double *xz) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return SLAB_DISPATCH(h, download_scalar_slices(sc, xy, xz));
}

extern "C" int elmm_slabs_project(elmm_slabs *h, double coef, elmm_stats *stats) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return SLAB_DISPATCH(h, project(coef, stats));
}

extern "C" int elmm_slabs_step(elmm_slabs *h, int32_t nsteps, elmm_stats *stats) {
  if (!h) return fail(ELMM_ERR_INVALID_ARG, "NULL handle");
  return SLAB_DISPATCH(h, step(nsteps, stats));
}
