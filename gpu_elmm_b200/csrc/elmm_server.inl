// elmm_server.inl -- the serving loop: continuous batching of dispersion
// requests (included by elmm_api.cu after BatchT).
//
// One worker thread owns the device work.  Each admitted request is a
// single-domain BatchT whose fields come from the server's HBM budget (an
// Arena over one allocation made at creation); the admitted requests step
// together through a view, a BatchT over their domains whose launch set and
// step graph are rebuilt whenever the set changes.  The loop:
//
//   launch a chunk of steps for the active set (asynchronous)
//   admit queued requests while the chunk runs: carve their memory from the
//     budget, upload their state and run their initial projection on their
//     own streams
//   wait for the chunk; requests that have run all their steps leave the
//     set, their averaged slices go to the host, their memory to the budget
//   admitted requests join the set (the next chunk rebuilds the view)
//
// A chunk is at most chunk_steps steps and never runs past the end of an
// active request, so requests finish exactly at their step count.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <thread>

template <typename T>
struct ServerT {
  struct Req {
    int64_t id = 0;
    elmm_config cfg;
    const double *U = nullptr, *V = nullptr, *W = nullptr, *Pr = nullptr, *S0 = nullptr;
    int nsteps = 0, done = 0;
    int64_t cells = 0;
    std::unique_ptr<BatchT<T>> dom;
    int64_t bytes = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    int status = ELMM_OK;
    std::string err;
    std::vector<double> xy, xz;
    double max_div = 0;
    bool finished = false;
  };

  elmm_server_config sc{};
  char *base = nullptr;          // the budget: one device allocation
  Arena arena;                   // request fields
  Arena tables;                  // launch tables of the views
  cudaStream_t stream = nullptr; // the stream the active set steps on
  cudaEvent_t c0 = nullptr, c1 = nullptr;
  std::chrono::steady_clock::time_point t_start;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stopping = false;
  int64_t next_id = 1;
  // guarded by mu
  std::deque<Req *> queue;
  std::deque<Req *> unreported;
  std::map<int64_t, std::unique_ptr<Req>> reqs;
  elmm_server_stats st{};
  // worker only
  std::vector<Req *> active, joining;
  std::unique_ptr<BatchT<T>> view;
  bool dirty = false;

  static constexpr size_t kTableBytes = 32u << 20;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  }

  int init(const elmm_server_config &c) {
    sc = c;
    t_start = std::chrono::steady_clock::now();
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= sc.device) return fail(ELMM_ERR_CUDA, "no CUDA device");
    CU(cudaSetDevice(sc.device));
    const size_t total = (size_t)sc.hbm_budget_bytes + kTableBytes;
    cudaError_t e = cudaMalloc((void **)&base, total);
    if (e != cudaSuccess) {
      base = nullptr;
      return fail(ELMM_ERR_OOM, std::string("cudaMalloc of the serving budget: ") + cudaGetErrorString(e));
    }
    arena.reset(base, (size_t)sc.hbm_budget_bytes);
    tables.reset(base + Arena::round((size_t)sc.hbm_budget_bytes), kTableBytes - Arena::kAlign);
    CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CU(cudaEventCreate(&c0));
    CU(cudaEventCreate(&c1));
    st.budget_bytes = sc.hbm_budget_bytes;
    worker = std::thread([this] { run(); });
    return ELMM_OK;
  }

  ~ServerT() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stopping = true;
    }
    cv_work.notify_all();
    if (worker.joinable()) worker.join();
    if (stream) cudaStreamSynchronize(stream);
    view.reset();
    for (auto &kv : reqs) kv.second->dom.reset();
    reqs.clear();
    if (c0) cudaEventDestroy(c0);
    if (c1) cudaEventDestroy(c1);
    if (stream) cudaStreamDestroy(stream);
    if (base) cudaFree(base);
  }

  int submit(const elmm_config &cfg, const double *U, const double *V, const double *W, const double *Pr,
             const double *S0, int nsteps, int64_t *id) {
    if (cfg.precision != sc.precision || cfg.device != sc.device)
      return fail(ELMM_ERR_INVALID_CONFIG, "a request must use the server's precision and device");
    if (nsteps < 1) return fail(ELMM_ERR_INVALID_ARG, "nsteps must be positive");
    if (!U || !V || !W) return fail(ELMM_ERR_INVALID_ARG, "NULL velocity array");
    if (S0 && cfg.num_scalars < 1) return fail(ELMM_ERR_INVALID_ARG, "an initial scalar needs num_scalars >= 1");
    if (cfg.zW) return fail(ELMM_ERR_INVALID_CONFIG, "the serving loop takes uniform grids");
    int r = check_config(cfg);
    if (r) return r;
    auto q = std::make_unique<Req>();
    q->cfg = cfg;
    q->U = U; q->V = V; q->W = W; q->Pr = Pr; q->S0 = S0;
    q->nsteps = nsteps;
    q->cells = (int64_t)cfg.Prnx * cfg.Prny * cfg.Prnz;
    {
      std::lock_guard<std::mutex> lk(mu);
      q->id = next_id++;
      q->t_submit = now();
      *id = q->id;
      queue.push_back(q.get());
      reqs[q->id] = std::move(q);
      st.submitted++;
      st.queued = (int32_t)queue.size();
    }
    cv_work.notify_all();
    return ELMM_OK;
  }

  int wait_any(int timeout_ms, elmm_request_info *info) {
    std::unique_lock<std::mutex> lk(mu);
    if (!cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return !unreported.empty(); }))
      return fail(ELMM_ERR_TIMEOUT, "no request finished in time");
    Req *r = unreported.front();
    unreported.pop_front();
    memset(info, 0, sizeof(*info));
    info->id = r->id;
    info->status = r->status;
    info->steps = r->done;
    info->t_submit = r->t_submit;
    info->t_admit = r->t_admit;
    info->t_done = r->t_done;
    info->bytes = r->bytes;
    info->max_div = r->max_div;
    info->cells = r->cells;
    if (r->status != ELMM_OK) g_err = r->err;
    return ELMM_OK;
  }

  int collect(int64_t id, double *xy, double *xz) {
    std::lock_guard<std::mutex> lk(mu);
    auto it = reqs.find(id);
    if (it == reqs.end()) return fail(ELMM_ERR_INVALID_ARG, "unknown request id");
    Req *r = it->second.get();
    if (!r->finished) return fail(ELMM_ERR_INVALID_ARG, "the request has not finished");
    if (r->status != ELMM_OK) {
      const std::string m = r->err;
      const int code = r->status;
      reqs.erase(it);
      return fail(code, m);
    }
    if ((xy && r->xy.empty()) || (xz && r->xz.empty()))
      return fail(ELMM_ERR_INVALID_ARG, "no such slice (avg_slice_k / avg_slice_j is 0)");
    if (xy) memcpy(xy, r->xy.data(), r->xy.size() * sizeof(double));
    if (xz) memcpy(xz, r->xz.data(), r->xz.size() * sizeof(double));
    reqs.erase(it);
    return ELMM_OK;
  }

  void stats(elmm_server_stats *out) {
    std::lock_guard<std::mutex> lk(mu);
    *out = st;
  }

  // ---------------------------------------------------------------- worker
  void finish(Req *r, int status, const std::string &err) {
    r->status = status;
    r->err = err;
    r->t_done = now();
    r->dom.reset();  // the memory returns to the budget
    {
      std::lock_guard<std::mutex> lk(mu);
      r->finished = true;
      unreported.push_back(r);
      if (status == ELMM_OK) st.finished++;
      else st.failed++;
      st.bytes_in_use = (int64_t)arena.in_use();
    }
    cv_done.notify_all();
  }

  void admit() {
    for (;;) {
      Req *r;
      size_t qi = 0;
      {
        std::lock_guard<std::mutex> lk(mu);
        if (queue.empty() || (int)(active.size() + joining.size()) >= sc.max_active) return;
        if (sc.policy == ELMM_SERVE_SHORTEST_FIRST)
          for (size_t q = 1; q < queue.size(); q++)
            if (queue[q]->cells * queue[q]->nsteps < queue[qi]->cells * queue[qi]->nsteps) qi = q;
        r = queue[qi];
      }
      auto b = std::make_unique<BatchT<T>>();
      b->arena = &arena;
      int rc = b->init(&r->cfg, 1);
      std::string err = rc ? g_err : std::string();
      if (rc == ELMM_ERR_ADMISSION) {
        b.reset();
        // with nothing else on the device the request can never fit
        if (!(active.empty() && joining.empty() && arena.empty())) return;
        err = "the request needs more device memory than the whole serving budget";
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        queue.erase(queue.begin() + qi);
        st.queued = (int32_t)queue.size();
      }
      if (rc) {
        finish(r, rc, err);
        continue;
      }
      rc = b->upload(0, r->U, r->V, r->W, r->Pr);
      if (!rc && r->S0) rc = b->upload_scalar(0, 1, r->S0);
      if (!rc) rc = b->project(1.0, nullptr);
      if (rc) {
        r->dom = std::move(b);
        finish(r, rc, g_err);
        continue;
      }
      b->drop_host_staging();
      r->bytes = (int64_t)b->arena_bytes;
      r->t_admit = now();
      r->dom = std::move(b);
      joining.push_back(r);
      std::lock_guard<std::mutex> lk(mu);
      st.admitted++;
      st.bytes_in_use = (int64_t)arena.in_use();
      st.bytes_peak = std::max<int64_t>(st.bytes_peak, (int64_t)arena.peak());
    }
  }

  int rebuild_view() {
    view.reset();
    dirty = false;
    if (active.empty()) return ELMM_OK;
    std::vector<BatchT<T> *> members;
    for (Req *r : active) members.push_back(r->dom.get());
    auto v = std::make_unique<BatchT<T>>();
    int rc = v->init_view(members, stream, &tables);
    if (rc) return rc;
    view = std::move(v);
    std::lock_guard<std::mutex> lk(mu);
    st.graph_builds++;
    return ELMM_OK;
  }

  int launch_chunk(int n) {
    CU(cudaEventRecord(c0, stream));
    int rc = view->step_launch(n);
    if (rc) return rc;
    CU(cudaEventRecord(c1, stream));
    return ELMM_OK;
  }

  // waits for the chunk; per-request checks of NaN and of bounded waits
  int finish_chunk(int n) {
    CU(cudaStreamSynchronize(stream));
    CU(cudaGetLastError());
    float ms = 0;
    cudaEventElapsedTime(&ms, c0, c1);
    int64_t cs = 0;
    std::vector<Req *> keep;
    for (int q = 0; q < (int)active.size(); q++) {
      Req *r = active[q];
      const Dom<T> &h = view->hdom[q];
      unsigned long long bits = 0;
      int fl[2] = {0, 0};
      CU(cudaMemcpy(&bits, h.maxdiv_bits, sizeof(bits), cudaMemcpyDeviceToHost));
      CU(cudaMemcpy(fl, h.flags, sizeof(fl), cudaMemcpyDeviceToHost));
      memcpy(&r->max_div, &bits, sizeof(double));
      r->done += n;
      cs += r->cells * n;
      if (!std::isfinite(r->max_div)) {
        finish(r, ELMM_ERR_NAN, "NaN or Inf in the velocity field");
      } else if (fl[1]) {
        finish(r, ELMM_ERR_TIMEOUT, "a device-side wait for a plane copy gave up; the step is incomplete");
      } else if (r->done >= r->nsteps) {
        int rc = ELMM_OK;
        if (r->cfg.num_scalars > 0 && r->cfg.avg_slice_k > 0) {
          r->xy.assign((size_t)r->cfg.Prnx * r->cfg.Prny, 0.0);
          rc = r->dom->download_scalar_slices(0, 1, r->xy.data(), nullptr);
        }
        if (!rc && r->cfg.num_scalars > 0 && r->cfg.avg_slice_j > 0) {
          r->xz.assign((size_t)r->cfg.Prnx * r->cfg.Prnz, 0.0);
          rc = r->dom->download_scalar_slices(0, 1, nullptr, r->xz.data());
        }
        finish(r, rc, rc ? g_err : std::string());
      } else {
        keep.push_back(r);
      }
    }
    if (keep.size() != active.size()) dirty = true;
    active.swap(keep);
    std::lock_guard<std::mutex> lk(mu);
    st.cell_steps += cs;
    st.chunks++;
    st.busy_s += ms * 1e-3;
    return ELMM_OK;
  }

  void fail_all(int rc, const std::string &err) {
    for (Req *r : active) finish(r, rc, err);
    for (Req *r : joining) finish(r, rc, err);
    active.clear();
    joining.clear();
    view.reset();
  }

  void run() {
    cudaSetDevice(sc.device);
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu);
        if (active.empty() && joining.empty())
          cv_work.wait(lk, [&] { return stopping || !queue.empty(); });
        if (stopping) break;
      }
      int n = 0;
      if (!active.empty()) {
        int rc = dirty || !view ? rebuild_view() : ELMM_OK;
        if (!rc) {
          n = sc.chunk_steps;
          for (Req *r : active) n = std::min(n, r->nsteps - r->done);
          rc = launch_chunk(n);
        }
        if (rc) {
          fail_all(rc, g_err);
          n = 0;
        }
      }
      admit();  // overlaps the chunk in flight
      if (n) {
        int rc = finish_chunk(n);
        if (rc) fail_all(rc, g_err);
      }
      // admitted requests join the set
      while (!joining.empty() && (int)active.size() < sc.max_active) {
        active.push_back(joining.front());
        joining.erase(joining.begin());
        dirty = true;
      }
      if (active.empty()) view.reset();
      std::lock_guard<std::mutex> lk(mu);
      st.active = (int32_t)active.size();
      st.peak_active = std::max<int32_t>(st.peak_active, st.active);
    }
    if (stream) cudaStreamSynchronize(stream);
    view.reset();
    for (Req *r : active) r->dom.reset();
    for (Req *r : joining) r->dom.reset();
  }
};

struct elmm_server {
  int precision = 0;
  std::unique_ptr<ServerT<double>> s64;
  std::unique_ptr<ServerT<float>> s32;
};
