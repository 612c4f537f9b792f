// Serving: continuous batching of DOS and Kubo-Bastin solves on one GPU.
//
// LinQT has no server (its drivers run one solve per process); this is the request
// loop of the B200 build.  Requests are queued at submit (states copied into pinned
// host blocks the server recycles), admitted in arrival order when an execution slot
// is free and their estimated device footprint fits in the HBM budget, and run on the
// slot's own CUDA stream, so solves admitted at different times overlap on the device.
// Workspaces come from the device's stream-ordered pool, which the server keeps
// populated up to its budget: a request's buffers are returned with cudaFreeAsync and
// reused by the next, with no device-wide synchronisation between requests.  Each
// request's chunking budget is its own footprint, which makes the chunking -- and with
// the fixed-order reductions the result -- independent of what else runs.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <unordered_map>

#include "internal.cuh"

namespace linqt {
// solver entry points of api.cu
void moments1d_for_server(Session *s, const DeviceOp &H, const DeviceOp *op, const double2 *states, int R, int M,
                          int precision, int block_width, double2 *mu);
void moments2d_for_server(Session *s, const DeviceOp &H, const DeviceOp *opl, const DeviceOp *opr,
                          const double2 *states, int R, int M, int precision, int block_width, double2 *mu);
void kubo_bastin_for_server(Session *s, const DeviceOp &H, const DeviceOp *op, const double2 *states, int R, int M,
                            int nump, double bw, double bc, int precision, int block_width, double2 *mu,
                            double *out);
}  // namespace linqt

using namespace linqt;

namespace {

typedef std::chrono::steady_clock clk;

// Fraction of the device the slots' persistent grids share (through the server's ledger):
// a little below 1 leaves room for CTAs of different kernels that do not pack evenly.
constexpr double kSlotShare = 0.9;
// Times per slot that a queued request waiting for memory may be passed by later ones.
constexpr int kMaxBypass = 4;

struct Job {
  long ticket = 0;
  linqt_request req{};
  void *states = nullptr;  // pinned host copy (server pool); NULL: generated on the device
  size_t states_cap = 0;
  size_t footprint = 0;
  int block_width = 1;
  int status = 0;  // 0 pending, 1 running, 2 done, <0 error
  bool alone = false;  // ran out of memory next to other requests: runs again with none beside it
  int bypassed = 0;    // requests admitted before it while it waited for memory
  double latency_ms = 0;
  std::string error;
  clk::time_point t_submit;
};

// Device bytes a request may hold: every workspace of the solver it runs (state copy,
// Chebyshev blocks, per-step partials, contraction partials) at vector-block width Rc.
size_t estimate_footprint(const linqt_request &r, int n, int sm_count, int Rc) {
  const size_t esz = r.precision == LINQT_PREC_FP64 ? sizeof(double2) : sizeof(float2);
  const size_t io = sizeof(double2) * ((size_t)r.R * n + (size_t)r.M * (r.kind == LINQT_REQ_DOS ? 1 : r.M));
  if (r.kind == LINQT_REQ_DOS) {
    const size_t steps = (size_t)r.M / 2 + 1, chunks = (r.R + Rc - 1) / Rc;
    return io + esz * (size_t)n * Rc * 3 +
           sizeof(double2) * (2 * steps * ((size_t)sm_count * 32 + 1) + 2 * steps * chunks) + (1 << 20);
  }
  // INT8 contraction planes: one K slab of them, as the solver's chunking counts them
  const size_t digits = i8_digit_bytes(i8_digits(r.precision), r.M, (long)n * Rc);
  // sigma(E): the per-site transforms' partial sums and the 3*nump outputs
  const size_t fft = r.sigma_out ? sizeof(double2) * 2 * (size_t)r.nump * 1024 + 3 * sizeof(double) * r.nump : 0;
  const size_t total = io + esz * (size_t)n * Rc * (2 * (size_t)r.M + 4) + digits +
                       sizeof(double2) * (size_t)r.M * r.M * 66 + fft + (1 << 20);
  return total + total / 20;  // 5 % for the buffers the estimate does not itemise
}

// Vector-block width of a request: the widest power of two up to R whose footprint fits in
// `cap` (the server's budget), as a solve alone on the device would choose: a large request
// then runs as efficiently as alone (and alone, when its footprint leaves no room), while
// smaller ones that fit pass it in the queue; width 1 when none does.
int pick_width(const linqt_request &r, int n, int sm_count, size_t cap) {
  int Rc = 1;
  while (Rc < r.R && Rc < 256) Rc <<= 1;
  while (Rc > 1 && estimate_footprint(r, n, sm_count, Rc) > cap) Rc >>= 1;
  return Rc;
}

}  // namespace

struct linqt_server {
  int device = 0;
  size_t budget = 0, in_use = 0;
  int max_active = 1, sm_count = 148;
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::deque<std::shared_ptr<Job>> queue;
  std::unordered_map<long, std::shared_ptr<Job>> jobs;
  long next_ticket = 1;
  int running = 0;
  long timeouts_retried = 0;  // requests re-run on the cooperative lane after a co-residency timeout
  long nomem_retried = 0;     // requests re-run alone after their workspaces did not fit
  bool stop = false;
  std::vector<std::thread> workers;
  // pinned host blocks by power-of-two capacity, recycled across requests
  std::multimap<size_t, void *> pinned_free;
  std::vector<void *> pinned_all;
  cudaMemPool_t pool = nullptr;
  uint64_t old_threshold = 0;
  CoopLedger ledger;  // the slots' persistent grids take their shares of the device from it

  void *pinned_get(size_t bytes, size_t *cap) {
    size_t c = 4096;
    while (c < bytes) c <<= 1;
    {
      std::lock_guard<std::mutex> g(mu);
      auto it = pinned_free.lower_bound(c);
      if (it != pinned_free.end() && it->first <= 4 * c) {
        void *p = it->second;
        *cap = it->first;
        pinned_free.erase(it);
        return p;
      }
    }
    void *p = nullptr;
    LQ_CUDA(cudaMallocHost(&p, c));
    {
      std::lock_guard<std::mutex> g(mu);
      pinned_all.push_back(p);
    }
    *cap = c;
    return p;
  }
  void pinned_put_locked(void *p, size_t cap) {
    if (p) pinned_free.emplace(cap, p);
  }

  void worker() {
    std::unique_ptr<linqt_session> sess(new linqt_session);
    {
      Session &s = sess->s;
      s.device = device;
      cudaSetDevice(device);
      cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
      s.own_stream = true;
      cudaDeviceGetAttribute(&s.sm_count, cudaDevAttrMultiProcessorCount, device);
      s.ledger = &ledger;
    }
    for (;;) {
      std::shared_ptr<Job> job;
      {
        std::unique_lock<std::mutex> g(mu);
        // admission: the oldest queued job whose footprint fits next to the running ones.  A
        // job that does not fit may be passed by later ones that do, at most kMaxBypass times
        // a slot; after that nothing behind it is admitted until it runs.  A job marked `alone`
        // (it ran out of memory next to others) waits at the head until none runs.
        const int max_bypass = kMaxBypass * max_active;
        auto pick = [&]() {
          for (auto it = queue.begin(); it != queue.end(); ++it) {
            const Job &f = **it;
            if (f.alone) return (it == queue.begin() && running == 0) ? it : queue.end();
            if (in_use + f.footprint <= budget) return it;
            if (f.bypassed >= max_bypass) return queue.end();
          }
          return queue.end();
        };
        cv.wait(g, [&] { return (stop && queue.empty()) || pick() != queue.end(); });
        if (queue.empty()) {  // stopping
          cudaStreamSynchronize(sess->s.stream);  // its share callbacks have run
          return;
        }
        const auto it = pick();
        for (auto p = queue.begin(); p != it; ++p) (*p)->bypassed++;
        job = *it;
        queue.erase(it);
        in_use += job->footprint;
        job->status = 1;
        running++;
      }
      if (job->alone) cudaMemPoolTrimTo(pool, 0);  // the pool's cached blocks back to the device
      int rc = 0;
      std::string err;
      void *res_host = nullptr;
      size_t res_cap = 0;
      // Persistent recursions of the slots run side by side: each grid takes what it needs of
      // the device from the server's ledger, up to what the other slots' running grids leave
      // free (at least a 1 / max_active part of kSlotShare, or all it needs, waiting for it
      // when less is free), and returns it when the kernel has finished; a request alone on
      // the device so gets all of it.  A grid that does not become co-resident in time (CTAs
      // of other kernels can hold SMs) ends its solve with LINQT_ERR_TIMEOUT; the request then
      // runs again at once on the device-wide cooperative lane.  A request whose workspaces
      // did not fit next to the others (LINQT_ERR_NOMEM: the footprint is an estimate) goes
      // back to the head of the queue to run alone.
      for (int attempt = 0; attempt < 2; ++attempt) {
        sess->s.coop_share = (attempt == 0 && max_active > 1 && !job->alone) ? kSlotShare / max_active : 1.0;
        rc = 0;
        err.clear();
        try {
          Session &s = sess->s;
          const DeviceOp &H = job->req.H->op;
          const DeviceOp *op = job->req.op ? &job->req.op->op : nullptr;
          const int n = H.n, R = job->req.R, M = job->req.M;
          const size_t sb = sizeof(double2) * (size_t)R * n;
          const size_t mb = sizeof(double2) * (size_t)M * (job->req.kind == LINQT_REQ_DOS ? 1 : M);
          s.hbm_budget = job->footprint;  // fixed per request: chunking independent of the other requests
          double2 *d_st = (double2 *)s.get("io_states", sb);
          double2 *d_mu = (double2 *)s.get("io_mu", mb);
          if (!res_host) res_host = pinned_get(mb, &res_cap);
          if (job->states)
            LQ_CUDA(cudaMemcpyAsync(d_st, job->states, sb, cudaMemcpyHostToDevice, s.stream));
          else
            random_phase_states(&s, n, R, job->req.seed, d_st);
          const bool sigma = job->req.kind == LINQT_REQ_KUBO_BASTIN && job->req.sigma_out;
          const size_t ob = sigma ? 3 * sizeof(double) * (size_t)job->req.nump : 0;
          double *d_out = sigma ? (double *)s.get("io_kubo", ob) : nullptr;
          if (job->req.kind == LINQT_REQ_DOS)
            moments1d_for_server(&s, H, op, d_st, R, M, job->req.precision, job->block_width, d_mu);
          else if (sigma)
            kubo_bastin_for_server(&s, H, op, d_st, R, M, job->req.nump, job->req.band_width,
                                   job->req.band_center, job->req.precision, job->block_width, d_mu, d_out);
          else
            moments2d_for_server(&s, H, op, op, d_st, R, M, job->req.precision, job->block_width, d_mu);
          LQ_CUDA(cudaMemcpyAsync(res_host, d_mu, mb, cudaMemcpyDeviceToHost, s.stream));
          if (sigma)
            LQ_CUDA(cudaMemcpyAsync(job->req.sigma_out, d_out, ob, cudaMemcpyDeviceToHost, s.stream));
          LQ_CUDA(cudaStreamSynchronize(s.stream));
          check_device_errors(&s);
          s.trim();  // stream-ordered frees back to the pool for the next request
          std::memcpy(job->req.mu_out, res_host, mb);
        } catch (const Error &e) {
          rc = e.code;
          err = e.what();
          coop_share_return(&sess->s);
          sess->s.trim();
        } catch (const std::exception &e) {
          rc = LINQT_ERR_INTERNAL;
          err = e.what();
          coop_share_return(&sess->s);
        }
        if (rc != LINQT_ERR_TIMEOUT || sess->s.coop_share >= 1.0) break;
        std::lock_guard<std::mutex> g(mu);
        timeouts_retried++;
      }
      if (rc == LINQT_ERR_NOMEM && !job->alone) {
        std::lock_guard<std::mutex> g(mu);
        nomem_retried++;
        in_use -= job->footprint;
        running--;
        pinned_put_locked(res_host, res_cap);
        job->alone = true;
        job->status = 0;
        queue.push_front(job);
        cv.notify_all();
        continue;
      }
      {
        std::lock_guard<std::mutex> g(mu);
        in_use -= job->footprint;
        running--;
        job->status = rc ? rc : 2;
        job->error = err;
        job->latency_ms = std::chrono::duration<double, std::milli>(clk::now() - job->t_submit).count();
        pinned_put_locked(job->states, job->states_cap);
        pinned_put_locked(res_host, res_cap);
        job->states = nullptr;
      }
      cv.notify_all();
      done_cv.notify_all();
    }
  }
};

extern "C" {

int linqt_server_create(int device, size_t hbm_budget_bytes, int max_active, linqt_server **out) {
  try {
    if (!out || max_active <= 0) fail(LINQT_ERR_INVALID, "server: bad argument");
    int n = 0;
    LQ_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) fail(LINQT_ERR_INVALID, "server: no such device");
    LQ_CUDA(cudaSetDevice(device));
    size_t fr = 0, tot = 0;
    LQ_CUDA(cudaMemGetInfo(&fr, &tot));
    std::unique_ptr<linqt_server> s(new linqt_server);
    s->device = device;
    s->budget = hbm_budget_bytes ? hbm_budget_bytes : (size_t)(fr * 0.8);
    s->max_active = max_active;
    s->ledger.free = s->ledger.capacity = kSlotShare;
    s->ledger.min_share = kSlotShare / max_active;
    LQ_CUDA(cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, device));
    // keep up to the budget cached in the device pool between requests (restored at destroy)
    LQ_CUDA(cudaDeviceGetDefaultMemPool(&s->pool, device));
    LQ_CUDA(cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &s->old_threshold));
    uint64_t thr = s->budget;
    LQ_CUDA(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &thr));
    for (int i = 0; i < max_active; ++i) s->workers.emplace_back([p = s.get()] { p->worker(); });
    *out = s.release();
    return LINQT_OK;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  }
}

int linqt_server_submit(linqt_server *srv, const linqt_request *req, long *ticket) {
  try {
    if (!srv || !req || !ticket || !req->H || !req->mu_out) fail(LINQT_ERR_INVALID, "server: NULL");
    if (req->R <= 0 || req->M <= 0) fail(LINQT_ERR_INVALID, "server: R and M must be positive");
    if (req->kind != LINQT_REQ_DOS && req->kind != LINQT_REQ_KUBO_BASTIN) fail(LINQT_ERR_INVALID, "server: kind");
    if (req->kind == LINQT_REQ_KUBO_BASTIN && req->sigma_out &&
        (req->nump < req->M || req->band_width <= 0 || !req->op))
      fail(LINQT_ERR_INVALID, "server: sigma needs nump >= M, band_width > 0 and a velocity operator");
    auto job = std::make_shared<Job>();
    job->req = *req;
    const int n = req->H->op.n;
    job->block_width = pick_width(*req, n, srv->sm_count, srv->budget);
    job->footprint = estimate_footprint(*req, n, srv->sm_count, job->block_width);
    if (job->footprint > srv->budget)
      fail(LINQT_ERR_NOMEM, "server: request footprint " + std::to_string(job->footprint >> 20) +
                                " MiB exceeds the HBM budget");
    if (req->states) {
      const size_t sb = sizeof(double2) * (size_t)req->R * n;
      job->states = srv->pinned_get(sb, &job->states_cap);
      std::memcpy(job->states, req->states, sb);
    }
    job->t_submit = clk::now();
    {
      std::lock_guard<std::mutex> g(srv->mu);
      job->ticket = srv->next_ticket++;
      srv->jobs[job->ticket] = job;
      srv->queue.push_back(job);
    }
    srv->cv.notify_all();
    *ticket = job->ticket;
    return LINQT_OK;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  }
}

int linqt_server_poll(linqt_server *srv, long ticket, int *status, double *latency_ms) {
  if (!srv || !status) {
    set_last_error("server: NULL");
    return LINQT_ERR_INVALID;
  }
  std::lock_guard<std::mutex> g(srv->mu);
  auto it = srv->jobs.find(ticket);
  if (it == srv->jobs.end()) {
    set_last_error("server: unknown ticket");
    return LINQT_ERR_INVALID;
  }
  *status = it->second->status;
  if (latency_ms) *latency_ms = it->second->latency_ms;
  if (it->second->status < 0) set_last_error(it->second->error);
  return LINQT_OK;
}

int linqt_server_wait_all(linqt_server *srv) {
  if (!srv) {
    set_last_error("server: NULL");
    return LINQT_ERR_INVALID;
  }
  std::unique_lock<std::mutex> g(srv->mu);
  srv->done_cv.wait(g, [&] { return srv->queue.empty() && srv->running == 0; });
  return LINQT_OK;
}

int linqt_server_cancel(linqt_server *srv, long ticket) {
  if (!srv) {
    set_last_error("server: NULL");
    return LINQT_ERR_INVALID;
  }
  std::shared_ptr<Job> job;
  {
    std::lock_guard<std::mutex> g(srv->mu);
    auto it = srv->jobs.find(ticket);
    if (it == srv->jobs.end()) {
      set_last_error("server: unknown ticket");
      return LINQT_ERR_INVALID;
    }
    job = it->second;
    if (job->status != 0) {
      set_last_error(job->status == 1 ? "server: the request is running and cannot be cancelled"
                                      : "server: the request has finished");
      return LINQT_ERR_INVALID;
    }
    for (auto q = srv->queue.begin(); q != srv->queue.end(); ++q)
      if (q->get() == job.get()) {
        srv->queue.erase(q);
        break;
      }
    job->status = LINQT_ERR_CANCELLED;
    job->error = "server: request cancelled before it started";
    job->latency_ms = std::chrono::duration<double, std::milli>(clk::now() - job->t_submit).count();
    srv->pinned_put_locked(job->states, job->states_cap);
    job->states = nullptr;
  }
  srv->cv.notify_all();  // the next queued request may fit now
  srv->done_cv.notify_all();
  return LINQT_OK;
}

int linqt_server_release(linqt_server *srv, long ticket) {
  if (!srv) {
    set_last_error("server: NULL");
    return LINQT_ERR_INVALID;
  }
  std::lock_guard<std::mutex> g(srv->mu);
  auto it = srv->jobs.find(ticket);
  if (it == srv->jobs.end() || it->second->status == 0 || it->second->status == 1) {
    set_last_error("server: release of an unknown or unfinished ticket");
    return LINQT_ERR_INVALID;
  }
  srv->jobs.erase(it);
  return LINQT_OK;
}

int linqt_server_stats(linqt_server *srv, long *timeouts_retried, long *nomem_retried) {
  if (!srv || !timeouts_retried) {
    set_last_error("server: NULL");
    return LINQT_ERR_INVALID;
  }
  std::lock_guard<std::mutex> g(srv->mu);
  *timeouts_retried = srv->timeouts_retried;
  if (nomem_retried) *nomem_retried = srv->nomem_retried;
  return LINQT_OK;
}

int linqt_server_destroy(linqt_server *srv) {
  if (!srv) return LINQT_OK;
  {
    std::lock_guard<std::mutex> g(srv->mu);
    srv->stop = true;
  }
  srv->cv.notify_all();
  for (auto &t : srv->workers) t.join();
  for (void *p : srv->pinned_all) cudaFreeHost(p);
  if (srv->pool) {
    cudaMemPoolSetAttribute(srv->pool, cudaMemPoolAttrReleaseThreshold, &srv->old_threshold);
    cudaMemPoolTrimTo(srv->pool, 0);
  }
  delete srv;
  return LINQT_OK;
}

}  // extern "C"
