// Serving: continuous batching of DOS and Kubo-Bastin solves on one GPU.
//
// LinQT has no server (its drivers run one solve per process); this is the request
// loop of the B200 build.  Requests are queued at submit (states copied to host
// memory the server owns), admitted in arrival order when an execution slot is free and their
// estimated device footprint fits in the HBM budget, and run on the slot's own CUDA
// stream, so solves admitted at different times overlap on the device.  Each slot
// owns a session whose workspace budget is fixed, which makes the chunking -- and
// with the fixed-order reductions the result -- independent of what else runs.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

#include "internal.cuh"

namespace linqt {
// solver entry points of api.cu
void moments1d_for_server(Session *s, const DeviceOp &H, const DeviceOp *op, const double2 *states, int R, int M,
                          int precision, double2 *mu);
void moments2d_for_server(Session *s, const DeviceOp &H, const DeviceOp *opl, const DeviceOp *opr,
                          const double2 *states, int R, int M, int precision, double2 *mu);
}  // namespace linqt

using namespace linqt;

namespace {

typedef std::chrono::steady_clock clk;

struct Job {
  long ticket = 0;
  linqt_request req{};
  std::vector<double2> states;  // host copy
  size_t footprint = 0;
  int status = 0;  // 0 pending, 1 running, 2 done, <0 error
  double latency_ms = 0;
  std::string error;
  clk::time_point t_submit;
};

// Device bytes a request may hold: every workspace of the solver it runs (state copy,
// Chebyshev blocks, per-step partials, contraction partials), with the same block width
// the solver picks when the budget allows it.
size_t estimate_footprint(const linqt_request &r, int n, int sm_count) {
  int Rc = 1;
  while (Rc < r.R && Rc < 256) Rc <<= 1;
  const size_t esz = r.precision == LINQT_PREC_FP64 ? sizeof(double2) : sizeof(float2);
  const size_t io = sizeof(double2) * ((size_t)r.R * n + (size_t)r.M * (r.kind == LINQT_REQ_DOS ? 1 : r.M));
  if (r.kind == LINQT_REQ_DOS) {
    const size_t steps = (size_t)r.M / 2 + 1;
    return io + esz * (size_t)n * Rc * 3 + sizeof(double2) * (2 * steps * ((size_t)sm_count * 32 + 1) + 2 * steps) +
           (1 << 20);
  }
  return io + esz * (size_t)n * Rc * (2 * (size_t)r.M + 4) + sizeof(double2) * (size_t)r.M * r.M * 66 + (1 << 20);
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
  bool stop = false;
  std::vector<std::thread> workers;

  void worker() {
    std::unique_ptr<linqt_session> sess(new linqt_session);
    {
      Session &s = sess->s;
      s.device = device;
      cudaSetDevice(device);
      cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
      s.own_stream = true;
      cudaDeviceGetAttribute(&s.sm_count, cudaDevAttrMultiProcessorCount, device);
    }
    for (;;) {
      std::shared_ptr<Job> job;
      {
        std::unique_lock<std::mutex> g(mu);
        // admission: the oldest queued job, once its footprint fits next to the running ones
        cv.wait(g, [&] { return stop || (!queue.empty() && in_use + queue.front()->footprint <= budget); });
        if (stop && queue.empty()) return;
        if (queue.empty()) continue;
        job = queue.front();
        queue.pop_front();
        in_use += job->footprint;
        job->status = 1;
        running++;
      }
      int rc = 0;
      std::string err;
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
        LQ_CUDA(cudaMemcpyAsync(d_st, job->states.data(), sb, cudaMemcpyHostToDevice, s.stream));
        if (job->req.kind == LINQT_REQ_DOS)
          moments1d_for_server(&s, H, op, d_st, R, M, job->req.precision, d_mu);
        else
          moments2d_for_server(&s, H, op, op, d_st, R, M, job->req.precision, d_mu);
        LQ_CUDA(cudaMemcpyAsync(job->req.mu_out, d_mu, mb, cudaMemcpyDeviceToHost, s.stream));
        LQ_CUDA(cudaStreamSynchronize(s.stream));
        check_device_errors(&s);
        s.trim();
      } catch (const Error &e) {
        rc = e.code;
        err = e.what();
        sess->s.trim();
      } catch (const std::exception &e) {
        rc = LINQT_ERR_INTERNAL;
        err = e.what();
      }
      {
        std::lock_guard<std::mutex> g(mu);
        in_use -= job->footprint;
        running--;
        job->status = rc ? rc : 2;
        job->error = err;
        job->latency_ms = std::chrono::duration<double, std::milli>(clk::now() - job->t_submit).count();
        job->states.clear();
        job->states.shrink_to_fit();
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
    LQ_CUDA(cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, device));
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
    if (!srv || !req || !ticket || !req->H || !req->states || !req->mu_out) fail(LINQT_ERR_INVALID, "server: NULL");
    if (req->R <= 0 || req->M <= 0) fail(LINQT_ERR_INVALID, "server: R and M must be positive");
    if (req->kind != LINQT_REQ_DOS && req->kind != LINQT_REQ_KUBO_BASTIN) fail(LINQT_ERR_INVALID, "server: kind");
    auto job = std::make_shared<Job>();
    job->req = *req;
    const int n = req->H->op.n;
    job->states.assign((const double2 *)req->states, (const double2 *)req->states + (size_t)req->R * n);
    job->footprint = estimate_footprint(*req, n, srv->sm_count);
    if (job->footprint > srv->budget)
      fail(LINQT_ERR_NOMEM, "server: request footprint " + std::to_string(job->footprint >> 20) +
                                " MiB exceeds the HBM budget");
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

int linqt_server_destroy(linqt_server *srv) {
  if (!srv) return LINQT_OK;
  {
    std::lock_guard<std::mutex> g(srv->mu);
    srv->stop = true;
  }
  srv->cv.notify_all();
  for (auto &t : srv->workers) t.join();
  delete srv;
  return LINQT_OK;
}

}  // extern "C"
