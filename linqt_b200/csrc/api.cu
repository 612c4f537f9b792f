// C ABI of liblinqt_gpu.so: sessions, operators and the solver orchestration.
//
// Every entry point catches linqt::Error (and std::exception) and turns it into a
// negative status plus a thread-local message; nothing aborts across the ABI.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>

#include "internal.cuh"

namespace linqt {

static thread_local std::string g_last_error;

void set_last_error(const std::string &msg) { g_last_error = msg; }

[[noreturn]] void fail(int code, const std::string &msg) { throw Error(code, msg); }


// ---------------------------------------------------------------------------
// sessions
// ---------------------------------------------------------------------------
struct EventPair {
  cudaEvent_t a, b;
  int phase;
};
static thread_local std::vector<EventPair> *g_pending = nullptr;

static void init_session(Session &s, int device) {
  s.device = device;
  LQ_CUDA(cudaSetDevice(device));
  LQ_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
  s.own_stream = true;
  int sms = 0;
  LQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  s.sm_count = sms;
}

// Workspaces come from the device's stream-ordered memory pool: growing or trimming a
// buffer is a cudaFreeAsync on the session stream, which (unlike cudaFree) does not
// synchronise the device, so sessions on other streams keep running.
void *Session::get(const std::string &name, size_t bytes) {
  if (bytes == 0) bytes = 16;
  auto it = ws.find(name);
  if (it != ws.end() && it->second.second >= bytes) return it->second.first;
  if (capturing) fail(LINQT_ERR_INTERNAL, "workspace '" + name + "' would be allocated inside a graph capture");
  if (it != ws.end()) {
    drop_graphs();  // they hold the old address
    LQ_CUDA(cudaFreeAsync(it->second.first, stream));
    ws.erase(it);
  }
  void *p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, bytes, stream);
  if (e == cudaErrorMemoryAllocation) {
    // Blocks freed earlier stay cached in the pool, each in its own address range, so a
    // larger buffer may not fit although the bytes are there: once this stream has reached
    // its frees, hand the pool's unused memory back and try once more.
    cudaGetLastError();
    cudaMemPool_t pool = nullptr;
    if (cudaStreamSynchronize(stream) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess)
      cudaMemPoolTrimTo(pool, 0);
    e = cudaMallocAsync(&p, bytes, stream);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(LINQT_ERR_NOMEM, "cudaMallocAsync(" + std::to_string(bytes) + ") for '" + name + "' failed: " +
                              cudaGetErrorString(e));
  }
  if ((uintptr_t)p & 255) {  // the TMA descriptors and vector loads rely on this
    cudaFreeAsync(p, stream);
    fail(LINQT_ERR_INTERNAL, "workspace '" + name + "' is not 256-byte aligned");
  }
  // counters used by the last-block reductions must start at zero
  if (name.find("counter") != std::string::npos || name.find("barrier") != std::string::npos)
    LQ_CUDA(cudaMemsetAsync(p, 0, bytes, stream));
  ws[name] = {p, bytes};
  return p;
}

void Session::drop_graphs() {
  for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
  graphs.clear();
  graph_calls.clear();
}

void Session::trim() {
  drop_graphs();
  for (auto &kv : ws) cudaFreeAsync(kv.second.first, stream);
  ws.clear();
  if (stream) cudaStreamSynchronize(stream);
}

Session::~Session() {
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(device);
  trim();
  if (own_stream && stream) cudaStreamDestroy(stream);
  cudaSetDevice(cur);
}

struct SessionPhaseLog {
  std::vector<EventPair> pending;
};
static std::map<Session *, SessionPhaseLog> &phase_logs() {
  static std::map<Session *, SessionPhaseLog> m;
  return m;
}
static std::mutex g_log_mu;

PhaseScope::PhaseScope(Session *s_, Phase p) : s(s_), ph(p) {
  if (!s->timing) return;
  LQ_CUDA(cudaEventCreate(&a));
  LQ_CUDA(cudaEventCreate(&b));
  LQ_CUDA(cudaEventRecord(a, s->stream));
}

PhaseScope::~PhaseScope() {
  if (!a) return;
  cudaEventRecord(b, s->stream);
  std::lock_guard<std::mutex> g(g_log_mu);
  phase_logs()[s].pending.push_back({a, b, (int)ph});
}

static void collect_phases(Session *s) {
  std::vector<EventPair> v;
  {
    std::lock_guard<std::mutex> g(g_log_mu);
    v.swap(phase_logs()[s].pending);
  }
  for (auto &e : v) {
    cudaEventSynchronize(e.b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e.a, e.b);
    s->phase_ms[e.phase] += ms;
    cudaEventDestroy(e.a);
    cudaEventDestroy(e.b);
  }
}

static std::map<int, std::unique_ptr<linqt_session>> &default_sessions() {
  static thread_local std::map<int, std::unique_ptr<linqt_session>> m;
  return m;
}

Session *default_session() {
  int dev = 0;
  LQ_CUDA(cudaGetDevice(&dev));
  auto &m = default_sessions();
  auto it = m.find(dev);
  if (it == m.end()) {
    std::unique_ptr<linqt_session> s(new linqt_session);
    init_session(s->s, dev);
    it = m.emplace(dev, std::move(s)).first;
  }
  return &it->second->s;
}

Session *resolve(linqt_session *s) {
  Session *r = s ? &s->s : default_session();
  LQ_CUDA(cudaSetDevice(r->device));
  return r;
}

// ---------------------------------------------------------------------------
// operators
// ---------------------------------------------------------------------------
// Hermitian expansion of an upper-stored CSR: entries with col >= row are used,
// the lower triangle is conj(upper) (include/sparse_matrix.hpp:52-54).  Rows come out
// sorted by column: the mirrored (lower) entries of row j are appended while
// scanning rows i < j, before row j's own entries.
static void expand_hermitian(int n, const std::vector<int> &urp, const std::vector<int> &ucol,
                             const std::vector<double2> &uval, std::vector<int> &rp, std::vector<int> &col,
                             std::vector<double2> &val) {
  std::vector<long> cnt(n + 1, 0);
  for (int i = 0; i < n; ++i)
    for (int k = urp[i]; k < urp[i + 1]; ++k) {
      const int j = ucol[k];
      cnt[i]++;
      if (j != i) cnt[j]++;
    }
  rp.assign(n + 1, 0);
  long tot = 0;
  for (int i = 0; i < n; ++i) {
    rp[i] = (int)tot;
    tot += cnt[i];
    if (tot > 0x7fffffffL) fail(LINQT_ERR_INVALID, "operator has more than 2^31-1 non-zeros");
  }
  rp[n] = (int)tot;
  col.resize(tot);
  val.resize(tot);
  std::vector<int> fill(rp.begin(), rp.end() - 1);
  for (int i = 0; i < n; ++i)
    for (int k = urp[i]; k < urp[i + 1]; ++k) {
      const int j = ucol[k];
      col[fill[i]] = j;
      val[fill[i]++] = uval[k];
      if (j != i) {
        col[fill[j]] = i;
        val[fill[j]++] = make_double2(uval[k].x, -uval[k].y);
      }
    }
}

void DeviceOp::free_device() {
  cudaFree(d_rowptr);
  cudaFree(d_col);
  cudaFree(d_val64);
  cudaFree(d_val32);
  d_rowptr = d_col = nullptr;
  d_val64 = nullptr;
  d_val32 = nullptr;
  for (auto &kv : sell) {
    cudaFree(kv.second.d_perm);
    cudaFree(kv.second.d_off);
    cudaFree(kv.second.d_col);
    cudaFree(kv.second.d_val64);
    cudaFree(kv.second.d_val32);
  }
  sell.clear();
  tuned.clear();
}

const float2 *DeviceOp::val32() {
  std::lock_guard<std::mutex> g(mu);
  if (!d_val32) {
    std::vector<float2> v32(std::max(1L, nnz));
    for (long k = 0; k < nnz; ++k) v32[k] = make_float2((float)val[k].x, (float)val[k].y);
    LQ_CUDA(cudaSetDevice(device));
    LQ_CUDA(cudaMalloc(&d_val32, sizeof(float2) * v32.size()));
    LQ_CUDA(cudaMemcpy(d_val32, v32.data(), sizeof(float2) * v32.size(), cudaMemcpyHostToDevice));
  }
  return d_val32;
}

void DeviceOp::upload() {
  if (hermitian)
    expand_hermitian(n, up_rowptr, up_col, up_val, rowptr, col, val);
  else {
    rowptr = up_rowptr;
    col = up_col;
    val = up_val;
  }
  nnz = rowptr[n];
  free_device();
  loc_order.clear();  // the pattern may have changed (a rescale can add diagonal entries)
  static std::atomic<unsigned long> next_uid{1};
  uid = next_uid++;
  LQ_CUDA(cudaSetDevice(device));
  LQ_CUDA(cudaMalloc(&d_rowptr, sizeof(int) * (n + 1)));
  LQ_CUDA(cudaMalloc(&d_col, sizeof(int) * std::max(1L, nnz)));
  LQ_CUDA(cudaMalloc(&d_val64, sizeof(double2) * std::max(1L, nnz)));
  LQ_CUDA(cudaMemcpy(d_rowptr, rowptr.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
  if (nnz) {
    LQ_CUDA(cudaMemcpy(d_col, col.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice));
    LQ_CUDA(cudaMemcpy(d_val64, val.data(), sizeof(double2) * nnz, cudaMemcpyHostToDevice));
  }
  version++;
}

// SELL-C-sigma: rows sorted by decreasing length inside windows of sigma = 8C rows
// (stable), slices of C rows, each slice stored column-major with width = its longest
// row; padding entries point at the row itself with value zero.  With kSellLocality in
// the key the windows are cut from the locality order of the rows.
const DeviceOp::Sell &DeviceOp::ensure_sell(int key, bool c64) {
  const int C = sell_height(key);
  LQ_REQUIRE(C > 0 && (key & ~(kSellLocality | (kSellLocality - 1))) == 0, "bad SELL layout key");
  std::lock_guard<std::mutex> g(mu);
  Sell &L = sell[key];
  if (!L.d_perm) {
    const int sigma = 8 * C;
    std::vector<int> order(n);
    if (key & kSellLocality) {
      if ((int)loc_order.size() != n) loc_order = locality_order(n, rowptr.data(), col.data(), kLocalityPart);
      order = loc_order;
    } else {
      for (int i = 0; i < n; ++i) order[i] = i;
    }
    auto len = [&](int r) { return rowptr[r + 1] - rowptr[r]; };
    for (int w0 = 0; w0 < n; w0 += sigma)
      std::stable_sort(order.begin() + w0, order.begin() + std::min(n, w0 + sigma),
                       [&](int a, int b) { return len(a) > len(b); });
    const int ns = (n + C - 1) / C;
    std::vector<int> off(ns + 1, 0);
    for (int sl = 0; sl < ns; ++sl) {
      int w = 0;
      for (int i = 0; i < C && sl * C + i < n; ++i) w = std::max(w, len(order[sl * C + i]));
      LQ_REQUIRE((long)off[sl] + (long)w * C < (1L << 31), "SELL layout exceeds 2^31 entries");
      off[sl + 1] = off[sl] + w * C;
    }
    L.len = std::max(1, off[ns]);
    std::vector<int> sc(L.len, 0);
    std::vector<double2> sv(L.len, make_double2(0, 0));
    for (int sl = 0; sl < ns; ++sl)
      for (int i = 0; i < C && sl * C + i < n; ++i) {
        const int r = order[sl * C + i], w = (off[sl + 1] - off[sl]) / C;
        for (int k = 0; k < w; ++k) {
          const size_t q = (size_t)off[sl] + (size_t)k * C + i;
          if (k < len(r)) {
            sc[q] = col[rowptr[r] + k];
            sv[q] = val[rowptr[r] + k];
          } else {
            sc[q] = r;
          }
        }
      }
    LQ_CUDA(cudaSetDevice(device));
    LQ_CUDA(cudaMalloc(&L.d_perm, sizeof(int) * std::max(1, n)));
    LQ_CUDA(cudaMalloc(&L.d_off, sizeof(int) * (ns + 1)));
    LQ_CUDA(cudaMalloc(&L.d_col, sizeof(int) * L.len));
    LQ_CUDA(cudaMalloc(&L.d_val64, sizeof(double2) * L.len));
    LQ_CUDA(cudaMemcpy(L.d_perm, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    LQ_CUDA(cudaMemcpy(L.d_off, off.data(), sizeof(int) * (ns + 1), cudaMemcpyHostToDevice));
    LQ_CUDA(cudaMemcpy(L.d_col, sc.data(), sizeof(int) * L.len, cudaMemcpyHostToDevice));
    LQ_CUDA(cudaMemcpy(L.d_val64, sv.data(), sizeof(double2) * L.len, cudaMemcpyHostToDevice));
  }
  if (c64 && !L.d_val32) {
    std::vector<double2> sv(L.len);
    LQ_CUDA(cudaSetDevice(device));
    LQ_CUDA(cudaMemcpy(sv.data(), L.d_val64, sizeof(double2) * L.len, cudaMemcpyDeviceToHost));
    std::vector<float2> s32(L.len);
    for (size_t q = 0; q < L.len; ++q) s32[q] = make_float2((float)sv[q].x, (float)sv[q].y);
    LQ_CUDA(cudaMalloc(&L.d_val32, sizeof(float2) * L.len));
    LQ_CUDA(cudaMemcpy(L.d_val32, s32.data(), sizeof(float2) * L.len, cudaMemcpyHostToDevice));
  }
  return L;
}

// ---------------------------------------------------------------------------
// block geometry
// ---------------------------------------------------------------------------
static int pow2_at_least(int r) {
  int p = 1;
  while (p < r) p <<= 1;
  return p;
}

static size_t free_device_bytes() {
  size_t fr = 0, tot = 0;
  LQ_CUDA(cudaMemGetInfo(&fr, &tot));
  return fr;
}

// states (R x N, device) -> chunk c of width Rc (power of two) as an N x Rc block
static void chunk_block(Session *s, const double2 *states, int N, int R, int c0, int Rc, void *blk, bool fp32) {
  const int w = std::min(Rc, R - c0);
  states_to_block(s, states + (size_t)c0 * N, blk, N, w, Rc, fp32);
}

static linqt_opts defaults(const linqt_opts *o) {
  linqt_opts d;
  std::memset(&d, 0, sizeof(d));
  if (o) d = *o;
  LQ_REQUIRE(d.format == LINQT_FORMAT_CSR || d.format == LINQT_FORMAT_SELL || d.format == LINQT_FORMAT_AUTO ||
                 d.format == LINQT_FORMAT_LOCAL,
             "opts.format: unknown sparse format");
  LQ_REQUIRE(d.operator_precision == 0 || d.operator_precision == 1, "opts.operator_precision must be 0 or 1");
  LQ_REQUIRE(d.thread_shape >= 0, "opts.thread_shape must be >= 0");
  return d;
}

// complex64 operator values are a 1D-recursion option (persistent CSR kernels)
static void require_c128_operators(const linqt_opts &o, const char *who) {
  if (o.operator_precision != 0)
    fail(LINQT_ERR_UNSUPPORTED, std::string(who) + ": complex64 operators (opts.operator_precision = 1) are "
                                                   "available for the 1D moments only");
}

// ---------------------------------------------------------------------------
// opts.use_graphs: a *_dev solve is enqueued eagerly on its first call with a given key (so
// that every workspace is allocated and any autotuning is done), captured into a CUDA graph
// on the second and replayed from the instantiated graph afterwards.  The key holds every
// pointer and size of the call and the operators' upload ids and versions; a workspace
// reallocation drops all graphs of the session.  While capturing, cooperative launches go on
// the session stream itself rather than the device lane.  Sessions on the legacy default
// stream, sessions with phase timing on, and keys whose capture failed run eagerly.
// ---------------------------------------------------------------------------
static std::string call_key(const char *name, std::initializer_list<const void *> ptrs,
                            std::initializer_list<const DeviceOp *> ops, std::initializer_list<double> nums,
                            const linqt_opts &o) {
  std::string k(name);
  char buf[64];
  for (const void *p : ptrs) {
    snprintf(buf, sizeof(buf), ":%p", p);
    k += buf;
  }
  for (const DeviceOp *d : ops) {
    snprintf(buf, sizeof(buf), ":%lu.%u", d ? d->uid : 0ul, d ? d->version : 0u);
    k += buf;
  }
  for (double x : nums) {
    snprintf(buf, sizeof(buf), ":%a", x);
    k += buf;
  }
  snprintf(buf, sizeof(buf), ":%d.%d.%d.%d.%d", o.precision, o.format, o.block_width, o.doubling, o.step_launches);
  return k + buf;
}

template <class F>
static void with_graph(Session *s, const linqt_opts &o, const std::string &key, F &&enqueue) {
  if (!o.use_graphs || s->timing || s->stream == nullptr) {
    enqueue();
    return;
  }
  auto g = s->graphs.find(key);
  if (g != s->graphs.end()) {
    LQ_CUDA(cudaGraphLaunch(g->second, s->stream));
    ++s->graph_replays;
    return;
  }
  int &calls = s->graph_calls[key];
  if (calls <= 0) {  // first call, or a capture that failed: eagerly
    if (calls == 0) calls = 1;
    enqueue();
    return;
  }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  LQ_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  s->capturing = true;
  bool ok = true;
  try {
    enqueue();
  } catch (const Error &) {
    ok = false;
  }
  s->capturing = false;
  cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
  if (ok && e == cudaSuccess && graph) e = cudaGraphInstantiate(&exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (!ok || e != cudaSuccess || !exec) {
    cudaGetLastError();
    s->graph_calls[key] = -1;
    enqueue();
    return;
  }
  s->graphs[key] = exec;
  LQ_CUDA(cudaGraphLaunch(exec, s->stream));
  ++s->graph_replays;
}

// ---------------------------------------------------------------------------
// Sparse layout and thread shape of a persistent recursion.  LINQT_FORMAT_CSR: the
// operator's CSR (whose per-CTA row slices the kernels keep in shared memory when they fit),
// thread shape 0; LINQT_FORMAT_SELL: SELL-C-sigma with C = 32, shape 0; LINQT_FORMAT_LOCAL:
// the CSR rows in the locality order (SELL with C = 1 over that order), shape 0;
// LINQT_FORMAT_AUTO: the autotuner times a short run of the same recursion (trial(C, shape))
// for every layout (CSR cached, CSR uncached, SELL with C = 8 and 32, and on large blocks
// the two locality layouts) and thread shape, keeps the fastest per
// operator pair, block width and precision, and returns it.  Each candidate runs once
// untimed (building its layout) and once timed.
// ---------------------------------------------------------------------------
struct RecCfg {
  int sellC = 0, shape = 0;
};

static RecCfg pick_layout(Session *s, const DeviceOp &H, const std::string &key, int format, int Rc,
                          const std::function<void(int, int)> &trial, float *best_ms = nullptr) {
  if (best_ms) *best_ms = -1;
  if (format == LINQT_FORMAT_CSR) return RecCfg{0, 0};
  if (format == LINQT_FORMAT_SELL || format == LINQT_FORMAT_LOCAL) {
    return RecCfg{format == LINQT_FORMAT_SELL ? 32 : 1 | kSellLocality, 0};
  }
  DeviceOp &Hm = const_cast<DeviceOp &>(H);
  {
    std::lock_guard<std::mutex> g(Hm.mu);
    auto it = Hm.tuned.find(key);
    if (it != Hm.tuned.end()) return RecCfg{it->second / 16 - 1, it->second % 16};
  }
  cudaEvent_t a, b;
  LQ_CUDA(cudaEventCreate(&a));
  LQ_CUDA(cudaEventCreate(&b));
  float best = 0;
  RecCfg pick;
  bool first = true;
  // 0: CSR, its row slices cached in shared memory when they fit; -1: CSR without the
  // cache (more resident CTAs per SM); 8, 32: SELL-C-sigma; 1 | kSellLocality (the CSR rows
  // copied in the locality order) and 32 | kSellLocality: tried when one block of the lattice
  // (8 bytes per value at least) exceeds 64 MB, i.e. when its neighbour rows can leave L2
  // between their reads
  const bool big = (double)H.n * Rc * sizeof(float2) > 64e6;
  for (int C : {0, -1, 8, 32, 1 | kSellLocality, 32 | kSellLocality})
    for (int sh = 0; sh < recur_shapes(Rc); ++sh) {
      if ((C & kSellLocality) && !big) continue;
      trial(C, sh);
      LQ_CUDA(cudaEventRecord(a, s->stream));
      trial(C, sh);
      LQ_CUDA(cudaEventRecord(b, s->stream));
      LQ_CUDA(cudaEventSynchronize(b));
      float ms = 0;
      LQ_CUDA(cudaEventElapsedTime(&ms, a, b));
      if (first || ms < best) {
        best = ms;
        pick = RecCfg{C, sh};
        first = false;
      }
    }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (best_ms) *best_ms = best;
  std::lock_guard<std::mutex> g(Hm.mu);
  Hm.tuned[key] = (pick.sellC + 1) * 16 + pick.shape;
  return pick;
}

static std::string layout_key(const char *kind, const DeviceOp *V, int Rc, bool fp32) {
  return std::string(kind) + ":" + std::to_string(Rc) + ":" + (fp32 ? "f32" : "f64") + ":" +
         std::to_string((unsigned long long)(uintptr_t)V) + ":" + std::to_string(V ? V->version : 0);
}

// ---------------------------------------------------------------------------
// 1D moments: chebyshev::SpectralMoments (src/chebyshev_solver.cpp:176-199)
// ---------------------------------------------------------------------------
static void moments1d_dev(Session *s, const DeviceOp &H, const DeviceOp *op, const double2 *states, int R, int M,
                          const linqt_opts &o, double2 *mu) {
  LQ_REQUIRE(R > 0 && M > 0, "moments1d: R and M must be positive");
  LQ_REQUIRE(!op || op->n == H.n, "moments1d: operator dimension mismatch");
  const int N = H.n;
  const bool fp32 = o.precision != LINQT_PREC_FP64;
  const bool c64 = o.operator_precision == 1;
  if (c64 && o.step_launches)
    fail(LINQT_ERR_UNSUPPORTED, "complex64 operators: the persistent recursion only (step_launches = 0)");
  const bool doubling = (o.doubling == 0 && op == nullptr) || o.doubling == 1;
  LQ_REQUIRE(!(doubling && op), "moments1d: the doubling identities need the identity operator");
  int Rc = o.block_width > 0 ? o.block_width : std::min(256, pow2_at_least(R));
  Rc = std::min(256, pow2_at_least(Rc));
  const int steps = doubling ? (M + 1) / 2 : M;
  const size_t esz = fp32 ? sizeof(float2) : sizeof(double2);
  char *T = (char *)s->get("m1_T", 3 * esz * (size_t)N * Rc);
  PhaseScope ph(s, PH_RECURSION);
  long launches = 0;
  // layout and thread shape for block width w, from short trials on the first w vectors
  auto tune = [&](int w, float *best_ms) {
    const size_t bw = esz * (size_t)N * w;
    const int Mt = std::min(M, 32), st = doubling ? (Mt + 1) / 2 : Mt;
    double2 *tdots = (double2 *)s->get("m1_trial_dots", sizeof(double2) * 2 * (size_t)st);
    return pick_layout(
        s, H, layout_key(c64 ? "1d64" : "1d", op, w, fp32), o.format, w,
        [&](int C, int shape) {
          // a short recursion on the first chunk (the real run below starts from scratch)
          void *b0 = T, *b1 = T + bw, *b2 = T + 2 * bw;
          chunk_block(s, states, N, R, 0, w, b2, fp32);
          void *x0 = b2;
          if (!doubling) {
            if (op)
              spmm(s, *op, make_double2(1, 0), b2, make_double2(0, 0), b0, w, fp32);
            else
              LQ_CUDA(cudaMemcpyAsync(b0, b2, bw, cudaMemcpyDeviceToDevice, s->stream));
            x0 = b0;
          }
          recur_1d(s, H, b2, x0, b1, st, Mt, doubling ? 2 : 1, w, fp32, tdots, C, shape, nullptr, 1, c64);
        },
        best_ms);
  };
  // LINQT_FORMAT_AUTO without a fixed block width: also the block width, among Rc, Rc/2, Rc/4
  // and Rc/8, by trial time per vector (a narrower block streams fewer bytes per row, which
  // can keep a large lattice's neighbour rows in L2), cached per operator pair, R and precision
  if (o.format == LINQT_FORMAT_AUTO && o.block_width <= 0 && !o.step_launches && Rc > 1) {
    DeviceOp &Hm = const_cast<DeviceOp &>(H);
    const std::string wkey = "1dw:" + std::to_string(R) + ":" + layout_key(c64 ? "c64" : "", op, Rc, fp32) +
                             (doubling ? ":d" : "");
    int w = 0;
    {
      std::lock_guard<std::mutex> g(Hm.mu);
      auto it = Hm.tuned.find(wkey);
      if (it != Hm.tuned.end()) w = it->second;
    }
    if (!w) {
      float best = 0;
      for (int c = Rc; c >= std::max(1, Rc / 8); c /= 2) {
        float ms = -1;
        tune(c, &ms);
        if (ms < 0) continue;  // tuned before at this width (another R): keep the widest so far
        if (!w || ms / c < 0.97f * best) {
          best = ms / c;
          w = c;
        }
      }
      if (!w) w = Rc;
      std::lock_guard<std::mutex> g(Hm.mu);
      Hm.tuned[wkey] = w;
    }
    Rc = w;
  }
  const int nchunks = (R + Rc - 1) / Rc;
  const size_t blk = esz * (size_t)N * Rc;
  double2 *dots = (double2 *)s->get("m1_dots", sizeof(double2) * 2 * (size_t)steps * nchunks);
  RecCfg cfg;
  if (!o.step_launches) {
    cfg = tune(Rc, nullptr);
    if (o.thread_shape > 0) {
      LQ_REQUIRE(o.thread_shape - 1 < recur_shapes(Rc), "opts.thread_shape: no such shape at this block width");
      cfg.shape = o.thread_shape - 1;
    }
  }
  LQ_CUDA(cudaMemsetAsync(dots, 0, sizeof(double2) * 2 * (size_t)steps * nchunks, s->stream));
  for (int c = 0; c < nchunks; ++c) {
    void *b0 = T, *b1 = T + blk, *b2 = T + 2 * blk;
    double2 *cd = dots + (size_t)2 * steps * c;
    void *phi = b2;
    chunk_block(s, states, N, R, c * Rc, Rc, phi, fp32);
    launches++;
    if (!o.step_launches) {
      void *x0 = phi;
      if (!doubling) {
        if (op) {
          spmm(s, *op, make_double2(1, 0), phi, make_double2(0, 0), b0, Rc, fp32);  // T_0 = OP phi
          launches++;
        } else {
          LQ_CUDA(cudaMemcpyAsync(b0, phi, blk, cudaMemcpyDeviceToDevice, s->stream));
        }
        x0 = b0;
      }
      recur_1d(s, H, phi, x0, b1, steps, M, doubling ? 2 : 1, Rc, fp32, cd, cfg.sellC, cfg.shape, nullptr, 1, c64);
      launches += 2;
      continue;
    }
    void *x;
    if (doubling) {
      x = phi;  // T_0 = phi
    } else if (op) {
      spmm(s, *op, make_double2(1, 0), phi, make_double2(0, 0), b0, Rc, fp32);  // T_0 = OP phi
      launches++;
      x = b0;
    } else {
      LQ_CUDA(cudaMemcpyAsync(b0, phi, blk, cudaMemcpyDeviceToDevice, s->stream));
      x = b0;
    }
    // step 0: T_1 = H T_0
    void *prev = nullptr, *cur = x;
    void *next = doubling ? b1 : (x == b0 ? b1 : b0);
    for (int st = 0; st < steps; ++st) {
      StepArgs a;
      a.x = cur;
      a.yprev = prev;
      const bool need_y = doubling ? (2 * st + 1 < M) : (st + 1 < M);
      a.y = need_y ? (prev ? (void *)prev : next) : nullptr;
      a.phi = phi;
      a.dot_mode = doubling ? 2 : 1;
      a.dots = cd + 2 * st;
      cheb_step(s, H, a, Rc, fp32, o.format);
      launches++;
      if (!need_y) break;
      void *ny = a.y;
      prev = cur;
      cur = ny;
      if (!doubling && st == 0) {
        // free buffer for the rest: the one that is neither prev nor cur nor phi
      }
    }
  }
  ph.launches(launches);
  // assemble (sum chunk dots first)
  if (nchunks > 1) {
    // fold chunk c>0 into chunk 0 (fixed order) with a tiny kernel via the GEMM reducer
    PhaseScope p2(s, PH_OTHER);
    sum_chunks(s, dots, 2 * steps, nchunks);
  }
  PhaseScope p3(s, PH_OTHER);
  moments1d_from_dots(s, dots, steps, M, R, doubling ? 2 : 1, mu);
}

// ---------------------------------------------------------------------------
// Disorder realisations in one block: S Hamiltonians with the same pattern (e.g. Anderson
// disorder seeds), Rs random vectors each, run as one R = S*Rs wide persistent recursion in
// which each realisation has its own group of CTAs, reading its own values (stacked [S][nnz]
// on the device) and its own Rs columns.  Moments per realisation (identity operator,
// doubling identities): mu[S][M].
// ---------------------------------------------------------------------------
// S realisations stacked in one persistent launch (S CTA groups, rows of R = S * Rs columns).
static void realisations_stacked(Session *s, const DeviceOp *const *Hs, int S, const double2 *states, int R, int M,
                                 const linqt_opts &o, double2 *mu) {
  const DeviceOp &H0 = *Hs[0];
  const int Rs = R / S;
  const bool fp32 = o.precision != LINQT_PREC_FP64;
  const int N = H0.n;
  const size_t esz = fp32 ? sizeof(float2) : sizeof(double2);
  // the S value sets side by side: complex128, or the complex64 copies with
  // opts.operator_precision = 1 (for either precision of the vectors)
  const bool c64 = o.operator_precision == 1;
  const size_t vsz = c64 ? sizeof(float2) : sizeof(double2);
  char *vals = (char *)s->get(c64 ? "real_vals32" : "real_vals", vsz * (size_t)S * std::max(1L, H0.nnz));
  for (int r = 0; r < S; ++r)
    LQ_CUDA(cudaMemcpyAsync(vals + vsz * (size_t)r * H0.nnz,
                            c64 ? (const void *)const_cast<DeviceOp *>(Hs[r])->val32() : (const void *)Hs[r]->d_val64,
                            vsz * H0.nnz, cudaMemcpyDeviceToDevice, s->stream));
  const int steps = (M + 1) / 2;  // doubling identities
  const size_t blk = esz * (size_t)N * R;
  char *T = (char *)s->get("m1_T", 3 * blk);
  double2 *dots = (double2 *)s->get("m1_dots", sizeof(double2) * 2 * (size_t)steps * S);
  void *b0 = T, *b1 = T + blk, *phi = T + 2 * blk;
  {
    PhaseScope ph(s, PH_RECURSION);
    chunk_block(s, states, N, R, 0, R, phi, fp32);
    LQ_CUDA(cudaMemcpyAsync(b0, phi, blk, cudaMemcpyDeviceToDevice, s->stream));
    recur_1d(s, H0, phi, b0, b1, steps, M, 2, R, fp32, dots, 0, 0, vals, S, c64);
    ph.launches(3);
  }
  PhaseScope p3(s, PH_OTHER);
  for (int r = 0; r < S; ++r)
    moments1d_from_dots(s, dots + (size_t)2 * steps * r, steps, M, Rs, 2, mu + (size_t)M * r);
}

// One 1D solve per realisation (each with its own autotuned layout).
static void realisations_separate(Session *s, const DeviceOp *const *Hs, int S, const double2 *states, int R, int M,
                                  const linqt_opts &o, double2 *mu) {
  const int Rs = R / S, N = Hs[0]->n;
  for (int r = 0; r < S; ++r)
    moments1d_dev(s, *Hs[r], nullptr, states + (size_t)r * Rs * N, Rs, M, o, mu + (size_t)r * M);
}

// linqt_moments1d_realisations: stacked or separate.  Stacking saves launches and barriers and
// fills the GPU when one realisation's block is narrow; on large lattices with wide blocks each
// separate solve already streams HBM with the whole GPU and the stacked rows (S times wider)
// cost more in the gathers.  opts.realisations = 0 times a 32-moment trial of both (after one
// untimed run each) and caches the faster per pattern owner, S, R/S and precision.
static void moments1d_realisations_dev(Session *s, const DeviceOp *const *Hs, int S, const double2 *states, int R,
                                       int M, const linqt_opts &o, double2 *mu) {
  LQ_REQUIRE(S >= 1 && R > 0 && M > 0 && R % S == 0, "realisations: R must be a positive multiple of S");
  const DeviceOp &H0 = *Hs[0];
  for (int r = 1; r < S; ++r)
    LQ_REQUIRE(Hs[r]->n == H0.n && Hs[r]->rowptr == H0.rowptr && Hs[r]->col == H0.col,
               "realisations: every Hamiltonian must have the sparsity pattern of the first");
  const int Rs = R / S;
  LQ_REQUIRE(Rs <= 256 && (Rs & (Rs - 1)) == 0, "realisations: R/S must be a power of two <= 256");
  LQ_REQUIRE(o.realisations >= 0 && o.realisations <= 2, "opts.realisations must be 0, 1 or 2");
  int mode = S == 1 ? 2 : o.realisations;
  if (mode == 0) {
    DeviceOp &Hm = const_cast<DeviceOp &>(H0);
    const std::string key = "real:" + std::to_string(S) + ":" + std::to_string(Rs) + ":" +
                            (o.precision != LINQT_PREC_FP64 ? "f32" : "f64") + (o.operator_precision ? ":c64" : "");
    {
      std::lock_guard<std::mutex> g(Hm.mu);
      auto it = Hm.tuned.find(key);
      if (it != Hm.tuned.end()) mode = it->second;
    }
    if (mode == 0) {
      const int Mt = std::min(M, 32);
      double2 *tmu = (double2 *)s->get("real_trial_mu", sizeof(double2) * (size_t)S * Mt);
      cudaEvent_t a, b;
      LQ_CUDA(cudaEventCreate(&a));
      LQ_CUDA(cudaEventCreate(&b));
      float best = 0;
      for (int c : {1, 2}) {
        auto run = [&] {
          if (c == 1)
            realisations_stacked(s, Hs, S, states, R, Mt, o, tmu);
          else
            realisations_separate(s, Hs, S, states, R, Mt, o, tmu);
        };
        run();
        LQ_CUDA(cudaEventRecord(a, s->stream));
        run();
        LQ_CUDA(cudaEventRecord(b, s->stream));
        LQ_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        LQ_CUDA(cudaEventElapsedTime(&ms, a, b));
        if (c == 1 || ms < best) {
          best = ms;
          mode = c;
        }
      }
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      std::lock_guard<std::mutex> g(Hm.mu);
      Hm.tuned[key] = mode;
    }
  }
  if (mode == 1)
    realisations_stacked(s, Hs, S, states, R, M, o, mu);
  else
    realisations_separate(s, Hs, S, states, R, M, o, mu);
}

// ---------------------------------------------------------------------------
// L/R Chebyshev vector blocks (shared by the 2D moments and the FFT solver)
//   L_m = T_m(H) OPL phi  (Moments::SetInitVectors(OP, phi) + Vectors::IterateAll,
//                          src/chebyshev_moments.cpp:5-22, src/chebyshev_vectors.cpp:4-21)
//   R_m = OPR T_m(H) phi  (+ Vectors::Multiply, src/chebyshev_vectors.cpp:24-51)
// Lstore/Rstore: M blocks of N x Rc (site-major) each.
// ---------------------------------------------------------------------------
static long lr_vectors(Session *s, const DeviceOp &H, const DeviceOp *opl, const DeviceOp *opr, void *phi, int M,
                       int Rc, bool fp32, char *Lstore, char *Rstore, char *tmp3, int format, bool step_launches) {
  const size_t esz = fp32 ? sizeof(float2) : sizeof(double2);
  const size_t blk = esz * (size_t)H.n * Rc;
  long launches = 0;
  if (!step_launches) {
    // one cooperative launch advances both recursions (recur.cu)
    auto start = [&]() {
      if (opl)
        spmm(s, *opl, make_double2(1, 0), phi, make_double2(0, 0), Lstore, Rc, fp32);
      else
        LQ_CUDA(cudaMemcpyAsync(Lstore, phi, blk, cudaMemcpyDeviceToDevice, s->stream));
      if (!opr) LQ_CUDA(cudaMemcpyAsync(Rstore, phi, blk, cudaMemcpyDeviceToDevice, s->stream));
    };
    const RecCfg cfg = pick_layout(s, H, layout_key("lr", opr, Rc, fp32), format, Rc, [&](int C, int shape) {
      start();
      recur_lr(s, H, opr, Lstore, Rstore, phi, tmp3, std::min(M, 16), Rc, fp32, C, shape);
    });
    start();
    recur_lr(s, H, opr, Lstore, Rstore, phi, tmp3, M, Rc, fp32, cfg.sellC, cfg.shape);
    return opl ? 2 : 1;
  }
  // ---- L side: the recursion runs in place inside the store
  if (opl) {
    spmm(s, *opl, make_double2(1, 0), phi, make_double2(0, 0), Lstore, Rc, fp32);
  } else {
    LQ_CUDA(cudaMemcpyAsync(Lstore, phi, blk, cudaMemcpyDeviceToDevice, s->stream));
  }
  launches++;
  for (int m = 0; m + 1 < M; ++m) {
    StepArgs a;
    a.x = Lstore + blk * m;
    a.yprev = m ? Lstore + blk * (m - 1) : nullptr;
    a.y = Lstore + blk * (m + 1);
    cheb_step(s, H, a, Rc, fp32, format);
    launches++;
  }
  // ---- R side
  if (!opr) {
    LQ_CUDA(cudaMemcpyAsync(Rstore, phi, blk, cudaMemcpyDeviceToDevice, s->stream));
    for (int m = 0; m + 1 < M; ++m) {
      StepArgs a;
      a.x = Rstore + blk * m;
      a.yprev = m ? Rstore + blk * (m - 1) : nullptr;
      a.y = Rstore + blk * (m + 1);
      cheb_step(s, H, a, Rc, fp32, format);
      launches++;
    }
    return launches;
  }
  // T_m live in three rotating buffers; each step also writes OPR T_m into Rstore[m]
  char *buf[3] = {tmp3, tmp3 + blk, tmp3 + 2 * blk};
  void *prev = nullptr, *cur = phi;
  int nb = 0;
  for (int m = 0; m < M; ++m) {
    StepArgs a;
    a.x = cur;
    a.yprev = prev;
    a.V = opr;
    a.vout = Rstore + blk * m;
    if (m + 1 < M) {
      void *dst = buf[nb % 3];
      if (dst == cur || dst == prev) dst = buf[(++nb) % 3];
      if (dst == cur || dst == prev) dst = buf[(++nb) % 3];
      a.y = dst;
      nb++;
    }
    cheb_step(s, H, a, Rc, fp32, format);
    launches++;
    prev = cur;
    cur = a.y;
  }
  return launches;
}

struct Chunking {
  int Rc, nchunks;
};

// pick the vector-chunk width so that 2 stores of M*N*Rc + buffers fit in memory, with the
// digit planes of the INT8 contraction (`digits` per value: 3 digits per float on the L side
// and 6 on the R side per digit, i.e. 3 * digits bytes per complex entry of each store)
static Chunking pick_chunks(Session *s, int N, int R, int M, size_t esz, const linqt_opts &o, size_t extra,
                            int digits = 0) {
  int Rc = o.block_width > 0 ? pow2_at_least(o.block_width) : pow2_at_least(R);
  Rc = std::min(Rc, 256);
  size_t avail;
  if (s->hbm_budget) {
    // a session with a fixed budget (serving) chunks by the budget alone, so the
    // result does not depend on what else occupies the device
    avail = s->hbm_budget;
  } else {
    avail = free_device_bytes();
    // plus what this session already holds in the buffers this solve reallocates (the L/R
    // stores and the digit planes); its other cached workspaces stay allocated
    for (auto &kv : s->ws)
      if (kv.first.rfind("lr_", 0) == 0 || kv.first.rfind("mu_i8_", 0) == 0) avail += kv.second.second;
    avail = (size_t)(avail * 0.90);
  }
  // the Chebyshev blocks (L and R stores, 4 scratch blocks) and, for the INT8 contraction,
  // one K slab of digit planes
  const auto need_at = [&](int rc) {
    return esz * (size_t)N * rc * (2 * (size_t)M + 4) + extra + i8_digit_bytes(digits, M, (long)N * rc);
  };
  while (Rc > 1) {
    if (need_at(Rc) <= avail) break;
    Rc >>= 1;
  }
  const size_t need = need_at(Rc);
  if (need > avail)
    fail(LINQT_ERR_NOMEM, "2D moments: " + std::to_string(need >> 20) + " MiB of Chebyshev blocks exceed the " +
                              std::to_string(avail >> 20) + " MiB available");
  return {Rc, (R + Rc - 1) / Rc};
}

// Whether the vector blocks are FP32 (the operators stay FP64 in every mode).
static bool prepare_precision(const linqt_opts &o, const DeviceOp &, const DeviceOp *, const DeviceOp *) {
  LQ_REQUIRE(o.precision >= LINQT_PREC_FP64 && o.precision <= LINQT_PREC_MIXED_FAST, "unknown precision");
  return o.precision != LINQT_PREC_FP64;
}

// ---------------------------------------------------------------------------
// 2D moments: chebyshev::CorrelationExpansionMoments (src/chebyshev_solver.cpp:86-172)
// ---------------------------------------------------------------------------
static void moments2d_dev(Session *s, const DeviceOp &H, const DeviceOp *opl, const DeviceOp *opr,
                          const double2 *states, int R, int M, const linqt_opts &o, double2 *mu) {
  LQ_REQUIRE(R > 0 && M > 0, "moments2d: R and M must be positive");
  LQ_REQUIRE((!opl || opl->n == H.n) && (!opr || opr->n == H.n), "moments2d: operator dimension mismatch");
  require_c128_operators(o, "moments2d");
  const bool fp32 = prepare_precision(o, H, opl, opr);
  const int N = H.n;
  const size_t esz = fp32 ? sizeof(float2) : sizeof(double2);
  const Chunking ch = pick_chunks(s, N, R, M, esz, o, sizeof(double2) * (size_t)M * M * 66, i8_digits(o.precision));
  const size_t blk = esz * (size_t)N * ch.Rc;
  char *Ls = (char *)s->get("lr_L", blk * M);
  char *Rs = (char *)s->get("lr_R", blk * M);
  char *tmp = (char *)s->get("lr_tmp", blk * 4);
  double2 *raw = (double2 *)s->get("mu_raw", sizeof(double2) * (size_t)M * M);
  LQ_CUDA(cudaMemsetAsync(raw, 0, sizeof(double2) * (size_t)M * M, s->stream));
  for (int c = 0; c < ch.nchunks; ++c) {
    void *phi = tmp + 3 * blk;
    {
      PhaseScope ph(s, PH_RECURSION);
      chunk_block(s, states, N, R, c * ch.Rc, ch.Rc, phi, fp32);
      ph.launches(1 + lr_vectors(s, H, opl, opr, phi, M, ch.Rc, fp32, Ls, Rs, tmp, o.format, o.step_launches != 0));
    }
    {
      PhaseScope ph(s, PH_CONTRACT);
      mu_contract(s, Ls, Rs, M, (long)N * ch.Rc, fp32, o.precision, raw);
      ph.launches(2);
    }
  }
  PhaseScope ph(s, PH_OTHER);
  mu_finalize(s, raw, M, R, mu);
  ph.launches(1);
}

// ---------------------------------------------------------------------------
// Kubo_solver_FFT::compute (src/Kubo_solver_FFT.cpp:12-136)
// ---------------------------------------------------------------------------

void moments1d_for_server(Session *s, const DeviceOp &H, const DeviceOp *op, const double2 *states, int R, int M,
                          int precision, int block_width, double2 *mu) {
  linqt_opts o = defaults(nullptr);
  o.precision = precision;
  o.block_width = block_width;
  moments1d_dev(s, H, op, states, R, M, o, mu);
}

void moments2d_for_server(Session *s, const DeviceOp &H, const DeviceOp *opl, const DeviceOp *opr,
                          const double2 *states, int R, int M, int precision, int block_width, double2 *mu) {
  linqt_opts o = defaults(nullptr);
  o.precision = precision;
  o.block_width = block_width;
  moments2d_dev(s, H, opl, opr, states, R, M, o, mu);
}

// ---------------------------------------------------------------------------
// One Kubo solve: the L/R blocks are computed once per vector chunk and feed the moment
// contraction (CorrelationExpansionMoments) and the per-site transforms of
// Kubo_solver_FFT (formula KUBO_BASTIN or KUBO_GREENWOOD).  mu or out may be NULL.
// ---------------------------------------------------------------------------
static void kubo_solve(Session *s, const DeviceOp &H, const DeviceOp *opl, const DeviceOp *opr,
                       const double2 *states, int R, int M, int nump, int formula, double bw, double bc,
                       const linqt_opts &o, double2 *mu, double *out) {
  LQ_REQUIRE(R > 0 && M > 0, "kubo: R and M must be positive");
  require_c128_operators(o, "kubo");
  LQ_REQUIRE(!out || nump >= M, "kubo: nump must be >= M (pre_factors are indexed m < M, src/Bastin_FFTs.cpp:18-21)");
  LQ_REQUIRE(formula == LINQT_KUBO_BASTIN || formula == LINQT_KUBO_GREENWOOD, "kubo: unknown formula");
  LQ_REQUIRE(bw > 0, "kubo: band_width must be positive");
  const bool fp32 = prepare_precision(o, H, opl, opr);
  const int N = H.n;
  const size_t esz = fp32 ? sizeof(float2) : sizeof(double2);
  size_t extra = 0;
  if (mu) extra += sizeof(double2) * (size_t)M * M * 66;
  if (out) extra += sizeof(double2) * 2 * (size_t)std::max(nump, 1) * 1024;
  const Chunking ch = pick_chunks(s, N, R, M, esz, o, extra, mu ? i8_digits(o.precision) : 0);
  const size_t blk = esz * (size_t)N * ch.Rc;
  char *Ls = (char *)s->get("lr_L", blk * M);
  char *Rs = (char *)s->get("lr_R", blk * M);
  char *tmp = (char *)s->get("lr_tmp", blk * 4);
  double2 *raw = nullptr, *acc = nullptr, *acc_c = nullptr;
  if (mu) {
    raw = (double2 *)s->get("mu_raw", sizeof(double2) * (size_t)M * M);
    LQ_CUDA(cudaMemsetAsync(raw, 0, sizeof(double2) * (size_t)M * M, s->stream));
  }
  if (out) {
    acc = (double2 *)s->get("kubo_acc", sizeof(double2) * 2 * (size_t)nump);
    LQ_CUDA(cudaMemsetAsync(acc, 0, sizeof(double2) * 2 * (size_t)nump, s->stream));
    acc_c = (double2 *)s->get("kubo_acc_c", sizeof(double2) * 2 * (size_t)nump);
  }
  for (int c = 0; c < ch.nchunks; ++c) {
    void *phi = tmp + 3 * blk;
    {
      PhaseScope ph(s, PH_RECURSION);
      chunk_block(s, states, N, R, c * ch.Rc, ch.Rc, phi, fp32);
      ph.launches(1 + lr_vectors(s, H, opl, opr, phi, M, ch.Rc, fp32, Ls, Rs, tmp, o.format, o.step_launches != 0));
    }
    if (mu) {
      PhaseScope ph(s, PH_CONTRACT);
      mu_contract(s, Ls, Rs, M, (long)N * ch.Rc, fp32, o.precision, raw);
      ph.launches(2);
    }
    if (out) {
      PhaseScope ph(s, PH_FFT);
      kubo_fft_sites(s, Ls, Rs, (long)N * ch.Rc, M, nump, formula, fp32, acc_c);
      add_into(s, acc, acc_c, 2 * nump);
      ph.launches(4);
    }
  }
  PhaseScope ph(s, PH_OTHER);
  if (mu) mu_finalize(s, raw, M, R, mu);
  if (out) kubo_postprocess(s, acc, R, nump, formula, N, bw, bc, out);
  ph.launches((mu ? 1 : 0) + (out ? 1 : 0));
}

// ---------------------------------------------------------------------------
// Time-domain correlations: chebyshev::TimeDependentCorrelations
// (src/chebyshev_solver.cpp:231-275) with MomentsTD::Evolve (src/chebyshev_momentsTD.cpp:4-46).
// Per block of states: PhiL = OPL Phi, PhiR = Phi; at time step n the 1D recursion from
// T_0 = OPR PhiR gives mu(m, n) = (2/R)(1/2)^[m=0] sum_r <PhiL|T_m>; both blocks then evolve
// by dt through one Chebyshev-Bessel series launch each.
// ---------------------------------------------------------------------------
// Coefficients of the evolution series: the reference's loop adds the terms n = 0, 1, ...
// and stops before the first n with |J_n(x)| <= 1e-10; c_n = e^{-i w0 dt} (2 - [n=0]) (-i)^n J_n(x).
static std::vector<double2> td_coefficients(double dt, double band_width, double band_center) {
  const double hbar = 0.6582119624;  // eV fs (MomentsTD::HBAR)
  const double x = dt * (0.5 * band_width) / hbar, w0dt = band_center / hbar * dt;
  const double2 e0 = make_double2(std::cos(w0dt), -std::sin(w0dt));
  auto J = [](int n, double z) { return n == 0 ? ::j0(z) : n == 1 ? ::j1(z) : ::jn(n, z); };
  std::vector<double2> c;
  double2 ip = make_double2(1, 0);  // (-i)^n
  double jn = 0.5 * J(0, x);
  for (int n = 0;; ++n) {
    const double a = 2.0 * jn;
    c.push_back(cmul(e0, make_double2(a * ip.x, a * ip.y)));
    ip = make_double2(ip.y, -ip.x);
    jn = J(n + 1, x);
    LQ_REQUIRE(n < 100000, "time correlations: the evolution series does not converge");
    if (!(std::fabs(jn) > 1e-10)) break;
  }
  return c;
}

static void moments_td_dev(Session *s, const DeviceOp &H, const DeviceOp *opl, const DeviceOp *opr,
                           const double2 *states, int R, int M, int NT, double dt, double band_width,
                           double band_center, const linqt_opts &o, double2 *mu) {
  LQ_REQUIRE(R > 0 && M > 0 && NT > 0, "time correlations: R, M and NT must be positive");
  require_c128_operators(o, "time correlations");
  LQ_REQUIRE((!opl || opl->n == H.n) && (!opr || opr->n == H.n), "time correlations: operator dimension mismatch");
  LQ_REQUIRE(band_width > 0 && dt >= 0, "time correlations: band_width > 0 and dt >= 0");
  LQ_REQUIRE(o.precision == LINQT_PREC_FP64, "time correlations: FP64 only");
  const int N = H.n;
  int Rc = o.block_width > 0 ? o.block_width : std::min(256, pow2_at_least(R));
  Rc = std::min(256, pow2_at_least(Rc));
  const int nchunks = (R + Rc - 1) / Rc;
  const size_t blk = sizeof(double2) * (size_t)N * Rc;
  char *W = (char *)s->get("td_blocks", 4 * blk);
  void *PR = W, *PL = W + blk, *X0 = W + 2 * blk, *X1 = W + 3 * blk;
  double2 *dots = (double2 *)s->get("td_dots", sizeof(double2) * 2 * (size_t)M * nchunks * NT);
  const std::vector<double2> c = td_coefficients(dt, band_width, band_center);
  double2 *coef = (double2 *)s->get("td_coef", sizeof(double2) * c.size());
  LQ_CUDA(cudaMemcpyAsync(coef, c.data(), sizeof(double2) * c.size(), cudaMemcpyHostToDevice, s->stream));
  const int sellC = o.format == LINQT_FORMAT_SELL ? 32 : o.format == LINQT_FORMAT_LOCAL ? 1 | kSellLocality : 0;
  {
    PhaseScope ph(s, PH_RECURSION);
    for (int ch = 0; ch < nchunks; ++ch) {
      chunk_block(s, states, N, R, ch * Rc, Rc, PR, false);
      if (opl)
        spmm(s, *opl, make_double2(1, 0), PR, make_double2(0, 0), PL, Rc, false);
      else
        LQ_CUDA(cudaMemcpyAsync(PL, PR, blk, cudaMemcpyDeviceToDevice, s->stream));
      for (int t = 0; t < NT; ++t) {
        if (opr)
          spmm(s, *opr, make_double2(1, 0), PR, make_double2(0, 0), X0, Rc, false);
        else
          LQ_CUDA(cudaMemcpyAsync(X0, PR, blk, cudaMemcpyDeviceToDevice, s->stream));
        recur_1d(s, H, PL, X0, X1, M, M, 1, Rc, false, dots + ((size_t)t * nchunks + ch) * 2 * M, sellC);
        if (t + 1 < NT) {  // the reference also evolves after the last step; nothing reads that
          cheb_series(s, H, PL, X0, X1, coef, (int)c.size(), Rc);
          cheb_series(s, H, PR, X0, X1, coef, (int)c.size(), Rc);
        }
      }
    }
    ph.launches((long)nchunks * (2 + (long)NT * 4));
  }
  PhaseScope p3(s, PH_OTHER);
  for (int t = 0; t < NT; ++t) {
    double2 *dt_dots = dots + (size_t)t * nchunks * 2 * M;
    if (nchunks > 1) sum_chunks(s, dt_dots, 2 * M, nchunks);
    moments1d_from_dots(s, dt_dots, M, M, R, 1, mu + t, NT);
  }
}

static void kubo_fft_dev(Session *s, const DeviceOp &H, const DeviceOp *opl, const DeviceOp *opr,
                         const double2 *states, int R, int M, int nump, int formula, double bw, double bc,
                         const linqt_opts &o, double *out) {
  kubo_solve(s, H, opl, opr, states, R, M, nump, formula, bw, bc, o, nullptr, out);
}

static void kubo_bastin_dev(Session *s, const DeviceOp &H, const DeviceOp *opl, const DeviceOp *opr,
                            const double2 *states, int R, int M, int nump, double bw, double bc,
                            const linqt_opts &o, double2 *mu, double *out) {
  kubo_solve(s, H, opl, opr, states, R, M, nump, LINQT_KUBO_BASTIN, bw, bc, o, mu, out);
}

void kubo_bastin_for_server(Session *s, const DeviceOp &H, const DeviceOp *op, const double2 *states, int R, int M,
                            int nump, double bw, double bc, int precision, int block_width, double2 *mu,
                            double *out) {
  linqt_opts o = defaults(nullptr);
  o.precision = precision;
  o.block_width = block_width;
  kubo_bastin_dev(s, H, op, op, states, R, M, nump, bw, bc, o, mu, out);
}

// ---------------------------------------------------------------------------
// host staging helpers
// ---------------------------------------------------------------------------
struct DevBuf {
  void *p = nullptr;
  explicit DevBuf(size_t bytes) {
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) {
      cudaGetLastError();
      fail(LINQT_ERR_NOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
    }
  }
  ~DevBuf() { cudaFree(p); }
};

static const DeviceOp *dop(const linqt_op *o) { return o ? &o->op : nullptr; }

static void check_op(const linqt_op *o, const char *what) {
  if (!o) fail(LINQT_ERR_INVALID, std::string(what) + " is NULL");
}

}  // namespace linqt

using namespace linqt;

// ===========================================================================
// C entry points
// ===========================================================================
extern "C" {

int linqt_abi_version(void) { return LINQT_ABI_VERSION; }

const char *linqt_last_error(void) { return g_last_error.c_str(); }

int linqt_session_create(int device, linqt_session **out) {
  return guarded([&] {
    LQ_REQUIRE(out, "out is NULL");
    int n = 0;
    LQ_CUDA(cudaGetDeviceCount(&n));
    LQ_REQUIRE(device >= 0 && device < n, "no such device");
    std::unique_ptr<linqt_session> s(new linqt_session);
    init_session(s->s, device);
    *out = s.release();
  });
}

int linqt_session_destroy(linqt_session *s) {
  return guarded([&] {
    if (!s) return;
    {
      std::lock_guard<std::mutex> g(g_log_mu);
      for (auto &e : phase_logs()[&s->s].pending) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
      }
      phase_logs().erase(&s->s);
    }
    delete s;
  });
}

int linqt_session_set_stream(linqt_session *s, void *stream) {
  return guarded([&] {
    Session *r = resolve(s);
    LQ_CUDA(cudaStreamSynchronize(r->stream));
    if (r->own_stream) LQ_CUDA(cudaStreamDestroy(r->stream));
    r->stream = (cudaStream_t)stream;
    r->own_stream = false;
  });
}

int linqt_session_get_stream(linqt_session *s, void **stream) {
  return guarded([&] {
    LQ_REQUIRE(stream, "stream is NULL");
    *stream = (void *)resolve(s)->stream;
  });
}

int linqt_session_synchronize(linqt_session *s) {
  return guarded([&] {
    Session *r = resolve(s);
    LQ_CUDA(cudaStreamSynchronize(r->stream));
    check_device_errors(r);
  });
}

int linqt_session_trim(linqt_session *s) {
  return guarded([&] { resolve(s)->trim(); });
}

int linqt_session_enable_timing(linqt_session *s, int on) {
  return guarded([&] { resolve(s)->timing = on != 0; });
}

int linqt_session_set_sm_share(linqt_session *s, double share) {
  return guarded([&] {
    LQ_REQUIRE(s, "NULL session");
    LQ_REQUIRE(share > 0.0 && share <= 1.0, "SM share must be in (0, 1]");
    Session *r = resolve(s);
    if (r->coop_share != share) r->drop_graphs();  // captured grids have the old size
    r->coop_share = share;
  });
}

int linqt_session_inject_barrier_timeout(linqt_session *s, int extra_arrivals, long long spin_limit) {
  return guarded([&] {
    LQ_REQUIRE(s, "NULL session");
    LQ_REQUIRE(extra_arrivals >= 0 && spin_limit >= 0, "bad argument");
    Session *r = resolve(s);
    r->inject_extra = extra_arrivals;
    r->inject_limit = spin_limit;
    r->barrier_cfg_dirty = true;
  });
}

int linqt_session_graph_stats(linqt_session *s, int *graphs, long *replays) {
  return guarded([&] {
    Session *r = resolve(s);
    if (graphs) *graphs = (int)r->graphs.size();
    if (replays) *replays = r->graph_replays;
  });
}

int linqt_session_phase_times(linqt_session *s, double ms[4], long launches[4], int reset) {
  return guarded([&] {
    Session *r = resolve(s);
    collect_phases(r);
    for (int i = 0; i < 4; ++i) {
      if (ms) ms[i] = r->phase_ms[i];
      if (launches) launches[i] = r->phase_launches[i];
      if (reset) {
        r->phase_ms[i] = 0;
        r->phase_launches[i] = 0;
      }
    }
  });
}

int linqt_csr_create(linqt_session *s, int n, const int *rowptr, const int *col, const double *val, int storage,
                     linqt_op **out) {
  return guarded([&] {
    LQ_REQUIRE(out && rowptr, "NULL argument");
    LQ_REQUIRE(n > 0, "dimension must be positive");
    LQ_REQUIRE(rowptr[n] == 0 || (col && val), "NULL col/val with non-zeros");
    LQ_REQUIRE(storage == LINQT_STORAGE_HERMITIAN_UPPER || storage == LINQT_STORAGE_GENERAL, "unknown storage");
    LQ_REQUIRE(rowptr[0] == 0, "rowptr[0] must be 0");
    for (int i = 0; i < n; ++i) LQ_REQUIRE(rowptr[i + 1] >= rowptr[i], "rowptr must be non-decreasing");
    const long nnz_in = rowptr[n];
    for (long k = 0; k < nnz_in; ++k)  // all host-side checks before the device is touched
      LQ_REQUIRE(col[k] >= 0 && col[k] < n, "column index " + std::to_string(col[k]) + " out of range at entry " +
                                                std::to_string(k));
    Session *r = resolve(s);
    std::unique_ptr<linqt_op> h(new linqt_op);
    DeviceOp &d = h->op;
    d.device = r->device;
    d.n = n;
    d.hermitian = storage == LINQT_STORAGE_HERMITIAN_UPPER;
    // keep the stored part the way the library interprets it, rows sorted by column
    d.up_rowptr.assign(n + 1, 0);
    std::vector<std::pair<int, double2>> row;
    for (int i = 0; i < n; ++i) {
      row.clear();
      for (long k = rowptr[i]; k < rowptr[i + 1]; ++k) {
        const int j = col[k];
        LQ_REQUIRE(j >= 0 && j < n, "column index out of range at row " + std::to_string(i));
        if (d.hermitian && j < i) continue;  // strictly lower entries are ignored
        row.push_back({j, make_double2(val[2 * k], val[2 * k + 1])});
      }
      std::stable_sort(row.begin(), row.end(),
                       [](const std::pair<int, double2> &a, const std::pair<int, double2> &b) { return a.first < b.first; });
      for (auto &e : row) {
        if (!d.up_col.empty() && (long)d.up_col.size() > d.up_rowptr[i] && d.up_col.back() == e.first) {
          d.up_val.back().x += e.second.x;  // duplicate entries are summed
          d.up_val.back().y += e.second.y;
          continue;
        }
        d.up_col.push_back(e.first);
        d.up_val.push_back(e.second);
      }
      d.up_rowptr[i + 1] = (int)d.up_col.size();
    }
    (void)nnz_in;
    d.upload();
    *out = h.release();
  });
}

int linqt_op_destroy(linqt_op *op) {
  return guarded([&] {
    if (!op) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(op->op.device);
    cudaDeviceSynchronize();
    op->op.free_device();
    cudaSetDevice(cur);
    delete op;
  });
}

int linqt_op_info(const linqt_op *op, int *n, long *nnz) {
  return guarded([&] {
    check_op(op, "op");
    if (n) *n = op->op.n;
    if (nnz) *nnz = op->op.nnz;
  });
}

int linqt_op_tuned(const linqt_op *op, char *buf, long cap, long *len) {
  return guarded([&] {
    check_op(op, "op");
    LQ_REQUIRE(cap >= 0 && (buf || cap == 0), "bad buffer");
    std::string out;
    {
      DeviceOp &d = const_cast<DeviceOp &>(op->op);
      std::lock_guard<std::mutex> g(d.mu);
      for (const auto &kv : d.tuned) {
        std::string v;
        if (kv.first.rfind("1dw:", 0) == 0) {
          v = "width " + std::to_string(kv.second);
        } else if (kv.first.rfind("real:", 0) == 0) {
          v = kv.second == 1 ? "stacked" : "separate";
        } else {
          const int key = kv.second / 16 - 1, shape = kv.second % 16;
          if (key == 0)
            v = "csr";
          else if (key < 0)
            v = "csr_nocache";
          else
            v = "sell" + std::to_string(sell_height(key)) + ((key & kSellLocality) ? "_local" : "");
          v += " shape " + std::to_string(shape);
        }
        out += kv.first + " " + v + "\n";
      }
    }
    if (len) *len = (long)out.size();
    if (cap > 0) {
      const size_t n = std::min((size_t)cap - 1, out.size());
      std::memcpy(buf, out.data(), n);
      buf[n] = 0;
    }
  });
}

// SparseMatrixType::Rescale (src/mkl_sparse_matrix.cpp:73-97): C = a*A + b*I on the stored
// entries (mkl_sparse_z_add); a missing diagonal entry is inserted.
int linqt_op_rescale(linqt_op *op, const double a[2], const double b[2]) {
  return guarded([&] {
    check_op(op, "op");
    LQ_REQUIRE(a && b, "NULL scale");
    DeviceOp &d = op->op;
    std::lock_guard<std::mutex> g(d.mu);
    LQ_CUDA(cudaSetDevice(d.device));
    LQ_CUDA(cudaDeviceSynchronize());
    const double2 A = make_double2(a[0], a[1]), B = make_double2(b[0], b[1]);
    std::vector<int> rp(d.n + 1, 0), cl;
    std::vector<double2> vl;
    cl.reserve(d.up_col.size() + d.n);
    vl.reserve(d.up_col.size() + d.n);
    for (int i = 0; i < d.n; ++i) {
      bool placed = false;
      for (int k = d.up_rowptr[i]; k < d.up_rowptr[i + 1]; ++k) {
        const int j = d.up_col[k];
        if (!placed && j > i) {
          cl.push_back(i);
          vl.push_back(B);
          placed = true;
        }
        double2 v = cmul(A, d.up_val[k]);
        if (j == i) {
          v = cadd(v, B);
          placed = true;
        }
        cl.push_back(j);
        vl.push_back(v);
      }
      if (!placed) {
        cl.push_back(i);
        vl.push_back(B);
      }
      rp[i + 1] = (int)cl.size();
    }
    d.up_rowptr.swap(rp);
    d.up_col.swap(cl);
    d.up_val.swap(vl);
    d.upload();
  });
}

int linqt_op_multiply(linqt_session *s, const linqt_op *op, const double a[2], const double *x, const double b[2],
                      double *y, int ncols) {
  return guarded([&] {
    check_op(op, "op");
    LQ_REQUIRE(a && b && x && y && ncols > 0, "bad argument");
    Session *r = resolve(s);
    const DeviceOp &d = op->op;
    const int N = d.n;
    const int Rc = std::min(256, pow2_at_least(ncols));
    DevBuf st(sizeof(double2) * (size_t)N * ncols), yt(sizeof(double2) * (size_t)N * ncols);
    DevBuf bx(sizeof(double2) * (size_t)N * Rc), by(sizeof(double2) * (size_t)N * Rc);
    LQ_CUDA(cudaMemcpyAsync(st.p, x, sizeof(double2) * (size_t)N * ncols, cudaMemcpyHostToDevice, r->stream));
    LQ_CUDA(cudaMemcpyAsync(yt.p, y, sizeof(double2) * (size_t)N * ncols, cudaMemcpyHostToDevice, r->stream));
    for (int c0 = 0; c0 < ncols; c0 += Rc) {
      const int w = std::min(Rc, ncols - c0);
      states_to_block(r, (const double2 *)st.p + (size_t)c0 * N, bx.p, N, w, Rc, false);
      states_to_block(r, (const double2 *)yt.p + (size_t)c0 * N, by.p, N, w, Rc, false);
      spmm(r, d, make_double2(a[0], a[1]), bx.p, make_double2(b[0], b[1]), by.p, Rc, false);
      block_to_states(r, by.p, (double2 *)yt.p + (size_t)c0 * N, N, w, Rc);
    }
    LQ_CUDA(cudaMemcpyAsync(y, yt.p, sizeof(double2) * (size_t)N * ncols, cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaStreamSynchronize(r->stream));
  });
}

int linqt_spectral_bounds(linqt_session *s, const linqt_op *op, double *lo, double *hi) {
  return guarded([&] {
    check_op(op, "op");
    LQ_REQUIRE(lo && hi, "NULL output");
    gershgorin(resolve(s), op->op, lo, hi);
  });
}

int linqt_random_phase_states_dev(linqt_session *s, int N, int R, unsigned long long seed, double *states_dev) {
  return guarded([&] {
    LQ_REQUIRE(states_dev, "NULL pointer");
    random_phase_states(resolve(s), N, R, seed, (double2 *)states_dev);
  });
}

int linqt_moments1d_dev(linqt_session *s, const linqt_op *H, const linqt_op *op, const double *states_dev, int R,
                        int M, const linqt_opts *opts, double *mu_dev) {
  return guarded([&] {
    check_op(H, "H");
    LQ_REQUIRE(states_dev && mu_dev, "NULL pointer");
    Session *ss = resolve(s);
    const linqt_opts o = defaults(opts);
    with_graph(ss, o, call_key("m1", {states_dev, mu_dev}, {&H->op, dop(op)}, {(double)R, (double)M}, o), [&] {
      moments1d_dev(ss, H->op, dop(op), (const double2 *)states_dev, R, M, o, (double2 *)mu_dev);
    });
  });
}

int linqt_moments1d(linqt_session *s, const linqt_op *H, const linqt_op *op, const double *states, int R, int M,
                    const linqt_opts *opts, double *mu) {
  return guarded([&] {
    check_op(H, "H");
    LQ_REQUIRE(states && mu && R > 0 && M > 0, "bad argument");
    Session *r = resolve(s);
    const size_t sb = sizeof(double2) * (size_t)R * H->op.n;
    double2 *d_st = (double2 *)r->get("io_states", sb);
    double2 *d_mu = (double2 *)r->get("io_mu", sizeof(double2) * (size_t)M);
    LQ_CUDA(cudaMemcpyAsync(d_st, states, sb, cudaMemcpyHostToDevice, r->stream));
    moments1d_dev(r, H->op, dop(op), d_st, R, M, defaults(opts), d_mu);
    LQ_CUDA(cudaMemcpyAsync(mu, d_mu, sizeof(double2) * (size_t)M, cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaStreamSynchronize(r->stream));
    check_device_errors(r);
  });
}

static void check_nonorth(const linqt_op *H, const linqt_op *S, const linqt_opts *opts, double tol, int maxit) {
  check_op(H, "H");
  check_op(S, "S");
  LQ_REQUIRE(tol > 0 && maxit > 0, "moments1d_nonorth: tolerance and iteration limit must be positive");
  if (opts && (opts->precision != LINQT_PREC_FP64 || opts->operator_precision != 0))
    fail(LINQT_ERR_UNSUPPORTED, "moments1d_nonorth: FP64 only (the BiCGSTAB solves run in FP64)");
}

int linqt_moments1d_nonorth_dev(linqt_session *s, const linqt_op *H, const linqt_op *op, const linqt_op *S,
                                const double *states_dev, int R, int M, double tol, int maxit,
                                const linqt_opts *opts, double *mu_dev, long *iterations) {
  return guarded([&] {
    check_nonorth(H, S, opts, tol, maxit);
    LQ_REQUIRE(states_dev && mu_dev && R > 0 && M > 0, "bad argument");
    Session *r = resolve(s);
    long long its = 0;
    moments1d_nonorth_dev(r, H->op, dop(op), S->op, (const double2 *)states_dev, R, M, tol, maxit,
                          (double2 *)mu_dev, iterations ? &its : nullptr);
    if (iterations) {
      check_device_errors(r);
      *iterations = (long)its;
    }
  });
}

int linqt_moments1d_nonorth(linqt_session *s, const linqt_op *H, const linqt_op *op, const linqt_op *S,
                            const double *states, int R, int M, double tol, int maxit, const linqt_opts *opts,
                            double *mu, long *iterations) {
  return guarded([&] {
    check_nonorth(H, S, opts, tol, maxit);
    LQ_REQUIRE(states && mu && R > 0 && M > 0, "bad argument");
    Session *r = resolve(s);
    const size_t sb = sizeof(double2) * (size_t)R * H->op.n;
    double2 *d_st = (double2 *)r->get("io_states", sb);
    double2 *d_mu = (double2 *)r->get("io_mu", sizeof(double2) * (size_t)M);
    LQ_CUDA(cudaMemcpyAsync(d_st, states, sb, cudaMemcpyHostToDevice, r->stream));
    long long its = 0;
    moments1d_nonorth_dev(r, H->op, dop(op), S->op, d_st, R, M, tol, maxit, d_mu, &its);
    LQ_CUDA(cudaMemcpyAsync(mu, d_mu, sizeof(double2) * (size_t)M, cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaStreamSynchronize(r->stream));
    check_device_errors(r);
    if (iterations) *iterations = (long)its;
  });
}

int linqt_moments1d_realisations(linqt_session *s, const linqt_op *const *H, int S, const double *states, int R,
                                 int M, const linqt_opts *opts, double *mu) {
  return guarded([&] {
    LQ_REQUIRE(H && states && mu && S >= 1 && R > 0 && M > 0, "bad argument");
    std::vector<const DeviceOp *> ops(S);
    for (int r = 0; r < S; ++r) {
      check_op(H[r], "H[r]");
      ops[r] = &H[r]->op;
    }
    Session *ss = resolve(s);
    const size_t sb = sizeof(double2) * (size_t)R * ops[0]->n;
    double2 *d_st = (double2 *)ss->get("io_states", sb);
    double2 *d_mu = (double2 *)ss->get("io_mu", sizeof(double2) * (size_t)M * S);
    LQ_CUDA(cudaMemcpyAsync(d_st, states, sb, cudaMemcpyHostToDevice, ss->stream));
    moments1d_realisations_dev(ss, ops.data(), S, d_st, R, M, defaults(opts), d_mu);
    LQ_CUDA(cudaMemcpyAsync(mu, d_mu, sizeof(double2) * (size_t)M * S, cudaMemcpyDeviceToHost, ss->stream));
    LQ_CUDA(cudaStreamSynchronize(ss->stream));
    check_device_errors(ss);
  });
}

int linqt_moments1d_realisations_dev(linqt_session *s, const linqt_op *const *H, int S, const double *states_dev,
                                     int R, int M, const linqt_opts *opts, double *mu_dev) {
  return guarded([&] {
    LQ_REQUIRE(H && states_dev && mu_dev && S >= 1, "bad argument");
    std::vector<const DeviceOp *> ops(S);
    for (int r = 0; r < S; ++r) {
      check_op(H[r], "H[r]");
      ops[r] = &H[r]->op;
    }
    moments1d_realisations_dev(resolve(s), ops.data(), S, (const double2 *)states_dev, R, M, defaults(opts),
                               (double2 *)mu_dev);
  });
}

int linqt_moments2d_dev(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                        const double *states_dev, int R, int M, const linqt_opts *opts, double *mu_dev) {
  return guarded([&] {
    check_op(H, "H");
    LQ_REQUIRE(states_dev && mu_dev, "NULL pointer");
    Session *ss = resolve(s);
    const linqt_opts o = defaults(opts);
    with_graph(ss, o, call_key("m2", {states_dev, mu_dev}, {&H->op, dop(opl), dop(opr)}, {(double)R, (double)M}, o),
               [&] { moments2d_dev(ss, H->op, dop(opl), dop(opr), (const double2 *)states_dev, R, M, o, (double2 *)mu_dev); });
  });
}

int linqt_moments2d(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                    const double *states, int R, int M, const linqt_opts *opts, double *mu) {
  return guarded([&] {
    check_op(H, "H");
    LQ_REQUIRE(states && mu && R > 0 && M > 0, "bad argument");
    Session *r = resolve(s);
    const size_t sb = sizeof(double2) * (size_t)R * H->op.n;
    const size_t mb = sizeof(double2) * (size_t)M * M;
    double2 *d_st = (double2 *)r->get("io_states", sb);
    double2 *d_mu = (double2 *)r->get("io_mu", mb);
    LQ_CUDA(cudaMemcpyAsync(d_st, states, sb, cudaMemcpyHostToDevice, r->stream));
    moments2d_dev(r, H->op, dop(opl), dop(opr), d_st, R, M, defaults(opts), d_mu);
    LQ_CUDA(cudaMemcpyAsync(mu, d_mu, mb, cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaStreamSynchronize(r->stream));
    check_device_errors(r);
  });
}

int linqt_moments_td_dev(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                         const double *states_dev, int R, int M, int NT, double dt, double band_width,
                         double band_center, const linqt_opts *opts, double *mu_dev) {
  return guarded([&] {
    check_op(H, "H");
    LQ_REQUIRE(states_dev && mu_dev, "NULL pointer");
    moments_td_dev(resolve(s), H->op, dop(opl), dop(opr), (const double2 *)states_dev, R, M, NT, dt, band_width,
                   band_center, defaults(opts), (double2 *)mu_dev);
  });
}

int linqt_moments_td(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                     const double *states, int R, int M, int NT, double dt, double band_width, double band_center,
                     const linqt_opts *opts, double *mu) {
  return guarded([&] {
    check_op(H, "H");
    LQ_REQUIRE(states && mu, "NULL pointer");
    LQ_REQUIRE(R > 0 && M > 0 && NT > 0, "time correlations: R, M and NT must be positive");
    Session *r = resolve(s);
    const int N = H->op.n;
    const size_t sb = sizeof(double2) * (size_t)R * N, mb = sizeof(double2) * (size_t)M * NT;
    double2 *d_st = (double2 *)r->get("td_io_states", sb);
    double2 *d_mu = (double2 *)r->get("td_io_mu", mb);
    LQ_CUDA(cudaMemcpyAsync(d_st, states, sb, cudaMemcpyHostToDevice, r->stream));
    moments_td_dev(r, H->op, dop(opl), dop(opr), d_st, R, M, NT, dt, band_width, band_center, defaults(opts), d_mu);
    LQ_CUDA(cudaMemcpyAsync(mu, d_mu, mb, cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaStreamSynchronize(r->stream));
    check_device_errors(r);
  });
}

int linqt_time_correlation_from_moments(linqt_session *s, const double *mu, int M, int NT, int N, double band_width,
                                        double band_center, double dt, double broad_meV, double energy, double *t,
                                        double *corr, int *M_used) {
  return guarded([&] {
    LQ_REQUIRE(mu && t && corr && M > 0 && NT > 0 && band_width > 0 && broad_meV > 0, "bad argument");
    Session *r = resolve(s);
    double2 *d_mu = (double2 *)r->get("tc_mu", sizeof(double2) * (size_t)M * NT);
    double *d_out = (double *)r->get("tc_out", sizeof(double) * 2 * (size_t)NT);
    LQ_CUDA(cudaMemcpyAsync(d_mu, mu, sizeof(double2) * (size_t)M * NT, cudaMemcpyHostToDevice, r->stream));
    int T = 0;
    time_correlation(r, d_mu, M, NT, N, band_width, band_center, dt, broad_meV, energy, d_out, d_out + NT, &T);
    LQ_CUDA(cudaMemcpyAsync(t, d_out, sizeof(double) * NT, cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaMemcpyAsync(corr, d_out + NT, sizeof(double) * NT, cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaStreamSynchronize(r->stream));
    if (M_used) *M_used = T;
  });
}

int linqt_kubo_fft_dev(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                       const double *states_dev, int R, int M, int nump, int formula, double band_width,
                       double band_center, const linqt_opts *opts, double *out_dev) {
  return guarded([&] {
    check_op(H, "H");
    LQ_REQUIRE(states_dev && out_dev, "NULL pointer");
    Session *ss = resolve(s);
    const linqt_opts o = defaults(opts);
    with_graph(ss, o,
               call_key("kf", {states_dev, out_dev}, {&H->op, dop(opl), dop(opr)},
                        {(double)R, (double)M, (double)nump, (double)formula, band_width, band_center}, o),
               [&] {
                 kubo_fft_dev(ss, H->op, dop(opl), dop(opr), (const double2 *)states_dev, R, M, nump, formula,
                              band_width, band_center, o, out_dev);
               });
  });
}

int linqt_kubo_fft(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                   const double *states, int R, int M, int nump, int formula, double band_width, double band_center,
                   const linqt_opts *opts, double *E, double *sigma, double *integrand) {
  return guarded([&] {
    check_op(H, "H");
    LQ_REQUIRE(states && E && sigma && R > 0 && M > 0 && nump > 0, "bad argument");
    Session *r = resolve(s);
    const size_t sb = sizeof(double2) * (size_t)R * H->op.n;
    double2 *d_st = (double2 *)r->get("io_states", sb);
    double *d_out = (double *)r->get("io_kubo", sizeof(double) * 3 * (size_t)nump);
    LQ_CUDA(cudaMemcpyAsync(d_st, states, sb, cudaMemcpyHostToDevice, r->stream));
    kubo_fft_dev(r, H->op, dop(opl), dop(opr), d_st, R, M, nump, formula, band_width, band_center, defaults(opts),
                 d_out);
    std::vector<double> h(3 * (size_t)nump);
    LQ_CUDA(cudaMemcpyAsync(h.data(), d_out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaStreamSynchronize(r->stream));
    check_device_errors(r);
    std::memcpy(E, h.data(), sizeof(double) * nump);
    std::memcpy(sigma, h.data() + nump, sizeof(double) * nump);
    if (integrand) std::memcpy(integrand, h.data() + 2 * (size_t)nump, sizeof(double) * nump);
  });
}

int linqt_kubo_bastin_dev(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                          const double *states_dev, int R, int M, int nump, double band_width, double band_center,
                          const linqt_opts *opts, double *mu_dev, double *out_dev) {
  return guarded([&] {
    check_op(H, "H");
    LQ_REQUIRE(states_dev && (mu_dev || out_dev), "NULL pointer");
    Session *ss = resolve(s);
    const linqt_opts o = defaults(opts);
    with_graph(ss, o,
               call_key("kb", {states_dev, mu_dev, out_dev}, {&H->op, dop(opl), dop(opr)},
                        {(double)R, (double)M, (double)nump, band_width, band_center}, o),
               [&] {
                 kubo_bastin_dev(ss, H->op, dop(opl), dop(opr), (const double2 *)states_dev, R, M, nump, band_width,
                                 band_center, o, (double2 *)mu_dev, out_dev);
               });
  });
}

int linqt_kubo_bastin(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                      const double *states, int R, int M, int nump, double band_width, double band_center,
                      const linqt_opts *opts, double *mu, double *E, double *sigma, double *integrand) {
  return guarded([&] {
    check_op(H, "H");
    LQ_REQUIRE(states && R > 0 && M > 0, "bad argument");
    LQ_REQUIRE(mu || (E && sigma), "nothing to compute");
    Session *r = resolve(s);
    const size_t sb = sizeof(double2) * (size_t)R * H->op.n;
    const size_t mb = sizeof(double2) * (size_t)M * M;
    const bool want_fft = E && sigma;
    double2 *d_st = (double2 *)r->get("io_states", sb);
    double2 *d_mu = mu ? (double2 *)r->get("io_mu", mb) : nullptr;
    double *d_out = want_fft ? (double *)r->get("io_kubo", sizeof(double) * 3 * (size_t)nump) : nullptr;
    LQ_CUDA(cudaMemcpyAsync(d_st, states, sb, cudaMemcpyHostToDevice, r->stream));
    kubo_bastin_dev(r, H->op, dop(opl), dop(opr), d_st, R, M, nump, band_width, band_center, defaults(opts), d_mu,
                    d_out);
    if (mu) LQ_CUDA(cudaMemcpyAsync(mu, d_mu, mb, cudaMemcpyDeviceToHost, r->stream));
    std::vector<double> h(want_fft ? 3 * (size_t)nump : 0);
    if (want_fft)
      LQ_CUDA(cudaMemcpyAsync(h.data(), d_out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaStreamSynchronize(r->stream));
    check_device_errors(r);
    if (want_fft) {
      std::memcpy(E, h.data(), sizeof(double) * nump);
      std::memcpy(sigma, h.data() + nump, sizeof(double) * nump);
      if (integrand) std::memcpy(integrand, h.data() + 2 * (size_t)nump, sizeof(double) * nump);
    }
  });
}

int linqt_jackson1d(double *mu, int M, double band_width, double broad_meV, int *M_out) {
  return guarded([&] {
    LQ_REQUIRE(mu && M > 0 && band_width > 0 && broad_meV > 0, "bad argument");
    const int Mt = jackson_cut(M, band_width, broad_meV);
    for (int m = 0; m < Mt; ++m) {
      const double g = jackson_factor(m, Mt);
      mu[2 * m] *= g;
      mu[2 * m + 1] *= g;
    }
    if (M_out) *M_out = Mt;
  });
}

int linqt_locality_order(int n, const int *rowptr, const int *col, int part_rows, int *order) {
  return guarded([&] {
    LQ_REQUIRE(n >= 0 && rowptr && order && part_rows >= 1 && (col || n == 0), "bad argument");
    LQ_REQUIRE(rowptr[0] == 0, "rowptr[0] must be 0");
    for (int i = 0; i < n; ++i) LQ_REQUIRE(rowptr[i + 1] >= rowptr[i], "rowptr must be non-decreasing");
    for (long k = 0; k < (long)rowptr[n]; ++k) LQ_REQUIRE(col[k] >= 0 && col[k] < n, "column index out of range");
    const std::vector<int> o = locality_order(n, rowptr, col, part_rows);
    std::copy(o.begin(), o.end(), order);
  });
}

int linqt_jackson2d(double *mu, int M0, int M1, double band_width, double b0, double b1, int *M0_out, int *M1_out) {
  return guarded([&] {
    LQ_REQUIRE(mu && M0 > 0 && M1 > 0 && band_width > 0 && b0 > 0 && b1 > 0, "bad argument");
    const int T0 = jackson_cut(M0, band_width, b0), T1 = jackson_cut(M1, band_width, b1);
    for (int i = 0; i < T0; ++i)
      for (int j = 0; j < T1; ++j) {
        const double g = jackson_factor(i, T0) * jackson_factor(j, T1);
        mu[2 * ((size_t)i * T1 + j)] = mu[2 * ((size_t)i * M1 + j)] * g;
        mu[2 * ((size_t)i * T1 + j) + 1] = mu[2 * ((size_t)i * M1 + j) + 1] * g;
      }
    if (M0_out) *M0_out = T0;
    if (M1_out) *M1_out = T1;
  });
}

int linqt_dos_from_moments(linqt_session *s, const double *mu, int M, int N, double band_width, double band_center,
                           double broad_meV, double *E, double *dos, int *num_out) {
  return guarded([&] {
    LQ_REQUIRE(mu && E && dos && M > 0 && band_width > 0 && broad_meV > 0, "bad argument");
    Session *r = resolve(s);
    const int Mt = jackson_cut(M, band_width, broad_meV);
    double2 *d_mu = (double2 *)r->get("dos_mu", sizeof(double2) * M);
    double2 *d_muj = (double2 *)r->get("dos_muj", sizeof(double2) * M);
    double *d_out = (double *)r->get("dos_out", sizeof(double) * 2 * M);
    LQ_CUDA(cudaMemcpyAsync(d_mu, mu, sizeof(double2) * M, cudaMemcpyHostToDevice, r->stream));
    jackson2d_dev(r, d_mu, 1, M, 1, Mt, d_muj);  // a 1 x M table: g(0, 1) = 1 on the first axis
    dos_grid(r, d_muj, Mt, N, band_width, band_center, d_out, d_out + Mt);
    LQ_CUDA(cudaMemcpyAsync(E, d_out, sizeof(double) * Mt, cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaMemcpyAsync(dos, d_out + Mt, sizeof(double) * Mt, cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaStreamSynchronize(r->stream));
    if (num_out) *num_out = Mt;
  });
}

int linqt_spectral_function_from_moments(linqt_session *s, const double *mu, int M, int N, double band_width,
                                         double band_center, double broad_meV, int grid, int num_div, double *E,
                                         double *out, int *num_out) {
  return guarded([&] {
    LQ_REQUIRE(mu && E && out && M > 0 && band_width > 0 && broad_meV > 0, "bad argument");
    LQ_REQUIRE(grid == LINQT_GRID_UNIFORM || grid == LINQT_GRID_CHEBYSHEV,
               "spectral function: grid must be LINQT_GRID_UNIFORM or LINQT_GRID_CHEBYSHEV");
    Session *r = resolve(s);
    const int Mt = jackson_cut(M, band_width, broad_meV);
    const int nd = num_div > 0 ? num_div : (grid == LINQT_GRID_UNIFORM ? 30 * Mt : Mt);
    LQ_REQUIRE(nd >= 2, "spectral function: at least two energies");
    double2 *d_mu = (double2 *)r->get("dos_mu", sizeof(double2) * M);
    double2 *d_muj = (double2 *)r->get("dos_muj", sizeof(double2) * M);
    double *d_out = (double *)r->get("spec_out", sizeof(double) * 2 * (size_t)nd);
    LQ_CUDA(cudaMemcpyAsync(d_mu, mu, sizeof(double2) * M, cudaMemcpyHostToDevice, r->stream));
    jackson2d_dev(r, d_mu, 1, M, 1, Mt, d_muj);  // a 1 x M table: g(0, 1) = 1 on the first axis
    spectral_grid(r, d_muj, Mt, N, band_width, band_center, grid, nd, d_out, d_out + nd);
    LQ_CUDA(cudaMemcpyAsync(E, d_out, sizeof(double) * nd, cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaMemcpyAsync(out, d_out + nd, sizeof(double) * nd, cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaStreamSynchronize(r->stream));
    if (num_out) *num_out = nd;
  });
}

int linqt_bastin_from_moments(linqt_session *s, const double *mu, int M0, int M1, int N, double band_width,
                              double band_center, double broad_meV, double xbound, int num_div, double *E,
                              double *sigma, int *num_out) {
  return guarded([&] {
    LQ_REQUIRE(mu && E && sigma && M0 > 0 && M1 > 0 && band_width > 0 && broad_meV > 0, "bad argument");
    LQ_REQUIRE(xbound > 0 && xbound < 1, "xbound must lie in (0, 1)");
    Session *r = resolve(s);
    const int T0 = jackson_cut(M0, band_width, broad_meV), T1 = jackson_cut(M1, band_width, broad_meV);
    const int nd = num_div > 0 ? num_div : 30 * std::max(T0, T1);
    LQ_REQUIRE(nd >= 2, "num_div must be >= 2");
    double2 *d_mu = (double2 *)r->get("bas_mu", sizeof(double2) * (size_t)M0 * M1);
    double2 *d_muj = (double2 *)r->get("bas_muj", sizeof(double2) * (size_t)T0 * T1);
    double *d_out = (double *)r->get("bas_out", sizeof(double) * 2 * (size_t)nd);
    LQ_CUDA(cudaMemcpyAsync(d_mu, mu, sizeof(double2) * (size_t)M0 * M1, cudaMemcpyHostToDevice, r->stream));
    jackson2d_dev(r, d_mu, M0, M1, T0, T1, d_muj);
    bastin_grid(r, d_muj, T0, T1, N, band_width, band_center, xbound, nd, d_out, d_out + nd);
    LQ_CUDA(cudaMemcpyAsync(E, d_out, sizeof(double) * (nd - 1), cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaMemcpyAsync(sigma, d_out + nd, sizeof(double) * (nd - 1), cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaStreamSynchronize(r->stream));
    if (num_out) *num_out = nd - 1;
  });
}

int linqt_kubo_from_moments(linqt_session *s, const double *mu, int M0, int M1, int N, double band_width,
                            double band_center, double broad_meV, int variant, int grid, double xbound, int num_div,
                            double *E, double *out, int *num_out) {
  return guarded([&] {
    LQ_REQUIRE(mu && E && out && M0 > 0 && M1 > 0 && band_width > 0 && broad_meV > 0, "bad argument");
    LQ_REQUIRE(variant >= LINQT_SUM_BASTIN && variant <= LINQT_SUM_BASTIN_SURF, "unknown variant");
    LQ_REQUIRE(grid >= LINQT_GRID_UNIFORM && grid <= LINQT_GRID_CHEBYSHEV_ASCENDING, "unknown grid");
    LQ_REQUIRE(grid != LINQT_GRID_UNIFORM || (xbound > 0 && xbound <= 1), "xbound must lie in (0, 1]");
    Session *r = resolve(s);
    const int T0 = jackson_cut(M0, band_width, broad_meV), T1 = jackson_cut(M1, band_width, broad_meV);
    const int Mt = std::max(T0, T1);
    const int nd = num_div > 0 ? num_div : (grid == LINQT_GRID_UNIFORM ? 30 * Mt : Mt);
    LQ_REQUIRE(nd >= 2, "num_div must be >= 2");
    double2 *d_mu = (double2 *)r->get("bas_mu", sizeof(double2) * (size_t)M0 * M1);
    double2 *d_muj = (double2 *)r->get("bas_muj", sizeof(double2) * (size_t)T0 * T1);
    double *d_out = (double *)r->get("bas_out", sizeof(double) * 2 * (size_t)nd);
    LQ_CUDA(cudaMemcpyAsync(d_mu, mu, sizeof(double2) * (size_t)M0 * M1, cudaMemcpyHostToDevice, r->stream));
    jackson2d_dev(r, d_mu, M0, M1, T0, T1, d_muj);
    energy_sums(r, d_muj, T0, T1, N, band_width, band_center, variant, grid, xbound, nd, d_out, d_out + nd);
    LQ_CUDA(cudaMemcpyAsync(E, d_out, sizeof(double) * (nd - 1), cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaMemcpyAsync(out, d_out + nd, sizeof(double) * (nd - 1), cudaMemcpyDeviceToHost, r->stream));
    LQ_CUDA(cudaStreamSynchronize(r->stream));
    if (num_out) *num_out = nd - 1;
  });
}

}  // extern "C"
