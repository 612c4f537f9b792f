// Internal declarations shared by the translation units of liblinqt_gpu.so.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/linqt_gpu.h"

namespace linqt {

// ---------------------------------------------------------------------------
// errors: internal code throws linqt::Error; every C entry point catches it
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const std::string &msg);
void set_last_error(const std::string &msg);

// body of a C entry point: runs f, turns an exception into a status and a message
template <class F>
inline int guarded(F &&f) {
  try {
    f();
    return LINQT_OK;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc &) {
    set_last_error("host allocation failed");
    return LINQT_ERR_NOMEM;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return LINQT_ERR_INTERNAL;
  }
}

#define LQ_CUDA(x)                                                                                    \
  do {                                                                                                \
    cudaError_t e_ = (x);                                                                             \
    if (e_ != cudaSuccess)                                                                            \
      ::linqt::fail(e_ == cudaErrorMemoryAllocation ? LINQT_ERR_NOMEM : LINQT_ERR_CUDA,               \
                    std::string(#x) + " failed: " + cudaGetErrorString(e_) + " (" + __FILE__ + ":" + \
                        std::to_string(__LINE__) + ")");                                              \
  } while (0)

#define LQ_REQUIRE(cond, msg)                                       \
  do {                                                              \
    if (!(cond)) ::linqt::fail(LINQT_ERR_INVALID, std::string(msg)); \
  } while (0)

// after a launch: surface configuration errors immediately
#define LQ_LAUNCHED() LQ_CUDA(cudaGetLastError())

// ---------------------------------------------------------------------------
// complex helpers on CUDA vector types
// ---------------------------------------------------------------------------
template <class T>
struct cplx_t;
template <>
struct cplx_t<double> {
  using type = double2;
};
template <>
struct cplx_t<float> {
  using type = float2;
};

__host__ __device__ inline double2 mk2(double x, double y) { return make_double2(x, y); }
__host__ __device__ inline float2 mk2(float x, float y) { return make_float2(x, y); }

// c + a*b
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
  c.x = fma(a.x, b.x, c.x);
  c.x = fma(-a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y);
  c.y = fma(a.y, b.x, c.y);
  return c;
}
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {
  c.x = fmaf(a.x, b.x, c.x);
  c.x = fmaf(-a.y, b.y, c.x);
  c.y = fmaf(a.x, b.y, c.y);
  c.y = fmaf(a.y, b.x, c.y);
  return c;
}
// c + conj(a)*b
__device__ __forceinline__ double2 cfma_conj(double2 a, double2 b, double2 c) {
  c.x = fma(a.x, b.x, c.x);
  c.x = fma(a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y);
  c.y = fma(-a.y, b.x, c.y);
  return c;
}
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

__device__ __forceinline__ double2 to_d2(double2 a) { return a; }
__device__ __forceinline__ double2 to_d2(float2 a) { return make_double2(a.x, a.y); }

// FP64 operator entry times a vector entry of either precision, accumulated in FP64: the
// recursions keep H and V in FP64 whatever the precision of their vector blocks (an FP32
// copy of H perturbs its spectrum coherently, and that error grows with the moment index).
__device__ __forceinline__ double2 cfma(double2 a, float2 b, double2 c) { return cfma(a, to_d2(b), c); }
template <class C>
__device__ __forceinline__ C from_d2(double2 v);
template <>
__device__ __forceinline__ double2 from_d2<double2>(double2 v) {
  return v;
}
template <>
__device__ __forceinline__ float2 from_d2<float2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}

// ---------------------------------------------------------------------------
// device operator: Hermitian-expanded CSR (plus optional FP32 copy and SELL-C)
// ---------------------------------------------------------------------------
// SELL layout keys: slice height C in the low bits, kSellLocality when the slices are cut
// from the locality order of the rows instead of their natural order
constexpr int kSellLocality = 1 << 12;
inline int sell_height(int key) { return key & (kSellLocality - 1); }
// rows of the leaves of the recursive bisection behind the locality order
constexpr int kLocalityPart = 8192;
// Locality order of the rows of a CSR pattern (recursive graph bisection into parts of at
// most `part` rows); order[pos] = row.
std::vector<int> locality_order(int n, const int *rp, const int *ci, int part);

struct SellView {
  int nslices = 0, C = 0;
  const long *slice_off = nullptr;  // [nslices+1], in entries
  const int *slice_w = nullptr;     // [nslices]
  const int *col = nullptr;         // padded, column-major per slice
  const void *val = nullptr;        // double2 or float2
};

struct CsrView {
  int n = 0;
  long nnz = 0;
  const int *rowptr = nullptr;
  const int *col = nullptr;
  const void *val = nullptr;  // double2 or float2
};

struct DeviceOp {
  int device = 0;
  int n = 0;
  // host copy of the operator as LinQT stores it (upper triangle incl. diagonal, sorted
  // by column); rescale acts here and the expansion is re-uploaded
  std::vector<int> up_rowptr, up_col;
  std::vector<double2> up_val;
  bool hermitian = true;
  // expanded CSR (host mirror + device)
  std::vector<int> rowptr, col;
  std::vector<double2> val;
  long nnz = 0;
  int *d_rowptr = nullptr, *d_col = nullptr;
  double2 *d_val64 = nullptr;
  unsigned version = 0;  // bumped by rescale
  unsigned long uid = 0;  // distinct for every upload (keys the replayable graphs)
  // SELL-C-sigma copies of the expanded operator, by layout key: the slice height C, plus
  // kSellLocality when the slices follow the locality order of the rows (built on first use)
  struct Sell {
    int *d_perm = nullptr, *d_off = nullptr, *d_col = nullptr;
    double2 *d_val64 = nullptr;
    float2 *d_val32 = nullptr;  // complex64 values (each rounded once), made on first use
    size_t len = 0;
  };
  std::map<int, Sell> sell;
  const Sell &ensure_sell(int key, bool c64 = false);
  std::vector<int> loc_order;  // locality order of the rows (made on first use)
  // format chosen by the autotuner, per (recursion kind, block width, precision, second operator)
  std::map<std::string, int> tuned;
  std::mutex mu;

  // complex64 copy of the expanded values (each FP64 value rounded once), made on first use
  float2 *d_val32 = nullptr;
  const float2 *val32();
  CsrView csr64() const { return CsrView{n, nnz, d_rowptr, d_col, d_val64}; }
  void free_device();
  void upload();
};

// ---------------------------------------------------------------------------
// sessions: stream + workspace cache + phase timing
// ---------------------------------------------------------------------------
// Index map of rearrange_crescent_order (src/Kubo_solver_FFT_postProcess.cpp:98-116): the
// reference interleaves x[k] and x[n-k-1] (k < n/2) and then reverses the array, so output j
// holds y[n-1-j] with y[2k] = x[k], y[2k+1] = x[n-k-1] and, for odd n, y[n-1] = x[n-1].
__host__ __device__ inline int rearranged_source(int j, int n) {
  const int i = n - 1 - j;
  const int h = n / 2;
  if ((i & 1) == 0 && i / 2 < h) return i / 2;
  if ((i & 1) == 1 && (i - 1) / 2 < h) return n - (i - 1) / 2 - 1;
  return i;
}

enum Phase { PH_RECURSION = 0, PH_CONTRACT = 1, PH_FFT = 2, PH_OTHER = 3 };

// Shares of a device's co-resident CTAs held by the persistent cooperative grids of the
// sessions that use it (the server's slots).  A grid takes what it needs, up to what is free,
// before its launch, and a host callback on its stream gives the share back when the kernel
// has finished, so the grids that run side by side always fit on the device together.
struct CoopLedger {
  std::mutex mu;
  std::condition_variable cv;
  double free = 0.9;       // 10 % slack for how CTAs of different grids pack into SMs
  double capacity = 0.9;   // what `free` is when no grid holds a share
  double min_share = 0.2;  // a grid waits until this much (or all it needs) is free
  long waits_expired = 0;  // waits that gave up (the grid then ran on what was free)
};

struct Session {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::map<std::string, std::pair<void *, size_t>> ws;
  bool timing = false;
  double phase_ms[4] = {0, 0, 0, 0};
  long phase_launches[4] = {0, 0, 0, 0};
  int sm_count = 148;
  size_t hbm_budget = 0;  // chunking budget; 0 = what the device has free
  bool barrier_used = false;  // a persistent kernel ran since the last error check
  // fault injection for tests (linqt_session_inject_barrier_timeout): grid barriers await
  // inject_extra more CTAs than launched and give up after inject_limit polls
  // fraction of the device's co-resident CTAs the session's persistent grids may use
  // (linqt_session_set_sm_share); below 1 they launch on the session stream, not the lane
  double coop_share = 1.0;
  // with a ledger (server slots) and coop_share < 1, each grid's share comes from the ledger
  CoopLedger *ledger = nullptr;
  double held_share = 0;  // taken for the grid about to launch, not yet handed to a callback
  int inject_extra = 0;
  long long inject_limit = 0;
  bool barrier_cfg_dirty = false;
  void *barrier_cfg_ptr = nullptr;
  // opts.use_graphs: solves replayed from instantiated CUDA graphs, by call key.  A graph holds
  // the workspace addresses it was captured with, so every workspace reallocation drops them.
  bool capturing = false;
  std::map<std::string, cudaGraphExec_t> graphs;
  std::map<std::string, int> graph_calls;  // calls seen per key (the first runs eagerly); -1: capture failed
  long graph_replays = 0;
  void drop_graphs();

  void *get(const std::string &name, size_t bytes);  // cached device buffer, >= bytes
  void trim();
  ~Session();
};

Session *default_session();
Session *resolve(linqt_session *s);

// scoped phase timer (CUDA events on the session stream when timing is on)
struct PhaseScope {
  Session *s;
  Phase ph;
  cudaEvent_t a = nullptr, b = nullptr;
  PhaseScope(Session *s_, Phase p);
  ~PhaseScope();
  void launches(long k) { s->phase_launches[ph] += k; }
};

// ---------------------------------------------------------------------------
// kernel launchers (spmm.cu, moments.cu, mu_gemm.cu, kubo_fft.cu, reconstruct.cu)
// ---------------------------------------------------------------------------
// y = alpha*A*x + beta*y on a block of R columns in site-major layout (x[i*R + r])
void spmm(Session *s, const DeviceOp &A, double2 alpha, const void *x, double2 beta, void *y, int R, bool fp32);

// one recursion step on a block: y = 2*H*x - yprev (yprev may alias y),
// optional fused V*x into vout, optional dot products into dots (see spmm.cu)
struct StepArgs {
  const void *x = nullptr;      // T_m
  const void *yprev = nullptr;  // T_{m-1} (nullptr: first step, y = H x)
  void *y = nullptr;            // T_{m+1} (nullptr: skip)
  const DeviceOp *V = nullptr;  // fused second operator
  void *vout = nullptr;         // V*x
  const void *phi = nullptr;    // for <phi|x> (direct 1D moments)
  double2 *dots = nullptr;      // per-step outputs: [0]=<x|x> or <phi|x>, [1]=<y|x>
  int dot_mode = 0;             // 0 none, 1 <phi|x>, 2 doubling (<x|x>, <y|x>)
};
void cheb_step(Session *s, const DeviceOp &H, const StepArgs &a, int R, bool fp32, int format);

// layout conversions between R x N (state-major, double) and N x R (site-major)
void states_to_block(Session *s, const double2 *states, void *block, int N, int R, int Rpad, bool fp32);

// 1D moments assembly from per-step dots
void moments1d_from_dots(Session *s, const double2 *dots, int steps, int M, int R, int mode, double2 *mu,
                         long stride = 1);

// mu_raw[M x M] += sum_k conj(L[m0][k]) * Rv[m1][k], FP64 (or FP32-input) operands
// C(i,j) (+)= sum_k conj(A[i][k]) B[j][k], FP64
void zgemm_cn(Session *s, const double2 *A, int MA, const double2 *B, int MB, long K, double2 *C, bool accumulate);
void mu_contract(Session *s, const void *L, const void *Rv, int M, long K, bool fp32_inputs, int precision,
                 double2 *mu_raw);
void mu_finalize(Session *s, const double2 *mu_raw, int M, int R, double2 *mu);
void reduce_parts_into(Session *s, const double2 *part, int S, long MM, double2 *dst);
// R random-phase states (R x N, state-major) from Philox4x32-10 with the given seed (states.cu)
void random_phase_states(Session *s, int N, int R, unsigned long long seed, double2 *out);
// tcgen05 split-TF32 contraction of FP32 Chebyshev blocks (mu_tc.cu)
bool mu_tc_supported(long K);
void mu_contract_tc(Session *s, const void *L, const void *Rv, int M, long K, double2 *mu_raw);
int mu_tc_check_error(Session *s);
// tcgen05 INT8 contraction of FP32 Chebyshev blocks split into 3 or 4 digits, exact accumulation (mu_i8.cu)
void mu_contract_i8(Session *s, const void *L, const void *Rv, int M, long K, int digits, double2 *mu_raw);
// digits per value of the INT8 contraction a precision mode uses (0: none)
inline int i8_digits(int precision) {
  return precision == LINQT_PREC_MIXED ? 4 : precision == LINQT_PREC_MIXED_FAST ? 3 : 0;
}
// The INT8 contraction splits K into slabs whose digit planes (6 * digits bytes per complex
// entry of one moment's block, L and R sides together) fit kI8DigitBudget; the planes are
// rewritten slab after slab.  i8_digit_bytes: the device bytes that takes for M moments of K.
constexpr size_t kI8DigitBudget = 8ull << 30;
inline long i8_slab(int digits, int M, long K) {
  const long per = 6L * digits * M;                       // bytes per complex column of K
  long slab = std::max(1024L, (long)(kI8DigitBudget / (size_t)per));
  slab = slab / 1024 * 1024;                              // keeps slab starts 16-byte aligned
  return std::min(K, slab);
}
inline size_t i8_digit_bytes(int digits, int M, long K) {
  return digits ? (size_t)6 * digits * M * (size_t)(i8_slab(digits, M, K) + 1024) : 0;
}

// FFT path: accumulate p/w over all sites into acc[2*nump] (complex)
// prefactors pf_m of Kubo_solver_FFT (kubo_fft.cu)
void kubo_prefactors(Session *s, int M, int nump, double2 *pf);
void kubo_fft_sites(Session *s, const void *L, const void *Rv, long nsites, int M, int nump, int formula,
                    bool fp32_inputs, double2 *acc);
void kubo_postprocess(Session *s, const double2 *acc, int R, int nump, int formula, int N, double band_width,
                      double band_center, double *out);

// reconstructions
void dos_grid(Session *s, const double2 *mu, int M, int N, double band_width, double band_center, double *E,
              double *dos);
// grid 0: num_div uniform points in [-1, 1], raw sums; grid 1: cos(pi (i+1/2)/num_div), |sum|
void spectral_grid(Session *s, const double2 *mu, int M, int N, double band_width, double band_center, int grid,
                   int num_div, double *E, double *out);
// LinQT's post-processor sums (variant 0 Bastin, 1 Greenwood, 2 Bastin I, 3 Bastin II, 4 sea,
// 5 surface) on a Jackson-damped device table; grid 0 uniform, 1 Chebyshev nodes, 2 ascending
void energy_sums(Session *s, const double2 *mu, int M0, int M1, int N, double band_width, double band_center,
                 int variant, int grid, double xbound, int num_div, double *E, double *out);
void bastin_grid(Session *s, const double2 *mu, int M0, int M1, int N, double band_width, double band_center,
                 double xbound, int num_div, double *E, double *sigma);

// bounds
void gershgorin(Session *s, const DeviceOp &A, double *lo, double *hi);

// Jackson kernel helpers (reconstruct.cu)
int jackson_cut(int M, double band_width, double broad);
double jackson_factor(int m, int Mom);
// timeCorrelationsFromChebmom on a device TD table mu[M x NT] (reconstruct.cu)
void time_correlation(Session *s, const double2 *mu, int M, int NT, int N, double band_width, double band_center,
                      double dt, double broad_meV, double energy, double *t_out, double *c_out, int *T_out);
void jackson2d_dev(Session *s, const double2 *mu, int M0, int M1, int M0t, int M1t, double2 *out);

// explicit-stream / caller-scratch launchers (spmm.cu, mu_gemm.cu) for the no-alloc entry point
int cheb_step_grid(int sm_count, int n, int R);
void cheb_step_scratch(cudaStream_t st, int sm_count, const DeviceOp &H, const StepArgs &a, int R,
                       double2 *partials, unsigned *counter);
void states_to_block_stream(cudaStream_t st, int sm_count, const double2 *states, void *block, int N, int R,
                            int Rpad);
void moments1d_from_dots_stream(cudaStream_t st, const double2 *dots, int steps, int M, int R, int mode,
                                double2 *mu);

// persistent recursions (recur.cu): one cooperative launch per recursion
// sellC = 0: the operator's CSR (row slices cached in shared memory when they fit); -1: CSR
// without the cache; sellC > 0: its SELL-C-sigma layout with slice height sellC.
// shape < recur_shapes(R): thread shape (shape s: min(R, 32) >> s threads per row)
int recur_shapes(int R);
void recur_lr(Session *s, const DeviceOp &H, const DeviceOp *V, void *Lstore, void *Rstore, const void *phi,
              void *tbuf, int M, int R, bool fp32, int sellC, int shape = 0);
// stacked != NULL: nreal realisations sharing H's pattern, values [nreal][nnz]; realisation r
// owns columns [r R/nreal, (r+1) R/nreal), served by its own group of CTAs, and dots becomes
// [nreal][steps][2]
// c64: the operator's complex64 value copy (FP32 values, FP64 accumulation); CSR layouts only,
// and `stacked` then holds float2 values
void recur_1d(Session *s, const DeviceOp &H, const void *phi, void *x0, void *b1, int steps, int M, int mode, int R,
              bool fp32, double2 *dots, int sellC, int shape = 0, const void *stacked = nullptr, int nreal = 1,
              bool c64 = false);
// X <- sum_{s<K} coef[s] T_s(H) X on an FP64 block of R columns (a, b: scratch blocks), one
// persistent launch (recur.cu)
void cheb_series(Session *s, const DeviceOp &H, void *X, void *a, void *b, const double2 *coef, int K, int R);
// after a stream synchronisation: fail with LINQT_ERR_TIMEOUT if a persistent kernel's barrier gave up
void check_device_errors(Session *s);
// chebyshev::SpectralMoments_nonOrth on the device (nonorth.cu): mu[M]; iterations (may be
// NULL; then nothing synchronises) gets the BiCGSTAB iterations summed over all solves
void moments1d_nonorth_dev(Session *s, const DeviceOp &H, const DeviceOp *op, const DeviceOp &S,
                           const double2 *states, int R, int M, double tol, int maxit, double2 *mu,
                           long long *iterations);
// the session's grid barrier for the next persistent launch (count and generation reset on
// the session stream; the error flag stays until check_device_errors reads it)
struct GridBarrier;
GridBarrier *barrier_for(Session *s);
// occupancy-sized cooperative grid and a launch through the device's cooperative lane (recur.cu)
int coop_grid(Session *s, const void *func, long max_blocks, size_t smem);
// The fraction of the co-resident CTAs a persistent grid of `s` may use, `want` being what it
// needs (at most 1): the session's fixed share, or with a ledger what it takes from it.
double coop_share_take(Session *s, double want);
void coop_share_return(Session *s);  // gives back a share taken for a grid that did not launch
// After a launch sized from coop_share_take: the share comes back (host callback on the
// session stream) once the work enqueued so far has finished.
void coop_share_hand_back(Session *s);
// SMs for a persistent non-cooperative kernel that occupies whole SMs (the per-site FFT):
// all of them, or with a ledger the share it takes (every SM when the ledger is all free),
// to be given back with coop_share_hand_back after the launch.
int sm_share_take(Session *s);
void coop_launch(Session *s, const void *f, int grid, void **args, size_t smem);

// small utilities (util.cu)
void sum_chunks_stream(cudaStream_t st, double2 *d, int len, int nchunks);
// Raise a kernel's dynamic shared-memory limit on the current device to at least `bytes`,
// never lowering it: the limit belongs to the function, and server slots on other threads
// launch the same kernels with other sizes, so a lowered limit could fail their launches.
void raise_smem_limit(const void *func, size_t bytes);
void sum_chunks(Session *s, double2 *d, int len, int nchunks);       // d[0:len] += sum_{c>0} d[c*len : ...]
void add_into(Session *s, double2 *dst, const double2 *src, int len); // dst += src
void block_to_states(Session *s, const void *blk, double2 *states, int N, int R, int Rpad);  // N x Rpad -> R x N

}  // namespace linqt

struct linqt_op {
  linqt::DeviceOp op;
};
struct linqt_session {
  linqt::Session s;
};
