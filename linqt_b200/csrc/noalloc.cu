// 1D Chebyshev moments with no device allocation.
//
// Who needs this: callers that must not call cudaMalloc or cudaFree while they run.
// The library's regular entry points keep a per-session workspace cache, and a cache
// miss calls cudaMalloc.  A resize calls cudaFree, which synchronises the whole device
// and stalls every other stream.  Some callers cannot accept that:
//   - a serving loop with a latency bound;
//   - a host thread that shares the GPU with a framework whose caching allocator owns
//     the device memory;
//   - code running where the CUDA allocation API may not be called.
// For them this entry point takes device pointers for its inputs and outputs, and keeps
// its scratch (Chebyshev blocks, per-step dot products, reduction partials) in one
// statically sized __device__ array that is part of the library image.  The array
// costs LINQT_NOALLOC_SCRATCH_BYTES of memory on every GPU that loads the library,
// held until the process exits.
#include <mutex>

#include "internal.cuh"

namespace linqt {

namespace {

// The scratch every call of linqt_moments1d_noalloc shares (one copy per device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[LINQT_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;

struct DeviceScratch {
  void *base = nullptr;  // device address of g_noalloc_scratch on this device
  int sm_count = 0;
};

std::mutex g_setup_mu;
DeviceScratch g_setup[kMaxDevices];

// Resolve the array's device address on the current device (once per device).  In host
// code g_noalloc_scratch names a host-side stand-in, not device memory, so the address
// must come from cudaGetSymbolAddress with the device current.
const DeviceScratch &setup_device(int dev) {
  LQ_REQUIRE(dev >= 0 && dev < kMaxDevices, "moments1d_noalloc: device index out of range");
  std::lock_guard<std::mutex> g(g_setup_mu);
  DeviceScratch &d = g_setup[dev];
  if (!d.base) {
    void *p = nullptr;
    LQ_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    int sms = 0;
    LQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    d.sm_count = sms;
    d.base = p;
  }
  return d;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

}  // namespace linqt

using namespace linqt;

extern "C" int linqt_moments1d_noalloc(const linqt_op *H, const double *states_dev, int R, int M, double *mu_dev,
                                       void *stream) {
  int prev_dev = -1;
  cudaGetDevice(&prev_dev);
  int rc = LINQT_OK;
  try {
    if (!H || !states_dev || !mu_dev) fail(LINQT_ERR_INVALID, "moments1d_noalloc: NULL argument");
    if (R <= 0 || M <= 0) fail(LINQT_ERR_INVALID, "moments1d_noalloc: R and M must be positive");
    const DeviceOp &op = H->op;
    if (op.device != prev_dev) LQ_CUDA(cudaSetDevice(op.device));
    const DeviceScratch &ds = setup_device(op.device);
    cudaStream_t st = (cudaStream_t)stream;
    if (st) {
      int sdev = -1;
      LQ_CUDA(cudaStreamGetDevice(st, &sdev));
      if (sdev != op.device)
        fail(LINQT_ERR_INVALID, "moments1d_noalloc: cuda_stream belongs to device " + std::to_string(sdev) +
                                    ", the operator to device " + std::to_string(op.device));
    }

    // Same block geometry and step count as linqt_moments1d with the identity operator
    // (doubling identities, block width = min(256, next power of two >= R)).
    int Rc = 1;
    while (Rc < R && Rc < 256) Rc <<= 1;
    const int nchunks = (R + Rc - 1) / Rc;
    const int steps = (M + 1) / 2;
    const int N = op.n;
    const int grid = cheb_step_grid(ds.sm_count, N, Rc);
    const size_t blk = sizeof(double2) * (size_t)N * Rc;
    // two Chebyshev blocks: the starting block (T_0, then every even T) and T_1 (every odd T)
    const size_t off_T = 0;
    const size_t off_dots = align256(off_T + 2 * blk);
    const size_t off_part = align256(off_dots + sizeof(double2) * 2 * (size_t)steps * nchunks);
    const size_t off_cnt = align256(off_part + sizeof(double2) * 2 * (size_t)grid);
    const size_t need = off_cnt + 256;
    if (need > (size_t)LINQT_NOALLOC_SCRATCH_BYTES)
      fail(LINQT_ERR_INVALID, "moments1d_noalloc: this solve needs " + std::to_string(need) +
                                  " bytes of scratch (2 Chebyshev blocks of N x " + std::to_string(Rc) +
                                  " complex doubles plus reductions), above the fixed LINQT_NOALLOC_SCRATCH_BYTES = " +
                                  std::to_string((size_t)LINQT_NOALLOC_SCRATCH_BYTES) +
                                  "; use linqt_moments1d_dev for larger systems");
    char *base = (char *)ds.base;
    char *T = base + off_T;
    double2 *dots = (double2 *)(base + off_dots);
    double2 *partials = (double2 *)(base + off_part);
    unsigned *counter = (unsigned *)(base + off_cnt);
    // the array keeps the previous call's contents: zero what must start at zero
    LQ_CUDA(cudaMemsetAsync(counter, 0, 256, st));
    LQ_CUDA(cudaMemsetAsync(dots, 0, sizeof(double2) * 2 * (size_t)steps * nchunks, st));

    for (int c = 0; c < nchunks; ++c) {
      void *phi = T, *b1 = T + blk;
      double2 *cd = dots + (size_t)2 * steps * c;
      const int w = std::min(Rc, R - c * Rc);
      states_to_block_stream(st, ds.sm_count, (const double2 *)states_dev + (size_t)c * Rc * N, phi, N, w, Rc);
      void *prev = nullptr, *cur = phi;
      for (int s = 0; s < steps; ++s) {
        StepArgs a;
        a.x = cur;
        a.yprev = prev;
        const bool need_y = 2 * s + 1 < M;
        a.y = need_y ? (prev ? prev : b1) : nullptr;
        a.dot_mode = 2;
        a.dots = cd + 2 * s;
        cheb_step_scratch(st, ds.sm_count, op, a, Rc, partials, counter);
        if (!need_y) break;
        prev = cur;
        cur = a.y;
      }
    }
    if (nchunks > 1) sum_chunks_stream(st, dots, 2 * steps, nchunks);
    moments1d_from_dots_stream(st, dots, steps, M, R, 2, (double2 *)mu_dev);
  } catch (const Error &e) {
    set_last_error(e.what());
    rc = e.code;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    rc = LINQT_ERR_INTERNAL;
  }
  if (prev_dev >= 0) cudaSetDevice(prev_dev);
  return rc;
}
