// Small device utilities shared by the solvers.
#include "internal.cuh"

namespace linqt {

namespace {

__global__ void k_sum_chunks(double2 *__restrict__ d, int len, int nchunks) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < len; t += gridDim.x * blockDim.x) {
    double2 s = d[t];
    for (int c = 1; c < nchunks; ++c) s = cadd(s, d[(size_t)c * len + t]);
    d[t] = s;
  }
}

__global__ void k_add_into(double2 *__restrict__ dst, const double2 *__restrict__ src, int len) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < len; t += gridDim.x * blockDim.x)
    dst[t] = cadd(dst[t], src[t]);
}

__global__ void k_block_to_states(const double2 *__restrict__ blk, double2 *__restrict__ st, int N, int R, int Rpad) {
  const long total = (long)N * R;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int r = (int)(t / N), i = (int)(t % N);
    st[t] = blk[(size_t)i * Rpad + r];
  }
}

}  // namespace

void sum_chunks(Session *s, double2 *d, int len, int nchunks) { sum_chunks_stream(s->stream, d, len, nchunks); }

void sum_chunks_stream(cudaStream_t st, double2 *d, int len, int nchunks) {
  k_sum_chunks<<<(len + 255) / 256, 256, 0, st>>>(d, len, nchunks);
  LQ_LAUNCHED();
}

void raise_smem_limit(const void *func, size_t bytes) {
  static std::mutex m;
  static std::map<std::pair<int, const void *>, size_t> limits;
  int dev = 0;
  LQ_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(m);
  size_t &cur = limits[{dev, func}];
  if (bytes <= cur) return;
  LQ_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  cur = bytes;
}

void add_into(Session *s, double2 *dst, const double2 *src, int len) {
  k_add_into<<<(len + 255) / 256, 256, 0, s->stream>>>(dst, src, len);
  LQ_LAUNCHED();
}

void block_to_states(Session *s, const void *blk, double2 *states, int N, int R, int Rpad) {
  const long total = (long)N * R;
  const int grid = (int)std::max(1L, std::min((total + 255) / 256, (long)s->sm_count * 16));
  k_block_to_states<<<grid, 256, 0, s->stream>>>((const double2 *)blk, states, N, R, Rpad);
  LQ_LAUNCHED();
}

}  // namespace linqt
