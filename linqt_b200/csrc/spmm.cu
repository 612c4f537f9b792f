// Sparse kernels of the Chebyshev recursion.
//
// Layout: a block of R vectors is stored site-major, x[i*R + r] (complex), so the
// R values a non-zero H_ij multiplies are one contiguous R*16-byte run (R*8 in
// FP32).  A group of TPR threads owns a row; thread `lane` owns the columns
// r = lane + TPR*u, u < VPT, so every x load of a group is one coalesced run and
// the row's column index / value loads are broadcast within the group.
//
// One launch performs one recursion step  T_{m+1} = 2 H T_m - T_{m-1}
// (Moments::Iterate, src/chebyshev_moments.cpp:157-162; the first step is
// T_1 = H T_0, src/chebyshev_moments.cpp:45-59) and, fused into the epilogue:
//   - V*T_m for a second operator sharing the x loads (the OPR application of
//     Vectors::Multiply, src/chebyshev_vectors.cpp:24-51);
//   - the moment dot products  <phi|T_m>  (chebyshev::SpectralMoments,
//     src/chebyshev_solver.cpp:193-195) or, with the doubling identities
//     T_{2m} = 2 T_m^2 - T_0 and T_{2m+1} = 2 T_{m+1} T_m - T_1,  <T_m|T_m> and <T_{m+1}|T_m>.
// Dot products are reduced per block (warp shuffles + shared memory), written to a
// partial array, and the last block to finish sums the partials in a fixed order
// (deterministic; no spin waits).
#include "internal.cuh"

namespace linqt {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double2 shfl_down2(double2 v, int o) {
  v.x = __shfl_down_sync(0xffffffffu, v.x, o);
  v.y = __shfl_down_sync(0xffffffffu, v.y, o);
  return v;
}

// Reduce (d0, d1) over the block; returns the sums in thread 0.
__device__ void block_reduce2(double2 &d0, double2 &d1) {
  __shared__ double2 sh[2][kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    d0 = cadd(d0, shfl_down2(d0, o));
    d1 = cadd(d1, shfl_down2(d1, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sh[0][w] = d0;
    sh[1][w] = d1;
  }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    d0 = l < nw ? sh[0][l] : make_double2(0, 0);
    d1 = l < nw ? sh[1][l] : make_double2(0, 0);
    for (int o = 16; o > 0; o >>= 1) {
      d0 = cadd(d0, shfl_down2(d0, o));
      d1 = cadd(d1, shfl_down2(d1, o));
    }
  }
  __syncthreads();
}

// Publish this block's partial sums; the last block reduces all partials in
// index order and writes out[0..1].  counter is reset to zero for the next launch.
__device__ void grid_reduce2(double2 d0, double2 d1, double2 *partials, unsigned *counter, double2 *out) {
  __shared__ bool am_last;
  block_reduce2(d0, d1);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = d0;
    partials[2 * blockIdx.x + 1] = d1;
    __threadfence();
    const unsigned t = atomicAdd(counter, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double2 s0 = make_double2(0, 0), s1 = make_double2(0, 0);
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    s0 = cadd(s0, __ldcg(partials + 2 * b));
    s1 = cadd(s1, __ldcg(partials + 2 * b + 1));
  }
  block_reduce2(s0, s1);
  if (threadIdx.x == 0) {
    out[0] = s0;
    out[1] = s1;
    *counter = 0u;
  }
}

template <class C>
__device__ __forceinline__ C ld(const C *p) {
  return __ldg(p);
}

// One recursion step on a CSR operator (FP64 values and accumulation for either vector
// precision; FP32 results are rounded once).  FUSE_V adds a second CSR operator applied
// to the same x.  dot_mode: 0 none, 1 <phi|x>, 2 <x|x> and <y|x>.
template <class T, int TPR, int VPT, bool FUSE_V>
__global__ void __launch_bounds__(kThreads)
    k_step_csr(int n, const int *__restrict__ rp, const int *__restrict__ ci, const double2 *__restrict__ hv,
               const int *__restrict__ vrp, const int *__restrict__ vci, const double2 *__restrict__ vv,
               const typename cplx_t<T>::type *__restrict__ x, const typename cplx_t<T>::type *yprev,
               typename cplx_t<T>::type *y, typename cplx_t<T>::type *__restrict__ vout,
               const typename cplx_t<T>::type *__restrict__ phi, int first, int dot_mode,
               double2 *__restrict__ partials, unsigned *__restrict__ counter, double2 *__restrict__ dots) {
  using C = typename cplx_t<T>::type;
  constexpr int R = TPR * VPT;
  const int lane = threadIdx.x % TPR;
  const int gpb = kThreads / TPR;
  double2 d0 = make_double2(0, 0), d1 = make_double2(0, 0);
  for (int row = blockIdx.x * gpb + threadIdx.x / TPR; row < n; row += gridDim.x * gpb) {
    double2 acc[VPT];
#pragma unroll
    for (int u = 0; u < VPT; ++u) acc[u] = make_double2(0, 0);
    {
      const int b = rp[row], e = rp[row + 1];
#pragma unroll 4
      for (int k = b; k < e; ++k) {
        const int j = __ldg(ci + k);
        const double2 h = ld(hv + k);
        const C *xr = x + (size_t)j * R + lane;
#pragma unroll
        for (int u = 0; u < VPT; ++u) acc[u] = cfma(h, ld(xr + u * TPR), acc[u]);
      }
    }
    const size_t base = (size_t)row * R + lane;
    if (FUSE_V) {
      double2 accv[VPT];
#pragma unroll
      for (int u = 0; u < VPT; ++u) accv[u] = make_double2(0, 0);
      const int b = vrp[row], e = vrp[row + 1];
#pragma unroll 4
      for (int k = b; k < e; ++k) {
        const int j = __ldg(vci + k);
        const double2 h = ld(vv + k);
        const C *xr = x + (size_t)j * R + lane;
#pragma unroll
        for (int u = 0; u < VPT; ++u) accv[u] = cfma(h, ld(xr + u * TPR), accv[u]);
      }
#pragma unroll
      for (int u = 0; u < VPT; ++u) vout[base + u * TPR] = from_d2<C>(accv[u]);
    }
#pragma unroll
    for (int u = 0; u < VPT; ++u) {
      const size_t idx = base + u * TPR;
      double2 ya = acc[u];
      if (!first) {
        const double2 p = to_d2(yprev[idx]);
        ya.x = 2 * ya.x - p.x;
        ya.y = 2 * ya.y - p.y;
      }
      const C yn = from_d2<C>(ya);
      if (y) y[idx] = yn;
      if (dot_mode == 1) {
        d0 = cfma_conj(to_d2(ld(phi + idx)), to_d2(ld(x + idx)), d0);
      } else if (dot_mode == 2) {
        const double2 xi = to_d2(ld(x + idx));
        d0 = cfma_conj(xi, xi, d0);
        d1 = cfma_conj(to_d2(yn), xi, d1);
      }
    }
  }
  if (dot_mode) grid_reduce2(d0, d1, partials, counter, dots);
}

// y = alpha*A*x + beta*y  (general SpMM on a site-major block)
template <class T, int TPR, int VPT>
__global__ void __launch_bounds__(kThreads)
    k_spmm_csr(int n, const int *__restrict__ rp, const int *__restrict__ ci, const double2 *__restrict__ av,
               const typename cplx_t<T>::type *__restrict__ x,
               typename cplx_t<T>::type *y, double2 alpha, double2 beta) {
  using C = typename cplx_t<T>::type;
  constexpr int R = TPR * VPT;
  const int lane = threadIdx.x % TPR;
  const int gpb = kThreads / TPR;
  for (int row = blockIdx.x * gpb + threadIdx.x / TPR; row < n; row += gridDim.x * gpb) {
    double2 acc[VPT];
#pragma unroll
    for (int u = 0; u < VPT; ++u) acc[u] = make_double2(0, 0);
    const int b = rp[row], e = rp[row + 1];
#pragma unroll 4
    for (int k = b; k < e; ++k) {
      const int j = __ldg(ci + k);
      const double2 h = __ldg(av + k);
      const C *xr = x + (size_t)j * R + lane;
#pragma unroll
      for (int u = 0; u < VPT; ++u) acc[u] = cfma(h, __ldg(xr + u * TPR), acc[u]);
    }
    const size_t base = (size_t)row * R + lane;
#pragma unroll
    for (int u = 0; u < VPT; ++u) {
      double2 r = cmul(alpha, acc[u]);
      if (beta.x != 0.0 || beta.y != 0.0) r = cadd(r, cmul(beta, to_d2(y[base + u * TPR])));
      y[base + u * TPR] = typename cplx_t<T>::type{(T)r.x, (T)r.y};
    }
  }
}

// R x N state-major doubles -> N x Rpad site-major block (zero columns r >= R)
template <class T>
__global__ void k_states_to_block(const double2 *__restrict__ st, typename cplx_t<T>::type *__restrict__ blk, int N,
                                  int R, int Rpad) {
  const long total = (long)N * Rpad;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t / Rpad), r = (int)(t % Rpad);
    double2 v = r < R ? st[(size_t)r * N + i] : make_double2(0, 0);
    blk[t] = typename cplx_t<T>::type{(T)v.x, (T)v.y};
  }
}

int grid_for(Session *s, long rows, int tpr) {
  const long need = (rows * tpr + kThreads - 1) / kThreads;
  const long cap = (long)s->sm_count * 8;
  return (int)std::max(1L, std::min(need, cap));
}

template <class T, int TPR, int VPT>
void launch_step(Session *s, const DeviceOp &H, const StepArgs &a) {
  using C = typename cplx_t<T>::type;
  const double2 *hv = H.d_val64;
  const int grid = grid_for(s, H.n, TPR);
  double2 *partials = nullptr;
  unsigned *counter = nullptr;
  if (a.dot_mode) {
    partials = (double2 *)s->get("step_partials", sizeof(double2) * 2 * (size_t)grid);
    counter = (unsigned *)s->get("step_counter", sizeof(unsigned) * 32);
  }
  const int first = a.yprev == nullptr;
  if (a.V) {
    const DeviceOp &V = *a.V;
    const double2 *vv = V.d_val64;
    k_step_csr<T, TPR, VPT, true><<<grid, kThreads, 0, s->stream>>>(
        H.n, H.d_rowptr, H.d_col, hv, V.d_rowptr, V.d_col, vv, (const C *)a.x, (const C *)a.yprev, (C *)a.y,
        (C *)a.vout, (const C *)a.phi, first, a.dot_mode, partials, counter, a.dots);
  } else {
    k_step_csr<T, TPR, VPT, false><<<grid, kThreads, 0, s->stream>>>(
        H.n, H.d_rowptr, H.d_col, hv, nullptr, nullptr, nullptr, (const C *)a.x, (const C *)a.yprev, (C *)a.y,
        nullptr, (const C *)a.phi, first, a.dot_mode, partials, counter, a.dots);
  }
  LQ_LAUNCHED();
}

template <class T, int TPR, int VPT>
void launch_spmm(Session *s, const DeviceOp &A, double2 alpha, const void *x, double2 beta, void *y) {
  using C = typename cplx_t<T>::type;
  const double2 *av = A.d_val64;
  const int grid = grid_for(s, A.n, TPR);
  k_spmm_csr<T, TPR, VPT><<<grid, kThreads, 0, s->stream>>>(A.n, A.d_rowptr, A.d_col, av, (const C *)x, (C *)y,
                                                            alpha, beta);
  LQ_LAUNCHED();
}

// dispatch over the (padded, power-of-two) block width
template <class T, template <class, int, int> class F, class... Args>
void dispatch_width(int R, Args &&...args) {
  switch (R) {
    case 1: return F<T, 1, 1>::run(args...);
    case 2: return F<T, 2, 1>::run(args...);
    case 4: return F<T, 4, 1>::run(args...);
    case 8: return F<T, 8, 1>::run(args...);
    case 16: return F<T, 16, 1>::run(args...);
    case 32: return F<T, 32, 1>::run(args...);
    case 64: return F<T, 32, 2>::run(args...);
    case 128: return F<T, 32, 4>::run(args...);
    case 256: return F<T, 32, 8>::run(args...);
    default: fail(LINQT_ERR_UNSUPPORTED, "block width must be a power of two <= 256, got " + std::to_string(R));
  }
}

template <class T, int TPR, int VPT>
struct StepF {
  static void run(Session *s, const DeviceOp &H, const StepArgs &a) { launch_step<T, TPR, VPT>(s, H, a); }
};
template <class T, int TPR, int VPT>
struct SpmmF {
  static void run(Session *s, const DeviceOp &A, double2 alpha, const void *x, double2 beta, void *y) {
    launch_spmm<T, TPR, VPT>(s, A, alpha, x, beta, y);
  }
};

}  // namespace

void cheb_step(Session *s, const DeviceOp &H, const StepArgs &a, int R, bool fp32, int /*format*/) {
  if (fp32)
    dispatch_width<float, StepF>(R, s, H, a);
  else
    dispatch_width<double, StepF>(R, s, H, a);
}

void spmm(Session *s, const DeviceOp &A, double2 alpha, const void *x, double2 beta, void *y, int R, bool fp32) {
  if (fp32)
    dispatch_width<float, SpmmF>(R, s, A, alpha, x, beta, y);
  else
    dispatch_width<double, SpmmF>(R, s, A, alpha, x, beta, y);
}

// ---------------------------------------------------------------------------
// Launchers with an explicit stream and caller-supplied scratch (used by the
// entry point that allocates nothing).  They launch the same kernels with the same
// grid as cheb_step / states_to_block, so results are bitwise identical.
// ---------------------------------------------------------------------------
namespace {
template <class T, int TPR, int VPT>
struct StepScratchF {
  static void run(cudaStream_t st, int sm_count, const DeviceOp &H, const StepArgs &a, double2 *partials,
                  unsigned *counter) {
    using C = typename cplx_t<T>::type;
    const long need = ((long)H.n * TPR + kThreads - 1) / kThreads;
    const int grid = (int)std::max(1L, std::min(need, (long)sm_count * 8));
    const int first = a.yprev == nullptr;
    k_step_csr<T, TPR, VPT, false><<<grid, kThreads, 0, st>>>(
        H.n, H.d_rowptr, H.d_col, (const C *)H.d_val64, nullptr, nullptr, nullptr, (const C *)a.x,
        (const C *)a.yprev, (C *)a.y, nullptr, (const C *)a.phi, first, a.dot_mode, partials, counter, a.dots);
    LQ_LAUNCHED();
  }
};
}  // namespace

int cheb_step_grid(int sm_count, int n, int R) {
  const int tpr = R >= 32 ? 32 : R;
  const long need = ((long)n * tpr + kThreads - 1) / kThreads;
  return (int)std::max(1L, std::min(need, (long)sm_count * 8));
}

void cheb_step_scratch(cudaStream_t st, int sm_count, const DeviceOp &H, const StepArgs &a, int R,
                       double2 *partials, unsigned *counter) {
  if (a.V) fail(LINQT_ERR_UNSUPPORTED, "cheb_step_scratch: no fused second operator");
  dispatch_width<double, StepScratchF>(R, st, sm_count, H, a, partials, counter);
}

void states_to_block_stream(cudaStream_t st, int sm_count, const double2 *states, void *block, int N, int R,
                            int Rpad) {
  const long total = (long)N * Rpad;
  const int grid = (int)std::max(1L, std::min((total + 255) / 256, (long)sm_count * 16));
  k_states_to_block<double><<<grid, 256, 0, st>>>(states, (double2 *)block, N, R, Rpad);
  LQ_LAUNCHED();
}

void states_to_block(Session *s, const double2 *states, void *block, int N, int R, int Rpad, bool fp32) {
  const long total = (long)N * Rpad;
  const int grid = (int)std::max(1L, std::min((total + 255) / 256, (long)s->sm_count * 16));
  if (fp32)
    k_states_to_block<float><<<grid, 256, 0, s->stream>>>(states, (float2 *)block, N, R, Rpad);
  else
    k_states_to_block<double><<<grid, 256, 0, s->stream>>>(states, (double2 *)block, N, R, Rpad);
  LQ_LAUNCHED();
}

}  // namespace linqt
