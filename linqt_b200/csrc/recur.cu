// Persistent recursion kernels: a whole Chebyshev recursion in one cooperative launch.
// (The grid barrier between steps is grid_sync.cuh's.)
//
// One launch per recursion step (spmm.cu) costs a launch gap and a cold start per step.
// At LinQT's sizes a step is 1-10 us of memory traffic, so the gaps are a large part of
// it.  Here every CTA owns a fixed contiguous range of rows and loops over the steps.
// Between steps the CTAs meet at a grid barrier with a bounded spin: after
// kSpinLimit polls a CTA sets the error flag and the kernel returns, so a bad launch
// cannot hang the GPU.  The host reports LINQT_ERR_TIMEOUT.
//
// Step semantics are those of spmm.cu (Moments::Iterate, src/chebyshev_moments.cpp:157-162;
// Vectors::IterateAll / Multiply, src/chebyshev_vectors.cpp:4-51).  k_recur_lr advances the
// L recursion (in place inside its store) and the R recursion (rotating blocks, V*T_m into
// its store) together.  They share the row's H loads.  k_recur_1d runs the 1D moment
// recursion with the dot products of every step written as per-CTA partials, reduced
// afterwards in a fixed order.
//
// Vectors written in one step are read by other CTAs in the next.  The grid barrier
// orders those writes before the next step's reads (release: bar.sync, fence, atomic;
// acquire: poll, fence, bar.sync) and its gpu-scope fence invalidates stale L1 lines, so
// vector loads may go through L1 (ld.global.ca), where a row's neighbours read by nearby
// rows of the same CTA hit.  Operators (read-only for the whole launch) use the
// read-only path.  The operators are FP64 for either vector precision: FP32 blocks are
// accumulated in FP64 and rounded once per entry and step.
#include <memory>
#include <unordered_map>

#include "grid_sync.cuh"
#include "internal.cuh"

namespace linqt {

namespace {

constexpr int kThreads = 256;

using Barrier = GridBarrier;

template <class C>
__device__ __forceinline__ C ldv(const C *p) {
  return __ldca(p);
}

// The V adjacent complex values a thread owns in a block row, loaded through L1 with the
// widest aligned accesses (p is aligned to min(32, V * sizeof(C)) bytes: rows hold a power
// of two >= V columns and blocks start 256-byte aligned).  One 32-byte access carries two
// FP64 or four FP32 complex numbers, so a gather of a neighbour row costs V/2 (FP64) or
// V/4 (FP32) loads per thread instead of V.  The loads are volatile asm so that they stay
// after the grid barrier that orders the previous step's stores before them.
template <int V>
__device__ __forceinline__ void ld_row(const double2 *p, double2 (&o)[V]) {
  if constexpr (V == 1) {
    o[0] = __ldca(p);
  } else {
#pragma unroll
    for (int q = 0; q < V; q += 2) {
      double a, b, c, d;
      asm volatile("ld.global.ca.v4.f64 {%0, %1, %2, %3}, [%4];"
                   : "=d"(a), "=d"(b), "=d"(c), "=d"(d)
                   : "l"(p + q));
      o[q] = make_double2(a, b);
      o[q + 1] = make_double2(c, d);
    }
  }
}

template <int V>
__device__ __forceinline__ void ld_row(const float2 *p, float2 (&o)[V]) {
  if constexpr (V == 1) {
    o[0] = __ldca(p);
  } else if constexpr (V == 2) {
    const float4 t = __ldca(reinterpret_cast<const float4 *>(p));
    o[0] = make_float2(t.x, t.y);
    o[1] = make_float2(t.z, t.w);
  } else {
#pragma unroll
    for (int q = 0; q < V; q += 4) {
      float a[8];
      asm volatile("ld.global.ca.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                   : "=f"(a[0]), "=f"(a[1]), "=f"(a[2]), "=f"(a[3]), "=f"(a[4]), "=f"(a[5]), "=f"(a[6]),
                     "=f"(a[7])
                   : "l"(p + q));
#pragma unroll
      for (int w = 0; w < 4; ++w) o[q + w] = make_float2(a[2 * w], a[2 * w + 1]);
    }
  }
}

// Ask L2 for the line holding p (a hint: no register, no wait), so that a load of p issued
// after other long-latency loads finds it there.
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

template <int V>
__device__ __forceinline__ void st_row(double2 *p, const double2 (&v)[V]) {
#pragma unroll
  for (int q = 0; q < V; ++q) p[q] = v[q];
}

template <int V>
__device__ __forceinline__ void st_row(float2 *p, const float2 (&v)[V]) {
  if constexpr (V == 1) {
    p[0] = v[0];
  } else {
#pragma unroll
    for (int q = 0; q < V; q += 2)
      *reinterpret_cast<float4 *>(p + q) = make_float4(v[q].x, v[q].y, v[q + 1].x, v[q + 1].y);
  }
}

// acc[u] += h * x[u]
template <class C, int V>
__device__ __forceinline__ void gather_fma(double2 h, const C *p, double2 (&acc)[V]) {
  C t[V];
  ld_row<V>(p, t);
#pragma unroll
  for (int u = 0; u < V; ++u) acc[u] = cfma(h, t[u], acc[u]);
}

__device__ __forceinline__ double2 shfl_down2(double2 v, int o) {
  v.x = __shfl_down_sync(0xffffffffu, v.x, o);
  v.y = __shfl_down_sync(0xffffffffu, v.y, o);
  return v;
}

// block sums of (d0, d1), valid in thread 0
__device__ void block_sum2(double2 &d0, double2 &d1) {
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
    d0 = l < kThreads / 32 ? sh[0][l] : make_double2(0, 0);
    d1 = l < kThreads / 32 ? sh[1][l] : make_double2(0, 0);
    for (int o = 16; o > 0; o >>= 1) {
      d0 = cadd(d0, shfl_down2(d0, o));
      d1 = cadd(d1, shfl_down2(d1, o));
    }
  }
  __syncthreads();
}


// The non-zeros of the row handled at position `pos`.  CSR: row = pos, entries
// rp[row] .. rp[row+1] - 1.  SELL-C-sigma (sperm != NULL): rows sorted by length inside
// windows of sigma rows, grouped in slices of C; slice s stores its entries column-major
// (entry k of its i-th row at soff[s] + k*C + i, short rows padded with zeros), so the
// rows of a warp read consecutive addresses at every k.  row = sperm[pos].
__device__ __forceinline__ void sell_or_csr(int pos, const int *__restrict__ sperm, const int *__restrict__ soff,
                                            int sC, const int *__restrict__ rp, int &row, int &b, int &e, int &st) {
  if (sperm) {
    const int sl = pos / sC, i = pos - sl * sC;
    row = sperm[pos];
    b = soff[sl] + i;
    e = soff[sl + 1];
    st = sC;
  } else {
    row = pos;
    b = rp[pos];
    e = rp[pos + 1];
    st = 1;
  }
}

// Copy this CTA's rows [r0, r1) of a CSR operator into shared memory at `dst` and return
// pointers that index like the global arrays (rowptr by global row, col/val by global
// entry).  `dst` is 16-byte aligned; returns the bytes used.
template <class C>
__device__ size_t cache_rows(const int *__restrict__ rp, const int *__restrict__ ci, const C *__restrict__ v, int r0,
                             int r1, unsigned char *dst, const int *&rp_o, const int *&ci_o, const C *&v_o) {
  const int k0 = rp[r0], k1 = rp[r1];
  const int nnz = k1 - k0, nr = r1 - r0;
  C *sv = reinterpret_cast<C *>(dst);
  int *sc = reinterpret_cast<int *>(sv + nnz);
  int *sr = sc + nnz;
  for (int k = threadIdx.x; k < nnz; k += blockDim.x) {
    sv[k] = v[k0 + k];
    sc[k] = ci[k0 + k];
  }
  for (int i = threadIdx.x; i <= nr; i += blockDim.x) sr[i] = rp[r0 + i];
  rp_o = sr - r0;
  ci_o = sc - k0;
  v_o = sv - k0;
  return ((size_t)nnz * (sizeof(C) + 4) + (size_t)(nr + 1) * 4 + 15) & ~(size_t)15;
}

// ---------------------------------------------------------------------------
// L and R recursions of CorrelationExpansionMoments / Kubo_solver_FFT.
//   L: Lst[0] given (OPL phi); Lst[m+1] = 2 H Lst[m] - Lst[m-1] (Lst[1] = H Lst[0]), m+1 < M.
//   R (HAS_V): T_0 = phi, T_{m+1} = tb[m % 3]; Rst[m] = V T_m for m < M.
//   R (!HAS_V): Rst[0] given (phi); in place like L.
// ---------------------------------------------------------------------------
template <class T, int TPR, int VPT, bool HAS_V>
__global__ void __launch_bounds__(kThreads)
    k_recur_lr(int n, const int *rp, const int *ci, const double2 *hv, const int *vrp, const int *vci,
               const double2 *vv, typename cplx_t<T>::type *Lst,
               typename cplx_t<T>::type *Rst, const typename cplx_t<T>::type *phi, typename cplx_t<T>::type *tb, int M,
               size_t blk, Barrier *bar, int cache, const int *__restrict__ sperm, const int *__restrict__ soff,
               int sC) {
  using C = typename cplx_t<T>::type;
  constexpr int R = TPR * VPT;
  const int c0 = (threadIdx.x % TPR) * VPT;  // this thread's VPT adjacent columns
  constexpr int gpb = kThreads / TPR;
  const int per = (n + gridDim.x - 1) / gridDim.x;
  const int r0 = min(n, blockIdx.x * per), r1 = min(n, r0 + per);
  if (cache) {
    // the operators do not change during the recursion: keep this CTA's rows on chip
    extern __shared__ __align__(16) unsigned char smc[];
    size_t off = cache_rows<double2>(rp, ci, hv, r0, r1, smc, rp, ci, hv);
    if (HAS_V) cache_rows<double2>(vrp, vci, vv, r0, r1, smc + off, vrp, vci, vv);
    __syncthreads();
  }
  // Rows: with the operators cached, this CTA's contiguous range; otherwise tiles of gpb
  // rows dealt round-robin, so that all CTAs sweep the rows together and a row's
  // neighbours (read by nearby tiles at about the same time) are still in L2.
  const int rfirst = cache ? r0 : blockIdx.x * gpb, rend = cache ? r1 : n;
  const int rstep = cache ? gpb : gridDim.x * gpb;
  for (int m = 0; m < M; ++m) {
    const bool doL = m + 1 < M;
    const C *xL = Lst + (size_t)m * blk;
    const C *pL = m ? Lst + (size_t)(m - 1) * blk : nullptr;
    C *yL = Lst + (size_t)(m + 1) * blk;
    const C *xR, *pR;
    C *yR;
    if (HAS_V) {
      xR = m == 0 ? phi : tb + (size_t)((m - 1) % 3) * blk;
      pR = m == 0 ? nullptr : (m == 1 ? phi : tb + (size_t)((m - 2) % 3) * blk);
      yR = doL ? tb + (size_t)(m % 3) * blk : nullptr;
    } else {
      xR = Rst + (size_t)m * blk;
      pR = m ? Rst + (size_t)(m - 1) * blk : nullptr;
      yR = doL ? Rst + (size_t)(m + 1) * blk : nullptr;
    }
    for (int pos = rfirst + threadIdx.x / TPR; pos < rend; pos += rstep) {
      int row, b, e, st;
      sell_or_csr(pos, sperm, soff, sC, rp, row, b, e, st);
      double2 aL[VPT], aR[VPT];
#pragma unroll
      for (int u = 0; u < VPT; ++u) aL[u] = aR[u] = make_double2(0, 0);
      const size_t base = (size_t)row * R + c0;
      // the previous vectors of this row, read after the gathers
      if (doL && pL) prefetch_l2(pL + base);
      if (yR && pR) prefetch_l2(pR + base);
#pragma unroll 4
      for (int k = b; k < e; k += st) {
        const int j = ci[k];
        const double2 h = hv[k];
        const size_t off = (size_t)j * R + c0;
        if (doL) gather_fma<C, VPT>(h, xL + off, aL);
        gather_fma<C, VPT>(h, xR + off, aR);
      }
      if (HAS_V) {
        double2 aV[VPT];
#pragma unroll
        for (int u = 0; u < VPT; ++u) aV[u] = make_double2(0, 0);
        const int vb = vrp[row], ve = vrp[row + 1];
#pragma unroll 4
        for (int k = vb; k < ve; ++k) gather_fma<C, VPT>(vv[k], xR + (size_t)vci[k] * R + c0, aV);
        C o[VPT];
#pragma unroll
        for (int u = 0; u < VPT; ++u) o[u] = from_d2<C>(aV[u]);
        st_row<VPT>(Rst + (size_t)m * blk + base, o);
      }
      if (doL) {
        C o[VPT];
        if (pL) {
          C p[VPT];
          ld_row<VPT>(pL + base, p);
#pragma unroll
          for (int u = 0; u < VPT; ++u) {
            const double2 q = to_d2(p[u]);
            o[u] = from_d2<C>(make_double2(2 * aL[u].x - q.x, 2 * aL[u].y - q.y));
          }
        } else {
#pragma unroll
          for (int u = 0; u < VPT; ++u) o[u] = from_d2<C>(aL[u]);
        }
        st_row<VPT>(yL + base, o);
      }
      if (yR) {
        C o[VPT];
        if (pR) {
          C p[VPT];
          ld_row<VPT>(pR + base, p);
#pragma unroll
          for (int u = 0; u < VPT; ++u) {
            const double2 q = to_d2(p[u]);
            o[u] = from_d2<C>(make_double2(2 * aR[u].x - q.x, 2 * aR[u].y - q.y));
          }
        } else {
#pragma unroll
          for (int u = 0; u < VPT; ++u) o[u] = from_d2<C>(aR[u]);
        }
        st_row<VPT>(yR + base, o);
      }
    }
    if (m + 1 < M && !grid_barrier(bar, gridDim.x)) return;
  }
}

// ---------------------------------------------------------------------------
// 1D moments (chebyshev::SpectralMoments, src/chebyshev_solver.cpp:176-199).
//   mode 1 (direct):   x_0 = T_0 in b0; partial[s] = <phi|T_s>.
//   mode 2 (doubling): x_0 = phi;      partial[s] = (<T_s|T_s>, <T_{s+1}|T_s>).
// The recursion runs in place: T_{s+1} overwrites T_{s-1}; T_1 goes to b1.
// partials: [steps][grid][2] per-CTA sums.
// ---------------------------------------------------------------------------
template <class T, class HV, int TPR, int VPT, bool STACKED>
__global__ void __launch_bounds__(kThreads)
    k_recur_1d(int n, const int *rp, const int *ci, const HV *hv, const typename cplx_t<T>::type *phi, typename cplx_t<T>::type *x0, typename cplx_t<T>::type *b1,
               int steps, int M, int mode, double2 *__restrict__ partials, Barrier *bar, int cache,
               const int *__restrict__ sperm, const int *__restrict__ soff, int sC, long vstride, int nreal,
               int ldx_rt) {
  using C = typename cplx_t<T>::type;
  constexpr int RW = TPR * VPT;  // columns handled by a CTA
  const int c0 = (threadIdx.x % TPR) * VPT;  // this thread's VPT adjacent columns
  constexpr int gpb = kThreads / TPR;
  // STACKED: nreal realisations (value sets at hv + r*vstride) share the sparsity pattern; the
  // grid is split into nreal equal groups of CTAs, group r serving columns [r*RW, (r+1)*RW) of
  // rows of ldx_rt columns.  Otherwise one group, rows of RW columns.
  const int ldx = STACKED ? ldx_rt : RW;
  const int G1 = STACKED ? (int)gridDim.x / nreal : (int)gridDim.x;
  const int real = STACKED ? (int)blockIdx.x / G1 : 0;
  const int bl = STACKED ? (int)blockIdx.x % G1 : (int)blockIdx.x;
  const int coff = real * RW;
  if (STACKED) hv += (size_t)real * vstride;
  const int per = (n + gridDim.x - 1) / gridDim.x;
  const int r0 = min(n, blockIdx.x * per), r1 = min(n, r0 + per);
  if (cache) {
    extern __shared__ __align__(16) unsigned char smc1[];
    cache_rows<HV>(rp, ci, hv, r0, r1, smc1, rp, ci, hv);
    __syncthreads();
  }
  const int rfirst = cache ? r0 : bl * gpb, rend = cache ? r1 : n;  // as in k_recur_lr
  const int rstep = cache ? gpb : G1 * gpb;
  C *prev = nullptr, *cur = x0;
  for (int s = 0; s < steps; ++s) {
    const bool need_y = mode == 2 ? (2 * s + 1 < M) : (s + 1 < M);
    C *y = need_y ? (prev ? prev : b1) : nullptr;
    double2 d0 = make_double2(0, 0), d1 = make_double2(0, 0);
    for (int pos = rfirst + threadIdx.x / TPR; pos < rend; pos += rstep) {
      int row, b, e, st;
      sell_or_csr(pos, sperm, soff, sC, rp, row, b, e, st);
      double2 acc[VPT];
#pragma unroll
      for (int u = 0; u < VPT; ++u) acc[u] = make_double2(0, 0);
      const size_t base = (size_t)row * ldx + coff + c0;
      if (prev) prefetch_l2(prev + base);  // T_{s-1} of this row, read after the gathers
#pragma unroll 4
      for (int k = b; k < e; k += st) gather_fma<C, VPT>(to_d2(hv[k]), cur + (size_t)ci[k] * ldx + coff + c0, acc);
      C pv[VPT], yv[VPT], xv[VPT];
      if (prev) ld_row<VPT>(prev + base, pv);
#pragma unroll
      for (int u = 0; u < VPT; ++u) {
        double2 ya = acc[u];
        if (prev) {
          const double2 p = to_d2(pv[u]);
          ya.x = 2 * ya.x - p.x;
          ya.y = 2 * ya.y - p.y;
        }
        yv[u] = from_d2<C>(ya);  // the value stored and used in the dot products
      }
      if (y) st_row<VPT>(y + base, yv);
      ld_row<VPT>(cur + base, xv);
      if (mode == 1) {
        C fv[VPT];
        ld_row<VPT>(phi + base, fv);
#pragma unroll
        for (int u = 0; u < VPT; ++u) d0 = cfma_conj(to_d2(fv[u]), to_d2(xv[u]), d0);
      } else {
#pragma unroll
        for (int u = 0; u < VPT; ++u) {
          const double2 xi = to_d2(xv[u]);
          d0 = cfma_conj(xi, xi, d0);
          d1 = cfma_conj(to_d2(yv[u]), xi, d1);
        }
      }
    }
    block_sum2(d0, d1);
    if (threadIdx.x == 0) {
      partials[((size_t)s * gridDim.x + blockIdx.x) * 2] = d0;
      partials[((size_t)s * gridDim.x + blockIdx.x) * 2 + 1] = d1;
    }
    if (!need_y) break;
    if (!grid_barrier(bar, gridDim.x)) return;
    prev = cur;
    cur = y;
  }
}

// ---------------------------------------------------------------------------
// Chebyshev series of H applied to a block (MomentsTD::Evolve, src/chebyshev_momentsTD.cpp:4-46):
//   X <- sum_{s < K} coef[s] T_s(H) X
// T_0 = X is copied to a, T_1 = H T_0 goes to b, then T_{s+1} = 2 H T_s - T_{s-1} in place
// over T_{s-1}; X accumulates coef[s] T_s as each T_s is produced (FP64).
// ---------------------------------------------------------------------------
template <int TPR, int VPT>
__global__ void __launch_bounds__(kThreads)
    k_cheb_series(int n, const int *rp, const int *ci, const double2 *hv, double2 *X, double2 *a, double2 *b,
                  const double2 *__restrict__ coef, int K, Barrier *bar, int cache) {
  constexpr int RW = TPR * VPT;
  const int c0 = (threadIdx.x % TPR) * VPT;  // this thread's VPT adjacent columns
  constexpr int gpb = kThreads / TPR;
  const int per = (n + gridDim.x - 1) / gridDim.x;
  const int r0 = min(n, blockIdx.x * per), r1 = min(n, r0 + per);
  if (cache) {
    extern __shared__ __align__(16) unsigned char smc2[];
    cache_rows<double2>(rp, ci, hv, r0, r1, smc2, rp, ci, hv);
    __syncthreads();
  }
  const int rfirst = cache ? r0 : blockIdx.x * gpb, rend = cache ? r1 : n;  // as in k_recur_lr
  const int rstep = cache ? gpb : gridDim.x * gpb;
  const double2 coef0 = coef[0];
  for (int pos = rfirst + threadIdx.x / TPR; pos < rend; pos += rstep)
#pragma unroll
    for (int u = 0; u < VPT; ++u) {
      const size_t idx = (size_t)pos * RW + c0 + u;
      const double2 x = X[idx];
      a[idx] = x;
      X[idx] = cmul(coef0, x);
    }
  double2 *prev = nullptr, *cur = a;
  for (int s = 1; s < K; ++s) {
    if (!grid_barrier(bar, gridDim.x)) return;
    double2 *y = prev ? prev : b;
    const double2 cs = coef[s];
    for (int pos = rfirst + threadIdx.x / TPR; pos < rend; pos += rstep) {
      double2 acc[VPT];
#pragma unroll
      for (int u = 0; u < VPT; ++u) acc[u] = make_double2(0, 0);
      const int kb = rp[pos], ke = rp[pos + 1];
#pragma unroll 4
      for (int k = kb; k < ke; ++k) gather_fma<double2, VPT>(hv[k], cur + (size_t)ci[k] * RW + c0, acc);
#pragma unroll
      for (int u = 0; u < VPT; ++u) {
        const size_t idx = (size_t)pos * RW + c0 + u;
        double2 yn = acc[u];
        if (prev) {
          const double2 p = ldv(prev + idx);
          yn.x = 2 * yn.x - p.x;
          yn.y = 2 * yn.y - p.y;
        }
        y[idx] = yn;
        X[idx] = cadd(X[idx], cmul(cs, yn));  // X rows are this thread's own: no barrier needed
      }
    }
    prev = cur;
    cur = y;
  }
}

// dots[2s + i] = sum_b partials[s][b][i]  (fixed order)
__global__ void k_reduce_step_partials(const double2 *__restrict__ partials, int steps, int nb,
                                       double2 *__restrict__ dots) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * steps; t += gridDim.x * blockDim.x) {
    const int s = t >> 1, i = t & 1;
    double2 acc = make_double2(0, 0);
    for (int b = 0; b < nb; ++b) acc = cadd(acc, partials[((size_t)s * nb + b) * 2 + i]);
    dots[t] = acc;
  }
}

// Stacked realisations: dots[(r*steps + s)*2 + i] = sum over the CTAs b of group r
// (b in [r*g1, (r+1)*g1)) of partials[s][b][i]  (fixed order)
__global__ void k_reduce_step_partials_split(const double2 *__restrict__ partials, int steps, int nb, int g1,
                                             int nreal, double2 *__restrict__ dots) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * steps * nreal; t += gridDim.x * blockDim.x) {
    const int i = t & 1, s = (t >> 1) % steps, r = (t >> 1) / steps;
    double2 acc = make_double2(0, 0);
    for (int b = r * g1; b < (r + 1) * g1; ++b) acc = cadd(acc, partials[((size_t)s * nb + b) * 2 + i]);
    dots[t] = acc;
  }
}

// Largest contiguous row slice (entries of one or two operators) a CTA owns for a given grid.
size_t max_slice_bytes(const DeviceOp &H, const DeviceOp *V, int grid, size_t esz) {
  const int n = H.n;
  const int per = (n + grid - 1) / grid;
  size_t worst = 0;
  for (int b = 0; b < grid; ++b) {
    const int r0 = std::min(n, b * per), r1 = std::min(n, r0 + per);
    size_t bytes = ((size_t)(H.rowptr[r1] - H.rowptr[r0]) * (esz + 4) + (size_t)(r1 - r0 + 1) * 4 + 15) & ~(size_t)15;
    if (V) bytes += ((size_t)(V->rowptr[r1] - V->rowptr[r0]) * (esz + 4) + (size_t)(r1 - r0 + 1) * 4 + 15) & ~(size_t)15;
    worst = std::max(worst, bytes);
  }
  return worst;
}

// Cooperative grid: as many co-resident CTAs as fit (at most one CTA's worth of rows per
// group of TPR threads).  The operator slices are cached in shared memory when they fit.
int coop_setup(Session *s, const void *func, const DeviceOp &H, const DeviceOp *V, int tpr, size_t esz,
               size_t *smem, bool allow_cache) {
  const int n = H.n, sm_count = s->sm_count;
  const long need = ((long)n * tpr + kThreads - 1) / kThreads;
  int per_sm = 0;
  LQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, kThreads, 0));
  if (per_sm <= 0) fail(LINQT_ERR_UNSUPPORTED, "persistent recursion: kernel does not fit on an SM");
  const double share = coop_share_take(s, std::min(1.0, (double)need / ((double)per_sm * sm_count)));
  // a session with an SM share (linqt_session_set_sm_share) keeps its grid to that fraction
  // of the co-resident CTAs, so that grids of sessions whose shares add up to 1 fit together
  const auto cap = [&](int p) { return std::max(1L, (long)(p * (double)sm_count * share)); };
  const int grid0 = (int)std::max(1L, std::min(cap(per_sm), need));
  const size_t limit = 96 * 1024;
  // 96 KB for every launch of these kernels, whichever thread launches them
  raise_smem_limit((const void *)func, limit);
  // Fewer CTAs fit with the cache, and fewer CTAs have larger slices: shrink the grid
  // until the slices of `grid` CTAs fit `grid` co-resident CTAs.
  int grid = grid0;
  for (int it = 0; allow_cache && it < 16; ++it) {
    const size_t bytes = max_slice_bytes(H, V, grid, esz);
    if (bytes > limit) break;
    int p = 0;
    LQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, func, kThreads, bytes));
    if (p <= 0) break;
    const int g = (int)std::max(1L, std::min(cap(p), need));
    if (g >= grid) {
      *smem = bytes;
      return grid;
    }
    grid = g;
  }
  *smem = 0;
  return grid0;
}

}  // namespace

// Co-resident CTAs of kThreads threads for func with smem bytes of dynamic shared memory,
// at most max_blocks.
int coop_grid(Session *s, const void *func, long max_blocks, size_t smem) {
  int per_sm = 0;
  LQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, kThreads, smem));
  if (per_sm <= 0) fail(LINQT_ERR_UNSUPPORTED, "persistent kernel does not fit on an SM");
  const double full = (double)per_sm * s->sm_count;
  const double share = coop_share_take(s, std::min(1.0, (double)max_blocks / full));
  const long cap = std::max(1L, (long)(full * share));
  return (int)std::max(1L, std::min(cap, max_blocks));
}

double coop_share_take(Session *s, double want) {
  if (!s->ledger || s->coop_share >= 1.0 || s->capturing) return s->coop_share;
  coop_share_return(s);  // a share left by a launch that failed before it was handed over
  CoopLedger &L = *s->ledger;
  std::unique_lock<std::mutex> g(L.mu);
  const double floor = std::min(want, L.min_share);
  // a share comes back when its kernel finishes; the wait is bounded in case a stream
  // stopped running callbacks (a device error), and the grid then sizes itself to what is free
  if (!L.cv.wait_for(g, std::chrono::seconds(120), [&] { return L.free >= floor - 1e-9; })) L.waits_expired++;
  // what is given back later is exactly what is taken here; a grid sized from a share near
  // zero (after an expired wait) still has one CTA
  const double share = std::max(0.0, std::min(want, L.free));
  L.free -= share;
  s->held_share = share;
  return std::max(share, 1e-9);
}

void coop_share_return(Session *s) {
  if (!s->ledger || s->held_share <= 0) return;
  std::lock_guard<std::mutex> g(s->ledger->mu);
  s->ledger->free += s->held_share;
  s->held_share = 0;
  s->ledger->cv.notify_all();
}

namespace {
struct ShareToken {
  CoopLedger *ledger;
  double share;
};
void CUDART_CB share_back(void *p) {  // host callback: no CUDA calls here
  ShareToken *t = static_cast<ShareToken *>(p);
  {
    std::lock_guard<std::mutex> g(t->ledger->mu);
    t->ledger->free += t->share;
  }
  t->ledger->cv.notify_all();
  delete t;
}
}  // namespace

void coop_share_hand_back(Session *s) {
  if (!s->ledger || s->held_share <= 0) return;
  ShareToken *t = new ShareToken{s->ledger, s->held_share};
  s->held_share = 0;
  const cudaError_t h = cudaLaunchHostFunc(s->stream, share_back, t);
  if (h != cudaSuccess) {
    share_back(t);
    LQ_CUDA(h);
  }
}

int sm_share_take(Session *s) {
  if (!s->ledger || s->coop_share >= 1.0 || s->capturing) return s->sm_count;
  const double share = coop_share_take(s, 1.0);
  if (share >= s->ledger->capacity - 1e-9) return s->sm_count;  // nothing else holds a share
  return std::max(1, (int)(share * s->sm_count));
}

// Cooperative kernels of all sessions on a device run one after another on one lane
// stream.  A grid barrier needs every CTA of its grid resident; two persistent grids
// that each fill the device, launched from two sessions' streams, could hold half the
// SMs each and wait on each other until the spin limit.  The session stream hands over
// to the lane with an event and waits for the kernel with another, so the order seen
// by the caller's stream is unchanged.
struct CoopLane {
  std::mutex mu;
  cudaStream_t stream = nullptr;
};

void coop_launch(Session *s, const void *f, int grid, void **args, size_t smem) {
  // a graph capture of this session's stream (api.cu, with_graph), or a session whose grids
  // are sized to its SM share: launched on the session's own stream
  if (s->capturing || s->coop_share < 1.0) {
    const cudaError_t e = cudaLaunchCooperativeKernel(f, dim3(grid), dim3(kThreads), args, smem, s->stream);
    if (e != cudaSuccess) {
      coop_share_return(s);
      LQ_CUDA(e);
    }
    coop_share_hand_back(s);  // the ledger's share comes back once the kernel has finished
    return;
  }
  static std::mutex table_mu;
  static std::unordered_map<int, std::unique_ptr<CoopLane>> lanes;
  CoopLane *lane;
  {
    std::lock_guard<std::mutex> g(table_mu);
    auto &p = lanes[s->device];
    if (!p) {
      p.reset(new CoopLane);
      LQ_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    }
    lane = p.get();
  }
  std::lock_guard<std::mutex> g(lane->mu);
  cudaEvent_t in, out;
  LQ_CUDA(cudaEventCreateWithFlags(&in, cudaEventDisableTiming));
  LQ_CUDA(cudaEventCreateWithFlags(&out, cudaEventDisableTiming));
  LQ_CUDA(cudaEventRecord(in, s->stream));
  LQ_CUDA(cudaStreamWaitEvent(lane->stream, in, 0));
  LQ_CUDA(cudaLaunchCooperativeKernel(f, dim3(grid), dim3(kThreads), args, smem, lane->stream));
  LQ_CUDA(cudaEventRecord(out, lane->stream));
  LQ_CUDA(cudaStreamWaitEvent(s->stream, out, 0));
  LQ_CUDA(cudaEventDestroy(in));
  LQ_CUDA(cudaEventDestroy(out));
}

namespace {

template <class T, int TPR, int VPT>
struct LRF {
  static void run(Session *s, const DeviceOp &H, const DeviceOp *V, void *Lst, void *Rst, const void *phi, void *tb,
                  int M, size_t blk, Barrier *bar, int sellC) {
    using C = typename cplx_t<T>::type;
    const double2 *hv = H.d_val64;
    const int *hci = H.d_col, *sperm = nullptr, *soff = nullptr;
    if (sellC > 0) {
      const DeviceOp::Sell &L = const_cast<DeviceOp &>(H).ensure_sell(sellC);
      hv = L.d_val64;
      hci = L.d_col;
      sperm = L.d_perm;
      soff = L.d_off;
    }
    const int *vrp = V ? V->d_rowptr : nullptr, *vci = V ? V->d_col : nullptr;
    const double2 *vv = V ? V->d_val64 : nullptr;
    int n = H.n;
    C *L = (C *)Lst, *Rs = (C *)Rst, *tbuf = (C *)tb;
    const C *ph = (const C *)phi;
    const void *f = V ? (const void *)k_recur_lr<T, TPR, VPT, true> : (const void *)k_recur_lr<T, TPR, VPT, false>;
    size_t smem = 0;
    const int grid = coop_setup(s, f, H, V, TPR, sizeof(double2), &smem, sellC == 0);
    sellC = std::max(sellC, 0);  // -1: CSR without the shared-memory cache
    int cache = smem > 0;
    int sc = sell_height(sellC);
    void *args[] = {&n,    (void *)&H.d_rowptr, (void *)&hci, (void *)&hv, (void *)&vrp, (void *)&vci,
                    (void *)&vv, &L, &Rs, (void *)&ph, &tbuf, &M, &blk, &bar, &cache,
                    (void *)&sperm, (void *)&soff, &sc};
    coop_launch(s, f, grid, args, smem);
  }
};

template <class T, int TPR, int VPT>
struct OneDF {
  static void run(Session *s, const DeviceOp &H, const void *phi, void *x0, void *b1, int steps, int M, int mode,
                  double2 *dots, Barrier *bar, int sellC, const void *stacked, int nreal, bool c64) {
    using C = typename cplx_t<T>::type;
    // complex64 operator values (FP32, accumulated in FP64) or the complex128 ones
    const void *hv = stacked ? stacked : (c64 ? (const void *)const_cast<DeviceOp &>(H).val32() : H.d_val64);
    long vstride = stacked ? H.nnz : 0;
    LQ_REQUIRE(!stacked || (nreal >= 1 && sellC <= 0), "stacked realisations: CSR layout only");
    const int *hci = H.d_col, *sperm = nullptr, *soff = nullptr;
    if (sellC > 0) {
      const DeviceOp::Sell &L = const_cast<DeviceOp &>(H).ensure_sell(sellC, c64);
      hv = c64 ? (const void *)L.d_val32 : (const void *)L.d_val64;
      hci = L.d_col;
      sperm = L.d_perm;
      soff = L.d_off;
    }
    const void *f = c64 ? (stacked ? (const void *)k_recur_1d<T, float2, TPR, VPT, true>
                                   : (const void *)k_recur_1d<T, float2, TPR, VPT, false>)
                        : (stacked ? (const void *)k_recur_1d<T, double2, TPR, VPT, true>
                                   : (const void *)k_recur_1d<T, double2, TPR, VPT, false>);
    size_t smem = 0;
    // the shared-memory operator cache holds one value set: not with stacked realisations
    int grid = coop_setup(s, f, H, nullptr, TPR, c64 ? sizeof(float2) : sizeof(double2), &smem,
                          sellC == 0 && !stacked);
    sellC = std::max(sellC, 0);  // -1: CSR without the shared-memory cache
    if (stacked) grid = std::max(nreal, grid / nreal * nreal);  // equal CTA groups per realisation
    int cache = smem > 0;
    int sc = sell_height(sellC);
    int ldx = TPR * VPT * (stacked ? nreal : 1);
    double2 *partials = (double2 *)s->get("rec1d_part", sizeof(double2) * 2 * (size_t)steps * grid);
    int n = H.n;
    const C *ph = (const C *)phi;
    C *xx = (C *)x0, *bb = (C *)b1;
    void *args[] = {&n,        (void *)&H.d_rowptr, (void *)&hci, (void *)&hv,    (void *)&ph, &xx, &bb, &steps,
                    &M,        &mode,               &partials,    &bar,           &cache,      (void *)&sperm,
                    (void *)&soff, &sc, &vstride, &nreal, &ldx};
    coop_launch(s, f, grid, args, smem);
    if (stacked)
      k_reduce_step_partials_split<<<(2 * steps * nreal + 255) / 256, 256, 0, s->stream>>>(
          partials, steps, grid, grid / nreal, nreal, dots);
    else
      k_reduce_step_partials<<<(2 * steps + 255) / 256, 256, 0, s->stream>>>(partials, steps, grid, dots);
    LQ_LAUNCHED();
  }
};

// Thread shape of a block of R columns: TPR threads per row, VPT = R / TPR columns per
// thread.  Shape 0 has TPR = min(R, 32); shape s halves TPR s times (VPT <= 8), so a warp
// serves 2^s times more rows at once with 2^s times more loads in flight per thread.
template <class T, int TPR, int VPT>
struct SeriesF {
  static void run(Session *s, const DeviceOp &H, void *X, void *a, void *b, const double2 *coef, int K, Barrier *bar) {
    const void *f = (const void *)k_cheb_series<TPR, VPT>;
    size_t smem = 0;
    const int grid = coop_setup(s, f, H, nullptr, TPR, sizeof(double2), &smem, true);
    int cache = smem > 0;
    int n = H.n;
    const double2 *hv = H.d_val64;
    double2 *x = (double2 *)X, *pa = (double2 *)a, *pb = (double2 *)b;
    void *args[] = {&n, (void *)&H.d_rowptr, (void *)&H.d_col, (void *)&hv, &x, &pa, &pb, (void *)&coef, &K, &bar,
                    &cache};
    coop_launch(s, f, grid, args, smem);
  }
};

template <class T, template <class, int, int> class F, class... Args>
void dispatch(int R, int shape, Args &&...args) {
#define LQ_SHAPE(r, s, tpr, vpt) \
  case (r) * 8 + (s): return F<T, tpr, vpt>::run(args...);
  switch (R * 8 + shape) {
    LQ_SHAPE(1, 0, 1, 1)
    LQ_SHAPE(2, 0, 2, 1) LQ_SHAPE(2, 1, 1, 2)
    LQ_SHAPE(4, 0, 4, 1) LQ_SHAPE(4, 1, 2, 2) LQ_SHAPE(4, 2, 1, 4)
    LQ_SHAPE(8, 0, 8, 1) LQ_SHAPE(8, 1, 4, 2) LQ_SHAPE(8, 2, 2, 4) LQ_SHAPE(8, 3, 1, 8)
    LQ_SHAPE(16, 0, 16, 1) LQ_SHAPE(16, 1, 8, 2) LQ_SHAPE(16, 2, 4, 4) LQ_SHAPE(16, 3, 2, 8)
    LQ_SHAPE(32, 0, 32, 1) LQ_SHAPE(32, 1, 16, 2) LQ_SHAPE(32, 2, 8, 4) LQ_SHAPE(32, 3, 4, 8)
    LQ_SHAPE(64, 0, 32, 2) LQ_SHAPE(64, 1, 16, 4) LQ_SHAPE(64, 2, 8, 8)
    LQ_SHAPE(128, 0, 32, 4) LQ_SHAPE(128, 1, 16, 8)
    LQ_SHAPE(256, 0, 32, 8)
    default: fail(LINQT_ERR_UNSUPPORTED, "block width must be a power of two <= 256 (thread shape " +
                                             std::to_string(shape) + ")");
  }
#undef LQ_SHAPE
}

}  // namespace

// The barrier's count/generation restart at zero for every launch; its error flag is
// sticky until check_device_errors reads it.
GridBarrier *barrier_for(Session *s) {
  Barrier *bar = (Barrier *)s->get("rec_barrier", sizeof(Barrier));
  LQ_CUDA(cudaMemsetAsync(bar, 0, kBarrierResetBytes, s->stream));
  if (s->barrier_cfg_dirty || (s->barrier_cfg_ptr != bar && (s->inject_extra || s->inject_limit))) {
    LQ_CUDA(cudaMemcpyAsync(&bar->extra, &s->inject_extra, sizeof(int), cudaMemcpyHostToDevice, s->stream));
    LQ_CUDA(cudaMemcpyAsync(&bar->spin_limit, &s->inject_limit, sizeof(long long), cudaMemcpyHostToDevice,
                            s->stream));
    LQ_CUDA(cudaStreamSynchronize(s->stream));  // the host fields may change after this call
    s->barrier_cfg_dirty = false;
  }
  s->barrier_cfg_ptr = bar;
  s->barrier_used = true;
  return bar;
}

int recur_shapes(int R) {
  switch (R) {
    case 1: return 1;
    case 2: return 2;
    case 4: return 3;
    case 8: case 16: case 32: return 4;
    case 64: return 3;
    case 128: return 2;
    default: return 1;
  }
}

void recur_lr(Session *s, const DeviceOp &H, const DeviceOp *V, void *Lstore, void *Rstore, const void *phi,
              void *tbuf, int M, int R, bool fp32, int sellC, int shape) {
  const size_t blk = (size_t)H.n * R;
  Barrier *bar = barrier_for(s);
  if (fp32)
    dispatch<float, LRF>(R, shape, s, H, V, Lstore, Rstore, phi, tbuf, M, blk, bar, sellC);
  else
    dispatch<double, LRF>(R, shape, s, H, V, Lstore, Rstore, phi, tbuf, M, blk, bar, sellC);
  LQ_LAUNCHED();
}

void recur_1d(Session *s, const DeviceOp &H, const void *phi, void *x0, void *b1, int steps, int M, int mode, int R,
              bool fp32, double2 *dots, int sellC, int shape, const void *stacked, int nreal, bool c64) {
  Barrier *bar = barrier_for(s);
  const int Rw = stacked ? R / nreal : R;  // columns per CTA
  if (fp32)
    dispatch<float, OneDF>(Rw, shape, s, H, phi, x0, b1, steps, M, mode, dots, bar, sellC, stacked, nreal, c64);
  else
    dispatch<double, OneDF>(Rw, shape, s, H, phi, x0, b1, steps, M, mode, dots, bar, sellC, stacked, nreal, c64);
}

void cheb_series(Session *s, const DeviceOp &H, void *X, void *a, void *b, const double2 *coef, int K, int R) {
  LQ_REQUIRE(K >= 1, "Chebyshev series: at least one term");
  Barrier *bar = barrier_for(s);
  dispatch<double, SeriesF>(R, 0, s, H, X, a, b, coef, K, bar);
  LQ_LAUNCHED();
}

void check_device_errors(Session *s) {
  if (!s->barrier_used) return;
  s->barrier_used = false;
  int err = 0;
  auto it = s->ws.find("rec_barrier");
  if (it != s->ws.end()) {
    Barrier *bar = (Barrier *)it->second.first;
    LQ_CUDA(cudaMemcpyAsync(&err, &bar->err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    LQ_CUDA(cudaStreamSynchronize(s->stream));
    if (err) LQ_CUDA(cudaMemsetAsync(&bar->err, 0, sizeof(int), s->stream));
  }
  if (err) fail(LINQT_ERR_TIMEOUT, "persistent recursion: a grid barrier wait expired; results of the solve are invalid");
  if (mu_tc_check_error(s))
    fail(LINQT_ERR_TIMEOUT, "tensor-core contraction: a pipeline wait expired; results of the solve are invalid");
}

}  // namespace linqt
