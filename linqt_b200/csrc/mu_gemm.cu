// Moment contraction  mu_raw(m0, m1) += sum_k conj(L[m0][k]) * Rv[m1][k].
//
// This is ComputeMomTable (src/chebyshev_solver.cpp:26-42: an M x M table of
// zdotc over the site index) written as the GEMM it is (the unused
// linalg::batch_vdot, src/mkl_linear_algebra.cpp:68-78, is the same product).
// Both operands are "K-major": moment m's block T_m is N*R contiguous complex
// numbers, so K = N*R and the contraction also sums over the R random vectors.
//
// FP64 path: FP64 tensor-core MMA (mma.sync m8n8k4 f64; there is no FP64 tcgen05 kind)
// on 64x64 complex output tiles per CTA (8 warps of 32x16), cp.async double-buffered
// 16-deep K slices in padded shared memory (conflict-free fragment loads), split-K over
// the long K axis with a fixed-order FP64 reduction (deterministic).
#include "internal.cuh"

namespace linqt {

namespace {

// LDS: smem row pitch in elements.  Fragment loads read rows fr = lane/4 (two per 8-lane
// phase) at k = lane%4; a pitch of 4 mod 8 puts those 8 accesses on distinct 16-byte bank
// groups, and the tile stores walk k fastest, which is conflict-free for any pitch.
constexpr int BM = 64, BN = 64, BK = 16, LDS = BK + 4;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}

// Load a BM x BK tile of rows [row0, row0+BM) and k in [k0, k0+BK) of a K-major matrix of
// complex values (double2, or float2 for FP32 Chebyshev blocks).
template <class Tc>
__device__ __forceinline__ void load_tile(Tc (*sm)[LDS], const Tc *__restrict__ g, int M, long K, int row0, long k0,
                                          long kend) {
  // 256 threads x 4 elements: element e = t + 256 q is row e / BK, k slot e % BK
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int e = threadIdx.x + 256 * q;
    const int r = e / BK, kk = e % BK;
    const int row = row0 + r;
    const long k = k0 + kk;
    const bool ok = row < M && k < kend;
    const Tc *src = ok ? g + (size_t)row * K + k : g;
    if constexpr (sizeof(Tc) == 16)
      cp_async16(&sm[r][kk], src, ok);
    else
      cp_async8(&sm[r][kk], src, ok);
  }
}

// D += A * B on an 8x8x4 FP64 tensor-core tile (mma.sync m8n8k4 f64).  Fragments:
// a = A[lane/4][lane%4], b = B[k = lane%4][n = lane/4], d = {D[lane/4][2(lane%4)], D[lane/4][2(lane%4)+1]}.
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// 64x64 complex output tile per CTA, 8 warps as 2 (rows) x 4 (cols), 32x16 complex per warp
// = 4 x 2 tiles of 8x8.  With a = conj(A) = ar + i ai (ai = -Im A) and b = br + i bi, three
// real DMMAs per tile (Gauss): t1 = ar br, t2 = ai bi, t3 = (ar + ai)(br + bi), and
// conj(A) B = (t1 - t2) + i (t3 - t1 - t2) in the epilogue -- 3/4 of the tensor-core work of
// the four-product form, at the cost of one rounding-level cancellation in the imaginary part.
template <class Tc>
__global__ void __launch_bounds__(256, 2) k_zgemm_cn_f64(const Tc *__restrict__ L, const Tc *__restrict__ Rv, int MA,
                                                         int MB, long K, long kchunk, double2 *__restrict__ part) {
  extern __shared__ double2 smem_d[];
  Tc *smem = reinterpret_cast<Tc *>(smem_d);
  Tc(*As)[BM][LDS] = reinterpret_cast<Tc(*)[BM][LDS]>(smem);
  Tc(*Bs)[BN][LDS] = reinterpret_cast<Tc(*)[BN][LDS]>(smem + 2 * BM * LDS);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp >> 2, wn = warp & 3;
  const int fr = lane >> 2, fk = lane & 3;
  const int m0 = blockIdx.y * BM, m1 = blockIdx.x * BN;
  const long kbeg = (long)blockIdx.z * kchunk;
  const long kend = min(K, kbeg + kchunk);
  double t1[4][2][2], t2[4][2][2], t3[4][2][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) t1[i][j][h] = t2[i][j][h] = t3[i][j][h] = 0.0;
  if (kbeg < kend) {
    const int nk = (int)((kend - kbeg + BK - 1) / BK);
    load_tile(As[0], L, MA, K, m0, kbeg, kend);
    load_tile(Bs[0], Rv, MB, K, m1, kbeg, kend);
    cp_async_commit();
    for (int it = 0; it < nk; ++it) {
      const int cur = it & 1;
      if (it + 1 < nk) {
        load_tile(As[cur ^ 1], L, MA, K, m0, kbeg + (long)(it + 1) * BK, kend);
        load_tile(Bs[cur ^ 1], Rv, MB, K, m1, kbeg + (long)(it + 1) * BK, kend);
      }
      cp_async_commit();
      cp_async_wait<1>();
      __syncthreads();
#pragma unroll
      for (int ks = 0; ks < BK / 4; ++ks) {
        double ar[4], ai[4], br[2], bi[2];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const double2 a = to_d2(As[cur][wm * 32 + i * 8 + fr][ks * 4 + fk]);
          ar[i] = a.x;
          ai[i] = -a.y;  // conj(A)
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const double2 b = to_d2(Bs[cur][wn * 16 + j * 8 + fr][ks * 4 + fk]);
          br[j] = b.x;
          bi[j] = b.y;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            dmma(t1[i][j][0], t1[i][j][1], ar[i], br[j]);
            dmma(t2[i][j][0], t2[i][j][1], ai[i], bi[j]);
          }
#pragma unroll
        for (int i = 0; i < 4; ++i) ar[i] += ai[i];
#pragma unroll
        for (int j = 0; j < 2; ++j) br[j] += bi[j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j) dmma(t3[i][j][0], t3[i][j][1], ar[i], br[j]);
      }
      __syncthreads();
    }
    cp_async_wait<0>();
  }
  double2 *out = part + (size_t)blockIdx.z * MA * MB;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = m0 + wm * 32 + i * 8 + fr;
    if (r >= MA) continue;
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = m1 + wn * 16 + j * 8 + 2 * fk + h;
        if (c < MB)
          out[(size_t)r * MB + c] = make_double2(t1[i][j][h] - t2[i][j][h], t3[i][j][h] - t1[i][j][h] - t2[i][j][h]);
      }
  }
}

// mu_raw += sum_z part[z]  (fixed order over z)
__global__ void k_reduce_parts(const double2 *__restrict__ part, int S, long MM, double2 *__restrict__ mu_raw) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < MM; t += (long)gridDim.x * blockDim.x) {
    double2 s = mu_raw[t];
    for (int z = 0; z < S; ++z) s = cadd(s, part[(size_t)z * MM + t]);
    mu_raw[t] = s;
  }
}

// Hermitian symmetrisation and scaling of CorrelationExpansionMoments
// (src/chebyshev_solver.cpp:143-162):
//   mu(i,j) = s_ij (raw(i,j) + conj(raw(j,i)))/2 for j >= i, mu(j,i) = conj(mu(i,j)),
//   s_ij = (4/R) (1/2)^{[i=0]} (1/2)^{[j=0]}
__global__ void k_mu_finalize(const double2 *__restrict__ raw, int M, double R, double2 *__restrict__ mu) {
  const long MM = (long)M * M;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < MM; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t / M), j = (int)(t % M);
    if (j < i) continue;
    double scal = 4.0 / R;
    if (i == 0) scal *= 0.5;
    if (j == 0) scal *= 0.5;
    const double2 a = raw[(size_t)i * M + j], b = raw[(size_t)j * M + i];
    const double2 v = make_double2(scal * (a.x + b.x) / 2.0, scal * (a.y - b.y) / 2.0);
    mu[(size_t)i * M + j] = v;
    mu[(size_t)j * M + i] = cconj(v);
  }
}

// 1D moments from per-step dot products (chebyshev::SpectralMoments scaling,
// src/chebyshev_solver.cpp:190-195: (2/R)(1/2)^{[m=0]}).
// mode 1: dots[2m] = <phi|T_m>; mode 2: dots[2s] = <T_s|T_s>, dots[2s+1] = <T_{s+1}|T_s>.
__global__ void k_moments1d(const double2 *__restrict__ dots, int steps, int M, double R, int mode,
                            double2 *__restrict__ mu, long stride) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
    double2 v;
    if (mode == 1) {
      v = dots[2 * m];
    } else {
      const int s = m >> 1;
      if (m & 1)
        v = s == 0 ? dots[1] : csub(cscale(dots[2 * s + 1], 2.0), dots[1]);
      else
        v = s == 0 ? dots[0] : csub(cscale(dots[2 * s], 2.0), dots[0]);
    }
    double scal = 2.0 / R;
    if (m == 0) scal *= 0.5;
    mu[(size_t)m * stride] = cscale(v, scal);
  }
}

template <class Tc>
void zgemm_cn_t(Session *s, const Tc *A, int MA, const Tc *B, int MB, long K, double2 *C, bool accumulate) {
  const int tiles = ((MA + BM - 1) / BM) * ((MB + BN - 1) / BN);
  const long target = (long)s->sm_count * 2 * 2;
  long S = std::max(1L, (target + tiles - 1) / tiles);
  const long min_chunk = 512;
  S = std::max(1L, std::min(std::min(S, 64L), (K + min_chunk - 1) / min_chunk));
  long kchunk = (K + S - 1) / S;
  kchunk = (kchunk + BK - 1) / BK * BK;
  S = (K + kchunk - 1) / kchunk;
  double2 *part = (double2 *)s->get("zgemm_parts", sizeof(double2) * (size_t)S * MA * MB);
  const size_t smem = sizeof(Tc) * 2 * (BM + BN) * LDS;
  raise_smem_limit((const void *)k_zgemm_cn_f64<Tc>, smem);
  dim3 grid((MB + BN - 1) / BN, (MA + BM - 1) / BM, (unsigned)S);
  k_zgemm_cn_f64<Tc><<<grid, 256, smem, s->stream>>>(A, B, MA, MB, K, kchunk, part);
  LQ_LAUNCHED();
  const long MM = (long)MA * MB;
  if (!accumulate) LQ_CUDA(cudaMemsetAsync(C, 0, sizeof(double2) * MM, s->stream));
  const int g2 = (int)std::max(1L, std::min((MM + 255) / 256, (long)s->sm_count * 8));
  k_reduce_parts<<<g2, 256, 0, s->stream>>>(part, (int)S, MM, C);
  LQ_LAUNCHED();
}

}  // namespace

// C(i, j) (+)= sum_k conj(A[i][k]) * B[j][k] for i < MA, j < MB  (FP64 MMA, deterministic split-K)
void zgemm_cn(Session *s, const double2 *A, int MA, const double2 *B, int MB, long K, double2 *C, bool accumulate) {
  zgemm_cn_t<double2>(s, A, MA, B, MB, K, C, accumulate);
}

// dst += sum_z part[z]  (fixed order over z)
void reduce_parts_into(Session *s, const double2 *part, int S, long MM, double2 *dst) {
  const int g2 = (int)std::max(1L, std::min((MM + 255) / 256, (long)s->sm_count * 8));
  k_reduce_parts<<<g2, 256, 0, s->stream>>>(part, S, MM, dst);
  LQ_LAUNCHED();
}

void mu_contract(Session *s, const void *L, const void *Rv, int M, long K, bool fp32_inputs, int precision,
                 double2 *mu_raw) {
  if (!fp32_inputs) {
    zgemm_cn_t<double2>(s, (const double2 *)L, M, (const double2 *)Rv, M, K, mu_raw, true);
  } else if (i8_digits(precision)) {
    mu_contract_i8(s, L, Rv, M, K, i8_digits(precision), mu_raw);  // tcgen05 INT8 digits, exact sums (mu_i8.cu)
  } else if (precision == LINQT_PREC_MIXED_TF32 && mu_tc_supported(K)) {
    mu_contract_tc(s, L, Rv, M, K, mu_raw);  // tcgen05 3xTF32 (mu_tc.cu)
  } else {
    zgemm_cn_t<float2>(s, (const float2 *)L, M, (const float2 *)Rv, M, K, mu_raw, true);  // FP64 MMA on FP32 data
  }
}

void mu_finalize(Session *s, const double2 *mu_raw, int M, int R, double2 *mu) {
  const long MM = (long)M * M;
  const int g = (int)std::max(1L, std::min((MM + 255) / 256, (long)s->sm_count * 8));
  k_mu_finalize<<<g, 256, 0, s->stream>>>(mu_raw, M, (double)R, mu);
  LQ_LAUNCHED();
}

void moments1d_from_dots_stream(cudaStream_t st, const double2 *dots, int steps, int M, int R, int mode,
                                double2 *mu) {
  k_moments1d<<<(M + 255) / 256, 256, 0, st>>>(dots, steps, M, (double)R, mode, mu, 1);
  LQ_LAUNCHED();
}

void moments1d_from_dots(Session *s, const double2 *dots, int steps, int M, int R, int mode, double2 *mu,
                         long stride) {
  k_moments1d<<<(M + 255) / 256, 256, 0, s->stream>>>(dots, steps, M, (double)R, mode, mu, stride);
  LQ_LAUNCHED();
}

}  // namespace linqt
