// Mixed-precision moment contraction with exact integer accumulation on the tcgen05
// tensor cores (kind::i8).
//
//   mu_raw(m0, m1) += sum_k conj(L[m0][k]) * Rv[m1][k]      (FP32 Chebyshev blocks)
//
// The 3xTF32 kernel (mu_tc.cu) accumulates in FP32 TMEM, whose additions truncate: the
// error of a K chunk grows linearly with its length (4e-5 of max|mu| at 2048 floats per
// chunk), and the Bastin sums over mu carry it into sigma.  Here every value is written as
// ND signed 7-bit digits under an exponent shared by its row and K chunk,
//
//   x = 2^(e - 6) (d_0 + d_1 2^-7 + ... + d_{ND-1} 2^-7(ND-1)),   |d_i| <= 64,
//
// exact for |x| < 2^e up to half a unit of the last digit (2^-(6 + 7(ND-1)) of 2^e).
// Products of digits are exact integers and INT32 accumulation is exact, so the only
// rounding is the digit truncation of each operand and the FP64 sums across K chunks.  The
// digit products d_i e_j with i + j < ND are kept in ND INT32 accumulators by weight
// w = i + j (ND = 3: 6 products, ND = 4: 10), and the epilogue forms
// 2^(ea + eb - 12) sum_w W_w 2^-7w in FP64.  A weight sums at most ND products of at most
// 64^2 per K element, which bounds the exact chunk length (MAX_CHUNK).
//
// ND = 4 keeps 27 bits of each row chunk's range, more than FP32 gives elements within a
// factor 8 of the chunk maximum; ND = 3 (21 bits) is cheaper and less accurate.
//
// Real form as in mu_tc.cu: with a, b the interleaved (re, im) floats of a row,
// Re mu = sum a b and Im mu = sum a b'' with b'' = (Bi, -Br); the digit planes of b'' are
// written beside those of b by the digit kernel, so the MMA's N = 128 rows of B are
// 64 rows of b followed by the same 64 rows of b''.
//
// CTA (192 threads): warp 0 issues the TMA loads (ND A digit tiles of 128 rows, ND + ND
// B tiles of 64 rows, BK bytes of K each), warp 1 owns TMEM and issues the MMAs
// (M = 128, N = 128, K = 32), warps 2-5 run the epilogue.  ND = 3: 128-byte K blocks
// (128-byte swizzle), 2 stages of 96 KB; ND = 4: 64-byte K blocks (64-byte swizzle),
// 3 stages of 64 KB.  Every mbarrier wait is bounded; on expiry the kernel raises the error
// flag, stops issuing, drains what it issued, frees TMEM and returns.  Every TMA load is issued by and for one CTA.
#include <cuda.h>

#include <cooperative_groups.h>

#include <cstdint>

#include "internal.cuh"
#include "tc_common.cuh"

namespace linqt {

namespace {

using namespace tc;
namespace cg = cooperative_groups;

constexpr int I8_BM = 128;         // A rows (m0) per CTA
constexpr int I8_BN = 64;          // complex output columns (m1) per CTA
constexpr int I8_ACC = 2 * I8_BN;  // TMEM columns per accumulator (N = 128: b and b'' rows)
constexpr int I8_TMEM_COLS = 512;
constexpr int I8_KPAD = 128;       // K of the digit planes is padded to a multiple of this

template <int ND>
struct I8Cfg {
  static constexpr int BK = ND == 3 ? 128 : 64;  // K bytes per block (one swizzle row)
  static constexpr int STAGES = ND == 3 ? 2 : 3;
  static constexpr int A_TILE = I8_BM * BK;
  static constexpr int B_HALF = I8_BN * BK;
  static constexpr int B_TILE = 2 * B_HALF;
  static constexpr int STAGE = ND * (A_TILE + B_TILE);
  static constexpr int NPROD = ND == 3 ? 6 : 10;
  // a weight sums at most ND products of at most 64^2 per K element
  static constexpr long MAX_CHUNK = ND == 3 ? 131072 : 65536;
};

template <int ND>
struct I8Shared {
  alignas(1024) uint8_t stage[I8Cfg<ND>::STAGES][I8Cfg<ND>::STAGE];
  alignas(8) unsigned long long full[I8Cfg<ND>::STAGES], empty[I8Cfg<ND>::STAGES], acc_full;
  uint32_t tmem_base;
  int abort;
};

// instruction descriptor: D S32, A and B signed 8-bit, both K-major, N = 128, M = 128
constexpr uint32_t kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(2 * I8_BN >> 3) << 17) |
                              ((uint32_t)(I8_BM >> 4) << 24);

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdescI8), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

template <int ND>
__device__ __forceinline__ uint64_t tile_desc(const void *p) {
  return ND == 3 ? smem_desc_sw128(p) : smem_desc_sw64(p);
}

template <int ND>
__global__ void __launch_bounds__(192, 1)
    k_mu_i8(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M0, int M1,
            long koff, long kfp, long kchunk, const int *__restrict__ expA, const int *__restrict__ expB, int nchunk,
            double2 *__restrict__ part, int *err) {
  using Cfg = I8Cfg<ND>;
  extern __shared__ uint8_t smem_raw[];
  I8Shared<ND> &sm =
      *reinterpret_cast<I8Shared<ND> *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * I8_BM, m1 = blockIdx.x * I8_BN;
  const long kbeg = koff + (long)blockIdx.z * kchunk;
  const long kend = min(kfp, kbeg + kchunk);
  const int nkb = kbeg < kend ? (int)((kend - kbeg) / Cfg::BK) : 0;  // kfp and kchunk are multiples of BK
  const int chunk = (int)(kbeg / kchunk);

  if (threadIdx.x == 0) {
    for (int s = 0; s < Cfg::STAGES; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
    }
    mbar_init(&sm.acc_full, 1);
    sm.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&sm.tmem_base)),
                 "r"(I8_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;

  if (warp == 0) {
    // ---------------- TMA producer
    if (lane == 0) {
      for (int kb = 0; kb < nkb && !*(volatile int *)&sm.abort; ++kb) {
        const int s = kb % Cfg::STAGES;
        const uint32_t ph = (kb / Cfg::STAGES) & 1;
        if (kb >= Cfg::STAGES && !mbar_wait(&sm.empty[s], ph ^ 1, err)) {
          sm.abort = 1;
          break;
        }
        mbar_arrive_expect_tx(&sm.full[s], Cfg::STAGE);
        // planes are stored per K chunk and this CTA's range starts on a chunk boundary
        // (koff is a multiple of kchunk), so x counts from the start of the chunk
        const int x = kb * Cfg::BK;
        const int za = chunk * ND, zb = chunk * 2 * ND;
        uint8_t *st = sm.stage[s];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
          tma_load_3d(st + d * Cfg::A_TILE, &tmA, x, m0, za + d, &sm.full[s]);
          uint8_t *bt = st + ND * Cfg::A_TILE + d * Cfg::B_TILE;
          tma_load_3d(bt, &tmB, x, m1, zb + d, &sm.full[s]);                     // digit d of b
          tma_load_3d(bt + Cfg::B_HALF, &tmB, x, m1, zb + ND + d, &sm.full[s]);  // digit d of b''
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      // digit products (a digit, b digit): accumulator w = i + j sums those of weight 2^-(12 + 7w);
      // the first product of each weight (i = 0) overwrites its accumulator on the first block
      constexpr int kPairA[10] = {0, 0, 1, 0, 1, 2, 0, 1, 2, 3};
      constexpr int kPairB[10] = {0, 1, 0, 2, 1, 0, 3, 2, 1, 0};
      for (int kb = 0; kb < nkb && !*(volatile int *)&sm.abort; ++kb) {
        const int s = kb % Cfg::STAGES;
        const uint32_t ph = (kb / Cfg::STAGES) & 1;
        if (!mbar_wait(&sm.full[s], ph, err)) {
          sm.abort = 1;
          break;
        }
        tc_fence_after();
        const uint8_t *st = sm.stage[s];
#pragma unroll
        for (int kk = 0; kk < Cfg::BK / 32; ++kk)
#pragma unroll
          for (int q = 0; q < Cfg::NPROD; ++q) {
            const int w = kPairA[q] + kPairB[q];
            const uint8_t *a = st + kPairA[q] * Cfg::A_TILE + kk * 32;
            const uint8_t *b = st + ND * Cfg::A_TILE + kPairB[q] * Cfg::B_TILE + kk * 32;
            const bool first = kb == 0 && kk == 0 && kPairA[q] == 0;
            umma_i8(tmem + w * I8_ACC, tile_desc<ND>(a), tile_desc<ND>(b), first ? 0u : 1u);
          }
        umma_commit(&sm.empty[s]);  // the stage may be reloaded once these MMAs have read it
      }
      umma_commit(&sm.acc_full);  // accumulators complete (also signals after an abort)
    }
  } else {
    // ---------------- epilogue (warps 2-5): TMEM -> FP64 partial tile
    const bool ok = mbar_wait(&sm.acc_full, 0, err);
    tc_fence_after();
    const bool aborted = *(volatile int *)&sm.abort;
    const int q = warp & 3;         // TMEM lane quarter this warp may access
    const int row = 32 * q + lane;  // accumulator row = TMEM lane
    const int r = m0 + row;
    double2 *out = part + (size_t)blockIdx.z * M0 * M1 + (size_t)r * M1;
    if (ok && !aborted && nkb > 0) {
      const int ea = r < M0 ? expA[(size_t)r * nchunk + chunk] : 0;
      const uint32_t lanebase = tmem + ((uint32_t)(32 * q) << 16);
#pragma unroll 1
      for (int cb = 0; cb < I8_BN; cb += 16) {
        double acc[2][16];  // [re, im][column], in units of 2^(ea + eb - 12)
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int j = 0; j < 16; ++j) acc[h][j] = 0;
#pragma unroll
        for (int w = ND - 1; w >= 0; --w) {  // smallest weights first
          uint32_t v[16];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            tmem_ld16_u32(lanebase + w * I8_ACC + h * I8_BN + cb, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[h][j] += ldexp((double)(int)v[j], -7 * w);
          }
        }
        if (r < M0) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int c = m1 + cb + j;
            if (c < M1) {
              const int sc = ea + expB[(size_t)c * nchunk + chunk] - 12;
              out[c] = make_double2(ldexp(acc[0][j], sc), ldexp(acc[1][j], sc));
            }
          }
        }
      }
    } else if (nkb == 0 && !aborted && r < M0) {
      for (int c = m1; c < min(M1, m1 + I8_BN); ++c) out[c] = make_double2(0, 0);
    }
  }
  tc_fence_before();
  __syncthreads();
  // after an abort, drain what this CTA issued before giving TMEM back
  if (*(volatile int *)&sm.abort && threadIdx.x == 0) {
    for (int s = 0; s < Cfg::STAGES; ++s) (void)mbar_wait(&sm.full[s], 0, err);
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(I8_TMEM_COLS));
  }
}

// y in (-64, 64) -> ND digits, y = sum_i d_i 2^-7i + O(2^-7(ND-1) / 2); every step exact in FP32
template <int ND>
__device__ __forceinline__ void digits(float y, int (&d)[ND]) {
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    const float f = rintf(y);
    d[i] = (int)f;
    y = (y - f) * 128.f;
  }
}

__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
  return (uint32_t)(a & 0xff) | ((uint32_t)(b & 0xff) << 8) | ((uint32_t)(c & 0xff) << 16) |
         ((uint32_t)(d & 0xff) << 24);
}

// Digit planes of both sides: z = 0 the L side (ND planes), z = 1 the R side (ND planes of b,
// then ND of b'' = (Bi, -Br)).  src: rows of kf floats, ld floats apart; dig: [nchunk][planes][rows][kchunk]
// int8, chunk-major so that the rows one K chunk's CTAs read at the same time lie kchunk
// bytes apart rather than the whole K apart (K padded with zeros to kfp; the part of the
// last chunk past kfp is never read); expo[row][chunk]: the exponent e with max |x| over
// the chunk < 2^e.  Grid (4 nchunk, rows, 2) in clusters of 4 CTAs: each CTA stages a quarter of a
// (row, chunk) in shared memory (kchunk / 4 floats, up to 64 KB), the cluster exchanges the
// quarter maxima through distributed shared memory, and the digits are written from the
// staged copy, so every value is read from HBM once.
constexpr int kDigitCluster = 4;

template <int ND>
__global__ void __cluster_dims__(kDigitCluster, 1, 1) __launch_bounds__(256)
    k_digits(const float *__restrict__ srcA, const float *__restrict__ srcB, long ld, long kf, long kfp, long kchunk,
             int rows, int nchunk, int8_t *__restrict__ digA, int8_t *__restrict__ digB, int *__restrict__ expA,
             int *__restrict__ expB) {
  extern __shared__ float4 stage_q[];
  __shared__ float red[8];
  __shared__ float qmax;
  cg::cluster_group cl = cg::this_cluster();
  const bool b_side = blockIdx.z == 1;
  const int row = blockIdx.y, c = blockIdx.x / kDigitCluster, quarter = blockIdx.x % kDigitCluster;
  const long q = kchunk / kDigitCluster;  // a multiple of 32 floats
  const long k0 = (long)c * kchunk + quarter * q, k1 = min(kfp, k0 + q), kd = min(k1, kf);
  const float *x = (b_side ? srcB : srcA) + (size_t)row * ld;  // rows ld floats apart, kf of them used
  // stage this quarter (kf is even: a pair (k, k+1) is all in or all out of [k0, kd))
  float mx = 0.f;
  const int nquad = (int)max(0L, (k1 - k0) / 4);
  for (int i = threadIdx.x; i < nquad; i += blockDim.x) {
    const long k = k0 + 4L * i;
    float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
    if (k < kd) {
      const float2 p = *reinterpret_cast<const float2 *>(x + k);
      t.x = p.x;
      t.y = p.y;
      if (k + 2 < kd) {
        const float2 r = *reinterpret_cast<const float2 *>(x + k + 2);
        t.z = r.x;
        t.w = r.y;
      }
    }
    stage_q[i] = t;
    mx = fmaxf(mx, fmaxf(fmaxf(fabsf(t.x), fabsf(t.y)), fmaxf(fabsf(t.z), fabsf(t.w))));
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = 0.f;
    for (int w = 0; w < 8; ++w) m = fmaxf(m, red[w]);
    qmax = m;
  }
  cl.sync();  // every quarter's maximum is written
  mx = 0.f;
#pragma unroll
  for (int r = 0; r < kDigitCluster; ++r) mx = fmaxf(mx, *cl.map_shared_rank(&qmax, r));
  cl.sync();  // no CTA leaves while another may still read its maximum
  int e = 0;
  if (mx > 0.f) (void)frexpf(mx, &e);  // mx = f 2^e, f in [0.5, 1): every |x| < 2^e
  if (threadIdx.x == 0 && quarter == 0) (b_side ? expB : expA)[(size_t)row * nchunk + c] = e;
  const size_t plane = (size_t)rows * kchunk;  // one digit plane of one K chunk
  const int nplanes = b_side ? 2 * ND : ND;
  int8_t *drow = (b_side ? digB : digA) + (size_t)c * nplanes * plane + (size_t)row * kchunk;
  for (int i = threadIdx.x; i < nquad; i += blockDim.x) {
    const long k = k0 + 4L * i - (long)c * kchunk;  // offset inside the chunk
    const float4 t = stage_q[i];
    int d[4][ND];
    digits<ND>(ldexpf(t.x, 6 - e), d[0]);
    digits<ND>(ldexpf(t.y, 6 - e), d[1]);
    digits<ND>(ldexpf(t.z, 6 - e), d[2]);
    digits<ND>(ldexpf(t.w, 6 - e), d[3]);
#pragma unroll
    for (int p = 0; p < ND; ++p) {
      *reinterpret_cast<uint32_t *>(drow + p * plane + k) = pack4(d[0][p], d[1][p], d[2][p], d[3][p]);
      if (b_side)  // b'' = (Bi, -Br): k is a multiple of 4, so (k, k+1) and (k+2, k+3) are (re, im) pairs
        *reinterpret_cast<uint32_t *>(drow + (ND + p) * plane + k) = pack4(d[1][p], -d[0][p], d[3][p], -d[2][p]);
    }
  }
}

// [planes][rows][kchunk] int8 (planes = chunks x digit planes per chunk), box bk bytes x
// box_rows x 1, swizzle of bk bytes; rows past the end of a plane read as zero
CUtensorMap make_map_i8(const void *base, int rows, long kchunk, int planes, int box_rows, int bk) {
  CUtensorMap m;
  const cuuint64_t dims[3] = {(cuuint64_t)kchunk, (cuuint64_t)rows, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)kchunk, (cuuint64_t)kchunk * rows};
  const cuuint32_t box[3] = {(cuuint32_t)bk, (cuuint32_t)box_rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void *>(base), dims, strides, box,
                                 estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 bk == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(LINQT_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return m;
}

// One slab of K: columns [0, K) of rows ld complex apart.
template <int ND>
void contract_i8_slab(Session *s, const void *L, const void *Rv, int M, long K, long ld, double2 *mu_raw) {
  using Cfg = I8Cfg<ND>;
  LQ_REQUIRE(((uintptr_t)L % 16) == 0 && ((uintptr_t)Rv % 16) == 0, "tensor-core operands must be 16-byte aligned");
  const long kf = 2 * K, kfp = (kf + I8_KPAD - 1) / I8_KPAD * I8_KPAD;
  const int tiles = ((M + I8_BM - 1) / I8_BM) * ((M + I8_BN - 1) / I8_BN);
  // K chunks (one exponent per row and chunk, one CTA per tile and chunk): at most
  // MAX_CHUNK floats, at least two CTAs per SM, and among the counts up to twice the least,
  // the one whose last wave of CTAs is fullest
  const long smin = std::max((kfp + Cfg::MAX_CHUNK - 1) / Cfg::MAX_CHUNK,
                             (long)(2 * s->sm_count + tiles - 1) / tiles);
  long best_s = smin;
  double best_fill = 0;
  for (long sc = smin; sc <= 2 * smin; ++sc) {
    const long ctas = (long)tiles * sc, waves = (ctas + s->sm_count - 1) / s->sm_count;
    const double fill = (double)ctas / ((double)waves * s->sm_count);
    if (fill > best_fill + 1e-9) {
      best_fill = fill;
      best_s = sc;
    }
  }
  long kchunk = (kfp + best_s - 1) / best_s;
  kchunk = std::min(Cfg::MAX_CHUNK, std::max((long)I8_KPAD, (kchunk + I8_KPAD - 1) / I8_KPAD * I8_KPAD));
  const int nchunk = (int)((kfp + kchunk - 1) / kchunk);
  const long kMaxSplit = 64;
  const long S = std::min<long>(nchunk, kMaxSplit);
  const long kcp = (long)nchunk * kchunk;  // K of the chunk-major planes (>= kfp)
  int8_t *dA = (int8_t *)s->get("mu_i8_a", (size_t)ND * M * kcp);
  int8_t *dB = (int8_t *)s->get("mu_i8_b", (size_t)2 * ND * M * kcp);
  int *eA = (int *)s->get("mu_i8_ea", sizeof(int) * (size_t)M * nchunk);
  int *eB = (int *)s->get("mu_i8_eb", sizeof(int) * (size_t)M * nchunk);
  double2 *part = (double2 *)s->get("mu_i8_parts", sizeof(double2) * (size_t)S * M * M);
  int *err = (int *)s->get("mu_tc_err_barrier", sizeof(int) * 4);  // read by mu_tc_check_error
  s->barrier_used = true;
  const size_t qsmem = sizeof(float) * (size_t)(kchunk / kDigitCluster);
  raise_smem_limit((const void *)k_digits<ND>, qsmem);
  k_digits<ND><<<dim3(kDigitCluster * nchunk, M, 2), 256, qsmem, s->stream>>>(
      (const float *)L, (const float *)Rv, 2 * ld, kf, kfp, kchunk, M, nchunk, dA, dB, eA, eB);
  LQ_LAUNCHED();
  const CUtensorMap ta = make_map_i8(dA, M, kchunk, ND * nchunk, I8_BM, Cfg::BK),
                    tb = make_map_i8(dB, M, kchunk, 2 * ND * nchunk, I8_BN, Cfg::BK);
  const size_t smem = sizeof(I8Shared<ND>) + 1024;
  raise_smem_limit((const void *)k_mu_i8<ND>, smem);
  for (long koff = 0; koff < kfp; koff += S * kchunk) {
    const int Sp = (int)std::min(S, (kfp - koff + kchunk - 1) / kchunk);
    dim3 grid((M + I8_BN - 1) / I8_BN, (M + I8_BM - 1) / I8_BM, (unsigned)Sp);
    k_mu_i8<ND><<<grid, 192, smem, s->stream>>>(ta, tb, M, M, koff, kfp, kchunk, eA, eB, nchunk, part, err);
    LQ_LAUNCHED();
    reduce_parts_into(s, part, Sp, (long)M * M, mu_raw);
  }
}

// K in slabs (i8_slab): each slab's digit planes overwrite the previous slab's, so the planes
// take at most kI8DigitBudget however long K is; the slabs' sums add into mu_raw in FP64.
template <int ND>
void contract_i8(Session *s, const void *L, const void *Rv, int M, long K, double2 *mu_raw) {
  const long slab = i8_slab(ND, M, K);
  for (long kb = 0; kb < K; kb += slab)
    contract_i8_slab<ND>(s, (const float2 *)L + kb, (const float2 *)Rv + kb, M, std::min(slab, K - kb), K, mu_raw);
}

}  // namespace

// mu_raw[M x M] += sum_k conj(L[m0][k]) Rv[m1][k] for FP32 complex L, Rv (K complex per row),
// with `digits` = 3 or 4 digits per value
void mu_contract_i8(Session *s, const void *L, const void *Rv, int M, long K, int digits, double2 *mu_raw) {
  LQ_REQUIRE(digits == 3 || digits == 4, "INT8 contraction: 3 or 4 digits");
  if (digits == 3)
    contract_i8<3>(s, L, Rv, M, K, mu_raw);
  else
    contract_i8<4>(s, L, Rv, M, K, mu_raw);
}

}  // namespace linqt
