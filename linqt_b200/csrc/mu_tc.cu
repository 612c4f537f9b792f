// Mixed-precision moment contraction on the 5th-generation tensor cores (tcgen05).
//
//   mu_raw(m0, m1) += sum_k conj(L[m0][k]) * Rv[m1][k]
// with L and Rv in FP32 (K complex = 2K floats per row, interleaved re/im).
//
// Real form.  With a[k'] the interleaved floats of L[m0] and b[k'] those of Rv[m1]:
//   Re mu = sum_k' a[k'] b[k']                      (Ar Br + Ai Bi)
//   Im mu = sum_k' a[k'] b''[k'],  b'' = (Bi, -Br)  (Ar Bi - Ai Br)
// so one GEMM with N = 2 * 128 computes both halves of a 128 x 128 complex tile.  B'' is
// built in shared memory from the loaded B tile.  Each operand is split into
// TF32 hi + lo parts (hi = value with the low 13 mantissa bits cleared, lo = value - hi,
// exact in FP32).  Three MMAs hi*hi + hi*lo + lo*hi keep about FP32 accuracy
// ("3xTF32").  Accumulation is FP32 in TMEM over one K chunk per CTA; chunks are
// summed in FP64 by the fixed-order split-K reduction of mu_gemm.cu.
//
// CTA roles (192 threads):
//   warp 0     TMA producer: 128 x 32-float tiles of L and Rv, 128-byte swizzle
//   warp 1     TMEM owner and MMA issuer (one elected thread, tcgen05.mma kind::tf32,
//              M = 128, N = 256, K = 8 per instruction)
//   warps 2-5  operand splitting (hi/lo, B''), then the epilogue
//              (tcgen05.ld 32x32b -> FP64 partial tile in global memory)
// Two pipeline stages of 96 KB (A hi/lo, B = [B'; B''] hi/lo).  Every mbarrier wait is
// bounded.  On expiry the kernel raises the error flag, stops issuing work, waits for its
// own copies and MMAs, frees TMEM and returns.
// Every TMA load fills the shared memory of the CTA that issues it.
#include <cuda.h>

#include <cstdint>

#include "internal.cuh"
#include "tc_common.cuh"

namespace linqt {

namespace {

using namespace tc;

constexpr int TC_BM = 128;           // output rows (m0) per CTA
constexpr int TC_BN = 128;           // output columns (m1) per CTA; MMA N = 2 * TC_BN
constexpr int TC_BK = 32;            // floats per K block (128 bytes: one swizzle row)
constexpr int TC_STAGES = 2;
constexpr int TILE = 128 * TC_BK * 4;  // 16 KB: 128 rows x 128 B
// stage layout: A_hi | A_lo | B'_hi | B''_hi | B'_lo | B''_lo
constexpr int OFF_AHI = 0, OFF_ALO = TILE, OFF_BHI = 2 * TILE, OFF_BLO = 4 * TILE;
constexpr int STAGE_BYTES = 6 * TILE;
constexpr int TMEM_COLS = 256;

struct TcShared {
  alignas(1024) uint8_t stage[TC_STAGES][STAGE_BYTES];
  alignas(8) unsigned long long full[TC_STAGES], ready[TC_STAGES], empty[TC_STAGES], acc_full;
  uint32_t tmem_base;
  int abort;
};

// instruction descriptor: D F32, A/B TF32, both K-major, N = 256, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(2 * TC_BN >> 3) << 17) |
                            ((uint32_t)(TC_BM >> 4) << 24);

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

__global__ void __launch_bounds__(192, 1)
    k_mu_tf32x3(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M0, int M1,
                long koff, long kf, long kchunk, double2 *__restrict__ part, int *err) {
  extern __shared__ uint8_t smem_raw[];
  TcShared &sm = *reinterpret_cast<TcShared *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * TC_BM, m1 = blockIdx.x * TC_BN;
  const long kbeg = koff + (long)blockIdx.z * kchunk;
  const long kend = min(kf, kbeg + kchunk);
  const int nkb = kbeg < kend ? (int)((kend - kbeg + TC_BK - 1) / TC_BK) : 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < TC_STAGES; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.ready[s], 4);
      mbar_init(&sm.empty[s], 1);
    }
    mbar_init(&sm.acc_full, 1);
    sm.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&sm.tmem_base)),
                 "r"(TMEM_COLS));
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
        const int s = kb % TC_STAGES;
        const uint32_t ph = (kb / TC_STAGES) & 1;
        if (kb >= TC_STAGES && !mbar_wait(&sm.empty[s], ph ^ 1, err)) {
          sm.abort = 1;
          break;
        }
        mbar_arrive_expect_tx(&sm.full[s], 2 * TILE);
        const int x = (int)(kbeg + (long)kb * TC_BK);
        tma_load_2d(sm.stage[s] + OFF_AHI, &tmA, x, m0, &sm.full[s]);
        tma_load_2d(sm.stage[s] + OFF_BHI, &tmB, x, m1, &sm.full[s]);
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      for (int kb = 0; kb < nkb && !*(volatile int *)&sm.abort; ++kb) {
        const int s = kb % TC_STAGES;
        const uint32_t ph = (kb / TC_STAGES) & 1;
        if (!mbar_wait(&sm.ready[s], ph, err)) {
          sm.abort = 1;
          break;
        }
        tc_fence_after();
        const uint8_t *st = sm.stage[s];
#pragma unroll
        for (int g = 0; g < 3; ++g) {  // hi*hi, hi*lo, lo*hi
          const uint8_t *a = st + (g == 2 ? OFF_ALO : OFF_AHI);
          const uint8_t *b = st + (g == 1 ? OFF_BLO : OFF_BHI);
#pragma unroll
          for (int kk = 0; kk < TC_BK / 8; ++kk)
            umma_tf32(tmem, smem_desc_sw128(a + kk * 32), smem_desc_sw128(b + kk * 32), (kb | g | kk) != 0);
        }
        umma_commit(&sm.empty[s]);  // the stage may be reloaded once these MMAs have read it
      }
      umma_commit(&sm.acc_full);  // accumulator complete (also signals after an abort)
    }
  } else {
    // ---------------- operand splitting (warps 2-5, 128 threads)
    const int t = threadIdx.x - 64;
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % TC_STAGES;
      const uint32_t ph = (kb / TC_STAGES) & 1;
      if (*(volatile int *)&sm.abort || !mbar_wait(&sm.full[s], ph, err)) {
        sm.abort = 1;
        break;
      }
      uint8_t *st = sm.stage[s];
      float4 *ahi = reinterpret_cast<float4 *>(st + OFF_AHI), *alo = reinterpret_cast<float4 *>(st + OFF_ALO);
      float4 *b1h = reinterpret_cast<float4 *>(st + OFF_BHI), *b2h = reinterpret_cast<float4 *>(st + OFF_BHI + TILE);
      float4 *b1l = reinterpret_cast<float4 *>(st + OFF_BLO), *b2l = reinterpret_cast<float4 *>(st + OFF_BLO + TILE);
      // a 16-byte chunk holds two complex numbers (re0, im0, re1, im1); the swizzle permutes whole
      // chunks, so elementwise work keeps every value at its swizzled position
      for (int i = t; i < TILE / 16; i += 128) {
        const float4 a = ahi[i];
        const float4 ah = make_float4(tf32_hi(a.x), tf32_hi(a.y), tf32_hi(a.z), tf32_hi(a.w));
        ahi[i] = ah;
        alo[i] = make_float4(a.x - ah.x, a.y - ah.y, a.z - ah.z, a.w - ah.w);
        const float4 b = b1h[i];
        const float4 bh = make_float4(tf32_hi(b.x), tf32_hi(b.y), tf32_hi(b.z), tf32_hi(b.w));
        const float4 bl = make_float4(b.x - bh.x, b.y - bh.y, b.z - bh.z, b.w - bh.w);
        b1h[i] = bh;
        b1l[i] = bl;
        b2h[i] = make_float4(bh.y, -bh.x, bh.w, -bh.z);  // (Bi, -Br)
        b2l[i] = make_float4(bl.y, -bl.x, bl.w, -bl.z);
      }
      fence_proxy_async();  // generic-proxy writes -> visible to the tensor cores
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.ready[s]);
    }
    // ---------------- epilogue: TMEM -> FP64 partial tile
    const bool ok = mbar_wait(&sm.acc_full, 0, err);
    tc_fence_after();
    const bool aborted = *(volatile int *)&sm.abort;
    if (ok && !aborted && nkb > 0) {
      const int q = warp & 3;          // TMEM lane quarter this warp may access
      const int row = 32 * q + lane;   // accumulator row = TMEM lane
      const int r = m0 + row;
      double2 *out = part + (size_t)blockIdx.z * M0 * M1 + (size_t)r * M1;
#pragma unroll 1
      for (int cb = 0; cb < TC_BN; cb += 16) {
        float re[16], im[16];
        tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + cb, re);
        tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + TC_BN + cb, im);
        if (r < M0) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int c = m1 + cb + j;
            if (c < M1) out[c] = make_double2((double)re[j], (double)im[j]);
          }
        }
      }
    } else if (nkb == 0 && !aborted) {
      const int q = warp & 3, row = 32 * q + lane, r = m0 + row;
      if (r < M0)
        for (int c = m1; c < min(M1, m1 + TC_BN); ++c)
          part[(size_t)blockIdx.z * M0 * M1 + (size_t)r * M1 + c] = make_double2(0, 0);
    }
  }
  tc_fence_before();
  __syncthreads();
  // after an abort, drain what this CTA issued before giving TMEM back
  if (*(volatile int *)&sm.abort && threadIdx.x == 0) {
    for (int s = 0; s < TC_STAGES; ++s) {
      (void)mbar_wait(&sm.full[s], 0, err);
    }
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// rows x kf floats, row-major (kf contiguous); box 32 floats x 128 rows, 128-byte swizzle
CUtensorMap make_map(const void *base, int rows, long kf) {
  CUtensorMap m;
  const cuuint64_t dims[2] = {(cuuint64_t)kf, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)kf * 4};
  const cuuint32_t box[2] = {(cuuint32_t)TC_BK, 128};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base), dims, strides, box,
                                 estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(LINQT_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return m;
}

}  // namespace

bool mu_tc_supported(long K) {
  // TMA: row stride 2K*4 bytes must be a multiple of 16, and the base 16-byte aligned
  return (K % 2) == 0;
}

// mu_raw[M x M] += sum_k conj(L[m0][k]) Rv[m1][k] for FP32 complex L, Rv (K complex per row)
void mu_contract_tc(Session *s, const void *L, const void *Rv, int M, long K, double2 *mu_raw) {
  LQ_REQUIRE(mu_tc_supported(K), "tensor-core contraction needs an even K");
  LQ_REQUIRE(((uintptr_t)L % 16) == 0 && ((uintptr_t)Rv % 16) == 0, "tensor-core operands must be 16-byte aligned");
  const long kf = 2 * K;
  const CUtensorMap ta = make_map(L, M, kf), tb = make_map(Rv, M, kf);
  const int tiles = ((M + TC_BM - 1) / TC_BM) * ((M + TC_BN - 1) / TC_BN);
  // FP32 accumulation in TMEM runs over at most kMaxChunk floats per CTA (measured: the
  // relative error of a chunk grows about linearly with its length, ~2e-9 per float); K is
  // covered in passes of at most kMaxSplit chunks, each reduced into mu_raw in FP64.
  const long kMaxChunk = 2048, kMaxSplit = 64;
  long S = std::max((long)(2 * s->sm_count + tiles - 1) / tiles, (kf + kMaxChunk - 1) / kMaxChunk);
  S = std::max(1L, std::min(S, kMaxSplit));
  long kchunk = std::min(kMaxChunk, (kf + S - 1) / S);
  kchunk = std::max((long)TC_BK, (kchunk + TC_BK - 1) / TC_BK * TC_BK);
  double2 *part = (double2 *)s->get("mu_tc_parts", sizeof(double2) * (size_t)S * M * M);
  int *err = (int *)s->get("mu_tc_err_barrier", sizeof(int) * 4);
  s->barrier_used = true;
  const size_t smem = sizeof(TcShared) + 1024;
  raise_smem_limit((const void *)k_mu_tf32x3, smem);
  for (long koff = 0; koff < kf; koff += S * kchunk) {
    const int Sp = (int)std::min(S, (kf - koff + kchunk - 1) / kchunk);
    dim3 grid((M + TC_BN - 1) / TC_BN, (M + TC_BM - 1) / TC_BM, (unsigned)Sp);
    k_mu_tf32x3<<<grid, 192, smem, s->stream>>>(ta, tb, M, M, koff, kf, kchunk, part, err);
    LQ_LAUNCHED();
    reduce_parts_into(s, part, Sp, (long)M * M, mu_raw);
  }
}

int mu_tc_check_error(Session *s) {
  auto it = s->ws.find("mu_tc_err_barrier");
  if (it == s->ws.end()) return 0;
  int h = 0;
  LQ_CUDA(cudaMemcpyAsync(&h, it->second.first, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  LQ_CUDA(cudaStreamSynchronize(s->stream));
  if (h) LQ_CUDA(cudaMemsetAsync(it->second.first, 0, sizeof(int), s->stream));
  return h;
}

}  // namespace linqt
