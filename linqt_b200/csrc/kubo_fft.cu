// Kubo_solver_FFT on the device: per-site DFTs of the Chebyshev vectors, the
// Bastin / Greenwood products, the sum over sites and the post-processing.
//
// Reference: src/Bastin_FFTs.cpp:6-173, src/Greenwood_FFTs.cpp:6-91,
// src/Kubo_solver_FFT_postProcess.cpp:8-397, include/Kubo_solver_FFT.hpp:93-107.
//
// For every site l (a (site, vector) pair of the block) and m < M the reference
// forms  pf_m = (2 - [m=0]) g_m exp(i pi m / (2 nump))  (g_m the Jackson factor of
// Kubo_solver_FFT::Jackson_kernel) and runs FFTW backward DFTs (exponent +1,
// unnormalised, zero padded to nump) of
//   pf_m Re(bra_m), pf_m Im(bra_m), pf_m Re(ket_m), pf_m Im(ket_m)
// and (Bastin) of the same four multiplied by m, with bra_m = L_m[l] (= T_m(H) OPL phi)
// and ket_m = R_m[l] (= OPR T_m(H) phi).  Products of the transforms are summed over
// sites into p[k] (and w[k]).
//
// Design: one CTA per site at a time (persistent, the CTAs interleaved over the sites),
// all 8 (or 4) transforms of the site in shared memory.  nump = 16 * 16 * R3,
// R3 in {1, 2, 4, 8}: pass 1 does 16-point DFTs in registers straight from the
// global loads, pass 2 16-point DFTs, pass 3 R3-point DFTs; every pass reads its
// inputs into registers, synchronises, and writes its outputs back in place
// (rows padded by one element to spread shared-memory banks).  The product stage
// then reads all transforms at a fixed set of frequencies per thread and keeps the
// per-frequency sums in registers across the CTA's sites; CTA partials are summed
// in a fixed order (deterministic).  Other nump use a direct DFT kernel.
#include <cmath>

#include "internal.cuh"

namespace linqt {

namespace {

__device__ __forceinline__ double2 mul_i(double2 a) { return make_double2(-a.y, a.x); }

__device__ __forceinline__ void dft2(double2 &a0, double2 &a1) {
  const double2 t = a0;
  a0 = cadd(t, a1);
  a1 = csub(t, a1);
}

// 4-point DFT with exponent +1 (in place)
__device__ __forceinline__ void dft4(double2 &a0, double2 &a1, double2 &a2, double2 &a3) {
  const double2 s02 = cadd(a0, a2), d02 = csub(a0, a2), s13 = cadd(a1, a3), d13 = mul_i(csub(a1, a3));
  a0 = cadd(s02, s13);
  a2 = csub(s02, s13);
  a1 = cadd(d02, d13);
  a3 = csub(d02, d13);
}

// exp(+2 pi i j / 16), j = 0..9
__device__ __forceinline__ double2 w16(int j) {
  constexpr double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173, h = 0.70710678118654752440;
  switch (j) {
    case 0: return make_double2(1.0, 0.0);
    case 1: return make_double2(c1, s1);
    case 2: return make_double2(h, h);
    case 3: return make_double2(s1, c1);
    case 4: return make_double2(0.0, 1.0);
    case 5: return make_double2(-s1, c1);
    case 6: return make_double2(-h, h);
    case 7: return make_double2(-c1, s1);
    case 8: return make_double2(-1.0, 0.0);
    default: return make_double2(-c1, -s1);
  }
}

// 16-point DFT, exponent +1.  On return v[4*q1 + q2] holds X[q1 + 4*q2].
__device__ __forceinline__ void dft16(double2 (&v)[16]) {
#pragma unroll
  for (int r2 = 0; r2 < 4; ++r2) dft4(v[r2], v[4 + r2], v[8 + r2], v[12 + r2]);
  // now v[4*q1 + r2] = Y_{r2}[q1]
#pragma unroll
  for (int q1 = 1; q1 < 4; ++q1)
#pragma unroll
    for (int r2 = 1; r2 < 4; ++r2) v[4 * q1 + r2] = cmul(v[4 * q1 + r2], w16(q1 * r2));
#pragma unroll
  for (int q1 = 0; q1 < 4; ++q1) dft4(v[4 * q1], v[4 * q1 + 1], v[4 * q1 + 2], v[4 * q1 + 3]);
}

// R-point DFT (R in 1, 2, 4, 8), exponent +1, natural output order
template <int R>
__device__ __forceinline__ void dft_small(double2 (&v)[R]) {
  if constexpr (R == 2) {
    dft2(v[0], v[1]);
  } else if constexpr (R == 4) {
    dft4(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    // r = 2 r1 + r2, q = q1 + 4 q2
    dft4(v[0], v[2], v[4], v[6]);  // Y_0[q1] at v[0], v[2], v[4], v[6]
    dft4(v[1], v[3], v[5], v[7]);  // Y_1[q1] at v[1], v[3], v[5], v[7]
    constexpr double h = 0.70710678118654752440;
    v[3] = cmul(v[3], make_double2(h, h));
    v[5] = mul_i(v[5]);
    v[7] = cmul(v[7], make_double2(-h, h));
    double2 o[8];
#pragma unroll
    for (int q1 = 0; q1 < 4; ++q1) {
      double2 a = v[2 * q1], b = v[2 * q1 + 1];
      dft2(a, b);
      o[q1] = a;
      o[q1 + 4] = b;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = o[q];
  }
}

// Sequence s of a site: source (0 bra, 1 ket), part (0 re, 1 im), derivative.
// Bastin order (src/Bastin_FFTs.cpp:40-52): re_bras, im_bras, re_kets, im_kets, re_D_bras,
// im_D_bras, re_D_kets, im_D_kets.  Greenwood uses the first four.
__device__ __forceinline__ double2 seq_input(int s, double2 bra, double2 ket, double2 pf, int m) {
  const double2 src = (s & 2) ? ket : bra;
  const double u = (s & 1) ? src.y : src.x;
  double f = u;
  if (s >= 4) f *= (double)m;
  return make_double2(pf.x * f, pf.y * f);
}

// Bastin products for one frequency (src/Bastin_FFTs.cpp:128-163), accumulated into p, w
__device__ __forceinline__ void bastin_products(int j, int nump, const double2 *X, int stride, double2 &p,
                                                double2 &w) {
  const double2 rb = X[0 * stride], ib = X[1 * stride], rk = X[2 * stride], ik = X[3 * stride];
  const double2 rDb = X[4 * stride], iDb = X[5 * stride], rDk = X[6 * stride], iDk = X[7 * stride];
  // Re(rb) - i Re(ib)
  const double2 ReG_b = make_double2(rb.x, -ib.x);
  // Re(rk) + i Re(ik)
  const double2 ReG_k = make_double2(rk.x, ik.x);
  double2 Gk, Gb, dGb, dGk;
  if (j < nump / 2) {
    Gk = cadd(rk, mul_i(ik));                           // rk + i ik
    Gb = csub(cconj(rb), mul_i(cconj(ib)));             // conj(rb) - i conj(ib)
    dGb = csub(cconj(rDb), mul_i(cconj(iDb)));          // conj(rDb) - i conj(iDb)
    dGk = cadd(rDk, mul_i(iDk));                        // rDk + i iDk
  } else {
    Gk = cadd(cconj(rk), mul_i(cconj(ik)));             // conj(rk) + i conj(ik)
    Gb = csub(rb, mul_i(ib));                           // rb - i ib
    dGb = csub(rDb, mul_i(iDb));                        // rDb - i iDb
    dGk = cadd(cconj(rDk), mul_i(cconj(iDk)));          // conj(rDk) + i conj(iDk)
  }
  p = cadd(p, cadd(cmul(ReG_b, Gk), cmul(Gb, ReG_k)));
  w = cadd(w, csub(cmul(dGb, ReG_k), cmul(ReG_b, dGk)));
}

// Greenwood product (src/Greenwood_FFTs.cpp:252-257): Re[(Re rb - i Re ib)(Re rk + i Re ik)]
__device__ __forceinline__ void greenwood_product(const double2 *X, int stride, double2 &p) {
  const double2 rb = X[0], ib = X[stride], rk = X[2 * stride], ik = X[3 * stride];
  p.x += rb.x * rk.x + ib.x * ik.x;
}

// prefactors pf_m (src/Bastin_FFTs.cpp:20-21, include/Kubo_solver_FFT.hpp:99-107)
__global__ void k_prefactors(int M, int nump, double2 *__restrict__ pf) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
    const double g = 1 / (M + 1.0) *
                     ((M - m + 1.0) * cos(M_PI * m / (M + 1.0)) + sin(M_PI * m / (M + 1.0)) / tan(M_PI / (M + 1.0)));
    const double amp = (2 - (m == 0)) * g;
    double sn, cs;
    sincos(M_PI * m / (2.0 * nump), &sn, &cs);
    pf[m] = make_double2(amp * cs, amp * sn);
  }
}

constexpr int kFftThreads = 512;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }
__device__ __forceinline__ void cp_async_el(double2 *smem, const double2 *g) { cp_async16(smem, g); }
__device__ __forceinline__ void cp_async_el(float2 *smem, const float2 *g) { cp_async8(smem, g); }

// Issue the asynchronous copies of site l's bra_m = L[m][l] and ket_m = Rv[m][l], m < M,
// into stage[0..M) and stage[M..2M).
template <class Tin>
__device__ __forceinline__ void stage_site(Tin *stage, const Tin *__restrict__ L, const Tin *__restrict__ Rv, long K,
                                           int M, long l) {
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    cp_async_el(stage + m, L + (size_t)m * K + l);
    cp_async_el(stage + M + m, Rv + (size_t)m * K + l);
  }
  cp_async_commit();
}

// 16-point DFT of a sequence whose upper half is zero (v[8..15] = 0 on entry), same
// output order as dft16.  The first radix-4 stage reduces to two-point sums.
__device__ __forceinline__ void dft16_half(double2 (&v)[16]) {
#pragma unroll
  for (int r2 = 0; r2 < 4; ++r2) {
    const double2 a0 = v[r2], a1 = v[4 + r2];
    v[r2] = cadd(a0, a1);
    v[8 + r2] = csub(a0, a1);
    v[4 + r2] = cadd(a0, mul_i(a1));
    v[12 + r2] = csub(a0, mul_i(a1));
  }
#pragma unroll
  for (int q1 = 1; q1 < 4; ++q1)
#pragma unroll
    for (int r2 = 1; r2 < 4; ++r2) v[4 * q1 + r2] = cmul(v[4 * q1 + r2], w16(q1 * r2));
#pragma unroll
  for (int q1 = 0; q1 < 4; ++q1) dft4(v[4 * q1], v[4 * q1 + 1], v[4 * q1 + 2], v[4 * q1 + 3]);
}

// Bastin / Greenwood products from the transforms of one frequency held in registers
__device__ __forceinline__ void bastin_products_reg(int k, int n, const double2 (&x)[8], double2 &p, double2 &w) {
  bastin_products(k, n, x, 1, p, w);
}
__device__ __forceinline__ void greenwood_product_reg(const double2 (&x)[4], double2 &p) { greenwood_product(x, 1, p); }

// Shared-memory layout (double2 units):
//   buf   NSEQ * 16 * (P + 1)   the transforms, 16 rows of P (+1 pad) per sequence
//   tw1   16 * P                w_n^{m1 k2} at [k2 * P + m1]   (pass 1)
//   tw2   16 * R3               w_P^{a c}   at [c * R3 + a]    (pass 2)
//   pfs   M                     prefactors
//   stage 2 * 2M                double-buffered bra/ket of the current and next site
//
// Per site: pass 1 (16-point DFTs over m2 from the staged site, twiddles w_n^{m1 k2},
// written to row k2), barrier, pass 2 (16-point DFTs over b within each row, in place:
// an item reads and writes the same 16 slots), barrier, then the last R3-point DFTs and
// the products straight from registers: thread pair (k2, c) computes the R3-point DFT of
// every sequence and keeps the outputs d = h, h + 2, ... (h = the thread's half), so no
// transform is written back.  Bank mapping: consecutive threads take consecutive m1 (pass
// 1) or consecutive rows k2 (pass 2, final) and the row pitch P + 1 is odd, so every
// 8-thread phase of a 16-byte access touches 8 distinct bank groups.
template <int R3, int NSEQ, bool HALF, class Tin>
__global__ void __launch_bounds__(kFftThreads)
    k_kubo_fft(const Tin *__restrict__ L, const Tin *__restrict__ Rv, long K, long chunk, int M,
               const double2 *__restrict__ pf_g, double2 *__restrict__ part) {
  constexpr int P = 16 * R3;     // n / 16
  constexpr int n = 16 * P;      // nump
  constexpr int ROW = P + 1;     // padded row of the 16 x P arrangement
  constexpr int SEQ = 16 * ROW;  // per-sequence footprint
  constexpr int ND = R3 >= 2 ? R3 / 2 : 1;  // final outputs per thread
  extern __shared__ double2 sm[];
  double2 *buf = sm;
  double2 *tw1 = buf + NSEQ * SEQ;
  double2 *tw2 = tw1 + 16 * P;
  double2 *pfs = tw2 + 16 * R3;
  Tin *stage = reinterpret_cast<Tin *>(pfs + M);  // 2 buffers of 2M
  // Sites blockIdx.x, blockIdx.x + gridDim.x, ...: at any time all CTAs work on neighbouring
  // sites, so each row m of the stores is read in one place (one page, L2 lines shared by the
  // CTAs) rather than at gridDim.x places K / gridDim.x sites apart (at K = 4e6 sites the
  // rows are 64 MB long and a contiguous split touched a different page per CTA and row).
  (void)chunk;
  const long lstep = gridDim.x;
  if ((long)blockIdx.x < K) stage_site(stage, L, Rv, K, M, blockIdx.x);
  for (int t = threadIdx.x; t < 16 * P; t += blockDim.x) {
    const int k2 = t / P, m1 = t % P;
    double sn, cs;
    sincospi(2.0 * (double)(m1 * k2) / n, &sn, &cs);
    tw1[t] = make_double2(cs, sn);
  }
  for (int t = threadIdx.x; t < 16 * R3; t += blockDim.x) {
    const int c = t / R3, a = t % R3;
    double sn, cs;
    sincospi(2.0 * (double)(a * c) / P, &sn, &cs);
    tw2[t] = make_double2(cs, sn);
  }
  for (int m = threadIdx.x; m < M; m += blockDim.x) pfs[m] = pf_g[m];
  // final-stage role of this thread: half h of the pair (k2f, cf)
  const int h = threadIdx.x & 1, pair = threadIdx.x >> 1;
  const int k2f = pair % 16, cf = pair / 16;  // pair < 256 for kFftThreads = 512
  const bool fin = (R3 >= 2 || h == 0);
  double2 accp[ND], accw[ND];
#pragma unroll
  for (int j = 0; j < ND; ++j) accp[j] = accw[j] = make_double2(0, 0);

  int cur = 0;
  for (long l = blockIdx.x; l < K; l += lstep) {
    cp_async_wait_all();
    __syncthreads();  // stage[cur] complete and visible; the previous site is fully consumed
    const Tin *bra = stage + cur * 2 * M, *ket = bra + M;
    if (l + lstep < K) stage_site(stage + (cur ^ 1) * 2 * M, L, Rv, K, M, l + lstep);
    // ---- pass 1: x_s[m1 + P m2], m2 < 16 -> 16-point DFT over m2, twiddle w_n^{m1 k2}
    for (int item = threadIdx.x; item < NSEQ * P; item += blockDim.x) {
      const int s = item / P, m1 = item % P;
      using Tr = decltype(Tin::x);
      const Tr *src = (const Tr *)((s & 2) ? ket : bra) + (s & 1);  // Re or Im part
      const bool deriv = s >= 4;
      double2 v[16];
#pragma unroll
      for (int m2 = 0; m2 < 16; ++m2) {
        const int m = m1 + P * m2;
        if ((!HALF || m2 < 8) && m < M) {
          double f = (double)src[2 * m];
          if (deriv) f *= (double)m;
          const double2 pf = pfs[m];
          v[m2] = make_double2(pf.x * f, pf.y * f);
        } else {
          v[m2] = make_double2(0, 0);
        }
      }
      if constexpr (HALF)
        dft16_half(v);
      else
        dft16(v);
      double2 *row = buf + s * SEQ;
#pragma unroll
      for (int q1 = 0; q1 < 4; ++q1)
#pragma unroll
        for (int q2 = 0; q2 < 4; ++q2) {
          const int k2 = q1 + 4 * q2;
          row[k2 * ROW + m1] = k2 ? cmul(v[4 * q1 + q2], tw1[k2 * P + m1]) : v[4 * q1 + q2];
        }
    }
    __syncthreads();
    // ---- pass 2: for row k2, m1 = a + R3 b: 16-point DFT over b, twiddle w_P^{a c}, in place
    for (int item = threadIdx.x; item < NSEQ * 16 * R3; item += blockDim.x) {
      const int k2 = item % 16, a = (item / 16) % R3, s = item / (16 * R3);
      double2 *row = buf + s * SEQ + k2 * ROW;
      double2 v[16];
#pragma unroll
      for (int b = 0; b < 16; ++b) v[b] = row[a + R3 * b];
      dft16(v);
#pragma unroll
      for (int q1 = 0; q1 < 4; ++q1)
#pragma unroll
        for (int q2 = 0; q2 < 4; ++q2) {
          const int c = q1 + 4 * q2;
          row[c * R3 + a] = (R3 == 1 || c == 0) ? v[4 * q1 + q2] : cmul(v[4 * q1 + q2], tw2[c * R3 + a]);
        }
    }
    __syncthreads();
    // ---- final: R3-point DFT over a of row k2f, column cf -> X[k2f + 16 cf + 256 d], and
    // the products for this thread's outputs d = h + 2 j
    if (fin) {
      double2 X[ND][NSEQ];
#pragma unroll
      for (int s = 0; s < NSEQ; ++s) {
        const double2 *row = buf + s * SEQ + k2f * ROW + cf * R3;
        double2 v[R3];
#pragma unroll
        for (int a = 0; a < R3; ++a) v[a] = row[a];
        if constexpr (R3 == 1) {
          X[0][s] = v[0];
        } else if constexpr (R3 == 2) {  // X_h = v0 + (-1)^h v1
          X[0][s] = h ? csub(v[0], v[1]) : cadd(v[0], v[1]);
        } else if constexpr (R3 == 4) {  // half h: {X0, X2} from v0 + v2, v1 + v3; {X1, X3} from the differences
          const double2 e = h ? csub(v[0], v[2]) : cadd(v[0], v[2]);
          const double2 o = h ? mul_i(csub(v[1], v[3])) : cadd(v[1], v[3]);
          X[0][s] = cadd(e, o);
          X[1][s] = csub(e, o);
        } else {
          dft_small<R3>(v);
#pragma unroll
          for (int j = 0; j < ND; ++j) X[j][s] = h ? v[2 * j + 1] : v[2 * j];  // constant indices
        }
      }
#pragma unroll
      for (int j = 0; j < ND; ++j) {
        const int k = k2f + 16 * cf + 256 * (R3 >= 2 ? h + 2 * j : 0);
        if constexpr (NSEQ == 8)
          bastin_products_reg(k, n, X[j], accp[j], accw[j]);
        else
          greenwood_product_reg(X[j], accp[j]);
      }
    }
    cur ^= 1;
  }
  cp_async_wait_all();
  double2 *out = part + (size_t)blockIdx.x * 2 * n;
  if (fin) {
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      const int k = k2f + 16 * cf + 256 * (R3 >= 2 ? h + 2 * j : 0);
      out[k] = accp[j];
      out[k + n] = accw[j];
    }
  }
}

// Direct DFT for any nump: one CTA per site at a time, thread per frequency.
template <int NSEQ, class Tin>
__global__ void __launch_bounds__(256)
    k_kubo_dft(const Tin *__restrict__ L, const Tin *__restrict__ Rv, long K, long chunk, int M, int nump,
               const double2 *__restrict__ pf_g, const double2 *__restrict__ twg, double2 *__restrict__ part) {
  extern __shared__ double2 sm[];
  double2 *bk = sm;  // bra[M], ket[M]
  const int kpt = (nump + blockDim.x - 1) / blockDim.x;
  double2 *acc_g = part + (size_t)blockIdx.x * 2 * nump;
  for (int q = 0; q < kpt; ++q) {
    const int k = threadIdx.x + q * blockDim.x;
    if (k < nump) acc_g[k] = acc_g[k + nump] = make_double2(0, 0);
  }
  const long lbeg = (long)blockIdx.x * chunk;
  const long lend = min(K, lbeg + chunk);
  for (long l = lbeg; l < lend; ++l) {
    __syncthreads();
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
      bk[m] = to_d2(L[(size_t)m * K + l]);
      bk[M + m] = to_d2(Rv[(size_t)m * K + l]);
    }
    __syncthreads();
    for (int q = 0; q < kpt; ++q) {
      const int k = threadIdx.x + q * blockDim.x;
      if (k >= nump) continue;
      double2 X[NSEQ];
#pragma unroll
      for (int s = 0; s < NSEQ; ++s) X[s] = make_double2(0, 0);
      for (int m = 0; m < M; ++m) {
        const double2 c = cmul(__ldg(pf_g + m), __ldg(twg + ((long)m * k) % nump));
#pragma unroll
        for (int s = 0; s < NSEQ; ++s) {
          const double2 src = (s & 2) ? bk[M + m] : bk[m];
          double u = (s & 1) ? src.y : src.x;
          if (s >= 4) u *= (double)m;
          X[s].x = fma(c.x, u, X[s].x);
          X[s].y = fma(c.y, u, X[s].y);
        }
      }
      double2 p = acc_g[k], w = acc_g[k + nump];
      if constexpr (NSEQ == 8)
        bastin_products(k, nump, X, 1, p, w);
      else
        greenwood_product(X, 1, p);
      acc_g[k] = p;
      acc_g[k + nump] = w;
    }
  }
}

__global__ void k_twiddles(int n, double2 *__restrict__ tw) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    double sn, cs;
    sincospi(2.0 * t / n, &sn, &cs);
    tw[t] = make_double2(cs, sn);
  }
}

// acc[t] = sum_b part[b][t]  (fixed order)
__global__ void k_sum_parts(const double2 *__restrict__ part, int nb, int len, double2 *__restrict__ acc) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < len; t += gridDim.x * blockDim.x) {
    double2 s = make_double2(0, 0);
    for (int b = 0; b < nb; ++b) s = cadd(s, part[(size_t)b * len + t]);
    acc[t] = s;
  }
}

// Post-processing: final_data = acc / R (the running mean of Kubo_solver_FFT::update_data
// over R states), then Bastin_postProcess (src/Kubo_solver_FFT_postProcess.cpp:120-273) or
// Greenwood_postProcess (:279-397).  out = [E (nump), sigma (nump), integrand (nump)].
// The integrand is evaluated in parallel; the left-rectangle cumulative integral
// (integration_linqt, :36-47) runs in index order on one thread.
__global__ void k_kubo_post(const double2 *__restrict__ acc, double R, int nump, int formula, double N, double a,
                            double b, double *__restrict__ out, double *__restrict__ scratch) {
  double *E = out, *sig = out + nump, *integ = out + 2 * nump;
  double *Er = scratch;  // rearranged reduced energies
  const double omega = N / (a * a);
  for (int j = threadIdx.x; j < nump; j += blockDim.x) {
    const int k = rearranged_source(j, nump);
    const double Ek = cos(M_PI * (2 * k + 0.5) / nump);
    Er[j] = Ek;
    if (formula == LINQT_KUBO_BASTIN) {
      const double pr = acc[k].x / R, wi = acc[k + nump].y / R;
      double v = Ek * pr - (sqrt(1.0 - Ek * Ek) * wi);
      v *= 1.0 / pow((1.0 - Ek * Ek), 2.0);
      v *= omega / (M_PI);
      integ[j] = v;
    } else {
      sig[j] = 2.0 * omega * (acc[k].x / R) / (1.0 - Ek * Ek) / (2 * M_PI);
      integ[j] = 0.0;
    }
  }
  __syncthreads();
  if (formula == LINQT_KUBO_BASTIN && threadIdx.x == 0) {
    double s = 0;
    for (int i = 0; i < nump - 1; ++i) {
      s += integ[i] * (Er[i + 1] - Er[i]);
      sig[i] = s;
    }
    sig[nump - 1] = 0.0;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < nump; j += blockDim.x) E[j] = a * Er[j] - b;
}

template <int R3, int NSEQ, class Tin>
void launch_fft(Session *s, const Tin *L, const Tin *Rv, long K, int M, const double2 *pf, double2 *acc) {
  constexpr int n = 256 * R3;
  const size_t smem = sizeof(double2) * ((size_t)NSEQ * 16 * (16 * R3 + 1) + 16 * 16 * R3 + 16 * R3 + (size_t)M) +
                      sizeof(Tin) * 4 * (size_t)M;
  if (smem > 227 * 1024) fail(LINQT_ERR_UNSUPPORTED, "kubo_fft: nump too large for the shared-memory FFT");
  // one CTA per SM (most of its shared memory), persistent over the sites; a server slot
  // takes its SMs from the server's ledger, so that the slots' persistent grids and this one
  // never wait for each other's SMs
  double2 *part = (double2 *)s->get("kubo_part", sizeof(double2) * 2 * (size_t)n * s->sm_count);
  const int nb = (int)std::max(1L, std::min(K, (long)sm_share_take(s)));
  const long chunk = (K + nb - 1) / nb;
  // every output k < n is written by exactly one thread of each CTA (pairs cover 16 x 16,
  // halves cover the R3 outputs), so the partials need no clearing
  if (2 * M <= n) {
    raise_smem_limit((const void *)k_kubo_fft<R3, NSEQ, true, Tin>, smem);
    k_kubo_fft<R3, NSEQ, true, Tin><<<nb, kFftThreads, smem, s->stream>>>(L, Rv, K, chunk, M, pf, part);
  } else {
    raise_smem_limit((const void *)k_kubo_fft<R3, NSEQ, false, Tin>, smem);
    k_kubo_fft<R3, NSEQ, false, Tin><<<nb, kFftThreads, smem, s->stream>>>(L, Rv, K, chunk, M, pf, part);
  }
  const cudaError_t le = cudaGetLastError();
  if (le != cudaSuccess) coop_share_return(s);
  LQ_CUDA(le);
  coop_share_hand_back(s);
  k_sum_parts<<<(2 * n + 255) / 256, 256, 0, s->stream>>>(part, nb, 2 * n, acc);
  LQ_LAUNCHED();
}

template <int NSEQ, class Tin>
void launch_dft(Session *s, const Tin *L, const Tin *Rv, long K, int M, int nump, const double2 *pf, double2 *acc) {
  double2 *tw = (double2 *)s->get("kubo_tw", sizeof(double2) * nump);
  k_twiddles<<<(nump + 255) / 256, 256, 0, s->stream>>>(nump, tw);
  LQ_LAUNCHED();
  const size_t smem = sizeof(double2) * 2 * (size_t)M;
  if (smem > 227 * 1024) fail(LINQT_ERR_UNSUPPORTED, "kubo_fft: M too large for the direct DFT");
  raise_smem_limit((const void *)k_kubo_dft<NSEQ, Tin>, smem);
  const int nb = (int)std::max(1L, std::min(K, (long)s->sm_count * 4));
  const long chunk = (K + nb - 1) / nb;
  double2 *part = (double2 *)s->get("kubo_part", sizeof(double2) * 2 * (size_t)nump * nb);
  k_kubo_dft<NSEQ, Tin><<<nb, 256, smem, s->stream>>>(L, Rv, K, chunk, M, nump, pf, tw, part);
  LQ_LAUNCHED();
  k_sum_parts<<<(2 * nump + 255) / 256, 256, 0, s->stream>>>(part, nb, 2 * nump, acc);
  LQ_LAUNCHED();
}

template <class Tin>
void kubo_fft_sites_t(Session *s, const Tin *L, const Tin *Rv, long nsites, int M, int nump, int formula,
                      const double2 *pf, double2 *acc) {
  const bool bastin = formula == LINQT_KUBO_BASTIN;
  const bool pow2 = nump >= 256 && nump <= 2048 && (nump & (nump - 1)) == 0;
  const bool fits = pow2 && (bastin ? nump <= 1024 : true);
  if (fits) {
    switch (nump) {
      case 256: bastin ? launch_fft<1, 8>(s, L, Rv, nsites, M, pf, acc) : launch_fft<1, 4>(s, L, Rv, nsites, M, pf, acc); return;
      case 512: bastin ? launch_fft<2, 8>(s, L, Rv, nsites, M, pf, acc) : launch_fft<2, 4>(s, L, Rv, nsites, M, pf, acc); return;
      case 1024: bastin ? launch_fft<4, 8>(s, L, Rv, nsites, M, pf, acc) : launch_fft<4, 4>(s, L, Rv, nsites, M, pf, acc); return;
      case 2048: launch_fft<8, 4>(s, L, Rv, nsites, M, pf, acc); return;
    }
  }
  if (bastin)
    launch_dft<8>(s, L, Rv, nsites, M, nump, pf, acc);
  else
    launch_dft<4>(s, L, Rv, nsites, M, nump, pf, acc);
}

}  // namespace

void kubo_prefactors(Session *s, int M, int nump, double2 *pf) {
  k_prefactors<<<(M + 255) / 256, 256, 0, s->stream>>>(M, nump, pf);
  LQ_LAUNCHED();
}

void kubo_fft_sites(Session *s, const void *Lv, const void *Rvv, long nsites, int M, int nump, int formula,
                    bool fp32_inputs, double2 *acc) {
  double2 *pf = (double2 *)s->get("kubo_pf", sizeof(double2) * M);
  kubo_prefactors(s, M, nump, pf);
  if (fp32_inputs)
    kubo_fft_sites_t(s, (const float2 *)Lv, (const float2 *)Rvv, nsites, M, nump, formula, pf, acc);
  else
    kubo_fft_sites_t(s, (const double2 *)Lv, (const double2 *)Rvv, nsites, M, nump, formula, pf, acc);
}

void kubo_postprocess(Session *s, const double2 *acc, int R, int nump, int formula, int N, double band_width,
                      double band_center, double *out) {
  double *scratch = (double *)s->get("kubo_post", sizeof(double) * 3 * (size_t)nump);
  k_kubo_post<<<1, 1024, 0, s->stream>>>(acc, (double)R, nump, formula, (double)N, band_width / 2.0, band_center,
                                         out, scratch);
  LQ_LAUNCHED();
}

}  // namespace linqt
