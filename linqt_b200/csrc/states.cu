// Random-phase states generated on the device.
//
// LinQT draws no random states itself: its default state is a delta at N/2
// (include/quantum_states.hpp:85-93) and its random-phase filler
// (FillWithRandomPhase, quantum_states.hpp:231-252) is never called, so phases are
// supplied from outside.  Here they come from Philox4x32-10 (Salmon et al., SC'11),
// restated from its published description and identical to the host generator of the
// Python package: key = (seed lo, seed hi), counter = (index lo, index hi, 0, 0) with
// index = r*N + i, x = (w0 << 32) | w1, u = (x >> 11) * 2^-53, and
// state r, site i = exp(2 pi i u) / sqrt(N).
#include "internal.cuh"

namespace linqt {

namespace {

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
    const uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += W0;
    k1 += W1;
  }
}

__global__ void k_random_phase(long total, int N, unsigned long long seed, double norm, double2 *out) {
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
    uint32_t c[4] = {(uint32_t)idx, (uint32_t)((unsigned long long)idx >> 32), 0u, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const unsigned long long x = ((unsigned long long)c[0] << 32) | c[1];
    const double u = (double)(x >> 11) * 0x1.0p-53;
    double sn, cs;
    sincos(6.283185307179586 * u, &sn, &cs);
    out[idx] = make_double2(cs / norm, sn / norm);
  }
}

}  // namespace

void random_phase_states(Session *s, int N, int R, unsigned long long seed, double2 *out) {
  LQ_REQUIRE(N > 0 && R > 0, "random_phase_states: N and R must be positive");
  const long total = (long)N * R;
  const int grid = (int)std::min<long>((total + 255) / 256, (long)s->sm_count * 16);
  k_random_phase<<<grid, 256, 0, s->stream>>>(total, N, seed, std::sqrt((double)N), out);
  LQ_LAUNCHED();
}

}  // namespace linqt
