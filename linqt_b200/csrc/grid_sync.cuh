// Grid-wide barrier of the persistent cooperative kernels (recur.cu, nonorth.cu).
//
// All CTAs of a cooperative launch are co-resident, so they can wait for each other.  The
// wait is bounded: after kSpinLimit polls a CTA sets the error flag and every waiting CTA
// gives up, so a bad launch ends instead of hanging the GPU; the host turns the flag into
// LINQT_ERR_TIMEOUT (check_device_errors).  For tests, a session can make its barriers wait
// for CTAs that were never launched, with a short poll limit
// (linqt_session_inject_barrier_timeout): the kernel then returns through the same path.  Release: bar.sync, fence, atomic arrival;
// acquire: poll the generation, fence, bar.sync.  The gpu-scope fence after the poll drops
// stale L1 lines, so data written by other CTAs before the barrier may be read through L1
// after it.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace linqt {

struct GridBarrier {
  unsigned count;  // arrivals
  unsigned gen;    // generation, bumped by the last arrival
  int err;
  int extra;              // fault injection (tests): arrivals awaited beyond the launched CTAs
  long long spin_limit;   // fault injection (tests): polls before giving up (0: kSpinLimit)
};
// bytes of GridBarrier that restart at zero for every launch (count, gen)
constexpr size_t kBarrierResetBytes = offsetof(GridBarrier, err);

constexpr long kSpinLimit = 1L << 24;  // polls of ~0.1 us: well above any step, far below a hang

// Returns false if the wait gave up (the error flag is then set).  One arrival counter: a
// two-level arrival (group counters, then a top counter) was measured slower at the grid
// sizes used here (256 CTAs: +0.4 ms over 512 steps), its extra round trip outweighing the
// shorter atomic queue.
__device__ inline bool grid_barrier(GridBarrier *bar, unsigned nblocks) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned *vgen = &bar->gen;
    const unsigned g = *vgen;
    const long long limit = bar->spin_limit > 0 ? bar->spin_limit : kSpinLimit;
    const unsigned need = nblocks + (unsigned)bar->extra;
    __threadfence();
    const unsigned arrived = atomicAdd(&bar->count, 1u);
    if (arrived == need - 1) {
      bar->count = 0;
      __threadfence();
      atomicAdd(&bar->gen, 1u);
    } else {
      long spins = 0;
      while (*vgen == g) {
        if (*(volatile int *)&bar->err) {
          ok = 0;
          break;
        }
        if (++spins > limit) {
          atomicExch(&bar->err, 1);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

}  // namespace linqt
