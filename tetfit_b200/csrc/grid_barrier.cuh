// Grid barrier of the persistent (cooperative-launch) CG kernels.
//
// bar[0] counts the blocks that arrived, bar[1] is the generation; the last
// block to arrive resets the count and advances the generation.  Both words
// start at 0 (the host clears them with *err).  The cooperative launch keeps
// every block resident, so in a correct kernel each wait ends within
// microseconds; the wait is still bounded: once `limit_ns` has passed, or as
// soon as another block has raised *err, the waiting block raises *err (bit
// value 2) and goes on.  After that every later barrier of the launch falls
// through at once, the kernel runs to its end (its loops are bounded by the
// iteration limit), and the host, which reads *err after the launch, reports
// the results as invalid instead of waiting for a launch that never ends.
#pragma once
#include <cstdint>

namespace tf {

constexpr int kBarrierTimedOut = 2;
constexpr uint64_t kBarrierLimitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void grid_barrier(unsigned int* bar, int* err, unsigned int nblocks,
                                             uint64_t limit_ns = kBarrierLimitNs) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* gen = bar + 1;
    const unsigned int g = *gen;  // read before arriving: the last arrival may advance it at once
    __threadfence();
    if (atomicAdd(bar, 1u) == nblocks - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const uint64_t t0 = global_ns();
      while (*gen == g) {
        if (*(volatile int*)err != 0 || global_ns() - t0 > limit_ns) {
          atomicOr(err, kBarrierTimedOut);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

}  // namespace tf
