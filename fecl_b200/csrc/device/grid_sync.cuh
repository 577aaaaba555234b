// Grid-wide barrier for the persistent decoders (a cooperative launch: every block of
// the grid is resident).
//
// The arrival counter only grows: each barrier adds gridDim.x, and `epoch` is the
// count a block waits for.  Every wait is bounded: after kBarrierNs of global time, or
// as soon as another block has given up (the shared failure flag), the block records
// the failure and the barrier returns false, so that the kernel ends instead of
// waiting for a block that will never arrive.
#pragma once

#include <cuda_runtime.h>

namespace fecl {

constexpr unsigned long long kBarrierNs = 2000000000ull;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned load_acquire(const unsigned* q) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(q) : "memory");
  return v;
}

// counter and error are two words in global memory, zeroed before the launch.
__device__ __forceinline__ bool grid_barrier(unsigned* counter, unsigned* error, unsigned& epoch) {
  __shared__ int ok;
  __syncthreads();
  epoch += gridDim.x;
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(counter, 1u);
    const unsigned long long t0 = global_ns();
    int good = 1;
    while (load_acquire(counter) < epoch) {
      if (load_acquire(error) != 0u) {
        good = 0;
        break;
      }
      __nanosleep(64);
      if (global_ns() - t0 > kBarrierNs) {
        atomicExch(error, 1u);
        good = 0;
        break;
      }
    }
    __threadfence();
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

}  // namespace fecl
