// Grid-wide barrier with a bounded wait, for persistent launches whose CTAs are all resident
// (cooperative launch).  No kernel spins without a limit: a wait that runs out sets the error
// word, every CTA then leaves at its next barrier, and the host reads and clears the word.
#pragma once

#include "topx_kernels.cuh"

namespace topx {

// polls of the barrier word before a CTA gives up (about a second in all)
constexpr unsigned kCoopSpinLimit = 1u << 20;

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_volatile_int(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

// bar->count only grows within a launch: barrier number i (1, 2, ...) is passed once it reaches
// i * gridDim.x, so an arrival is one fire-and-forget release add and the wait polls that single
// word (no reset round trip).  The last CTA to leave the kernel (coop_exit) zeroes the words for
// the next launch.  Returns false in every thread of the CTA once any CTA has given up; the
// kernel then returns, so it always ends.
__device__ __forceinline__ bool coop_barrier(CoopBarrier* bar, unsigned& epoch) {
  __shared__ int s_ok;
  __syncthreads();
  ++epoch;
  if (threadIdx.x == 0) {
    int ok = ld_volatile_int(&bar->err) == 0;
    if (ok) {
      const unsigned target = epoch * gridDim.x;
      asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&bar->count) : "memory");
      unsigned it = 0;
      while (ld_acquire_gpu(&bar->count) < target) {
        if (++it > kCoopSpinLimit || ld_volatile_int(&bar->err)) {
          atomicCAS(&bar->err, 0, kCoopErrBarrier);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Called once by every CTA on every exit path after its first barrier: the last one out
// re-arms the barrier words (all other CTAs have left their waits by then).
__device__ __forceinline__ void coop_exit(CoopBarrier* bar) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&bar->gen, 1u) == gridDim.x - 1) {
      atomicExch(&bar->count, 0u);
      atomicExch(&bar->gen, 0u);
    }
  }
}

}  // namespace topx
