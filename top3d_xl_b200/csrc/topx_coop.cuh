// Bounded waits of persistent launches whose CTAs are all resident (cooperative launch).  No
// kernel spins without a limit: a wait that runs out sets the error word, the CTAs waiting after
// it give up too, and the host reads and clears the word.
#pragma once

#include "topx_kernels.cuh"

namespace topx {

// polls of a counter before a CTA gives up (about a second in all)
constexpr unsigned kCoopSpinLimit = 1u << 20;

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_volatile_int(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

// Thread 0 of a CTA waits until the counter *p has reached `need` (counters only grow within a
// launch; producers add with release semantics, the poll loads with acquire).  Gives up after
// kCoopSpinLimit polls, or soon after another CTA gave up, with ctl->err set to kCoopErrWait.
__device__ __forceinline__ bool coop_wait_count(const unsigned* p, unsigned need, CoopControl* ctl) {
  unsigned it = 0;
  while (ld_acquire_gpu(p) < need) {
    if ((++it & 31u) == 0u && (it > kCoopSpinLimit || ld_volatile_int(&ctl->err))) {
      atomicCAS(&ctl->err, 0, kCoopErrWait);
      return false;
    }
  }
  return true;
}
__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

}  // namespace topx
