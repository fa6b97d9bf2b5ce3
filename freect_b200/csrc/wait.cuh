// Bounded mbarrier waits shared by the kernels that wait on one (TMA rings,
// the tensor-core pipeline): a wait gives up after a wall-clock limit read
// from %globaltimer (and after a hard cap of polls), returning false, so a
// producer that never arrives ends the kernel with an error word set
// instead of hanging the GPU.
#pragma once

#include <stdint.h>

constexpr uint64_t WFBP_WAIT_LIMIT_NS = 4000000000ull;  // 4 s; a healthy stage completes in microseconds
constexpr uint32_t WFBP_WAIT_MAX_POLLS = 1u << 30;

__device__ __forceinline__ uint64_t wfbp_globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool wfbp_mbar_wait(uint64_t* bar, uint32_t parity,
                                               uint64_t limit_ns = WFBP_WAIT_LIMIT_NS) {
  const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(bar));
  uint64_t t0 = 0;
  for (uint32_t it = 0; it < WFBP_WAIT_MAX_POLLS; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 63u) == 0) {
      const uint64_t now = wfbp_globaltimer();
      if (it == 0) t0 = now;
      else if (now - t0 > limit_ns) return false;
    }
  }
  return false;
}
