// SPDX-License-Identifier: GPL-3.0-or-later
// Tensor-memory-accelerator copies of field tiles into shared memory (cp.async.bulk.tensor, completed on an
// mbarrier of the block), the bounded wait on them, and the descriptor of a scalar species' tensor maps.
//
// No copy here multicasts across a cluster: every load reads this GPU's own field arrays into the issuing block's
// shared memory.
#pragma once

#include <cuda.h>

#include <cstdint>

namespace cw {

// the tensor maps of one scalar species' two q_2 buffers (q_2 and q_new swap after every update, so a kernel takes
// the map of the buffer that q_2's view points into). A map covers the buffer's whole allocation as (x, y, z) =
// (pitch, rows, levels); x0, y0 are the map coordinates of i = 0 and j = 0.
struct alignas(64) QMap {
  CUtensorMap a, b;
  const void* pa;  // the view origin of buffer a
  int x0, y0;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// the initialised barriers made visible to the copies (the async proxy) before any copy completes on them
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// one arrival that also announces the bytes the phase's copies will deliver
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t done;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// wait for the phase of the given parity to complete, for at most `cycles` SM clock cycles: false if it did not
constexpr long long kWaitCycles = 2000000000ll;  // about one second at the B200's clocks
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, long long cycles = kWaitCycles) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > cycles) return false;
  return true;
}

// one box of a 3-D tensor map at coordinates (x, y, z) into shared memory; its bytes complete on bar. The caller
// guarantees x * element size to be a multiple of 16 bytes (the tile's x start) and dst 128-byte aligned (a tensor
// copy's shared-memory destination must be).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace cw
