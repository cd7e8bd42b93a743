// elmm_stream.cuh -- plane streaming into shared memory with the tensor
// memory accelerator (TMA): one cp.async.bulk.tensor box per field and
// plane, completion counted on an mbarrier per ring slot.  Planes are
// requested several planes ahead of their use, so the bytes in flight per SM
// do not depend on registers or on the number of resident warps, and one
// thread issues every copy of a tile.
//
// Alignment: the innermost box coordinate times the element size is a
// multiple of 16 bytes and every shared-memory destination is 128-byte
// aligned.  Every copy lands in the issuing block's own shared memory.
#pragma once

#include <cuda.h>

#include <cstdint>

namespace elmm {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// make the initialised barriers and prior shared-memory accesses visible to
// the async (bulk-copy) proxy
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// One box of a 3-D tensor map (tile mode) into this block's shared memory;
// x is the innermost element coordinate and must be a multiple of 16 bytes.
// Boxes that reach past the tensor are zero-filled by the hardware.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_addr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// Bounded wait: every try_wait already suspends for a while in hardware; a
// phase that has not completed after `limit` tries (kWaitLimit unless a test
// of the failure path lowered it) is reported as a timeout instead of
// spinning for ever.
constexpr int kWaitLimit = 1 << 20;

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int limit = kWaitLimit) {
  for (int n = 0; n < limit; n++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

}  // namespace elmm
