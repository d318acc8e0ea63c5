// tma.cuh -- tensor-memory-accelerator (TMA) tile copies with mbarrier
// completion, for kernels that stream tiles of a padded field through shared
// memory (sm_90+ PTX: cp.async.bulk.tensor, mbarrier, fence.proxy.async).
//
// Only plain (non-multicast) loads and stores of this GPU's own memory are
// used.  Every wait on an mbarrier is bounded: tma_wait() gives up after a
// fixed number of try_wait rounds and returns false, and the kernel then
// records an error word that the host reads (a TMA copy of local memory always
// completes, so this is a safety net, not an expected path).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace nse {

// host: a tiled 3-D tensor map over a padded field (x fastest): extents
// (e0, e1, e2) elements, row and plane pitches in bytes, box (b0, b1, b2)
// elements; out-of-range box elements read as zero and are not stored.
// Returns false when the driver entry point is missing or rejects the map.
bool tma_encode_3d(CUtensorMap* map, const void* base, bool fp64, long e0, long e1, long e2,
                   long pitch1, long pitch2, int b0, int b1, int b2);

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// bounded wait for the phase with parity `parity` of bar to complete
__device__ __forceinline__ bool tma_wait(uint64_t* bar, unsigned parity) {
  const unsigned a = smem_u32(bar);
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// load the box at element coordinates (x, y, z) into smem; completes on bar
__device__ __forceinline__ void tma_load_3d(void* smem, const CUtensorMap* map, int x, int y,
                                            int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_u32(smem)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
// store the box at (x, y, z) from smem (bulk group of the issuing thread)
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int x, int y, int z,
                                             const void* smem) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];\n" ::"l"(
          reinterpret_cast<uint64_t>(map)),
      "r"(x), "r"(y), "r"(z), "r"(smem_u32(smem))
      : "memory");
}
__device__ __forceinline__ void tma_store_commit() {
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
// the issuing thread's committed stores have finished reading shared memory
__device__ __forceinline__ void tma_store_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}
// ... and are complete in global memory
__device__ __forceinline__ void tma_store_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
}
// generic-proxy writes to shared memory become visible to TMA (async proxy)
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

}  // namespace nse
