// sqg_tma.cuh -- tensor-memory-accelerator (TMA) tile loads of the column
// passes: the raw half columns of a column pair are copied from a field
// stack (nf x (N/2+1) x N complex, row-major, this GPU's memory) into shared
// memory by cp.async.bulk.tensor, completion counted on an mbarrier.
//
// Tensor map (encoded on the host, one per field stack): 32-bit elements,
// dims {N * sizeof(C) / 4, N/2 + 1, nf}, strides {N * sizeof(C), (N/2+1) N
// sizeof(C)} bytes, box {2 sizeof(C) / 4, min(N/2, 256), 1}: one box is a
// column pair over up to 256 rows, 16 (float) or 32 (double) bytes a row,
// written densely -- the layout the column pass keeps its raw half columns
// in.  The x coordinate of a box is (first column) sizeof(C) / 4 with an even
// first column, so x * 4 bytes is a multiple of 16.  No multicast.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sqg {

// Iterations of try_wait before a wait gives up (each returns after at most
// a short hardware time limit).
constexpr uint32_t kTmaWaitLimit = 1u << 22;
// Status bit set by a column pass whose tile copies did not complete.
constexpr unsigned kStatusTmaTimeout = 2u;

__device__ __forceinline__ uint32_t tma_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_bar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(tma_smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tma_bar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// Orders this thread's earlier generic-proxy shared-memory accesses (made
// visible to it by a block barrier) before its later async-proxy copies.
__device__ __forceinline__ void tma_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// Adds the bytes of copies about to be issued to the current phase.
__device__ __forceinline__ void tma_bar_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;\n" ::"r"(tma_smem_u32(bar)), "r"(bytes)
               : "memory");
}
// The one arrival of a phase (after every expect of the phase).
__device__ __forceinline__ void tma_bar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(tma_smem_u32(bar)) : "memory");
}
// Bounded wait for the phase of the given parity; false on time-out.
__device__ __forceinline__ bool tma_bar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = tma_smem_u32(bar);
  for (uint32_t it = 0; it < kTmaWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];\n" ::"r"(tma_smem_u32(dst)),
      "l"(map), "r"(tma_smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

}  // namespace sqg
