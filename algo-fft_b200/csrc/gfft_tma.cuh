// Tensor Memory Accelerator (TMA) helpers: tile copies between global and
// shared memory by the copy engine, completion on an mbarrier (loads) or a
// bulk group (stores), and host-side tensor-map encoding.
//
// Every copy here is a plain CTA-local tile copy: no cluster multicast.
// The innermost coordinate of every copy is a multiple of 4 FP32 words
// (16 bytes); callers guarantee it by copying whole complex elements of
// tiles whose first column is even.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace gfft {

__device__ __forceinline__ uint32_t sm_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sm_addr(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation and generic-proxy shared-memory accesses
// visible to the copy engine.
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm_addr(bar)), "r"(bytes)
               : "memory");
}

// Bounded wait for the phase of this parity; false once `limit` rounds of
// try_wait (each with the hardware's own short suspend) have passed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned limit) {
  for (unsigned it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(sm_addr(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];" ::"r"(sm_addr(dst)),
      "l"(map), "r"(sm_addr(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z,
                                            int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, "
      "%6}], [%2];" ::"r"(sm_addr(dst)),
      "l"(map), "r"(sm_addr(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
      : "memory");
}

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int x, int y, int z) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(map),
               "r"(sm_addr(src)), "r"(x), "r"(y), "r"(z)
               : "memory");
}

__device__ __forceinline__ void tma_store_4d(const CUtensorMap* map, const void* src, int x, int y, int z, int w) {
  asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%2, %3, %4, %5}], [%1];" ::"l"(map),
               "r"(sm_addr(src)), "r"(x), "r"(y), "r"(z), "r"(w)
               : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Waits until the committed stores have finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// Waits until the committed stores are complete.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Host side.  A tensor of complex elements of `elem_bytes` (8 or 16) viewed
// as FP32 words: dims[0] complex elements along the contiguous axis, then up
// to three outer axes with strides in elements; the box is box[0] elements
// by box[1..] along the outer axes.  Returns cudaErrorInvalidValue when the
// copy engine cannot address it (alignment, sizes), so the caller can take
// its plain path.
// swizzle128: the box's rows are 128 bytes and land in shared memory in the
// 128-byte swizzle pattern (16-byte chunk j of row r at chunk j ^ (r mod 8)).
cudaError_t encode_tile_map(CUtensorMap* map, const void* base, int elem_bytes, int rank, const int64_t* dims,
                            const int64_t* strides_elems, const int* box, bool swizzle128 = false);

}  // namespace gfft
