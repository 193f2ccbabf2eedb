// Tensor-memory-accelerator loads (cp.async.bulk.tensor) with mbarrier
// completion, for sm_100a: a host helper that encodes a 2D tile map through
// the driver's cuTensorMapEncodeTiled (reached with cudaGetDriverEntryPoint,
// so the library does not link libcuda), and device wrappers around the PTX.
// Every wait is bounded.  Loads only, from this GPU's own memory, without
// cluster multicast.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace scy {

// 2D map over a row-major array of `rows` x `cols` elements (row stride
// `stride_bytes`, a multiple of 16) with a box of box_rows x box_cols; reads
// outside the array return zeros.  Returns 0 on success.
int tma_map_2d(CUtensorMap* map, const void* base, CUtensorMapDataType type, int esize, long cols, long rows,
               long stride_bytes, int box_cols, int box_rows);

// 3D map over d0 x d1 x d2 elements (d0 innermost, strides of dimensions 1
// and 2 in bytes, multiples of 16) with a box of box0 x box1 x box2
int tma_map_3d(CUtensorMap* map, const void* base, CUtensorMapDataType type, long d0, long d1, long d2,
               long stride1_bytes, long stride2_bytes, int box0, int box1, int box2);

// the same with 64-byte swizzling of the box's rows in shared memory (box0
// elements of the innermost dimension must span exactly 64 bytes; the
// destination must be 512-byte aligned): the K-major canonical layout
// tcgen05.mma reads through a SWIZZLE_64B shared-memory descriptor
int tma_map_3d_sw64(CUtensorMap* map, const void* base, CUtensorMapDataType type, long d0, long d1, long d2,
                    long stride1_bytes, long stride2_bytes, int box0, int box1, int box2);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// true once the phase with the given parity has completed; false after
// max_polls unsuccessful polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int max_polls) {
  const uint32_t a = smem_u32(bar);
  for (int k = 0; k < max_polls; ++k) {
    uint32_t done = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// box at element coordinates (x = column, y = row) into dst, completion on bar
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// box at element coordinates (x, y, z) of a 3D map into dst, completion on bar
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// orders this thread's earlier global stores before later async-proxy (TMA) reads
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

}  // namespace scy
