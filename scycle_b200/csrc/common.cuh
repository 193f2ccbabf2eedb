// Shared helpers for the SCycle B200 kernels: status codes, launch checks,
// deterministic block reductions.
#pragma once
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdint>
#include <string>

#include "../../include/scycle_b200.h"

namespace scy {

// Last error message of this thread, returned through scy_get_last_error().
void set_error(const char* fmt, ...);
// Counts kernel launches of this library (read by scy_launch_count()).
void count_launch();
void count_launches(long long n);  // n kernels launched at once (a CUDA graph replay)

#define SCY_CUDA_TRY(call)                                                     \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      ::scy::set_error("%s:%d: %s failed: %s", __FILE__, __LINE__, #call,      \
                       cudaGetErrorString(e_));                                \
      return SCY_ERR_CUDA;                                                     \
    }                                                                          \
  } while (0)

#define SCY_LAUNCH_CHECK()                                                     \
  do {                                                                         \
    ::scy::count_launch();                                                     \
    cudaError_t e_ = cudaGetLastError();                                       \
    if (e_ != cudaSuccess) {                                                   \
      ::scy::set_error("%s:%d: kernel launch failed: %s", __FILE__, __LINE__,  \
                       cudaGetErrorString(e_));                                \
      return SCY_ERR_CUDA;                                                     \
    }                                                                          \
  } while (0)

#define SCY_TRY(call)                                                          \
  do {                                                                         \
    int s_ = (call);                                                           \
    if (s_ != SCY_OK) return s_;                                               \
  } while (0)

constexpr int kBlock = 256;
constexpr int kNumSMs = 148;

inline int grid_for(long n, int block = kBlock, int max_blocks = 148 * 16) {
  long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > max_blocks) g = max_blocks;
  return (int)g;
}

// Warp + block sum; every thread of the block receives the total.
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T w = __shfl_xor_sync(0xffffffffu, v, o);
    v = v > w ? v : w;
  }
  return v;
}

// Sum over the block in a fixed order (deterministic for a fixed launch shape).
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* sh /* >= 32 entries */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  T t = (threadIdx.x < nw) ? sh[threadIdx.x] : T(0);
  if (wid == 0) t = warp_sum(t);
  if (threadIdx.x == 0) sh[0] = t;
  __syncthreads();
  t = sh[0];
  __syncthreads();
  return t;
}

// Grid-wide deterministic reduction over the blocks of one z-slice of the
// grid (the whole grid when gridDim.z == 1; batched launches give each
// instance its own slice and pass that slice's partials, counter and out):
// each block stores its partial sum in partials[block id within the slice];
// the last block of the slice to finish adds them in index order and writes
// *out.  `counter` must be zero on entry and is reset to zero.
__device__ __forceinline__ void grid_reduce_finish(double block_total, double* partials,
                                                   unsigned int* counter, double* out,
                                                   double* sh) {
  __shared__ bool am_last;
  const unsigned int nblocks = gridDim.x * gridDim.y;
  const unsigned int bid = blockIdx.x + gridDim.x * blockIdx.y;
  if (threadIdx.x == 0) {
    partials[bid] = block_total;
    __threadfence();
    unsigned int prev = atomicAdd(counter, 1u);
    am_last = (prev == nblocks - 1);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)nblocks; i += blockDim.x) s += ((volatile double*)partials)[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) {
      *out = s;
      *counter = 0u;
    }
  }
}

}  // namespace scy
