// Banded Cholesky sweeps along y of the fast-diagonalisation
// preconditioner, fed by TMA (shared by the batched ensemble and the
// single-instance driver).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "tma.cuh"

namespace scy {
namespace {

template <typename T>
__device__ __forceinline__ T fma_t(T a, T b, T c);
template <>
__device__ __forceinline__ double fma_t<double>(double a, double b, double c) {
  return fma(a, b, c);
}
template <>
__device__ __forceinline__ float fma_t<float>(float a, float b, float c) {
  return fmaf(a, b, c);
}

// After the z transform: for every z mode j and instance k, the banded
// solve (Ky + lz_j My) x = t along y with the Cholesky factor L (forward
// L y = t, back L^T x = y), in place in t (rows of Nzp values, instance k
// at rows k Ny ..).  The factor tables hold, per row i and mode j, nine
// values in the order the row is processed: [0] 1 / L_ii, [1] the coupling
// to the row processed just before, already divided by L_ii (forward
// L(i, i-1) / L_ii, back L(i+1, i) / L_ii), [2..8] the contributions of
// row i to the rows 2..8 further on (forward L(i+m, i), back L(i, i-m)).
// With the coupling folded in, a row costs one dependent FMA on the chain:
//   x_i = (t_i - b_i) / L_ii - c1_i x_prev
// where b_i collects the contributions of the rows before x_prev.
//
// Tensor-memory-accelerator feed: a block owns YS_C = 16 consecutive z
// modes of B = 2 W I instances: lane c + 16 h of warp w carries the chains
// of mode j0 + c for the I instances (2 w + h) I + s, so one read of a
// factor value from shared memory serves I chains, and lanes c and c + 16
// read the same value (a broadcast).  Per chunk of YS_R = 16 rows one 2D
// copy brings the factor (16 rows x 9 table rows x 16 modes) and one 3D copy
// the transform of the block's instances (16 modes x 16 rows x B); YS_S = 3
// stages, so two chunks are in flight while one is swept.  Every chunk is
// swept over all 16 rows: rows outside 0..Ny-1 arrive as zeros (factor and
// data), give zero and only shift the accumulators, and are not stored.  A
// wait that runs out sets status bit 4 of the block's instances (their solve
// is then repeated) and the block stops.
constexpr int YS_R = 16, YS_C = 16, YS_S = 3;
constexpr int YS_I = 2, YS_W = 2;          // chains per lane, warps per block
constexpr int YS_B = 2 * YS_W * YS_I;      // instances per block

template <typename T, int I, int W>
__global__ void __launch_bounds__(32 * W) b_ysolve_tma_kernel(const __grid_constant__ CUtensorMap mLcol,
                                                              const __grid_constant__ CUtensorMap mLrow,
                                                              const __grid_constant__ CUtensorMap mT,
                                                              T* __restrict__ t, int Ny, int Nz, int Nzp, int K,
                                                              unsigned* __restrict__ status,
                                                              int first_polls = 1 << 18, int drop_first = 0) {
  constexpr int B = 2 * W * I;
  extern __shared__ __align__(128) unsigned char ys_smem[];
  constexpr int CT = YS_R * 9 * YS_C, DT = B * YS_R * YS_C;  // elements per tile
  T* coef = reinterpret_cast<T*>(ys_smem);                   // [YS_S][YS_R][9][YS_C]
  T* dat = coef + YS_S * CT;                                 // [YS_S][B][YS_R][YS_C]
  uint64_t* bar = reinterpret_cast<uint64_t*>(dat + YS_S * DT);
  const int lane = threadIdx.x & 31, c = lane % YS_C, h = lane / YS_C, wv = threadIdx.x >> 5;
  const int j0 = blockIdx.x * YS_C, j = j0 + c, kb = blockIdx.y * B;
  const int kk0 = (wv * 2 + h) * I;  // the lane's first instance in the block
  bool valid[I];
  T* colp[I];
#pragma unroll
  for (int s = 0; s < I; ++s) {
    const int k = kb + kk0 + s;
    valid[s] = j < Nz && k < K;
    colp[s] = t + (long)min(k, K - 1) * Ny * Nzp + j;
  }
  constexpr uint32_t bytes = (uint32_t)((CT + DT) * sizeof(T));
  const int nch = (Ny + YS_R - 1) / YS_R;
  constexpr int kPolls = 1 << 18;
  const bool leader = threadIdx.x == 0;
  if (leader) {
    for (int st = 0; st < YS_S; ++st) mbar_init(&bar[st], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // chunk g of the 2 * nch chunks (forward 0..nch-1 from row 0, back
  // nch..2nch-1 from row Ny-1) into stage g % YS_S
  // drop_first (a test hook): the first chunk's copy is never issued, so
  // its wait runs out (no copy of it is in flight to await afterwards)
  auto issue = [&](int g) {
    if (drop_first && g == 0) return;
    const int st = g % YS_S;
    mbar_expect_tx(&bar[st], bytes);
    const bool fwd = g < nch;
    const int lo = fwd ? g * YS_R : Ny - (g - nch + 1) * YS_R;  // first row (may be < 0)
    tma_load_2d(coef + st * CT, fwd ? &mLcol : &mLrow, &bar[st], j0, lo * 9);
    tma_load_3d(dat + st * DT, &mT, &bar[st], j0, lo, kb);
  };
  if (leader)
    for (int q = 0; q < YS_S && q < nch; ++q) issue(q);
  bool ok = true;
  // per chain: the previous row's value, the contributions b to the current
  // row, and a[m] the contributions to the rows m + 1 .. 7 further on
  T xp[I], b[I], a[I][7];
  auto reset = [&]() {
#pragma unroll
    for (int s = 0; s < I; ++s) {
      xp[s] = b[s] = T(0);
#pragma unroll
      for (int m = 0; m < 7; ++m) a[s][m] = T(0);
    }
  };
  reset();
  // one row r of the chunk in stage st; stored at colp[s] + off when in range
  auto row = [&](const T* cf, const T* dv, int r, long off, bool in) {
    const T* cr = cf + r * 9 * YS_C;
    T cm[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) cm[m] = cr[m * YS_C];
#pragma unroll
    for (int s = 0; s < I; ++s) {
      const T tt = (dv[((kk0 + s) * YS_R + r) * YS_C] - b[s]) * cm[0];
      const T x = fma_t<T>(-cm[1], xp[s], tt);
      if (valid[s] && in) colp[s][off] = x;
      b[s] = a[s][0];
#pragma unroll
      for (int m = 0; m < 6; ++m) a[s][m] = fma_t<T>(cm[m + 2], x, a[s][m + 1]);
      a[s][6] = cm[8] * x;
      xp[s] = x;
    }
  };
  int g = 0;
  for (; g < 2 * nch; ++g) {
    if (g == nch) {
      // the back sweep reads the forward result through the TMA: order the
      // stores first, then start its chunks
      fence_proxy_async_global();
      __syncthreads();
      if (leader)
        for (int q = nch; q < nch + YS_S && q < 2 * nch; ++q) issue(q);
      reset();
    }
    const int st = g % YS_S;
    ok = mbar_wait(&bar[st], (g / YS_S) & 1, first_polls);
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    const T* cf = coef + st * CT + c;
    const T* dv = dat + st * DT + c;
    if (g < nch) {
      const int i0 = g * YS_R;
      long off = (long)i0 * Nzp;
#pragma unroll
      for (int r = 0; r < YS_R; ++r) {
        row(cf, dv, r, off, i0 + r < Ny);
        off += Nzp;
      }
    } else {
      const int lo = Ny - (g - nch + 1) * YS_R;
      long off = (long)(lo + YS_R - 1) * Nzp;
#pragma unroll
      for (int r = YS_R - 1; r >= 0; --r) {
        row(cf, dv, r, off, lo + r >= 0);
        off -= Nzp;
      }
    }
    __syncthreads();  // every warp is done with stage st
    const int nx = g + YS_S;
    if (leader && (nx < nch || (nx >= nch + YS_S && nx < 2 * nch))) issue(nx);
  }
  if (!ok) {
    if (leader) {
      for (int q = 0; q < B && kb + q < K; ++q) atomicOr(status + kb + q, 4u);
      // let the loads already issued land before the block's shared memory goes
      for (int q = g; q < g + YS_S && q < 2 * nch; ++q)
        if (!(drop_first && q == 0)) mbar_wait(&bar[q % YS_S], (q / YS_S) & 1, kPolls);
    }
    __syncthreads();
  }
}

inline int ys_smem_bytes(int esize) { return YS_S * (YS_R * 9 * YS_C + YS_B * YS_R * YS_C) * esize + YS_S * 8; }

}  // namespace
}  // namespace scy
