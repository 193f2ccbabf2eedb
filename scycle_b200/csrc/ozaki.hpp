// FP64-accurate dense products on the integer tensor cores (tcgen05.mma
// kind::i8), for the z transforms of the fast-diagonalisation
// preconditioner.
//
// Each row of an FP64 operand is scaled by a power of two 2^e (e chosen so
// that max|x| 2^-e lies in [1/4, 1/2)) and written as S signed 8-bit digits,
//     x = 2^e * sum_{i=1..S} d_i 2^(-7 i) + r,   d_i in [-64, 64],
//     |r| <= 2^(e - 7 S - 1),
// extracted exactly in FP64 by repeated round-to-nearest (the splitting of
// Ozaki, Ogita, Oishi and Rump, "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59 (2012), with integer digits).  A
// product of two digit planes is exact in 32-bit integers (|d w| <= 2^12,
// at most 2^10 terms), so
//     sum_k X[r,k] W[c,k] ~= 2^(ex_r + ew_c) sum_{g=0..S-1} 2^(-7 (g+2)) P_g,
//     P_g = sum_{i+j = g+2} D_i W_j^T,
// where the S(S+1)/2 digit products with i + j <= S + 1 are accumulated
// group by group in tensor memory and combined in FP64 by the epilogue.
// The dropped products and the digit remainders leave a relative error of
// about 100^-S per row (S = 7: ~1e-13; S = 4: ~1e-7).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "sbp_solver.hpp"

namespace scy {

// One operand in digit form: S planes of rows x Kp digits (signed bytes,
// or bf16; Kp = K rounded up to 32 bytes of digits, zero beyond K), a
// power-of-two exponent per row, and the 3D TMA map (digits of a row, rows,
// planes) with a box of 64 bytes x box_rows rows x S planes (zero-filled
// past Kp) and 64-byte swizzling (the K-major canonical layout the tensor
// cores read).
struct OzkOperand {
  DevBuf dig, expo;
  int S = 0, rows = 0, K = 0, Kp = 0, box_rows = 0, box_rows_pair = 0;
  int esz = 1;  // bytes of a digit: 1 (signed 8-bit) or 2 (bf16)
  long plane = 0;  // digits of one plane (rows x Kp)
  CUtensorMap map, map_pair;
  // box_rows: 128 for the row operand (X), the column tile width of S
  // (ozk_cols_per_tile) for the weights (W); Kp = K rounded up to 32 bytes
  // of digits (one MMA K step)
  int alloc(int S, int rows, int K, int box_rows, int esz = 1);
  // the weights' operand (W) with the maps of both product shapes
  int alloc_weights(int S, int rows, int K, int esz = 1);
};

// bf16 digits give exact FP32 accumulation for S planes and K (every
// partial sum below 2^24: S * 64 * 64 * Kp < 2^24, Kp = K rounded up to 16)
bool ozk_bf16_exact(int S, int K);

// column tile width of the product for S digit planes: one CTA per SM
// (S * width <= 512 tensor-memory columns) or, for S <= 5, two CTAs per SM
// (S * width <= 256; 0 for S > 5)
int ozk_cols_per_tile(int S);
int ozk_cols_per_tile_pair(int S);

// sets the kernels' shared-memory limit for S planes on the current device
// (done by the first product too; call it before capturing one in a graph)
int ozk_prepare(int S);

// digits of the rows of a device matrix X (rows x K, row stride ldx)
int ozk_split(OzkOperand& o, const double* X, long ldx, cudaStream_t s);
int ozk_split(OzkOperand& o, const float* X, long ldx, cudaStream_t s);
// digits of the rows of a host matrix W (rows x K, row stride ldw); set-up
int ozk_set_host(OzkOperand& o, const double* W, long ldw, cudaStream_t s);

// D[r, c] = sum_k X[r, k] W[c, k] for r < x.rows, c < cout (<= w.rows),
// D of row stride ldd.  x.S == w.S.  A wait inside the kernel that runs out
// (2^20 polls) sets `bit` in status[r / rows_per_status] for the rows of its
// tile when status is given.  pair = 1 takes the two-CTAs-per-SM shape, pair
// = 2 the persistent shape with double-buffered accumulators (both S <= 5,
// W made by alloc_weights); the shapes give identical results.
int ozk_gemm(const OzkOperand& x, const OzkOperand& w, double* D, long ldd, int cout, cudaStream_t s,
             unsigned* status = nullptr, int rows_per_status = 1, unsigned bit = 4u, int pair = 0);
int ozk_gemm(const OzkOperand& x, const OzkOperand& w, float* D, long ldd, int cout, cudaStream_t s,
             unsigned* status = nullptr, int rows_per_status = 1, unsigned bit = 4u, int pair = 0);

}  // namespace scy
