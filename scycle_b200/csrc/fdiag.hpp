// Fast-diagonalisation preconditioner for K = -A.
//
// K is approximated by its separable part K_sep = (-Ly) (x) Mz + My (x) (-Lz)
// with 1D SBP-SAT operators Ly, Lz (coefficients averaged across the other
// direction) and diagonal weights My = Hy*yq, Mz = Hz*zr.  For constant mu
// on a grid whose y depends only on iy and z only on iz, K_sep differs from
// K only in the flattened-index mu3 average of the last z column.  With the
// generalised eigendecompositions (-Ly) Vy = My Vy Ly_lambda (Vy^T My Vy = I)
// and likewise for z,
//     K_sep^-1 = (Vy (x) Vz) diag(1/(ly_i + lz_j)) (Vy^T (x) Vz^T),
// applied to a body vector R (Ny x Nz, z fastest) either as four dense
// GEMMs, Z = Vy [ (Vy^T R Vz) ./ (ly_i + lz_j) ] Vz^T (when the y operator
// is not banded), or, in the banded form every order-2/4 SBP operator has,
// as Z = Vz [ per z mode j: (Ky + lz_j My)^-1 along y ] Vz^T R with the two
// z transforms on the integer tensor cores (ozaki.hpp).
#pragma once
#include <cublas_v2.h>

#include "ozaki.hpp"
#include "sbp_solver.hpp"

namespace scy {

struct FDPrecond {
  int Ny = 0, Nz = 0;
  int ready = 0;
  cublasHandle_t blas = nullptr;
  DevBuf Vy, Vz, inv_lam, t1, t2;          // FP64
  DevBuf Vy32, Vz32, inv_lam32, t1f, t2f;  // FP32 copies for the mixed path
  DevBuf r32;                              // FP32 copy of the residual
  // Banded form of the y part (ybanded = 1 when the symmetric part of the y
  // line operator has half-bandwidth <= 8): after the z transform the
  // operator splits into one banded SPD system per z mode j,
  // Ky + lz_j My, solved with its Cholesky factor L_j.  The factors are
  // kept for the TMA-fed sweeps, rows padded to Nzp (a multiple of 4)
  // values: row form [(i * 9 + m) * Nzp + j] = L_j(i, i - m) (Ny + 8
  // rows), column form [(i * 9 + m) * Nzp + j] = L_j(i + m, i) (Ny rows)
  // for m = 2..8; slot m = 0 holds 1 / L_j(i, i) in both, slot 1 the
  // coupling to the row a sweep processes just before row i over L_j(i, i):
  // L_j(i + 1, i) / L_j(i, i) in the row form (back sweep, rows going up),
  // L_j(i, i - 1) / L_j(i, i) in the column form (forward sweep).
  int ybanded = 0;
  int Nzp = 0;
  DevBuf Lrow, Lcol, Lrow32, Lcol32;
  // With the banded form, apply / apply32 run the z transforms on the
  // integer tensor cores (digit planes: kPlanes64 for apply, kPlanes32 for apply32) and the
  // TMA-fed sweeps of the batched ensemble (one instance) on the padded
  // transform t1p (Ny rows of Nzp values); no library GEMM.  A sweep wait
  // that runs out sets ys_status (the CG convergence test then fails).
  static constexpr int kPlanes64 = 7, kPlanes32 = 4;  // digit planes of apply (FP64-accurate) / apply32
  OzkOperand zx64, zx32, zw1_64, zw2_64, zw1_32, zw2_32;
  DevBuf t1p, t1pf, ys_status;
  CUtensorMap mLcol, mLrow, mT, mLcol32, mLrow32, mT32;
  ~FDPrecond();
  int build(const LevelHost& L, cudaStream_t s);
  // z = K_sep^-1 r (FP64)
  int apply(const double* r, double* z, cudaStream_t s);
  // z = K_sep^-1 r with FP32 GEMMs (z in FP32)
  int apply32(const double* r, float* z, cudaStream_t s);
};

}  // namespace scy
