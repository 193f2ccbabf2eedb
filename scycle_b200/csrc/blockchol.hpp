// Direct solve of an SBP-SAT operator by block Cholesky, for set-up solves
// whose operator is too ill-conditioned for an iterative method to match a
// direct solve (the power-law steady state, whose viscosity spans up to
// fourteen decades).  It is the device counterpart of the reference's
// KSPSolve with a direct Cholesky factorisation (linSolver = MUMPSCHOLESKY,
// PowerLaw::setupKSP powerLaw.cpp:1162-1215, used for the steady-state
// operator at :2111-2116).
//
// K = -A (symmetric positive definite; A as the cross form of
// build_cross_planes) is block tridiagonal once the y lines are grouped in
// blocks of 8 (the cross form couples lines at most 8 apart): diagonal
// blocks D_I and sub-diagonal blocks E_I = K[I][I-1], dense on the device
// (column-major), assembled there from the cross planes.  The factor is
//   Lc_0 Lc_0^T = D_0,  B_I = E_I Lc_{I-1}^-T,  Lc_I Lc_I^T = D_I - B_I B_I^T
// (cuBLAS trsm and syrk, cuSOLVER potrf), and K x = f is the forward and
// backward block substitution (trsv and gemv).  Memory: about 16 m^2 bytes
// per block of m = 8 Nz rows; 8.4 GB at 401 x 401.
#pragma once
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <vector>

#include "sbp_host.hpp"
#include "sbp_solver.hpp"

namespace scy {

struct BlockChol {
  static constexpr int kLines = 8;
  int Ny = 0, Nz = 0, nb = 0, mmax = 0;
  std::vector<int> l0, nl;  // first line and lines of each block
  DevBuf Lc, B;             // nb factors and nb - 1 couplings, mmax x mmax each (column-major)
  DevBuf planes, work, info, tmp;
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t sol = nullptr;
  ~BlockChol();
  // bytes the factor of an Ny x Nz operator holds
  static double bytes_for(int Ny, int Nz);
  // factorises K = -A of level h on stream s
  int factor(const LevelHost& h, cudaStream_t s);
  // x = A^-1 rhs (device vectors of Ny*Nz; x may not alias rhs)
  int solve(const double* rhs, double* x, cudaStream_t s);
};

}  // namespace scy
