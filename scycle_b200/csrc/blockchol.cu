// Block Cholesky direct solve of an SBP-SAT operator (see blockchol.hpp).
#include "blockchol.hpp"

#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace scy {

#define BC_BLAS(call)                                                                      \
  do {                                                                                     \
    cublasStatus_t b_ = (call);                                                            \
    if (b_ != CUBLAS_STATUS_SUCCESS) {                                                     \
      ::scy::set_error("%s:%d: %s failed (%d)", __FILE__, __LINE__, #call, (int)b_);      \
      return SCY_ERR_CUDA;                                                                 \
    }                                                                                      \
  } while (0)
#define BC_SOLVER(call)                                                                    \
  do {                                                                                     \
    cusolverStatus_t c_ = (call);                                                          \
    if (c_ != CUSOLVER_STATUS_SUCCESS) {                                                   \
      ::scy::set_error("%s:%d: %s failed (%d)", __FILE__, __LINE__, #call, (int)c_);      \
      return SCY_ERR_CUDA;                                                                 \
    }                                                                                      \
  } while (0)

namespace {

// Dense block of K = -A: rows = nodes of lines [ri, ri + rn), columns =
// nodes of lines [cj, cj + cn), column-major with leading dimension ld
// (zero-filled beforehand).  One thread per row node writes its row's
// entries from the cross form (C: 33 planes of N; y offsets -8..8 in planes
// 0..16, z offsets -8..-1 in 17..24 and 1..8 in 25..32).
__global__ void bc_assemble_kernel(const double* __restrict__ C, int Ny, int Nz, int ri, int rn, int cj, int cn,
                                   double* __restrict__ out, long ld) {
  const long N = (long)Ny * Nz;
  const long rows = (long)rn * Nz;
  for (long r = blockIdx.x * (long)blockDim.x + threadIdx.x; r < rows; r += (long)gridDim.x * blockDim.x) {
    const int iy = ri + (int)(r / Nz), iz = (int)(r % Nz);
    const long node = (long)iy * Nz + iz;
    for (int o = -8; o <= 8; ++o) {
      const int jy = iy + o;
      if (jy < cj || jy >= cj + cn || jy >= Ny) continue;
      const long c = (long)(jy - cj) * Nz + iz;
      out[c * ld + r] = -C[(long)(o + 8) * N + node];
    }
    if (iy >= cj && iy < cj + cn) {
      for (int o = -8; o <= 8; ++o) {
        const int jz = iz + o;
        if (o == 0 || jz < 0 || jz >= Nz) continue;
        const long c = (long)(iy - cj) * Nz + jz;
        out[c * ld + r] = -C[(long)(o < 0 ? 25 + o : 24 + o) * N + node];
      }
    }
  }
}

__global__ void bc_negate_kernel(const double* __restrict__ a, double* __restrict__ b, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) b[i] = -a[i];
}

}  // namespace

BlockChol::~BlockChol() {
  if (blas) cublasDestroy(blas);
  if (sol) cusolverDnDestroy(sol);
}

double BlockChol::bytes_for(int Ny, int Nz) {
  const int nb = (Ny + kLines - 1) / kLines;
  const double m = (double)std::min(Ny, kLines) * Nz;
  return (2.0 * nb - 1.0) * m * m * 8.0;
}

int BlockChol::factor(const LevelHost& h, cudaStream_t s) {
  Ny = h.Ny;
  Nz = h.Nz;
  nb = (Ny + kLines - 1) / kLines;
  l0.assign(nb, 0);
  nl.assign(nb, 0);
  for (int I = 0; I < nb; ++I) {
    l0[I] = I * kLines;
    nl[I] = std::min(kLines, Ny - l0[I]);
  }
  mmax = std::min(Ny, kLines) * Nz;
  const long mm = (long)mmax * mmax;
  {
    std::vector<double> C;
    build_cross_planes(h, C);
    SCY_TRY(planes.alloc(C.size() * sizeof(double)));
    SCY_CUDA_TRY(cudaMemcpyAsync(planes.p, C.data(), C.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    SCY_CUDA_TRY(cudaStreamSynchronize(s));
  }
  SCY_TRY(Lc.alloc((size_t)nb * mm * sizeof(double)));
  SCY_TRY(B.alloc((size_t)std::max(1, nb - 1) * mm * sizeof(double)));
  SCY_TRY(info.alloc(sizeof(int)));
  SCY_TRY(tmp.alloc((size_t)Ny * Nz * sizeof(double)));
  if (!blas) BC_BLAS(cublasCreate(&blas));
  if (!sol) BC_SOLVER(cusolverDnCreate(&sol));
  BC_BLAS(cublasSetStream(blas, s));
  BC_SOLVER(cusolverDnSetStream(sol, s));
  int lwork = 0;
  BC_SOLVER(cusolverDnDpotrf_bufferSize(sol, CUBLAS_FILL_MODE_LOWER, mmax, Lc.as<double>(), mmax, &lwork));
  SCY_TRY(work.alloc((size_t)std::max(1, lwork) * sizeof(double)));
  const double* Cp = planes.as<double>();
  const double one = 1.0, mone = -1.0;
  for (int I = 0; I < nb; ++I) {
    const int m = nl[I] * Nz;
    double* D = Lc.as<double>() + (long)I * mm;
    SCY_CUDA_TRY(cudaMemsetAsync(D, 0, mm * sizeof(double), s));
    bc_assemble_kernel<<<grid_for((long)m), kBlock, 0, s>>>(Cp, Ny, Nz, l0[I], nl[I], l0[I], nl[I], D, mmax);
    SCY_LAUNCH_CHECK();
    if (I > 0) {
      const int mp = nl[I - 1] * Nz;
      double* E = B.as<double>() + (long)(I - 1) * mm;
      SCY_CUDA_TRY(cudaMemsetAsync(E, 0, mm * sizeof(double), s));
      bc_assemble_kernel<<<grid_for((long)m), kBlock, 0, s>>>(Cp, Ny, Nz, l0[I], nl[I], l0[I - 1], nl[I - 1], E,
                                                               mmax);
      SCY_LAUNCH_CHECK();
      const double* Lp = Lc.as<double>() + (long)(I - 1) * mm;
      // B_I = E_I Lc_{I-1}^-T ; D_I -= B_I B_I^T
      BC_BLAS(cublasDtrsm(blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT, m, mp,
                          &one, Lp, mmax, E, mmax));
      BC_BLAS(cublasDsyrk(blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, m, mp, &mone, E, mmax, &one, D, mmax));
    }
    BC_SOLVER(cusolverDnDpotrf(sol, CUBLAS_FILL_MODE_LOWER, m, D, mmax, work.as<double>(), lwork, info.as<int>()));
    int hinfo = 0;
    SCY_CUDA_TRY(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SCY_CUDA_TRY(cudaStreamSynchronize(s));
    if (hinfo != 0) {
      set_error("block Cholesky: block %d of %d is not positive definite (potrf info %d)", I, nb, hinfo);
      return SCY_ERR_NONFINITE;
    }
  }
  planes.release();
  return SCY_OK;
}

int BlockChol::solve(const double* rhs, double* x, cudaStream_t s) {
  if (!nb) {
    set_error("block Cholesky: not factorised");
    return SCY_ERR_STATE;
  }
  const long N = (long)Ny * Nz, mm = (long)mmax * mmax;
  BC_BLAS(cublasSetStream(blas, s));
  // K x = -rhs (K = -A): forward y_I = Lc_I^-1 (f_I - B_I y_{I-1}), then
  // backward x_I = Lc_I^-T (y_I - B_{I+1}^T x_{I+1}), in place in x
  bc_negate_kernel<<<grid_for(N), kBlock, 0, s>>>(rhs, x, N);
  SCY_LAUNCH_CHECK();
  const double one = 1.0, mone = -1.0;
  for (int I = 0; I < nb; ++I) {
    const int m = nl[I] * Nz;
    double* xi = x + (long)l0[I] * Nz;
    if (I > 0) {
      const int mp = nl[I - 1] * Nz;
      BC_BLAS(cublasDgemv(blas, CUBLAS_OP_N, m, mp, &mone, B.as<double>() + (long)(I - 1) * mm, mmax,
                          x + (long)l0[I - 1] * Nz, 1, &one, xi, 1));
    }
    BC_BLAS(cublasDtrsv(blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, m,
                        Lc.as<double>() + (long)I * mm, mmax, xi, 1));
  }
  for (int I = nb - 1; I >= 0; --I) {
    const int m = nl[I] * Nz;
    double* xi = x + (long)l0[I] * Nz;
    if (I < nb - 1) {
      const int mn = nl[I + 1] * Nz;
      BC_BLAS(cublasDgemv(blas, CUBLAS_OP_T, mn, m, &mone, B.as<double>() + (long)I * mm, mmax,
                          x + (long)l0[I + 1] * Nz, 1, &one, xi, 1));
    }
    BC_BLAS(cublasDtrsv(blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT, m,
                        Lc.as<double>() + (long)I * mm, mmax, xi, 1));
  }
  return SCY_OK;
}

}  // namespace scy
