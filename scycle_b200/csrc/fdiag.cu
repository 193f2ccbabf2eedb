// Fast-diagonalisation preconditioner (see fdiag.hpp).
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "common.cuh"
#include "fdiag.hpp"
#include "tma.cuh"
#include "ysolve.cuh"

namespace scy {

#define SCY_BLAS_TRY(call)                                                   \
  do {                                                                       \
    cublasStatus_t b_ = (call);                                              \
    if (b_ != CUBLAS_STATUS_SUCCESS) {                                       \
      ::scy::set_error("%s:%d: %s failed (%d)", __FILE__, __LINE__, #call,   \
                       (int)b_);                                             \
      return SCY_ERR_CUDA;                                                   \
    }                                                                        \
  } while (0)

namespace {

// Dense 1D operator of one direction with averaged coefficients c1, m31
// (column-major n x n, symmetric): the y or z part of A restricted to a line,
// SAT terms included.  Entry (i, l) of L = sum_k Q[i,k] c1_k D[k,l]
//   - R3T[i,k] w3_k m31_k R3[k,l] - R4T[i,k] w4_k c1_k R4[k,l] + SAT.
std::vector<double> dense_line_operator(const DirTables& t, const std::vector<double>& c1,
                                        const std::vector<double>& m31, int bc_lo, int bc_hi) {
  const int n = t.n;
  std::vector<double> Lm((size_t)n * n, 0.0);
  auto at = [&](int i, int l) -> double& { return Lm[(size_t)l * n + i]; };
  auto band = [&](const std::vector<double>& b, int row, int col) {
    int off = col - row;
    if (off < -kHalf || off > kHalf || b.empty()) return 0.0;
    return b[(size_t)row * kBand + off + kHalf];
  };
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < kBand; ++j) {
      int k = i + j - kHalf;
      if (k < 0 || k >= n) continue;
      const double q = t.Q[(size_t)i * kBand + j], r3 = t.R3T[(size_t)i * kBand + j],
                   r4 = t.R4T[(size_t)i * kBand + j];
      for (int jj = 0; jj < kBand; ++jj) {
        int l = k + jj - kHalf;
        if (l < 0 || l >= n) continue;
        double v = q * c1[k] * band(t.D, k, l) - r3 * t.w3[k] * m31[k] * band(t.R3, k, l) -
                   r4 * t.w4[k] * c1[k] * band(t.R4, k, l);
        at(i, l) += v;
      }
    }
  if (bc_lo == 0) {
    for (int i = 0; i < kBand && i < n; ++i) at(i, 0) += (t.bs0[i] + (i == 0 ? t.alphaD : 0.0)) * c1[0];
  } else {
    for (int l = 0; l < n; ++l) at(0, l) += c1[0] * band(t.D, 0, l);
  }
  if (bc_hi == 0) {
    for (int i = std::max(0, n - kBand); i < n; ++i)
      at(i, n - 1) += (t.bsN[i - (n - kBand)] + (i == n - 1 ? t.alphaD : 0.0)) * c1[n - 1];
  } else {
    for (int l = 0; l < n; ++l) at(n - 1, l) -= c1[n - 1] * band(t.D, n - 1, l);
  }
  return Lm;
}

// Generalised eigendecomposition of (-L, M): returns V (column-major,
// V^T M V = I) and the eigenvalues.
int gen_eig(std::vector<double>& negL, const std::vector<double>& M, int n, std::vector<double>& V,
            std::vector<double>& lam, cudaStream_t s) {
  std::vector<double> S((size_t)n * n);
  for (int l = 0; l < n; ++l)
    for (int i = 0; i < n; ++i) {
      double a = negL[(size_t)l * n + i], b = negL[(size_t)i * n + l];
      S[(size_t)l * n + i] = 0.5 * (a + b) / std::sqrt(M[i] * M[l]);
    }
  cusolverDnHandle_t h = nullptr;
  if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) {
    set_error("cusolverDnCreate failed");
    return SCY_ERR_CUDA;
  }
  cusolverDnSetStream(h, s);
  DevBuf dS, dW, dinfo, dwork;
  int rc = SCY_OK;
  do {
    if ((rc = dS.alloc(S.size() * 8)) != SCY_OK) break;
    if ((rc = dW.alloc((size_t)n * 8)) != SCY_OK) break;
    if ((rc = dinfo.alloc(16)) != SCY_OK) break;
    if (cudaMemcpyAsync(dS.p, S.data(), S.size() * 8, cudaMemcpyHostToDevice, s) != cudaSuccess) {
      rc = SCY_ERR_CUDA;
      set_error("copy to the eigensolver failed");
      break;
    }
    int lwork = 0;
    if (cusolverDnDsyevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, dS.as<double>(), n,
                                    dW.as<double>(), &lwork) != CUSOLVER_STATUS_SUCCESS) {
      rc = SCY_ERR_CUDA;
      set_error("cusolverDnDsyevd_bufferSize failed");
      break;
    }
    if ((rc = dwork.alloc((size_t)std::max(lwork, 1) * 8)) != SCY_OK) break;
    if (cusolverDnDsyevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, dS.as<double>(), n,
                         dW.as<double>(), dwork.as<double>(), lwork, dinfo.as<int>()) != CUSOLVER_STATUS_SUCCESS) {
      rc = SCY_ERR_CUDA;
      set_error("cusolverDnDsyevd failed");
      break;
    }
    int info = 0;
    lam.resize(n);
    cudaMemcpyAsync(&info, dinfo.p, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(lam.data(), dW.p, (size_t)n * 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(S.data(), dS.p, S.size() * 8, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      rc = SCY_ERR_CUDA;
      set_error("eigensolver synchronisation failed");
      break;
    }
    if (info != 0) {
      rc = SCY_ERR_ARG;
      set_error("eigensolver reported info = %d", info);
      break;
    }
  } while (0);
  cusolverDnDestroy(h);
  if (rc != SCY_OK) return rc;
  V.resize((size_t)n * n);
  for (int c = 0; c < n; ++c)
    for (int i = 0; i < n; ++i) V[(size_t)c * n + i] = S[(size_t)c * n + i] / std::sqrt(M[i]);
  return SCY_OK;
}

template <typename T>
__global__ void scale_by_kernel(T* __restrict__ x, const T* __restrict__ s, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) x[i] *= s[i];
}

__global__ void to_f32_kernel(const double* __restrict__ a, float* __restrict__ b, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

template <typename T>
int upload_as(DevBuf& b, const std::vector<double>& v, cudaStream_t s) {
  std::vector<T> t(v.begin(), v.end());
  SCY_TRY(b.alloc(t.size() * sizeof(T)));
  SCY_CUDA_TRY(cudaMemcpyAsync(b.p, t.data(), t.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  return SCY_OK;
}
}  // namespace

FDPrecond::~FDPrecond() {
  if (blas) cublasDestroy(blas);
}

namespace {
// Product fit mu(y, z) ~ a(y) b(z) for a non-constant shear modulus (or
// viscosity): log mu ~ alpha(iy) + beta(iz) by alternating midranges, which
// drives down the largest log misfit (the spread of mu / (a b) bounds the
// condition number of the preconditioned operator).  a = b = 1 for constant
// or non-positive mu, so the averaged coefficients below are then the
// plain means.
void product_fit(const LevelHost& L, std::vector<double>& a, std::vector<double>& b) {
  const int Ny = L.Ny, Nz = L.Nz;
  a.assign(Ny, 1.0);
  b.assign(Nz, 1.0);
  bool varies = false;
  for (size_t i = 0; i < L.mu.size(); ++i) {
    if (!(L.mu[i] > 0)) return;
    if (L.mu[i] != L.mu[0]) varies = true;
  }
  if (!varies) return;
  std::vector<double> lg(L.mu.size()), al(Ny, 0.0), be(Nz, 0.0);
  for (size_t i = 0; i < lg.size(); ++i) lg[i] = std::log(L.mu[i]);
  for (int round = 0; round < 60; ++round) {
    for (int iy = 0; iy < Ny; ++iy) {
      double lo = INFINITY, hi = -INFINITY;
      for (int iz = 0; iz < Nz; ++iz) {
        const double v = lg[(size_t)iy * Nz + iz] - be[iz];
        lo = std::min(lo, v);
        hi = std::max(hi, v);
      }
      al[iy] = 0.5 * (lo + hi);
    }
    for (int iz = 0; iz < Nz; ++iz) {
      double lo = INFINITY, hi = -INFINITY;
      for (int iy = 0; iy < Ny; ++iy) {
        const double v = lg[(size_t)iy * Nz + iz] - al[iy];
        lo = std::min(lo, v);
        hi = std::max(hi, v);
      }
      be[iz] = 0.5 * (lo + hi);
    }
  }
  for (int iy = 0; iy < Ny; ++iy) a[iy] = std::exp(al[iy]);
  for (int iz = 0; iz < Nz; ++iz) b[iz] = std::exp(be[iz]);
}
}  // namespace

int FDPrecond::build(const LevelHost& L, cudaStream_t s) {
  Ny = L.Ny;
  Nz = L.Nz;
  const size_t N = (size_t)Ny * Nz;
  // Averaged 1D coefficients and weights of the separable operator
  // Ly(cy1) x Mz + My x Lz(cz1).  Both directions' coefficients carry mu
  // (cy = mu qy, cz = mu rz); with the product fit mu ~ a(y) b(z) the y
  // operator takes cy / b and the z mass b, the z operator cz / a and the y
  // mass a, which is exact when mu is a product and the metrics separate.
  std::vector<double> fa, fb;
  product_fit(L, fa, fb);
  std::vector<double> cy1(Ny, 0), m3y1(Ny, 0), My(Ny, 0), cz1(Nz, 0), m3z1(Nz, 0), Mz(Nz, 0);
  for (int iy = 0; iy < Ny; ++iy)
    for (int iz = 0; iz < Nz; ++iz) {
      size_t i = (size_t)iy * Nz + iz;
      cy1[iy] += L.cy[i] / fb[iz] / Nz;
      m3y1[iy] += L.m3y[i] / fb[iz] / Nz;
      My[iy] += L.wz[i] / Nz;
      cz1[iz] += L.cz[i] / fa[iy] / Ny;
      m3z1[iz] += L.m3z[i] / fa[iy] / Ny;
      Mz[iz] += L.wy[i] / Ny;
    }
  for (int iy = 0; iy < Ny; ++iy) My[iy] *= fa[iy];
  for (int iz = 0; iz < Nz; ++iz) Mz[iz] *= fb[iz];
  std::vector<double> Ly = dense_line_operator(L.ty, cy1, m3y1, L.bc[2], L.bc[0]);
  std::vector<double> Lz = dense_line_operator(L.tz, cz1, m3z1, L.bc[1], L.bc[3]);
  for (auto& v : Ly) v = -v;
  for (auto& v : Lz) v = -v;
  std::vector<double> Vyh, Vzh, ly, lz;
  SCY_TRY(gen_eig(Ly, My, Ny, Vyh, ly, s));
  SCY_TRY(gen_eig(Lz, Mz, Nz, Vzh, lz, s));
  std::vector<double> il(N);
  for (int iy = 0; iy < Ny; ++iy)
    for (int iz = 0; iz < Nz; ++iz) {
      double d = ly[iy] + lz[iz];
      if (!(d > 0)) {
        set_error("separable operator is singular (eigenvalue sum %g): no Dirichlet boundary?", d);
        return SCY_ERR_ARG;
      }
      il[(size_t)iy * Nz + iz] = 1.0 / d;
    }
  // banded Cholesky factors of Ky + lz_j My, Ky = (Ly + Ly^T) / 2
  {
    const int bw = 8;
    bool banded = true;
    auto ks = [&](int i, int l) { return 0.5 * (Ly[(size_t)l * Ny + i] + Ly[(size_t)i * Ny + l]); };
    for (int l = 0; l < Ny && banded; ++l)
      for (int i = 0; i < Ny; ++i)
        if (std::abs(i - l) > bw && ks(i, l) != 0.0) {
          banded = false;
          break;
        }
    if (banded) {
      std::vector<double> Lbh((size_t)(Ny + bw) * 9 * Nz, 0.0);
      std::vector<double> c((size_t)Ny * (bw + 1));  // c[i*(bw+1) + k] = L(i, i-k)
      bool spd = true;
      for (int j = 0; j < Nz && spd; ++j) {
        for (int i = 0; i < Ny && spd; ++i)
          for (int col = std::max(0, i - bw); col <= i; ++col) {
            double sum = ks(i, col) + (i == col ? lz[j] * My[i] : 0.0);
            for (int p = std::max(0, i - bw); p < col; ++p) {
              if (col - p > bw) continue;
              sum -= c[(size_t)i * (bw + 1) + (i - p)] * c[(size_t)col * (bw + 1) + (col - p)];
            }
            if (col == i) {
              if (!(sum > 0)) {
                spd = false;
                break;
              }
              c[(size_t)i * (bw + 1)] = std::sqrt(sum);
            } else {
              c[(size_t)i * (bw + 1) + (i - col)] = sum / c[(size_t)col * (bw + 1)];
            }
          }
        for (int i = 0; i < Ny && spd; ++i)
          for (int k = 0; k <= bw; ++k) {
            double v = c[(size_t)i * (bw + 1) + k];
            if (k == 0) v = 1.0 / v;
            if (i - k < 0 && k > 0) v = 0.0;
            Lbh[((size_t)i * 9 + k) * Nz + j] = v;
          }
      }
      if (spd) {
        // padded row and column forms for the TMA-fed sweeps
        Nzp = (Nz + 3) / 4 * 4;
        std::vector<double> Lr((size_t)(Ny + bw) * 9 * Nzp, 0.0), Lc((size_t)Ny * 9 * Nzp, 0.0);
        // slot 1 holds the coupling to the row processed just before,
        // divided by L_ii: L(i+1, i) / L_ii going up (row form), L(i, i-1) /
        // L_ii going down (column form)
        for (int i = 0; i < Ny + bw; ++i)
          for (int k = 0; k < 9; ++k)
            for (int j = 0; j < Nz; ++j) {
              double v = Lbh[((size_t)i * 9 + k) * Nz + j];
              if (k == 1)
                v = i + 1 < Ny + bw ? Lbh[((size_t)(i + 1) * 9 + 1) * Nz + j] * Lbh[((size_t)i * 9) * Nz + j] : 0.0;
              Lr[((size_t)i * 9 + k) * Nzp + j] = v;
            }
        for (int i = 0; i < Ny; ++i)
          for (int j = 0; j < Nz; ++j) {
            Lc[((size_t)i * 9) * Nzp + j] = Lbh[((size_t)i * 9) * Nz + j];
            Lc[((size_t)i * 9 + 1) * Nzp + j] = Lbh[((size_t)i * 9 + 1) * Nz + j] * Lbh[((size_t)i * 9) * Nz + j];
            for (int m = 2; m <= bw; ++m) Lc[((size_t)i * 9 + m) * Nzp + j] = Lbh[((size_t)(i + m) * 9 + m) * Nz + j];
          }
        SCY_TRY(upload_as<double>(Lrow, Lr, s));
        SCY_TRY(upload_as<double>(Lcol, Lc, s));
        SCY_TRY(upload_as<float>(Lrow32, Lr, s));
        SCY_TRY(upload_as<float>(Lcol32, Lc, s));
        ybanded = 1;
      }
    }
  }
  SCY_TRY(upload_as<double>(Vy, Vyh, s));
  SCY_TRY(upload_as<double>(Vz, Vzh, s));
  SCY_TRY(upload_as<double>(inv_lam, il, s));
  SCY_TRY(upload_as<float>(Vy32, Vyh, s));
  SCY_TRY(upload_as<float>(Vz32, Vzh, s));
  SCY_TRY(upload_as<float>(inv_lam32, il, s));
  if (ybanded) {
    SCY_TRY(t1p.alloc((size_t)Ny * Nzp * 8));
    SCY_TRY(t1pf.alloc((size_t)Ny * Nzp * 4));
    SCY_CUDA_TRY(cudaMemset(t1p.p, 0, (size_t)Ny * Nzp * 8));
    SCY_CUDA_TRY(cudaMemset(t1pf.p, 0, (size_t)Ny * Nzp * 4));
    std::vector<double> vzt((size_t)Nz * Nz);
    for (int k = 0; k < Nz; ++k)
      for (int m = 0; m < Nz; ++m) vzt[(size_t)k * Nz + m] = Vzh[(size_t)m * Nz + k];
    for (int S : {kPlanes64, kPlanes32}) {
      OzkOperand& x = S == kPlanes64 ? zx64 : zx32;
      OzkOperand& w1 = S == kPlanes64 ? zw1_64 : zw1_32;
      OzkOperand& w2 = S == kPlanes64 ? zw2_64 : zw2_32;
      SCY_TRY(x.alloc(S, Ny, Nz, 128));
      SCY_TRY(w1.alloc(S, Nz, Nz, ozk_cols_per_tile(S)));
      SCY_TRY(w2.alloc(S, Nz, Nz, ozk_cols_per_tile(S)));
      SCY_TRY(ozk_set_host(w1, Vzh.data(), Nz, s));  // rows of Vz^T: the columns of Vz
      SCY_TRY(ozk_set_host(w2, vzt.data(), Nz, s));  // rows of Vz
      SCY_TRY(ozk_prepare(S));
    }
    // tile maps of the TMA-fed sweeps over the one instance's transform
    const CUtensorMapDataType d64 = CU_TENSOR_MAP_DATA_TYPE_FLOAT64, d32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    SCY_TRY(tma_map_2d(&mLcol, Lcol.p, d64, 8, Nz, (long)Ny * 9, (long)Nzp * 8, YS_C, YS_R * 9));
    SCY_TRY(tma_map_2d(&mLrow, Lrow.p, d64, 8, Nz, (long)(Ny + 8) * 9, (long)Nzp * 8, YS_C, YS_R * 9));
    SCY_TRY(tma_map_3d(&mT, t1p.p, d64, Nz, Ny, 1, (long)Nzp * 8, (long)Ny * Nzp * 8, YS_C, YS_R, YS_B));
    SCY_TRY(tma_map_2d(&mLcol32, Lcol32.p, d32, 4, Nz, (long)Ny * 9, (long)Nzp * 4, YS_C, YS_R * 9));
    SCY_TRY(tma_map_2d(&mLrow32, Lrow32.p, d32, 4, Nz, (long)(Ny + 8) * 9, (long)Nzp * 4, YS_C, YS_R * 9));
    SCY_TRY(tma_map_3d(&mT32, t1pf.p, d32, Nz, Ny, 1, (long)Nzp * 4, (long)Ny * Nzp * 4, YS_C, YS_R, YS_B));
    SCY_CUDA_TRY(cudaFuncSetAttribute(b_ysolve_tma_kernel<double, YS_I, YS_W>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, ys_smem_bytes(8)));
    SCY_CUDA_TRY(cudaFuncSetAttribute(b_ysolve_tma_kernel<float, YS_I, YS_W>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, ys_smem_bytes(4)));
    SCY_TRY(ys_status.alloc(sizeof(unsigned)));
    SCY_CUDA_TRY(cudaMemset(ys_status.p, 0, sizeof(unsigned)));
  }
  SCY_TRY(t1.alloc(N * 8));
  SCY_TRY(t2.alloc(N * 8));
  SCY_TRY(t1f.alloc(N * 4));
  SCY_TRY(t2f.alloc(N * 4));
  SCY_TRY(r32.alloc(N * 4));
  if (!blas) SCY_BLAS_TRY(cublasCreate(&blas));
  ready = 1;
  return SCY_OK;
}

int FDPrecond::apply(const double* r, double* z, cudaStream_t s) {
  if (ybanded) {
    double* t = t1p.as<double>();
    SCY_TRY(ozk_split(zx64, r, Nz, s));
    SCY_TRY(ozk_gemm(zx64, zw1_64, t, Nzp, Nz, s));
    b_ysolve_tma_kernel<double, YS_I, YS_W><<<dim3((Nz + YS_C - 1) / YS_C, 1), 32 * YS_W, ys_smem_bytes(8), s>>>(
        mLcol, mLrow, mT, t, Ny, Nz, Nzp, 1, ys_status.as<unsigned>());
    SCY_LAUNCH_CHECK();
    SCY_TRY(ozk_split(zx64, (const double*)t, Nzp, s));
    SCY_TRY(ozk_gemm(zx64, zw2_64, z, Nz, Nz, s));
    return SCY_OK;
  }
  SCY_BLAS_TRY(cublasSetStream(blas, s));
  SCY_BLAS_TRY(cublasSetMathMode(blas, CUBLAS_DEFAULT_MATH));
  const double one = 1.0, zero = 0.0;
  double* a = t1.as<double>();
  double* b = t2.as<double>();
  const double* vy = Vy.as<double>();
  const double* vz = Vz.as<double>();
  // column-major views: body vector = Nz x Ny matrix (z fastest)
  SCY_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, Nz, Ny, Nz, &one, vz, Nz, r, Nz, &zero, a, Nz));
  SCY_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, Nz, Ny, Ny, &one, a, Nz, vy, Ny, &zero, b, Nz));
  count_launch();
  count_launch();
  long n = (long)Ny * Nz;
  scale_by_kernel<double><<<grid_for(n), 256, 0, s>>>(b, inv_lam.as<double>(), n);
  SCY_LAUNCH_CHECK();
  SCY_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_T, Nz, Ny, Ny, &one, b, Nz, vy, Ny, &zero, a, Nz));
  SCY_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, Nz, Ny, Nz, &one, vz, Nz, a, Nz, &zero, z, Nz));
  count_launch();
  count_launch();
  return SCY_OK;
}

int FDPrecond::apply32(const double* r, float* z, cudaStream_t s) {
  if (ybanded) {
    float* t = t1pf.as<float>();
    SCY_TRY(ozk_split(zx32, r, Nz, s));
    SCY_TRY(ozk_gemm(zx32, zw1_32, t, Nzp, Nz, s));
    b_ysolve_tma_kernel<float, YS_I, YS_W><<<dim3((Nz + YS_C - 1) / YS_C, 1), 32 * YS_W, ys_smem_bytes(4), s>>>(
        mLcol32, mLrow32, mT32, t, Ny, Nz, Nzp, 1, ys_status.as<unsigned>());
    SCY_LAUNCH_CHECK();
    SCY_TRY(ozk_split(zx32, (const float*)t, Nzp, s));
    SCY_TRY(ozk_gemm(zx32, zw2_32, z, Nz, Nz, s));
    return SCY_OK;
  }
  SCY_BLAS_TRY(cublasSetStream(blas, s));
  // full FP32 GEMMs: TF32 inputs (10-bit mantissa) cost CG two to three
  // times the iterations on these operators
  SCY_BLAS_TRY(cublasSetMathMode(blas, CUBLAS_DEFAULT_MATH));
  const float one = 1.0f, zero = 0.0f;
  long n = (long)Ny * Nz;
  float* rf = r32.as<float>();
  to_f32_kernel<<<grid_for(n), 256, 0, s>>>(r, rf, n);
  SCY_LAUNCH_CHECK();
  float* a = t1f.as<float>();
  float* b = t2f.as<float>();
  const float* vy = Vy32.as<float>();
  const float* vz = Vz32.as<float>();
  SCY_BLAS_TRY(cublasSgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, Nz, Ny, Nz, &one, vz, Nz, rf, Nz, &zero, a, Nz));
  SCY_BLAS_TRY(cublasSgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, Nz, Ny, Ny, &one, a, Nz, vy, Ny, &zero, b, Nz));
  count_launch();
  count_launch();
  scale_by_kernel<float><<<grid_for(n), 256, 0, s>>>(b, inv_lam32.as<float>(), n);
  SCY_LAUNCH_CHECK();
  SCY_BLAS_TRY(cublasSgemm(blas, CUBLAS_OP_N, CUBLAS_OP_T, Nz, Ny, Ny, &one, b, Nz, vy, Ny, &zero, a, Nz));
  SCY_BLAS_TRY(cublasSgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, Nz, Ny, Nz, &one, vz, Nz, a, Nz, &zero, z, Nz));
  count_launch();
  count_launch();
  return SCY_OK;
}

}  // namespace scy
