// Per-node device code of the power-law viscoelastic rates, shared by the
// single-instance driver (powerlaw.cu) and the batched ensemble (batch.cu):
// the viscous source B gVxy + C gVxz (PowerLaw::initializeMomBalMats,
// computeViscStrainSourceTerms, source/powerLaw.cpp:1239-1318, :1651-1671) and
// the strains, stresses, dislocation-creep viscosity and viscous strain rates
// (computeTotalStrains, computeStresses / computeSDev, computeViscosity,
// computeViscStrainRates with computeViscousStrainRateSAT, :1674-1887,
// DislocationCreep::computeInvEffVisc :438-474).
#pragma once
#include <cmath>

#include "sbp_dev.cuh"

namespace scy {

__device__ __forceinline__ double band_row_y(const LevelDev<double>& L, const double* __restrict__ x,
                                             const double* __restrict__ w, int iy, int iz) {
  // sum_k D[iy][k] * (w ? w[k,iz] : 1) * x[k,iz]
  const double* row = L.y.D + (long)iy * BAND;
  const int Nz = L.Nz;
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < BAND; ++j) {
    const int k = iy + j - HALF;
    if (k >= 0 && k < L.Ny) {
      const long n = (long)k * Nz + iz;
      acc += row[j] * (w ? w[n] * x[n] : x[n]);
    }
  }
  return acc;
}

__device__ __forceinline__ double band_row_z(const LevelDev<double>& L, const double* __restrict__ x,
                                             const double* __restrict__ w, int iy, int iz) {
  const double* row = L.z.D + (long)iz * BAND;
  const int Nz = L.Nz;
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < BAND; ++j) {
    const int k = iz + j - HALF;
    if (k >= 0 && k < Nz) {
      const long n = (long)iy * Nz + k;
      acc += row[j] * (w ? w[n] * x[n] : x[n]);
    }
  }
  return acc;
}

// B gVxy + C gVxz at one node.  B = (yq zr H) Dy mu + SAT and C = (yq zr H)
// Dz mu + SAT matrix-free: yq zr H = wy * wz, zr Hz = wy and yq Hy = wz in
// terms of the operator's outer weights, Dy = qy Dq and Dz = rz Dr.
__device__ __forceinline__ double pl_source_node(const LevelDev<double>& L, const double* __restrict__ gxy,
                                                 const double* __restrict__ gxz, long node) {
  const int Ny = L.Ny, Nz = L.Nz;
  const int iy = (int)(node / Nz), iz = (int)(node - (long)iy * Nz);
  const double wyz = L.wy[node] * L.wz[node];  // yq zr H
  double dy = band_row_y(L, gxy, L.mu, iy, iz);
  double dz = band_row_z(L, gxz, L.mu, iy, iz);
  if (L.var) {
    dy *= L.qy[node];
    dz *= L.rz[node];
  }
  double b = wyz * dy;
  // Neumann SATs: + zr Hz mu E0y, - zr Hz mu ENy; + yq Hy mu E0z, - yq Hy mu ENz
  if (L.y.bc_lo == 1 && iy == 0) b += L.wy[node] * L.mu[node] * gxy[node];
  if (L.y.bc_hi == 1 && iy == Ny - 1) b -= L.wy[node] * L.mu[node] * gxy[node];
  double c = wyz * dz;
  if (L.z.bc_lo == 1 && iz == 0) c += L.wz[node] * L.mu[node] * gxz[node];
  if (L.z.bc_hi == 1 && iz == Nz - 1) c -= L.wz[node] * L.mu[node] * gxz[node];
  return b + c;
}

struct PLRatesArgs {
  LevelDev<double> L;
  const double *u, *gxy, *gxz, *bcL, *bcR;
  const double *c1, *e1, *n;
  double inv_cap;
  double *dgxy, *dgxz, *sxy, *sxz, *sdev, *effVisc;
};

// Strains, stresses, viscosity and viscous strain rates at one node; the
// level is passed apart from the pointers so that batched launches can share it.
__device__ __forceinline__ void pl_rates_node(const LevelDev<double>& L, const PLRatesArgs& a, long node) {
  const int Ny = L.Ny, Nz = L.Nz;
  const int iy = (int)(node / Nz), iz = (int)(node - (long)iy * Nz);
  double gTxy = band_row_y(L, a.u, nullptr, iy, iz);
  double gTxz = band_row_z(L, a.u, nullptr, iy, iz);
  if (L.var) {
    gTxy *= L.qy[node];
    gTxz *= L.rz[node];
  }
  const double mu = L.mu[node];
  const double sxy = (gTxy + (-1.0) * a.gxy[node]) * mu;
  const double sxz = (gTxz + (-1.0) * a.gxz[node]) * mu;
  const double sdev = sqrt(fabs(sxy * sxy + 1.0 * (sxz * sxz)));
  const double inv = a.c1[node] * pow(sdev, a.n[node] - 1.0) * a.e1[node];
  const double visc = 1.0 / (a.inv_cap + 1.0 * inv);
  // SAT of the viscous strain rate at Dirichlet y boundaries
  double sat = 0.0;
  if (L.y.bc_lo == 0 && iy == 0) {
    const double hinv = L.y.Hinvd[0];
    sat = sat + 1.0 * (hinv * a.u[node]);
    sat = sat + (-1.0) * (hinv * a.bcL[iz]);
  }
  if (L.y.bc_hi == 0 && iy == Ny - 1) {
    const double hinv = L.y.Hinvd[Ny - 1];
    sat = sat + (-1.0) * (hinv * a.u[node]);
    sat = sat + 1.0 * (hinv * a.bcR[iz]);
  }
  if (L.var) sat = L.qy[node] * sat;
  a.dgxy[node] = (mu * sat + 1.0 * sxy) / visc;
  a.dgxz[node] = sxz / visc;
  a.sxy[node] = sxy;
  a.sxz[node] = sxz;
  a.sdev[node] = sdev;
  a.effVisc[node] = visc;
}

}  // namespace scy
