// Power-law viscoelastic d_dt: StrikeSlip_PowerLaw_qd::d_dt and
// solveMomentumBalance (source/strikeSlip_powerLaw_qd.cpp:633-690, :787-823)
// with PowerLaw's viscous source, strains, stresses, dislocation-creep
// viscosity and strain rates (source/powerLaw.cpp:1239-1318, :1651-1887).
//
// Per d_dt: boundary data, rhs = setRhs + B gVxy + C gVxz (pl_source_kernel),
// the elliptic solve, one fused per-node kernel for the strains, stresses,
// viscosity and strain rates (pl_rates_kernel), and the fault update with
// tau from sxy on the fault row (pl_fault_kernel).
//
// B = (yq zr H) Dy mu + SAT and C = (yq zr H) Dz mu + SAT are applied
// matrix-free: yq zr H = wy * wz, zr Hz = wy and yq Hy = wz in terms of the
// operator's outer weights (wy = Hz zr, wz = Hy yq; zr = yq = 1 on the
// constant grid), Dy = qy Dq and Dz = rz Dr.
#include <cmath>

#include "common.cuh"
#include "fault_node.cuh"
#include "qd.hpp"
#include "powerlaw_dev.cuh"
#include "sbp_dev.cuh"

namespace scy {

// rhs += B gVxy + C gVxz (computeViscStrainSourceTerms, initializeMomBalMats)
__global__ void pl_source_kernel(LevelDev<double> L, const double* __restrict__ gxy, const double* __restrict__ gxz,
                                 double* __restrict__ rhs) {
  const long N = (long)L.Ny * L.Nz;
  for (long node = blockIdx.x * (long)blockDim.x + threadIdx.x; node < N; node += (long)gridDim.x * blockDim.x)
    rhs[node] = rhs[node] + 1.0 * pl_source_node(L, gxy, gxz, node);
}

// computeTotalStrains, computeStresses / computeSDev, computeViscosity and
// computeViscStrainRates (with computeViscousStrainRateSAT) per node
__global__ void pl_rates_kernel(PLRatesArgs a) {
  const long N = (long)a.L.Ny * a.L.Nz;
  for (long node = blockIdx.x * (long)blockDim.x + threadIdx.x; node < N; node += (long)gridDim.x * blockDim.x)
    pl_rates_node(a.L, a, node);
}

// Fault_qd::d_dt with tauQS from the material's sxy on the fault row
__global__ void pl_fault_kernel(const double* __restrict__ sxy, FaultParams fp, const double* __restrict__ var,
                                double* __restrict__ f, double* __restrict__ slipVel, double* __restrict__ tauQSP,
                                double* __restrict__ tauP, double* __restrict__ strength, unsigned* flags,
                                unsigned long long* its_total) {
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  if (iz >= fp.Nz) return;
  fault_node_update(iz, sxy[iz], fp, var, f, slipVel, tauQSP, tauP, strength, flags, its_total);
}

int pl_d_dt(QDContext& q, double t, const double* var, double* f) {
  cudaStream_t s = q.sbp.stream;
  const long N = q.N;
  const int Nz = q.Nz;
  const LevelDev<double>& L = q.sbp.fine->dev;
  SCY_TRY(qd_bc_launch(q, t, var));
  SCY_TRY(q.sbp.set_rhs(q.bcL.as<double>(), q.bcR.as<double>(), q.bcT.as<double>(), q.bcB.as<double>(),
                        q.rhs.as<double>()));
  const double* gxy = var + q.key_off[SCY_KEY_GVXY];
  const double* gxz = var + q.key_off[SCY_KEY_GVXZ];
  const int gb = grid_for(N, 256, 148 * 8);
  pl_source_kernel<<<gb, 256, 0, s>>>(L, gxy, gxz, q.rhs.as<double>());
  SCY_LAUNCH_CHECK();
  scy_solve_opts o = q.solve_opts;
  o.nonzero_guess = 1;
  scy_solve_stats st{};
  SCY_TRY(q.sbp.solve(q.rhs.as<double>(), q.u.as<double>(), o, st));
  q.n_solve_its += st.iterations;
  q.n_solves += 1;
  q.last_rnorm = st.rnorm;
  PLRatesArgs a{};
  a.L = L;
  a.u = q.u.as<double>();
  a.gxy = gxy;
  a.gxz = gxz;
  a.bcL = q.bcL.as<double>();
  a.bcR = q.bcR.as<double>();
  a.c1 = q.pl_c1.as<double>();
  a.e1 = q.pl_e1.as<double>();
  a.n = q.pl_n.as<double>();
  a.inv_cap = q.inv_visc_cap;
  a.dgxy = f + q.key_off[SCY_KEY_GVXY];
  a.dgxz = f + q.key_off[SCY_KEY_GVXZ];
  a.sxy = q.sxy.as<double>();
  a.sxz = q.sxz.as<double>();
  a.sdev = q.sdev.as<double>();
  a.effVisc = q.effVisc.as<double>();
  pl_rates_kernel<<<gb, 256, 0, s>>>(a);
  SCY_LAUNCH_CHECK();
  const int tb = 64, fb = (Nz + tb - 1) / tb;
  pl_fault_kernel<<<fb, tb, 0, s>>>(q.sxy.as<double>(), q.fp, var, f, q.slipVel.as<double>(), q.tauQSP.as<double>(),
                                    q.tauP.as<double>(), q.strength.as<double>(), q.flags.as<unsigned>(),
                                    q.fault_its.as<unsigned long long>());
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

}  // namespace scy
