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
#include "blockchol.hpp"
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "fault_node.cuh"
#include "qd.hpp"
#include "infile.hpp"
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

__global__ void pl_axpy_kernel(double* __restrict__ x, const double* __restrict__ d, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) x[i] += d[i];
}

// ---------------------------------------------------------------------------
// The steady-state initial guess of guessSteadyStateICs = 1:
// StrikeSlip_PowerLaw_qd::solveSS(0) (strikeSlip_powerLaw_qd.cpp:922-955)
// with Fault::guessSS (fault.cpp:633-672), PowerLaw::guessSteadyStateEffVisc
// (powerLaw.cpp:1999-2037; DislocationCreep::guessInvEffVisc :399-433),
// guessTauSS (:888-918), solveSSViscoelasticProblem (:1018-1107; setSSRHS,
// updateSSa and updateSSb, powerLaw.cpp:2040-2195) and setSSBCs
// (:1295-1342).  Every iteration builds the SBP operator with mu = effVisc
// and the boundary types R Dirichlet, T / L / B Neumann, solves for the
// steady velocity v on the GPU and applies Dy and Dz there; the per-node
// viscosity update (stresses, dislocation-creep viscosity, log10 damping)
// is host arithmetic on the read-back strain rates.  The fault's slip
// velocity is seeded with vL (guessSS); the root find the reference runs
// after guessTauSS only moves the first root find's starting point.
int QDContext::pl_steady_state(const QDProblem& P, std::vector<double>& psi, std::vector<double>& slip,
                               double* gVxy, double* gVxz, int* its_out, double* err_out) {
  cudaStream_t s = sbp.stream;
  const double dg = P.ss_gss_t, cap = P.pdesc.visc_cap;
  // Fault::guessSS
  std::vector<double> tau(Nz), vel(Nz, vL);
  for (int i = 0; i < Nz; ++i) {
    if (!P.stateVals_given) psi[i] = f0 - h_b[i] * std::log(std::fabs(vL) / v0);
    tau[i] = h_sN[i] * h_a[i] * std::asinh(0.5 * vL * std::exp(psi[i] / h_a[i]) / v0);
  }
  // guessSteadyStateEffVisc: 1 / effVisc = 1 / cap + dg / (dg / (A e^(-B/T)))^(1/n)
  std::vector<double> eff((size_t)N);
  for (long k = 0; k < N; ++k) {
    const double temp = P.plA[k] * std::exp(-P.plB[k] / P.plT[k]);
    const double sk = std::pow(dg / temp, 1.0 / P.pln[k]);
    eff[k] = 1.0 / (1.0 / cap + dg / sk);
  }
  if (!P.ss_effvisc.empty()) eff = P.ss_effvisc;
  // guessTauSS: tauSS = min(tauRS, dg * effVisc on the fault)
  if (!P.ss_tau.empty())
    tau = P.ss_tau;
  else
    for (int i = 0; i < Nz; ++i) tau[i] = std::min(tau[i], eff[i] * dg);
  SCY_CUDA_TRY(cudaMemcpyAsync(slipVel.p, vel.data(), Nz * 8, cudaMemcpyHostToDevice, s));
  // solveSSViscoelasticProblem: bcL = tauSS (traction), bcR = vL / 2
  DevBuf dbcL, dbcR, dzero, drhs, dv, dgxy, dgxz;
  SCY_TRY(dbcL.alloc(Nz * 8));
  SCY_TRY(dbcR.alloc(Nz * 8));
  SCY_TRY(dzero.alloc((size_t)std::max(Ny, Nz) * 8));
  SCY_TRY(drhs.alloc(N * 8));
  SCY_TRY(dv.alloc(N * 8));
  SCY_TRY(dgxy.alloc(N * 8));
  SCY_TRY(dgxz.alloc(N * 8));
  const std::vector<double> half(Nz, vL / 2.0);
  SCY_CUDA_TRY(cudaMemcpyAsync(dbcL.p, tau.data(), Nz * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(dbcR.p, half.data(), Nz * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemsetAsync(dzero.p, 0, (size_t)std::max(Ny, Nz) * 8, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  scy_grid_desc g = P.desc.grid;
  g.bcR = SCY_BC_DIRICHLET;
  g.bcT = SCY_BC_NEUMANN;
  g.bcL = SCY_BC_NEUMANN;
  g.bcB = SCY_BC_NEUMANN;
  // The viscosity spans many decades (up to the cap, 1e30 by default,
  // powerLaw.cpp:757) and is far from separable; the stresses the update
  // reads are products of that viscosity with small velocity gradients, so
  // the velocity is needed to the accuracy of a direct solve, which is what
  // the reference runs here (MUMPS Cholesky, powerLaw.cpp:2111-2116).  Each
  // solve is a defect correction: the residual in double-double arithmetic
  // (SbpContext::residual_dd) and a correction by the block Cholesky
  // factorisation of this iteration's operator (BlockChol; by
  // preconditioned CG to a relative 1e-6 when the caller chose a
  // preconditioner or the factor would not fit in a third of the free
  // device memory), repeated until the residual meets the solve tolerance
  // or stops falling, and at least once.  The first residual of each
  // iteration is that of the previous iteration's velocity (a warm start).
  const int kMaxRefine = 30;
  scy_solve_opts o = solve_opts;
  o.verify = 1;
  o.nonzero_guess = 0;
  o.rtol = 1e-6;
  o.atol = 0.0;
  o.max_its = std::max(o.max_its, 4000);
  ss_cg_its = 0;
  ss_trace.clear();
  DevBuf dres, dcor, dkeep, dzN;
  SCY_TRY(dres.alloc(N * 8));
  SCY_TRY(dcor.alloc(N * 8));
  SCY_TRY(dkeep.alloc(N * 8));
  SCY_TRY(dzN.alloc(N * 8));
  SCY_CUDA_TRY(cudaMemsetAsync(dzN.p, 0, N * 8, s));
  SCY_CUDA_TRY(cudaMemsetAsync(dv.p, 0, N * 8, s));
  std::vector<double> gxy((size_t)N), gxz((size_t)N), v((size_t)N), sxy_h((size_t)N), sxz_h((size_t)N);
  bool direct = solve_opts.precond == SCY_PC_AUTO;
  if (direct) {
    size_t fr = 0, tot = 0;
    SCY_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    direct = BlockChol::bytes_for(Ny, Nz) < (double)fr / 3.0;
  }
  int it = 0;
  double err = 1e10;
  while (it < P.ss_max_its && err >= P.ss_atol) {
    g.mu = eff.data();
    SbpContext eta;  // initializeSSMatrices: the operator of this iteration's viscosity
    SCY_TRY(eta.create(g));
    SCY_CUDA_TRY(cudaDeviceSynchronize());
    eta.stream = s;
    SCY_TRY(eta.set_rhs(dbcL.as<double>(), dbcR.as<double>(), dzero.as<double>(), dzero.as<double>(),
                        drhs.as<double>()));
    BlockChol chol;
    if (direct) SCY_TRY(chol.factor(eta.hosts[0], s));
    double b2 = 0.0;
    SCY_TRY(eta.residual_dd(drhs.as<double>(), dzN.as<double>(), dres.as<double>(), &b2));
    const double tol = std::max(solve_opts.rtol * std::sqrt(b2), solve_opts.atol);
    double prev = INFINITY, first_rn = -1.0, last_rn = -1.0;
    long its_here = 0;
    int steps = 0;
    for (int m = 0; m <= kMaxRefine; ++m) {
      double r2 = 0.0;
      SCY_TRY(eta.residual_dd(drhs.as<double>(), dv.as<double>(), dres.as<double>(), &r2));
      const double rn = std::sqrt(r2);
      if (first_rn < 0) first_rn = rn;
      if (rn > prev) {
        // the last correction made it worse (rounding floor): keep the one before
        SCY_CUDA_TRY(cudaMemcpyAsync(dv.p, dkeep.p, N * 8, cudaMemcpyDeviceToDevice, s));
        break;
      }
      last_rn = rn;
      // at least one correction: with this contrast the relative residual
      // barely sees the soft region, so a warm start that already meets the
      // tolerance can still be far from this iteration's velocity there
      if ((m > 0 && rn <= tol) || rn > 0.9 * prev || m == kMaxRefine) break;
      prev = rn;
      if (direct) {
        SCY_TRY(chol.solve(dres.as<double>(), dcor.as<double>(), s));
      } else {
        scy_solve_stats st{};
        const int rc = eta.solve(dres.as<double>(), dcor.as<double>(), o, st);
        ss_cg_its += st.iterations;
        its_here += st.iterations;
        if (rc != SCY_OK && rc != SCY_ERR_CG_NOCONV) return rc;
      }
      ++steps;
      SCY_CUDA_TRY(cudaMemcpyAsync(dkeep.p, dv.p, N * 8, cudaMemcpyDeviceToDevice, s));
      pl_axpy_kernel<<<grid_for(N), kBlock, 0, s>>>(dv.as<double>(), dcor.as<double>(), N);
      SCY_LAUNCH_CHECK();
    }
    SCY_TRY(eta.apply(SCY_OP_DY, dv.as<double>(), dgxy.as<double>()));
    SCY_TRY(eta.apply(SCY_OP_DZ, dv.as<double>(), dgxz.as<double>()));
    SCY_CUDA_TRY(cudaMemcpyAsync(gxy.data(), dgxy.p, N * 8, cudaMemcpyDeviceToHost, s));
    SCY_CUDA_TRY(cudaMemcpyAsync(gxz.data(), dgxz.p, N * 8, cudaMemcpyDeviceToHost, s));
    SCY_CUDA_TRY(cudaMemcpyAsync(v.data(), dv.p, N * 8, cudaMemcpyDeviceToHost, s));
    SCY_CUDA_TRY(cudaStreamSynchronize(s));
    // updateSSa: stresses, deviatoric stress, the new viscosity; then the
    // damped update log10(eff) = (1 - f) log10(old) + f log10(new)
    // (MyVecLog10AXPBY, genFuncs.cpp:339-365) and the change
    // |eff - old| / |old| (computeNormDiff_L2_scaleL2, genFuncs.cpp:221-238)
    double dn = 0.0, on = 0.0;
    for (long k = 0; k < N; ++k) {
      const double old = eff[k];
      sxy_h[k] = old * gxy[k];
      sxz_h[k] = old * gxz[k];
      const double sdev = std::sqrt(std::fabs(sxy_h[k] * sxy_h[k] + sxz_h[k] * sxz_h[k]));
      const double inv = 1e3 * P.plA[k] * std::pow(sdev, P.pln[k] - 1.0) * std::exp(-P.plB[k] / P.plT[k]);
      const double nw = 1.0 / (1.0 / cap + 1.0 * inv);
      const double damped = std::pow(10.0, (1.0 - P.ss_fss) * std::log10(old) + P.ss_fss * std::log10(nw));
      dn += (damped - old) * (damped - old);
      on += old * old;
      eff[k] = damped;
    }
    err = std::sqrt(dn) / std::sqrt(on);
    const double bn = std::sqrt(b2) > 0 ? std::sqrt(b2) : 1.0;
    ss_trace.insert(ss_trace.end(), {(double)steps, first_rn / bn, last_rn / bn, (double)its_here, err});
    ++it;
  }
  // updateSSb at initTime: u = v t0 (made non-negative), viscous strains
  // gV = gV_t t0 - s / mu; setSSBCs: bcRShift = bcR = u at y = Ly, slip =
  // u at y = 0 (times 2 for a symmetric fault)
  const double t0 = P.init_time;
  std::vector<double> hu((size_t)N);
  for (long k = 0; k < N; ++k) hu[k] = v[k] * t0;
  double mn = *std::min_element(hu.begin(), hu.end());
  if (mn < 0)
    for (auto& x : hu) x += std::fabs(mn);
  if (it > 0)
    for (long k = 0; k < N; ++k) {
      gVxy[k] = gxy[k] * t0 - sxy_h[k] / P.mu[k];
      gVxz[k] = gxz[k] * t0 - sxz_h[k] / P.mu[k];
    }
  std::vector<double> shift(hu.end() - Nz, hu.end());
  slip.assign(hu.begin(), hu.begin() + Nz);
  for (auto& x : slip) x *= fts;
  SCY_CUDA_TRY(cudaMemcpyAsync(u.p, hu.data(), N * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(bcRShift.p, shift.data(), Nz * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(bcR.p, shift.data(), Nz * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  if (its_out) *its_out = it;
  if (err_out) *err_out = err;
  return SCY_OK;
}

}  // namespace scy
