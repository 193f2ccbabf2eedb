// Heat equation of the thermal quasi-dynamic driver on the device (see
// thermal.hpp): one backward-Euler step after every accepted RK step.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "qd.hpp"
#include "sbp_host.hpp"
#include "thermal_dev.hpp"

namespace scy {

namespace {

constexpr int kRedBlocks = 296;  // blocks of the reductions (two per SM)

// frictional heating (computeFrictionalShearHeating :1543-1576): with a
// zero-width shear zone the fault flux bcL = -tau V / 2; otherwise the body
// source Q = Gw * (tau V) of the node's fault row (node i takes fault value
// i mod Nz)
__global__ void th_fric_flux_kernel(const double* __restrict__ tau, const double* __restrict__ V,
                                    double* __restrict__ bcL, int Nz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < Nz) bcL[i] = -0.5 * (tau[i] * V[i]);
}

// rhs = dt (temp + [var] Iw Q) + rc Iw (T - Tamb), with temp = setRhs(bcL)
// already in rhs; Q = sgn Gw (tau V) when the shear zone has width
__global__ void th_transient_rhs_kernel(double* __restrict__ rhs, const double* __restrict__ T,
                                        const double* __restrict__ Tamb, const double* __restrict__ rc,
                                        const double* __restrict__ Iw, const double* __restrict__ Gw,
                                        const double* __restrict__ tau, const double* __restrict__ V, double dt,
                                        int body_source, int Nz, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double t = rhs[i];
    if (body_source) {
      const int iz = (int)(i % Nz);
      t += Iw[i] * (Gw[i] * (tau[iz] * V[iz]));
    }
    rhs[i] = dt * t + (Iw[i] * (T[i] - Tamb[i])) * rc[i];
  }
}

// rhs = setRhs(bcL) - Iw Q (be_steadyState: the frictional source enters
// negated, on both grids)
__global__ void th_steady_rhs_kernel(double* __restrict__ rhs, const double* __restrict__ Iw,
                                     const double* __restrict__ Gw, const double* __restrict__ tau,
                                     const double* __restrict__ V, int Nz, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int iz = (int)(i % Nz);
    rhs[i] -= Iw[i] * (Gw[i] * (tau[iz] * V[iz]));
  }
}

// deterministic block sums of a[i] * b[i] into part[blockIdx.x]
__global__ void th_dot_kernel(const double* __restrict__ a, const double* __restrict__ b, long n,
                              double* __restrict__ part) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    acc += a[i] * b[i];
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// q = rc Iw p - dt (A p)   (Ap holds A p on entry)
__global__ void th_mop_kernel(const double* __restrict__ p, double* __restrict__ q, const double* __restrict__ rc,
                              const double* __restrict__ Iw, double dt, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    q[i] = (rc[i] * Iw[i]) * p[i] - dt * q[i];
}

// r = rhs - q (q = M x0); z = r / diag M, diag M = rc Iw + dt diag(-A)
__global__ void th_res_kernel(const double* __restrict__ rhs, const double* __restrict__ q, double* __restrict__ r,
                              double* __restrict__ z, double* __restrict__ p, const double* __restrict__ rc,
                              const double* __restrict__ Iw, const double* __restrict__ dK, double dt, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double rv = rhs[i] - q[i];
    r[i] = rv;
    const double zv = rv / (rc[i] * Iw[i] + dt * dK[i]);
    z[i] = zv;
    p[i] = zv;
  }
}

__global__ void th_update_kernel(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                                 const double* __restrict__ q, double alpha, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    r[i] -= alpha * q[i];
  }
}

__global__ void th_precond_kernel(const double* __restrict__ r, double* __restrict__ z, const double* __restrict__ rc,
                                  const double* __restrict__ Iw, const double* __restrict__ dK, double dt, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    z[i] = r[i] / (rc[i] * Iw[i] + dt * dK[i]);
}

__global__ void th_pdir_kernel(double* __restrict__ p, const double* __restrict__ z, double beta, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

__global__ void th_sum_kernel(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ c,
                              long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    c[i] = a[i] + b[i];
}

__global__ void th_gather_fault_kernel(const double* __restrict__ T, double* __restrict__ Tf, int Nz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < Nz) Tf[i] = T[i];  // the fault is the body's first Nz nodes (iy = 0)
}

int upload(DevBuf& b, const std::vector<double>& v, cudaStream_t s) {
  SCY_TRY(b.alloc(v.size() * sizeof(double)));
  SCY_CUDA_TRY(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  return SCY_OK;
}

}  // namespace

int ThermalContext::create(QDContext& q, const HeatProblem& H) {
  Ny = q.Ny;
  Nz = q.Nz;
  N = q.N;
  coupled = H.coupling == 2;
  steady = H.steady;
  fric = H.fric;
  ksp_tol = H.ksp_tol;
  wMax = H.wMax;
  cudaStream_t s = q.sbp.stream;
  // the operator of k: R, T, B Dirichlet, L Neumann (setUpTransientProblem)
  scy_grid_desc g = q.sbp.desc;
  g.mu = H.k.data();
  g.y = q.sbp.y.empty() ? nullptr : q.sbp.y.data();
  g.z = q.sbp.z.empty() ? nullptr : q.sbp.z.data();
  g.bcR = SCY_BC_DIRICHLET;
  g.bcT = SCY_BC_DIRICHLET;
  g.bcL = SCY_BC_NEUMANN;
  g.bcB = SCY_BC_DIRICHLET;
  SCY_TRY(sbp.create(g));
  sbp.stream = s;
  const LevelHost& L = sbp.hosts[0];
  const bool var = L.grid_type == 1;
  var_grid = var ? 1 : 0;
  std::vector<double> iw((size_t)N), rcv((size_t)N);
  for (int iy = 0; iy < Ny; ++iy)
    for (int iz = 0; iz < Nz; ++iz) {
      const size_t i = (size_t)iy * Nz + iz;
      iw[i] = L.ty.Hd[iy] * L.tz.Hd[iz] * (var ? L.yq[i] * L.zr[i] : 1.0);  // I = (J) H
      rcv[i] = H.rho[i] * H.c[i];
    }
  SCY_TRY(upload(Iw, iw, s));
  SCY_TRY(upload(rc, rcv, s));
  SCY_TRY(upload(diagK, L.diagK, s));
  SCY_TRY(upload(Tamb, H.Tamb, s));
  SCY_TRY(upload(T, H.T, s));
  SCY_TRY(upload(dT, H.dT, s));
  SCY_TRY(upload(Gw, H.Gw, s));
  SCY_TRY(upload(Qrad, H.Qrad, s));
  std::vector<double> zeros((size_t)std::max(Ny, Nz), 0.0);
  SCY_TRY(upload(bcL, zeros, s));
  SCY_TRY(upload(zNz, zeros, s));
  SCY_TRY(upload(zNy, zeros, s));
  for (DevBuf* b : {&r, &z, &p, &q_, &rhs}) SCY_TRY(b->alloc((size_t)N * sizeof(double)));
  SCY_TRY(sc.alloc(sizeof(double) * kRedBlocks));
  // the fault: temperature the friction law reads, rho c and k there, Tw
  std::vector<double> Tf0(H.T.begin(), H.T.begin() + Nz), rcf(Nz), kf(H.k.begin(), H.k.begin() + Nz);
  SCY_TRY(upload(Tf, Tf0, s));
  SCY_TRY(upload(k_f, kf, s));
  if (H.flash) {
    for (int i = 0; i < Nz; ++i) rcf[i] = H.rho_f[i] * H.c[i];
    SCY_TRY(upload(rc_f, rcf, s));
    SCY_TRY(upload(Tw, H.Tw, s));
    std::vector<double> vw(Nz, H.Vw);
    SCY_TRY(upload(Vw, vw, s));
    FaultParams& fp = q.fp;
    fp.Tf = Tf.as<double>();
    fp.rc_f = rc_f.as<double>();
    fp.k_f = k_f.as<double>();
    fp.Tw = Tw.as<double>();
    fp.Vw = Vw.as<double>();
    fp.fl_D = H.D;
    fp.fl_tau_c = H.tau_c;
    fp.fl_fw = H.fw;
  }
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  return SCY_OK;
}

int ThermalContext::set_fault_temperature() {
  th_gather_fault_kernel<<<(Nz + 127) / 128, 128, 0, sbp.stream>>>(T.as<double>(), Tf.as<double>(), Nz);
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

// HeatEquation::be (heatEquation.cpp:1108-1143) with be_transient
// (:1146-1240) or be_steadyState (:1242-1318)
int ThermalContext::step(QDContext& qd, double dt) {
  cudaStream_t s = sbp.stream;
  const int gN = grid_for(N);
  const double* tau = qd.tauP.as<double>();
  const double* V = qd.slipVel.as<double>();
  double* bl = bcL.as<double>();
  SCY_CUDA_TRY(cudaMemsetAsync(bl, 0, Nz * sizeof(double), s));
  const int zero_width = wMax == 0.0;
  if (fric && zero_width) {
    th_fric_flux_kernel<<<(Nz + 127) / 128, 128, 0, s>>>(tau, V, bl, Nz);
    SCY_LAUNCH_CHECK();
  }
  double* R = rhs.as<double>();
  SCY_TRY(sbp.set_rhs(bl, zNz.as<double>(), zNy.as<double>(), zNy.as<double>(), R));
  double* x = dT.as<double>();
  if (steady) {
    if (fric && !zero_width) {
      th_steady_rhs_kernel<<<gN, 256, 0, s>>>(R, Iw.as<double>(), Gw.as<double>(), tau, V, Nz, N);
      SCY_LAUNCH_CHECK();
    }
    scy_solve_opts o{};
    o.rtol = ksp_tol;
    o.atol = 0.0;
    o.max_its = 20000;
    o.precision = SCY_PREC_FP64;
    o.nonzero_guess = 1;
    o.check_every = 1;
    o.precond = SCY_PC_AUTO;
    o.verify = 1;
    scy_solve_stats st{};
    SCY_TRY(sbp.solve(R, x, o, st));
    its += st.iterations;
  } else {
    th_transient_rhs_kernel<<<gN, 256, 0, s>>>(R, T.as<double>(), Tamb.as<double>(), rc.as<double>(),
                                               Iw.as<double>(), Gw.as<double>(), tau, V, dt,
                                               (fric && !zero_width && var_grid) ? 1 : 0, Nz, N);
    SCY_LAUNCH_CHECK();
    SCY_TRY(pcg(dt));
  }
  th_sum_kernel<<<gN, 256, 0, s>>>(Tamb.as<double>(), x, T.as<double>(), N);
  SCY_LAUNCH_CHECK();
  ++solves;
  return SCY_OK;
}

// Jacobi-preconditioned CG on (rc I - dt A) dT = rhs from the previous dT;
// stops at ||r|| <= ksp_tol ||rhs|| (relative, as KSP's default test)
int ThermalContext::pcg(double dt) {
  cudaStream_t s = sbp.stream;
  const int gN = grid_for(N);
  double *X = dT.as<double>(), *R = r.as<double>(), *Z = z.as<double>(), *P = p.as<double>(),
         *Q = q_.as<double>(), *B = rhs.as<double>();
  const double *rcp = rc.as<double>(), *iw = Iw.as<double>(), *dk = diagK.as<double>();
  std::vector<double> part(kRedBlocks);
  auto dot = [&](const double* a, const double* b, double* out) -> int {
    th_dot_kernel<<<kRedBlocks, 256, 0, s>>>(a, b, N, sc.as<double>());
    SCY_LAUNCH_CHECK();
    SCY_CUDA_TRY(cudaMemcpyAsync(part.data(), sc.p, kRedBlocks * sizeof(double), cudaMemcpyDeviceToHost, s));
    SCY_CUDA_TRY(cudaStreamSynchronize(s));
    double t = 0.0;
    for (double v : part) t += v;
    *out = t;
    return SCY_OK;
  };
  auto mop = [&](const double* in, double* out) -> int {
    SCY_TRY(sbp.apply(SCY_OP_A, in, out));
    th_mop_kernel<<<gN, 256, 0, s>>>(in, out, rcp, iw, dt, N);
    SCY_LAUNCH_CHECK();
    return SCY_OK;
  };
  double bb = 0.0;
  SCY_TRY(dot(B, B, &bb));
  const double tol = ksp_tol * std::sqrt(bb);
  SCY_TRY(mop(X, Q));
  th_res_kernel<<<gN, 256, 0, s>>>(B, Q, R, Z, P, rcp, iw, dk, dt, N);
  SCY_LAUNCH_CHECK();
  double rr = 0.0, rz = 0.0;
  SCY_TRY(dot(R, R, &rr));
  if (std::sqrt(rr) <= tol) return SCY_OK;
  SCY_TRY(dot(R, Z, &rz));
  const int max_its = 50000;
  for (int it = 1; it <= max_its; ++it) {
    SCY_TRY(mop(P, Q));
    double pq = 0.0;
    SCY_TRY(dot(P, Q, &pq));
    if (!(pq > 0.0)) {
      set_error("heat-equation CG: p.Mp = %g (operator not positive definite?)", pq);
      return SCY_ERR_NONFINITE;
    }
    const double alpha = rz / pq;
    th_update_kernel<<<gN, 256, 0, s>>>(X, R, P, Q, alpha, N);
    SCY_LAUNCH_CHECK();
    ++its;
    SCY_TRY(dot(R, R, &rr));
    if (!std::isfinite(rr)) {
      set_error("non-finite residual in the heat-equation solve");
      return SCY_ERR_NONFINITE;
    }
    if (std::sqrt(rr) <= tol) return SCY_OK;
    th_precond_kernel<<<gN, 256, 0, s>>>(R, Z, rcp, iw, dk, dt, N);
    SCY_LAUNCH_CHECK();
    double rz_new = 0.0;
    SCY_TRY(dot(R, Z, &rz_new));
    th_pdir_kernel<<<gN, 256, 0, s>>>(P, Z, rz_new / rz, N);
    SCY_LAUNCH_CHECK();
    rz = rz_new;
  }
  set_error("heat-equation CG stopped at ||r|| = %g after %d iterations (target %g)", std::sqrt(rr), max_its, tol);
  return SCY_ERR_CG_NOCONV;
}

}  // namespace scy
