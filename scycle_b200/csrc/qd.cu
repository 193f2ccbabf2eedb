// Linear-elastic quasi-dynamic driver on the device.
//
// d_dt follows StrikeSlip_LinearElastic_qd::d_dt
// (source/strikeSlip_linearElastic_qd.cpp:756-798) and Fault_qd::d_dt
// (source/fault.cpp:861-918); the integrators follow RK32::integrate and
// RK43::integrate (source/odeSolver.cpp:505-627, :973-1175) with their step
// control (:395-445, :846-898), including the reference's handling of the
// 100-attempt cap and of a step that falls to the minimum size.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "fault_node.cuh"
#include "infile.hpp"
#include "qd.hpp"
#include "thermal_dev.hpp"

namespace scy {

// ---------------------------------------------------------------------------
// bcL = slip/faultTypeScale, bcR = vL t/faultTypeScale + bcRShift
__global__ void qd_bc_kernel(const double* __restrict__ slip, int Nz, double t, double vL, double inv_fts,
                             int bcL_from_slip, int bcR_remote, const double* __restrict__ shift,
                             double* __restrict__ bcL, double* __restrict__ bcR) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Nz) return;
  if (bcL_from_slip) bcL[i] = slip[i] * inv_fts;
  if (bcR_remote) bcR[i] = vL * t * inv_fts + shift[i];
}

// Fault column: sxy = mu*Dy*u at iy = 0 (body2L scatter of muxDy), then the
// fault update.
__global__ void qd_fault_kernel(LevelDev<double> L, const double* __restrict__ u, FaultParams fp,
                                const double* __restrict__ var, double* __restrict__ f,
                                double* __restrict__ slipVel, double* __restrict__ tauQSP,
                                double* __restrict__ tauP, double* __restrict__ strength, unsigned* flags,
                                unsigned long long* its_total) {
  int iz = blockIdx.x * blockDim.x + threadIdx.x;
  if (iz >= fp.Nz) return;
  const double sxy = fault_row_sxy(L, u, iz);
  fault_node_update(iz, sxy, fp, var, f, slipVel, tauQSP, tauP, strength, flags, its_total);
}

// Fault_qd::d_dt with the body's shear stress on the fault given by the
// caller (the fault-row sxy a driver gets from its own solve and muxDy).
__global__ void qd_fault_given_tau_kernel(const double* __restrict__ tau_body, FaultParams fp,
                                          const double* __restrict__ var, double* __restrict__ f,
                                          double* __restrict__ slipVel, double* __restrict__ tauQSP,
                                          double* __restrict__ tauP, double* __restrict__ strength, unsigned* flags,
                                          unsigned long long* its_total) {
  int iz = blockIdx.x * blockDim.x + threadIdx.x;
  if (iz >= fp.Nz) return;
  fault_node_update(iz, tau_body[iz], fp, var, f, slipVel, tauQSP, tauP, strength, flags, its_total);
}

int QDContext::fault_d_dt(const double* var, const double* tau_body, double* f) {
  const int tb = 64, gb = (Nz + tb - 1) / tb;
  qd_fault_given_tau_kernel<<<gb, tb, 0, sbp.stream>>>(tau_body, fp, var, f, slipVel.as<double>(),
                                                       tauQSP.as<double>(), tauP.as<double>(),
                                                       strength.as<double>(), flags.as<unsigned>(),
                                                       fault_its.as<unsigned long long>());
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

// Fault column stress of a body displacement, for building the response
// matrices: out[iz * ld + col] = mu * Dy u at (0, iz); surf[iy * ld + col] = u(iy, 0).
__global__ void qd_response_column_kernel(LevelDev<double> L, const double* __restrict__ u, double* __restrict__ out,
                                          double* __restrict__ surf, int ld, int col) {
  const int Ny = L.Ny, Nz = L.Nz;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < Nz) {
    double d = 0.0;
#pragma unroll
    for (int j = HALF; j < BAND; ++j) {
      int k = j - HALF;
      if (k < Ny) d += L.y.D[j] * u[(long)k * Nz + i];
    }
    if (L.var) d *= L.qy[i];
    out[(long)i * ld + col] = L.mu[i] * d;
  }
  if (i < Ny && surf) surf[(long)i * ld + col] = u[(long)i * Nz];
}

// Fault-response d_dt: one warp per fault node forms
// tau = GL[iz,:] . (slip/faultTypeScale) + c g1[iz] + gs[iz], lane 0 then
// runs the fault update.
__global__ void qd_green_kernel(const double* __restrict__ GL, const double* __restrict__ g1,
                                const double* __restrict__ gs, double c, double inv_fts, FaultParams fp,
                                const double* __restrict__ var, double* __restrict__ f, double* __restrict__ slipVel,
                                double* __restrict__ tauQSP, double* __restrict__ tauP, double* __restrict__ strength,
                                double* __restrict__ bcL, unsigned* flags, unsigned long long* its_total) {
  const int Nz = fp.Nz;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= Nz) return;
  const double* row = GL + (long)warp * Nz;
  const double* slip = var + fp.slip_off;
  double acc = 0.0;
  for (int j = lane; j < Nz; j += 32) acc += row[j] * (slip[j] * inv_fts);
  acc = warp_sum(acc);
  if (lane == 0) {
    bcL[warp] = slip[warp] * inv_fts;  // kept for output fields
    const double tau = acc + (c * g1[warp] + gs[warp]);
    fault_node_update(warp, tau, fp, var, f, slipVel, tauQSP, tauP, strength, flags, its_total);
  }
}

// surface displacement from the response matrices and the last bcL
__global__ void qd_green_surf_kernel(const double* __restrict__ SL, const double* __restrict__ s1,
                                     const double* __restrict__ ss, double c, int Ny, int Nz,
                                     const double* __restrict__ bcL, double* __restrict__ out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= Ny) return;
  const double* row = SL + (long)warp * Nz;
  double acc = 0.0;
  for (int j = lane; j < Nz; j += 32) acc += row[j] * bcL[j];
  acc = warp_sum(acc);
  if (lane == 0) out[warp] = acc + (c * s1[warp] + ss[warp]);
}

int qd_green_surf_launch(QDContext& q, double c, double* host_out) {
  cudaStream_t s = q.sbp.stream;
  const int wpb = 4;
  qd_green_surf_kernel<<<(q.Ny + wpb - 1) / wpb, 32 * wpb, 0, s>>>(q.SL.as<double>(), q.s1.as<double>(),
                                                                   q.ss.as<double>(), c, q.Ny, q.Nz,
                                                                   q.bcL.as<double>(), q.sxy.as<double>());
  SCY_LAUNCH_CHECK();
  SCY_CUDA_TRY(cudaMemcpyAsync(host_out, q.sxy.p, (size_t)q.Ny * 8, cudaMemcpyDeviceToHost, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  return SCY_OK;
}

// Body displacement for output in response mode: one full solve with the
// boundary data of the last d_dt.
int QDContext::full_solve_for_output() {
  cudaStream_t s = sbp.stream;
  const int tb = 64, gb = (Nz + tb - 1) / tb;
  qd_bc_kernel<<<gb, tb, 0, s>>>(rk[0].as<double>() + fp.slip_off, Nz, last_t, vL, 1.0 / fts, 0, bcR_remote,
                                 bcRShift.as<double>(), bcL.as<double>(), bcR.as<double>());
  SCY_LAUNCH_CHECK();
  SCY_TRY(sbp.set_rhs(bcL.as<double>(), bcR.as<double>(), bcT.as<double>(), bcB.as<double>(), rhs.as<double>()));
  scy_solve_opts o = solve_opts;
  o.nonzero_guess = 1;
  scy_solve_stats st{};
  return sbp.solve(rhs.as<double>(), u.as<double>(), o, st);
}

// out = ((var + c0 f0) + c1 f1) + ... in the reference's WAXPY/AXPY order
struct Combo {
  const double* f[5];
  double c[5];
  int nf;
};

__global__ void rk_combine_kernel(double* __restrict__ out, const double* __restrict__ var, Combo cb, long n) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v = cb.c[0] * cb.f[0][i] + var[i];
  for (int j = 1; j < cb.nf; ++j) v = v + cb.c[j] * cb.f[j][i];
  out[i] = v;
}

// Per integrated field (block b handles SCY_KEY b at [off[b], off[b]+len[b])):
// sum (lo-hi)^2, sum hi^2, max(|lo-hi|/hi) into out[3b .. 3b+2].
struct KeyTable {
  long off[4], len[4];
};

__global__ void rk_error_kernel(const double* __restrict__ lo, const double* __restrict__ hi, KeyTable kt,
                                double* __restrict__ out) {
  __shared__ double sh[32];
  const int key = blockIdx.x;
  const long off = kt.off[key], len = kt.len[key];
  double ss = 0.0, sh2 = 0.0, mx = -INFINITY;
  for (long i = threadIdx.x; i < len; i += blockDim.x) {
    double h = hi[off + i];
    double d = lo[off + i] - h;
    ss += d * d;
    sh2 += h * h;
    double r = fabs(d) / h;
    mx = fmax(mx, r);
  }
  ss = block_sum(ss, sh);
  sh2 = block_sum(sh2, sh);
  double m = warp_max(mx);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < (blockDim.x + 31) / 32 ? sh[threadIdx.x] : -INFINITY;
    t = warp_max(t);
    if (threadIdx.x == 0) {
      out[key * 3 + 0] = ss;
      out[key * 3 + 1] = sh2;
      out[key * 3 + 2] = t;
    }
  }
}

// ---------------------------------------------------------------------------
template <typename T>
static int upload_vec(DevBuf& b, const T* src, size_t n, cudaStream_t s) {
  SCY_TRY(b.alloc(n * sizeof(T)));
  SCY_CUDA_TRY(cudaMemcpyAsync(b.p, src, n * sizeof(T), cudaMemcpyHostToDevice, s));
  return SCY_OK;
}

static int upload_or_fill(DevBuf& b, const double* src, size_t n, double fill, cudaStream_t s) {
  std::vector<double> v(n, fill);
  if (src) std::copy(src, src + n, v.begin());
  SCY_TRY(upload_vec(b, v.data(), n, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  return SCY_OK;
}

int QDContext::create(const scy_qd_desc& d, const scy_pl_desc* pld) {
  pl = pld ? 1 : 0;
  if (pl && (!pld->A || !pld->B || !pld->n || !pld->T || !(pld->visc_cap > 0))) {
    set_error("power-law descriptor needs A, B, n, T and visc_cap > 0");
    return SCY_ERR_ARG;
  }
  SCY_TRY(sbp.create(d.grid));
  Ny = d.grid.Ny;
  Nz = d.grid.Nz;
  N = (long)Ny * Nz;
  const scy_fault_desc& f = d.fault;
  if (f.Nz != Nz) {
    set_error("fault Nz (%d) differs from grid Nz (%d)", f.Nz, Nz);
    return SCY_ERR_ARG;
  }
  if (!f.a || !f.b || !f.sN || !f.Dc || !f.eta) {
    set_error("fault arrays a, b, sN, Dc, eta are required");
    return SCY_ERR_ARG;
  }
  if (f.state_law < 0 || f.state_law > 3) {
    set_error("unknown state law %d", f.state_law);
    return SCY_ERR_ARG;
  }
  if (!(f.v0 > 0) || !(f.root_tol > 0) || f.max_its < 1) {
    set_error("fault needs v0 > 0, root_tol > 0, max_its >= 1");
    return SCY_ERR_ARG;
  }
  cudaStream_t s = sbp.stream;
  SCY_TRY(upload_or_fill(fa, f.a, Nz, 0, s));
  SCY_TRY(upload_or_fill(fb, f.b, Nz, 0, s));
  SCY_TRY(upload_or_fill(fsN, f.sN, Nz, 0, s));
  SCY_TRY(upload_or_fill(fDc, f.Dc, Nz, 0, s));
  SCY_TRY(upload_or_fill(feta, f.eta, Nz, 0, s));
  SCY_TRY(upload_or_fill(flocked, f.locked, Nz, 0, s));
  SCY_TRY(upload_or_fill(fprestress, f.prestress, Nz, 0, s));
  for (DevBuf* b : {&slipVel, &tauQSP, &tauP, &strength}) SCY_TRY(upload_or_fill(*b, nullptr, Nz, 0, s));
  SCY_TRY(upload_or_fill(bcL, d.bcL0, Nz, 0, s));
  SCY_TRY(upload_or_fill(bcR, nullptr, Nz, 0, s));
  SCY_TRY(upload_or_fill(bcRShift, d.bcRShift, Nz, 0, s));
  SCY_TRY(upload_or_fill(bcT, nullptr, Ny, 0, s));
  SCY_TRY(upload_or_fill(bcB, nullptr, Ny, 0, s));
  SCY_TRY(rhs.alloc(N * 8));
  SCY_TRY(u.alloc(N * 8));
  SCY_TRY(sxy.alloc(N * 8));
  SCY_CUDA_TRY(cudaMemset(u.p, 0, N * 8));
  SCY_TRY(flags.alloc(16));
  SCY_CUDA_TRY(cudaMemset(flags.p, 0, 16));
  SCY_TRY(fault_its.alloc(16));
  SCY_CUDA_TRY(cudaMemset(fault_its.p, 0, 16));
  h_a.assign(f.a, f.a + Nz);
  h_b.assign(f.b, f.b + Nz);
  h_sN.assign(f.sN, f.sN + Nz);
  f0 = f.f0;
  v0 = f.v0;
  fp.Nz = Nz;
  fp.a = fa.as<double>();
  fp.b = fb.as<double>();
  fp.sN = fsN.as<double>();
  fp.Dc = fDc.as<double>();
  fp.eta = feta.as<double>();
  fp.locked = flocked.as<double>();
  fp.prestress = fprestress.as<double>();
  fp.f0 = f.f0;
  fp.v0 = f.v0;
  fp.vL = f.vL;
  fp.root_tol = f.root_tol;
  fp.max_its = f.max_its;
  fp.state_law = f.state_law;
  fp.jacobian = f.exact_jacobian ? 1 : 0;
  vL = d.vL;
  fts = d.fault_type_scale;
  if (!(fts > 0)) {
    set_error("fault_type_scale must be positive");
    return SCY_ERR_ARG;
  }
  bcL_from_slip = d.bcL_from_slip;
  bcR_remote = d.bcR_remote;
  solve_opts = d.solve;
  if (solve_opts.max_its < 1) solve_opts.max_its = 200;
  if (solve_opts.check_every < 1) solve_opts.check_every = 1;
  // integrated state layout (the std::map's key order)
  for (int k = 0; k < 4; ++k) key_off[k] = key_len[k] = 0;
  if (pl) {
    key_off[SCY_KEY_GVXY] = 0;
    key_len[SCY_KEY_GVXY] = N;
    key_off[SCY_KEY_GVXZ] = N;
    key_len[SCY_KEY_GVXZ] = N;
    key_off[SCY_KEY_PSI] = 2 * N;
    key_off[SCY_KEY_SLIP] = 2 * N + Nz;
    nvar = 2 * N + 2 * (long)Nz;
  } else {
    key_off[SCY_KEY_PSI] = 0;
    key_off[SCY_KEY_SLIP] = Nz;
    nvar = 2 * (long)Nz;
  }
  key_len[SCY_KEY_PSI] = key_len[SCY_KEY_SLIP] = Nz;
  fp.psi_off = key_off[SCY_KEY_PSI];
  fp.slip_off = key_off[SCY_KEY_SLIP];
  if (pl) {
    // DislocationCreep::computeInvEffVisc evaluates 1e3*A*pow(s, n-1)*exp(-B/T)
    // left to right; 1e3*A and exp(-B/T) are fixed without thermal coupling
    std::vector<double> c1(N), e1(N);
    for (long i = 0; i < N; ++i) {
      c1[i] = 1e3 * pld->A[i];
      e1[i] = std::exp(-pld->B[i] / pld->T[i]);
    }
    SCY_TRY(upload_vec(pl_c1, c1.data(), N, s));
    SCY_TRY(upload_vec(pl_e1, e1.data(), N, s));
    SCY_TRY(upload_vec(pl_n, pld->n, N, s));
    inv_visc_cap = 1.0 / pld->visc_cap;
    SCY_TRY(sxz.alloc(N * 8));
    SCY_TRY(sdev.alloc(N * 8));
    SCY_TRY(effVisc.alloc(N * 8));
    SCY_CUDA_TRY(cudaMemsetAsync(sxz.p, 0, N * 8, s));
    SCY_CUDA_TRY(cudaMemsetAsync(sdev.p, 0, N * 8, s));
    SCY_CUDA_TRY(cudaMemsetAsync(effVisc.p, 0, N * 8, s));
    SCY_CUDA_TRY(cudaStreamSynchronize(s));
  }
  for (auto& b : rk) {
    SCY_TRY(b.alloc((size_t)nvar * 8));
    SCY_CUDA_TRY(cudaMemset(b.p, 0, (size_t)nvar * 8));
  }
  SCY_TRY(errbuf.alloc(16 * 8));
  return SCY_OK;
}

int QDContext::read_flags() {
  unsigned h = 0;
  SCY_CUDA_TRY(cudaMemcpyAsync(&h, flags.p, sizeof(unsigned), cudaMemcpyDeviceToHost, sbp.stream));
  SCY_CUDA_TRY(cudaStreamSynchronize(sbp.stream));
  if (h) {
    SCY_CUDA_TRY(cudaMemsetAsync(flags.p, 0, sizeof(unsigned), sbp.stream));
    if (h & FAULT_NONFINITE) {
      set_error("non-finite value in the fault root bracket or state rate");
      return SCY_ERR_NONFINITE;
    }
    set_error("rootFinder BracketedNewton did not converge within %d iterations", fp.max_its);
    return SCY_ERR_ROOT_NOCONV;
  }
  return SCY_OK;
}

int qd_bc_launch(QDContext& q, double t, const double* var) {
  const int tb = 64, gb = (q.Nz + tb - 1) / tb;
  qd_bc_kernel<<<gb, tb, 0, q.sbp.stream>>>(var + q.fp.slip_off, q.Nz, t, q.vL, 1.0 / q.fts, q.bcL_from_slip,
                                            q.bcR_remote, q.bcRShift.as<double>(), q.bcL.as<double>(),
                                            q.bcR.as<double>());
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

int QDContext::d_dt(double t, const double* var, double* f) {
  cudaStream_t s = sbp.stream;
  if (fp.state_law == SCY_LAW_FLASH && !fp.Tf) {
    set_error("the flash-heating law needs the heat equation's fault fields (a driver with thermalCoupling)");
    return SCY_ERR_STATE;
  }
  if (pl) {
    if (mode == SCY_QD_MODE_RESPONSE) {
      set_error("the fault-response mode does not apply to the power-law material");
      return SCY_ERR_STATE;
    }
    SCY_TRY(pl_d_dt(*this, t, var, f));
    last_t = t;
    ++n_d_dt;
    return SCY_OK;
  }
  if (mode == SCY_QD_MODE_RESPONSE) {
    if (!green_ready) SCY_TRY(build_green());
    const double c = bcR_remote ? vL * t * (1.0 / fts) : 0.0;
    const int wpb = 4;
    qd_green_kernel<<<(Nz + wpb - 1) / wpb, 32 * wpb, 0, s>>>(
        GL.as<double>(), g1.as<double>(), gs.as<double>(), c, 1.0 / fts, fp, var, f, slipVel.as<double>(),
        tauQSP.as<double>(), tauP.as<double>(), strength.as<double>(), bcL.as<double>(), flags.as<unsigned>(),
        fault_its.as<unsigned long long>());
    SCY_LAUNCH_CHECK();
    last_t = t;
    ++n_d_dt;
    return SCY_OK;
  }
  const int tb = 64, gb = (Nz + tb - 1) / tb;
  qd_bc_kernel<<<gb, tb, 0, s>>>(var + fp.slip_off, Nz, t, vL, 1.0 / fts, bcL_from_slip, bcR_remote,
                                 bcRShift.as<double>(), bcL.as<double>(), bcR.as<double>());
  SCY_LAUNCH_CHECK();
  SCY_TRY(sbp.set_rhs(bcL.as<double>(), bcR.as<double>(), bcT.as<double>(), bcB.as<double>(), rhs.as<double>()));
  scy_solve_opts o = solve_opts;
  o.nonzero_guess = 1;  // the previous stage's displacement is the initial guess
  scy_solve_stats st{};
  SCY_TRY(sbp.solve(rhs.as<double>(), u.as<double>(), o, st));
  n_solve_its += st.iterations;
  n_solves += 1;
  last_rnorm = st.rnorm;
  qd_fault_kernel<<<gb, tb, 0, s>>>(sbp.fine->dev, u.as<double>(), fp, var, f, slipVel.as<double>(),
                                    tauQSP.as<double>(), tauP.as<double>(), strength.as<double>(),
                                    flags.as<unsigned>(), fault_its.as<unsigned long long>());
  SCY_LAUNCH_CHECK();
  last_t = t;
  ++n_d_dt;
  return SCY_OK;
}

// Response of the fault stress and the surface displacement to unit boundary
// data: Nz solves with bcL = e_j, one with bcR = 1 and one with the current
// fixed part of bcR (bcRShift when the right boundary is loaded, else bcR).
int QDContext::build_green() {
  cudaStream_t s = sbp.stream;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  SCY_TRY(GL.alloc((size_t)Nz * Nz * 8));
  SCY_TRY(SL.alloc((size_t)Ny * Nz * 8));
  DevBuf cols, scol;
  SCY_TRY(cols.alloc((size_t)Nz * 2 * 8));
  SCY_TRY(scol.alloc((size_t)Ny * 2 * 8));
  SCY_TRY(g1.alloc((size_t)Nz * 8));
  SCY_TRY(gs.alloc((size_t)Nz * 8));
  SCY_TRY(s1.alloc((size_t)Ny * 8));
  SCY_TRY(ss.alloc((size_t)Ny * 8));
  DevBuf bL, bR, uu;
  SCY_TRY(bL.alloc((size_t)Nz * 8));
  SCY_TRY(bR.alloc((size_t)Nz * 8));
  SCY_TRY(uu.alloc((size_t)N * 8));
  scy_solve_opts o = solve_opts;
  o.rtol = std::min(o.rtol, 1e-13);
  o.nonzero_guess = 0;
  o.max_its = std::max(o.max_its, 500);
  const LevelDev<double>& L = sbp.fine->dev;
  const int tb = 128, gb = (std::max(Ny, Nz) + tb - 1) / tb;
  std::vector<double> e(Nz, 0.0);
  SCY_CUDA_TRY(cudaMemsetAsync(bR.p, 0, (size_t)Nz * 8, s));
  for (int j = 0; j < Nz; ++j) {
    e[j] = 1.0;
    SCY_CUDA_TRY(cudaMemcpyAsync(bL.p, e.data(), (size_t)Nz * 8, cudaMemcpyHostToDevice, s));
    e[j] = 0.0;
    SCY_TRY(sbp.set_rhs(bL.as<double>(), bR.as<double>(), bcT.as<double>(), bcB.as<double>(), rhs.as<double>()));
    scy_solve_stats st{};
    SCY_TRY(sbp.solve(rhs.as<double>(), uu.as<double>(), o, st));
    qd_response_column_kernel<<<gb, tb, 0, s>>>(L, uu.as<double>(), GL.as<double>(), SL.as<double>(), Nz, j);
    SCY_LAUNCH_CHECK();
  }
  // bcR = 1 and the fixed part of bcR
  SCY_CUDA_TRY(cudaMemsetAsync(bL.p, 0, (size_t)Nz * 8, s));
  for (int k = 0; k < 2; ++k) {
    if (k == 0) {
      std::vector<double> ones(Nz, 1.0);
      SCY_CUDA_TRY(cudaMemcpyAsync(bR.p, ones.data(), (size_t)Nz * 8, cudaMemcpyHostToDevice, s));
      SCY_CUDA_TRY(cudaStreamSynchronize(s));
    } else {
      const DevBuf& fixed = bcR_remote ? bcRShift : bcR;
      SCY_CUDA_TRY(cudaMemcpyAsync(bR.p, fixed.p, (size_t)Nz * 8, cudaMemcpyDeviceToDevice, s));
    }
    SCY_TRY(sbp.set_rhs(bL.as<double>(), bR.as<double>(), bcT.as<double>(), bcB.as<double>(), rhs.as<double>()));
    scy_solve_stats st{};
    SCY_TRY(sbp.solve(rhs.as<double>(), uu.as<double>(), o, st));
    qd_response_column_kernel<<<gb, tb, 0, s>>>(L, uu.as<double>(), cols.as<double>(), scol.as<double>(), 2, k);
    SCY_LAUNCH_CHECK();
  }
  // split the two columns into g1/gs and s1/ss
  std::vector<double> hc((size_t)Nz * 2), hs((size_t)Ny * 2), a(Nz), b(Nz), c(Ny), d(Ny);
  SCY_CUDA_TRY(cudaMemcpyAsync(hc.data(), cols.p, hc.size() * 8, cudaMemcpyDeviceToHost, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(hs.data(), scol.p, hs.size() * 8, cudaMemcpyDeviceToHost, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  for (int i = 0; i < Nz; ++i) {
    a[i] = hc[(size_t)i * 2];
    b[i] = hc[(size_t)i * 2 + 1];
  }
  for (int i = 0; i < Ny; ++i) {
    c[i] = hs[(size_t)i * 2];
    d[i] = hs[(size_t)i * 2 + 1];
  }
  SCY_CUDA_TRY(cudaMemcpyAsync(g1.p, a.data(), (size_t)Nz * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(gs.p, b.data(), (size_t)Nz * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(s1.p, c.data(), (size_t)Ny * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(ss.p, d.data(), (size_t)Ny * 8, cudaMemcpyHostToDevice, s));
  cudaEventRecord(e1, s);
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  green_build_ms = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  green_ready = 1;
  return SCY_OK;
}

// ---------------------------------------------------------------------------
int QDContext::steady_state_guess(std::vector<double>& psi, int keep_psi, std::vector<double>& slip) {
  cudaStream_t s = sbp.stream;
  // Fault::guessSS / computePsiSS (fault.cpp:619-672)
  std::vector<double> tau(Nz), vel(Nz, vL);
  for (int i = 0; i < Nz; ++i) {
    if (!keep_psi) psi[i] = f0 - h_b[i] * std::log(std::fabs(vL) / v0);
    tau[i] = h_sN[i] * h_a[i] * std::asinh(0.5 * vL * std::exp(psi[i] / h_a[i]) / v0);
  }
  SCY_CUDA_TRY(cudaMemcpyAsync(slipVel.p, vel.data(), Nz * 8, cudaMemcpyHostToDevice, s));
  // solve with a traction (Neumann) condition at the fault, bcL = tau
  // (strikeSlip_linearElastic_qd.cpp:60-62, :895-930)
  const int saved[4] = {sbp.bc[0], sbp.bc[1], sbp.bc[2], sbp.bc[3]};
  SCY_TRY(sbp.change_bc(saved[0], saved[1], SCY_BC_NEUMANN, saved[3]));
  std::vector<double> zeros((size_t)std::max(Ny, Nz), 0.0);
  SCY_CUDA_TRY(cudaMemcpyAsync(bcL.p, tau.data(), Nz * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(bcR.p, zeros.data(), Nz * 8, cudaMemcpyHostToDevice, s));
  SCY_TRY(sbp.set_rhs(bcL.as<double>(), bcR.as<double>(), bcT.as<double>(), bcB.as<double>(), rhs.as<double>()));
  scy_solve_opts o = solve_opts;
  o.nonzero_guess = 0;
  o.max_its = std::max(o.max_its, 500);
  scy_solve_stats st{};
  int rc = sbp.solve(rhs.as<double>(), u.as<double>(), o, st);
  if (rc != SCY_OK) {
    sbp.change_bc(saved[0], saved[1], saved[2], saved[3]);
    return rc;
  }
  std::vector<double> hu((size_t)N);
  SCY_CUDA_TRY(cudaMemcpyAsync(hu.data(), u.p, N * 8, cudaMemcpyDeviceToHost, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  // solveSSb (strikeSlip_linearElastic_qd.cpp:934-1006): shift u to be
  // non-negative, take bcRShift from y = Ly and slip from y = 0
  double mn = *std::min_element(hu.begin(), hu.end());
  if (mn < 0) {
    double add = std::fabs(mn);
    for (auto& v : hu) v += add;
  }
  std::vector<double> shift(hu.end() - Nz, hu.end()), uL(hu.begin(), hu.begin() + Nz);
  slip.resize(Nz);
  for (int i = 0; i < Nz; ++i) slip[i] = uL[i] * fts;
  SCY_CUDA_TRY(cudaMemcpyAsync(u.p, hu.data(), N * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(bcRShift.p, shift.data(), Nz * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(bcR.p, shift.data(), Nz * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(bcL.p, uL.data(), Nz * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  SCY_TRY(sbp.change_bc(saved[0], saved[1], saved[2], saved[3]));
  return SCY_OK;
}

double QDContext::compute_min_dt(const std::vector<double>& cs, double Ly, double Lz) const {
  const LevelHost& h = sbp.hosts[0];
  double m = INFINITY;
  const double ry = 1.0 / (Ny - 1), rz_ = 1.0 / (Nz - 1);
  for (long i = 0; i < N; ++i) {
    double dy = h.grid_type == 1 ? h.yq[i] * ry : Ly / (Ny - 1.0);
    double dz = h.grid_type == 1 ? h.zr[i] * rz_ : Lz / (Nz - 1.0);
    m = std::min(m, std::min(dy / cs[i], dz / cs[i]));
  }
  return m;
}

double QDContext::compute_step_size(double totErr) {
  const double ord = ode.method == SCY_RK32 ? 3.0 : 4.0;
  const double kappa = 0.9;
  double ratio;
  if (ode.control == SCY_CTRL_P) {
    ratio = kappa * std::pow(totTol / totErr, 1.0 / (1.0 + ord));
  } else {
    const double alpha = 0.49 / ord, beta = 0.34 / ord, gamma = 0.1 / ord;
    if (stepCount < 4)
      ratio = kappa * std::pow(totTol / totErr, 1.0 / (1.0 + ord));
    else
      ratio = kappa * std::pow(totTol / totErr, alpha) * std::pow(errA[0] / totTol, beta) *
              std::pow(totTol / errA[1], gamma);
  }
  double dt = ratio * deltaT;
  dt = std::min(deltaT * 5.0, dt);
  dt = std::min(ode.max_dt, dt);
  dt = std::max(ode.min_dt, dt);
  if (ode.min_dt == dt)
    ++numMin;
  else if (ode.max_dt == dt)
    ++numMax;
  return dt;
}

int QDContext::compute_error(const double* lo, const double* hi, double* err) {
  cudaStream_t s = sbp.stream;
  KeyTable kt;
  for (int k = 0; k < 4; ++k) {
    kt.off[k] = key_off[k];
    kt.len[k] = key_len[k];
  }
  rk_error_kernel<<<pl ? 4 : 2, 1024, 0, s>>>(lo, hi, kt, errbuf.as<double>());
  SCY_LAUNCH_CHECK();
  double h[12];
  SCY_CUDA_TRY(cudaMemcpyAsync(h, errbuf.p, (pl ? 12 : 6) * sizeof(double), cudaMemcpyDeviceToHost, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  *err = error_from(h);
  return SCY_OK;
}

double QDContext::error_from(const double* h) const {
  double tot = 0.0;
  for (int i = 0; i < ode.n_err; ++i) {
    int key = ode.err_keys[i];
    double scale = ode.err_scale[i];
    double ss = h[key * 3 + 0], sh = h[key * 3 + 1], mx = h[key * 3 + 2];
    if (ode.norm == SCY_NORM_L2_ABS) {
      tot += std::sqrt(ss) / (std::sqrt((double)key_len[key]) * scale);
    } else if (ode.method == SCY_RK32) {
      tot += std::sqrt(ss) / (std::sqrt(sh) * scale);
    } else {
      tot += mx / scale;
    }
  }
  return tot;
}

static Combo combo(std::initializer_list<std::pair<const double*, double>> terms) {
  Combo c{};
  int i = 0;
  for (auto& t : terms) {
    c.f[i] = t.first;
    c.c[i] = t.second;
    ++i;
  }
  c.nf = i;
  return c;
}


int QDContext::attempt(double dt, double** lo, double** hi) {
  cudaStream_t s = sbp.stream;
  const long n = nvar;
  const int tb = 256, gb = (int)((n + tb - 1) / tb);
  double* var = rk[V_VAR].as<double>();
  double* f0 = rk[V_DVAR].as<double>();
  double* k = rk[V_K].as<double>();
  double* L = rk[V_LO].as<double>();
  double* H = rk[V_HI].as<double>();
  const double t = currT;
  if (ode.method == SCY_RK32) {
    double* fa = rk[V_F1].as<double>();
    double* fb = rk[V_F2].as<double>();
    rk_combine_kernel<<<gb, tb, 0, s>>>(k, var, combo({{f0, 0.5 * dt}}), n);
    SCY_LAUNCH_CHECK();
    SCY_TRY(d_dt(t + 0.5 * dt, k, fa));
    rk_combine_kernel<<<gb, tb, 0, s>>>(k, var, combo({{f0, -dt}, {fa, 2 * dt}}), n);
    SCY_LAUNCH_CHECK();
    SCY_TRY(d_dt(t + dt, k, fb));
    rk_combine_kernel<<<gb, tb, 0, s>>>(L, var, combo({{f0, 0.5 * dt}, {fb, 0.5 * dt}}), n);
    SCY_LAUNCH_CHECK();
    rk_combine_kernel<<<gb, tb, 0, s>>>(H, var, combo({{f0, dt / 6.0}, {fa, 2 * dt / 3.0}, {fb, dt / 6.0}}), n);
    SCY_LAUNCH_CHECK();
  } else {
    using namespace rk43;
    double* f2 = rk[V_F2].as<double>();
    double* f3 = rk[V_F3].as<double>();
    double* f4 = rk[V_F4].as<double>();
    double* f5 = rk[V_F5].as<double>();
    double* f6 = rk[V_F6].as<double>();
    rk_combine_kernel<<<gb, tb, 0, s>>>(k, var, combo({{f0, a21 * dt}}), n);
    SCY_LAUNCH_CHECK();
    SCY_TRY(d_dt(t + c2 * dt, k, f2));
    rk_combine_kernel<<<gb, tb, 0, s>>>(k, var, combo({{f0, a31 * dt}, {f2, a32 * dt}}), n);
    SCY_LAUNCH_CHECK();
    SCY_TRY(d_dt(t + c3 * dt, k, f3));
    rk_combine_kernel<<<gb, tb, 0, s>>>(k, var, combo({{f0, a41 * dt}, {f2, a42 * dt}, {f3, a43 * dt}}), n);
    SCY_LAUNCH_CHECK();
    SCY_TRY(d_dt(t + c4 * dt, k, f4));
    rk_combine_kernel<<<gb, tb, 0, s>>>(k, var,
                                        combo({{f0, a51 * dt}, {f2, a52 * dt}, {f3, a53 * dt}, {f4, a54 * dt}}), n);
    SCY_LAUNCH_CHECK();
    SCY_TRY(d_dt(t + c5 * dt, k, f5));
    rk_combine_kernel<<<gb, tb, 0, s>>>(
        k, var, combo({{f0, a61 * dt}, {f2, a62 * dt}, {f3, a63 * dt}, {f4, a64 * dt}, {f5, a65 * dt}}), n);
    SCY_LAUNCH_CHECK();
    SCY_TRY(d_dt(t + c6 * dt, k, f6));
    rk_combine_kernel<<<gb, tb, 0, s>>>(
        L, var, combo({{f0, hb1 * dt}, {f3, hb3 * dt}, {f4, hb4 * dt}, {f5, hb5 * dt}, {f6, hb6 * dt}}), n);
    SCY_LAUNCH_CHECK();
    rk_combine_kernel<<<gb, tb, 0, s>>>(
        H, var, combo({{f0, b1 * dt}, {f3, b3 * dt}, {f4, b4 * dt}, {f5, b5 * dt}, {f6, b6 * dt}}), n);
    SCY_LAUNCH_CHECK();
  }
  *lo = L;
  *hi = H;
  return SCY_OK;
}

// setErrInds: an empty list means every integrated field in the map's
// sorted key order (odeSolver.cpp:77-95)
int QDContext::check_err_keys(scy_ode_opts& o) const {
  if (o.n_err <= 0) {
    const int le[2] = {SCY_KEY_PSI, SCY_KEY_SLIP};
    const int pk[4] = {SCY_KEY_GVXY, SCY_KEY_GVXZ, SCY_KEY_PSI, SCY_KEY_SLIP};
    o.n_err = pl ? 4 : 2;
    for (int i = 0; i < o.n_err; ++i) {
      o.err_keys[i] = pl ? pk[i] : le[i];
      o.err_scale[i] = 1.0;
    }
  }
  if (o.n_err > 4) {
    set_error("at most four error indices");
    return SCY_ERR_ARG;
  }
  for (int i = 0; i < o.n_err; ++i)
    if (o.err_keys[i] < 0 || o.err_keys[i] > 3 || key_len[o.err_keys[i]] == 0) {
      set_error("error index %d names no integrated variable", o.err_keys[i]);
      return SCY_ERR_ARG;
    }
  return SCY_OK;
}

int QDContext::integrate_begin(const scy_ode_opts& o) {
  ode = o;
  if (ode.method != SCY_RK32 && ode.method != SCY_RK43) {
    set_error("unsupported integrator %d", ode.method);
    return SCY_ERR_ARG;
  }
  SCY_TRY(check_err_keys(ode));
  totTol = o.tol;
  currT = o.t0;
  deltaT = o.init_dt;
  newDeltaT = o.init_dt;
  stepCount = 0;
  numRejected = numMin = numMax = 0;
  errA[0] = errA[1] = 0.0;
  if (deltaT == 0) deltaT = (o.t1 - o.t0) / (double)o.max_steps;
  ode_ready = 1;
  // the driver's timeMonitor(initTime, initDeltaT, 0) before integrating
  // (strikeSlip_linearElastic_qd.cpp:733-735)
  if (out) SCY_TRY(out->on_step(*this, 0, currT, o.init_dt));
  if (ckpt > 0) SCY_TRY(write_checkpoint());  // stepCount 0: 0 % interval == 0
  // first evaluation of the rates (odeSolver.cpp:545)
  SCY_TRY(d_dt(currT, rk[V_VAR].as<double>(), rk[V_DVAR].as<double>()));
  return read_flags();
}

int QDContext::phase_begin(double t0, double t1, double init_dt, double min_dt, double max_dt, long step0,
                           long max_rel) {
  if (ode.method != SCY_RK32 && ode.method != SCY_RK43) {
    set_error("phase_begin: integrator settings missing");
    return SCY_ERR_STATE;
  }
  ode.t0 = t0;
  ode.t1 = t1;
  ode.init_dt = init_dt;
  ode.min_dt = min_dt;
  ode.max_dt = max_dt;
  ode.max_steps = step0 + max_rel;
  totTol = ode.tol;
  currT = t0;
  deltaT = init_dt;
  newDeltaT = init_dt;
  stepCount = step0;
  numRejected = numMin = numMax = 0;
  errA[0] = errA[1] = 0.0;
  phase_stopped = 0;
  if (deltaT == 0) deltaT = (t1 - t0) / (double)ode.max_steps;
  ode_ready = 1;
  if (ode.max_steps == 0) return SCY_OK;
  SCY_TRY(d_dt(currT, rk[V_VAR].as<double>(), rk[V_DVAR].as<double>()));
  return read_flags();
}

int QDContext::integrate_steps(long nsteps, scy_ode_stats* st) {
  if (!ode_ready) {
    set_error("integrate_steps called before integrate_begin");
    return SCY_ERR_STATE;
  }
  cudaStream_t s = sbp.stream;
  double* var = rk[V_VAR].as<double>();
  double* dvar = rk[V_DVAR].as<double>();
  const long n = nvar;
  ckpt_stopped = 0;
  long done_steps = 0;
  double totErr = 0.0, used_dt = 0.0;
  while (done_steps < nsteps && stepCount < ode.max_steps && currT < ode.t1) {
    ++stepCount;
    int attemptCount = 0;
    double *lo = nullptr, *hi = nullptr;
    while (attemptCount < 100) {
      ++attemptCount;
      if (currT + deltaT > ode.t1) deltaT = ode.t1 - currT;
      bool forced = forced_pos < forced_dt.size();
      int forced_accept = 0;
      if (forced) {
        deltaT = forced_dt[forced_pos];
        forced_accept = forced_acc[forced_pos];
        ++forced_pos;
      }
      SCY_TRY(attempt(deltaT, &lo, &hi));
      used_dt = deltaT;
      SCY_TRY(compute_error(lo, hi, &totErr));
      SCY_TRY(read_flags());
      bool acc = (ode.method == SCY_RK32 && !imex) ? (totErr <= totTol) : (totErr < totTol);
      if (forced) acc = forced_accept != 0;
      if (record) {
        log_dt.push_back(deltaT);
        log_acc.push_back(acc ? 1 : 0);
      }
      if (acc) break;
      double nd = compute_step_size(totErr);
      if (!forced) deltaT = nd;
      if (ode.min_dt == deltaT) break;
      ++numRejected;
    }
    // accept the higher-order solution (odeSolver.cpp:599-603, :1148-1152)
    if (record) log_step_dt.push_back(used_dt);
    currT = currT + deltaT;
    SCY_CUDA_TRY(cudaMemcpyAsync(var, hi, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    // the IMEX d_dt (strikeSlip_linearElastic_qd.cpp:800-870): coupled, the
    // fault takes the heat equation's temperature first; after the rates,
    // one backward-Euler heat step with the new slip velocity and tauP
    if (th && th->coupled) SCY_TRY(th->set_fault_temperature());
    SCY_TRY(d_dt(currT, var, dvar));
    SCY_TRY(read_flags());
    if (th) SCY_TRY(th->step(*this, deltaT));
    if (totErr != 0.0) newDeltaT = compute_step_size(totErr);
    errA[1] = errA[0];
    errA[0] = totErr;
    last_dt = deltaT;
    ++done_steps;
    // timeMonitor (odeSolver.cpp:608): output, then a checkpoint that ends the run
    if (out) SCY_TRY(out->on_step(*this, stepCount, currT, deltaT));
    if (ckpt > 0 && ((ckpt_interval > 0 && stepCount % ckpt_interval == 0) || stepCount >= ode.max_steps ||
                     currT >= ode.t1)) {
      SCY_TRY(write_checkpoint());
      ckpt_stopped = 1;
      deltaT = newDeltaT;  // as a run restarted from the checkpoint would take it
      break;
    }
    if (monitor) {
      int stop = 0;
      SCY_TRY(monitor(&stop));
      if (stop) {
        phase_stopped = 1;
        break;
      }
    }
    deltaT = newDeltaT;
  }
  if (st) {
    st->t = currT;
    st->dt = last_dt;
    st->new_dt = newDeltaT;
    st->step_count = stepCount;
    st->rejected = numRejected;
    st->d_dt_evals = n_d_dt;
    st->solve_its = n_solve_its;
    st->solves = n_solves;
    st->errA[0] = errA[0];
    st->errA[1] = errA[1];
    st->done = ckpt_stopped ? 2 : (stepCount >= ode.max_steps || currT >= ode.t1) ? 1 : 0;
  }
  return SCY_OK;
}

// StrikeSlip_LinearElastic_qd::writeCheckpoint (:527-556), LinearElastic::
// writeCheckpoint (linearElastic.cpp:689-702) and Fault::writeCheckpoint
// (fault.cpp:561-578): the step's scalars as ASCII, the fields as PETSc
// binary Vecs, all under ckpt_dir.
int QDContext::write_checkpoint() {
  cudaStream_t s = sbp.stream;
  if (out) SCY_TRY(out->flush());
  auto get = [&](const void* src, size_t n, std::vector<double>& h) -> int {
    h.resize(n);
    SCY_CUDA_TRY(cudaMemcpyAsync(h.data(), src, n * 8, cudaMemcpyDeviceToHost, s));
    return SCY_OK;
  };
  std::vector<double> slip, vel, psi, sn, tau, tq, pre, bR, bS, bT, bL, bB;
  const double* var = rk[V_VAR].as<double>();
  SCY_TRY(get(var + fp.slip_off, Nz, slip));
  SCY_TRY(get(slipVel.p, Nz, vel));
  SCY_TRY(get(var + fp.psi_off, Nz, psi));
  SCY_TRY(get(fsN.p, Nz, sn));
  SCY_TRY(get(tauP.p, Nz, tau));
  SCY_TRY(get(tauQSP.p, Nz, tq));
  SCY_TRY(get(fprestress.p, Nz, pre));
  SCY_TRY(get(bcR.p, Nz, bR));
  SCY_TRY(get(bcRShift.p, Nz, bS));
  SCY_TRY(get(bcT.p, Ny, bT));
  SCY_TRY(get(bcL.p, Nz, bL));
  SCY_TRY(get(bcB.p, Ny, bB));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  ++ckpt_number;
  auto ascii = [&](const char* name, const char* fmt, double v, bool integer) -> int {
    FILE* f = fopen((ckpt_dir + name).c_str(), "w");
    if (!f) {
      set_error("cannot write %s%s", ckpt_dir.c_str(), name);
      return SCY_ERR_IO;
    }
    if (integer)
      fprintf(f, fmt, (long)v);
    else
      fprintf(f, fmt, v);
    fclose(f);
    return SCY_OK;
  };
  SCY_TRY(ascii("ckptNumber", "%ld\n", ckpt_number, true));
  SCY_TRY(ascii("chkpt_currT", "%.15e\n", currT, false));
  SCY_TRY(ascii("chkpt_stepCount", "%ld\n", (double)stepCount, true));
  SCY_TRY(ascii("chkpt_prevErr", "%.15e\n", errA[1], false));
  SCY_TRY(ascii("chkpt_currErr", "%.15e\n", errA[0], false));
  SCY_TRY(ascii("chkpt_deltaT", "%.15e\n", newDeltaT, false));
  try {
    const std::string c = ckpt_dir + "chkpt_";
    write_petsc_vec(c + "momBal_bcR", bR.data(), Nz, 0);
    write_petsc_vec(c + "momBal_bcRShift", bS.data(), Nz, 0);
    write_petsc_vec(c + "momBal_bcT", bT.data(), Ny, 0);
    write_petsc_vec(c + "momBal_bcL", bL.data(), Nz, 0);
    write_petsc_vec(c + "momBal_bcB", bB.data(), Ny, 0);
    write_petsc_vec(c + "slip", slip.data(), Nz, 0);
    write_petsc_vec(c + "slipVel", vel.data(), Nz, 0);
    write_petsc_vec(c + "psi", psi.data(), Nz, 0);
    write_petsc_vec(c + "sNEff", sn.data(), Nz, 0);
    write_petsc_vec(c + "sN", sn.data(), Nz, 0);
    write_petsc_vec(c + "tau", tau.data(), Nz, 0);
    write_petsc_vec(c + "tauQS", tq.data(), Nz, 0);
    write_petsc_vec(c + "prestress", pre.data(), Nz, 0);
  } catch (const std::exception& e) {
    set_error("%s", e.what());
    return SCY_ERR_IO;
  }
  return SCY_OK;
}

}  // namespace scy
