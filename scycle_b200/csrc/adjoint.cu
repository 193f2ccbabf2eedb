// Discrete adjoint of the quasi-dynamic RK32 integration (see adjoint.hpp).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "adjoint.hpp"
#include "capi_types.hpp"
#include "common.cuh"

namespace scy {

namespace {

// out = c0 f0 + y (+ c_j f_j ...), in the single driver's order
struct AxCombo {
  const double* f[3];
  double c[3];
  int nf;
};

__global__ void adj_combine_kernel(double* __restrict__ out, const double* __restrict__ y, AxCombo cb, long n) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v = cb.c[0] * cb.f[0][i] + y[i];
  for (int j = 1; j < cb.nf; ++j) v = v + cb.c[j] * cb.f[j][i];
  out[i] = v;
}

// y += a x over n entries
__global__ void adj_axpy_kernel(double* __restrict__ y, const double* __restrict__ x, double a, long n) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) y[i] += a * x[i];
}

// y = a x over n entries
__global__ void adj_scale_kernel(double* __restrict__ y, const double* __restrict__ x, double a, long n) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * x[i];
}

// psi, V and tau of an evaluation (3 Nz); the surface displacement (Ny) for
// evaluations at accepted states
__global__ void adj_capture_kernel(const double* __restrict__ y, long psi_off, const double* __restrict__ V,
                                   const double* __restrict__ tq, const double* __restrict__ u, int Ny, int Nz,
                                   double* __restrict__ ev, double* __restrict__ evs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < Nz) {
    ev[i] = y[psi_off + i];
    ev[Nz + i] = V[i];
    ev[2 * Nz + i] = tq[i];
  }
  if (evs && i < Ny) evs[i] = u[(long)i * Nz];
}

// observations of an accepted state and its misfit term
__global__ void adj_misfit_kernel(const double* __restrict__ V, const double* __restrict__ u, int Ny, int Nz,
                                  const double* __restrict__ ts, const double* __restrict__ tv, double ws, double wv,
                                  double* __restrict__ obs_s, double* __restrict__ obs_v, double* __restrict__ Jn) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < Ny; i += blockDim.x) {
    const double s = u[(long)i * Nz];
    obs_s[i] = s;
    if (ts) {
      const double d = s - ts[i];
      acc += ws * d * d;
    }
  }
  for (int i = threadIdx.x; i < Nz; i += blockDim.x) {
    obs_v[i] = V[i];
    if (tv) {
      const double d = V[i] - tv[i];
      acc += wv * d * d;
    }
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) *Jn = acc;
}

// Per fault node: the reverse of Fault_qd::d_dt.  Cotangents in: of dpsi and
// dslip (lf) and of V from the misfit; out: of psi (added to ly), of tau
// (ltau), and of a, b, Dc (added to grad).
__global__ void adj_fault_kernel(const double* __restrict__ ev, FaultParams fp, const double* __restrict__ lf,
                                 const double* __restrict__ tv, double wv, double* __restrict__ ly,
                                 double* __restrict__ ltau, double* __restrict__ grad) {
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  const int Nz = fp.Nz;
  if (iz >= Nz) return;
  const double psi = ev[iz], V = ev[Nz + iz];
  const double a = fp.a[iz], b = fp.b[iz], Dc = fp.Dc[iz], sN = fp.sN[iz], eta = fp.eta[iz];
  const double v0 = fp.v0, f0 = fp.f0;
  const double l_dpsi = lf[fp.psi_off + iz];
  double lV = lf[fp.slip_off + iz];
  if (tv) lV += 2.0 * wv * (V - tv[iz]);
  // state law partials g_V, g_psi, g_a, g_b, g_Dc
  double gV = 0.0, gpsi = 0.0, ga = 0.0, gb = 0.0, gDc = 0.0;
  if (fp.state_law == 0) {
    const double A = exp((f0 - psi) / b);
    if (!isinf(A) && b > 1e-3) {
      const double g = (b * v0 / Dc) * (A - V / v0);
      gV = -b / Dc;
      gpsi = -(v0 / Dc) * A;
      gb = (v0 / Dc) * (A - V / v0) - (v0 / Dc) * A * (f0 - psi) / b;
      gDc = -g / Dc;
    }
  } else if (fp.state_law == 1 && V != 0.0) {
    const double absV = fabs(V), sg = V > 0.0 ? 1.0 : -1.0;
    const double X = (absV / 2.0 / v0) * exp(psi / a), S = sqrt(1.0 + X * X);
    const double h = a * asinh(X) - (f0 + (a - b) * log(absV / v0));
    const double g = -absV / Dc * h;
    gV = sg * (-h / Dc - (a * X / S - (a - b)) / Dc);
    gpsi = -(absV / Dc) * X / S;
    ga = -(absV / Dc) * (asinh(X) - X * psi / (a * S) - log(absV / v0));
    gb = -(absV / Dc) * log(absV / v0);
    gDc = -g / Dc;
  }
  lV += l_dpsi * gV;
  double lpsi = l_dpsi * gpsi, la = l_dpsi * ga, lt = 0.0;
  const double lk = fp.locked[iz];
  if (!(lk > 0.5) && !(lk < -0.5)) {
    // V from F(V) = a sN asinh(X) - (tau - eta V) = 0, X = V/(2 v0) e^(psi/a)
    const double E = exp(psi / a);
    const double X = (0.5 * V / v0) * E, S = sqrt(1.0 + X * X);
    const double FV = a * sN * (0.5 * E / v0) / S + eta;
    const double Fpsi = sN * X / S;
    const double Fa = sN * asinh(X) - sN * X * psi / (a * S);
    const double m = lV / FV;
    lt = m;
    lpsi -= m * Fpsi;
    la -= m * Fa;
  }
  ly[fp.psi_off + iz] += lpsi;
  ltau[iz] = lt;
  grad[iz] += la;
  grad[Nz + iz] += l_dpsi * gb;
  grad[2 * Nz + iz] += l_dpsi * gDc;
}

// lu = d tau / d u ^T ltau: tau(iz) = mu(iz) [qy(iz)] sum_k D0[k] u(k, iz), k = 0..4
__global__ void adj_tau_scatter_kernel(LevelDev<double> L, const double* __restrict__ ltau, double* __restrict__ lu) {
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  const int Nz = L.Nz;
  if (iz >= Nz) return;
  double s = L.mu[iz] * ltau[iz];
  if (L.var) s *= L.qy[iz];
#pragma unroll
  for (int j = HALF; j < BAND; ++j) {
    const int k = j - HALF;
    if (k < L.Ny) lu[(long)k * Nz + iz] += L.y.D[j] * s;
  }
}

// lu(iy, 0) += 2 ws (surfDisp(iy) - target(iy))
__global__ void adj_surf_kernel(const double* __restrict__ us, const double* __restrict__ ts, double ws, int Ny,
                                int Nz, double* __restrict__ lu) {
  const int iy = blockIdx.x * blockDim.x + threadIdx.x;
  if (iy < Ny) lu[(long)iy * Nz] += 2.0 * ws * (us[iy] - ts[iy]);
}

// ly[slip] += (M_L^T w) / faultTypeScale: the setRhs column of bcL
__global__ void adj_bcl_kernel(LevelDev<double> L, const double* __restrict__ w, double inv_fts, long slip_off,
                               double* __restrict__ ly) {
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  const int Ny = L.Ny, Nz = L.Nz;
  if (iz >= Nz) return;
  double s = 0.0;
  if (L.y.bc_lo == 0) {
    for (int iy = 0; iy < BAND && iy < Ny; ++iy) {
      const long node = (long)iy * Nz + iz;
      s += L.wy[node] * (L.y.bs0[iy] + (iy == 0 ? L.y.alphaD : 0.0)) * L.cy[iz] * w[node];
    }
  } else {
    s = L.wy[iz] * w[iz];
  }
  ly[slip_off + iz] += inv_fts * s;
}

int blocks(long n, int tb) { return (int)((n + tb - 1) / tb); }

}  // namespace

int AdjointContext::create(QDContext* qd, int checkpoint_every) {
  q = qd;
  ck = checkpoint_every;
  if (q->pl || q->mode != SCY_QD_MODE_SOLVE) {
    set_error("the adjoint covers the linear-elastic driver in solve mode");
    return SCY_ERR_ARG;
  }
  if (q->ode.method != SCY_RK32 || !q->ode_ready) {
    set_error("the adjoint needs a begun RK32 driver");
    return SCY_ERR_STATE;
  }
  if (ck < 1) {
    set_error("checkpoint interval must be >= 1");
    return SCY_ERR_ARG;
  }
  const long nv = q->nvar, Nz = q->Nz, Ny = q->Ny, N = q->N;
  t0 = q->currT;
  SCY_TRY(y0.alloc(nv * 8));
  SCY_CUDA_TRY(cudaMemcpy(y0.p, q->rk[V_VAR].p, nv * 8, cudaMemcpyDeviceToDevice));
  // the slip velocity at the start is the root finder's first guess
  SCY_TRY(v0.alloc(Nz * 8));
  SCY_CUDA_TRY(cudaMemcpy(v0.p, q->slipVel.p, Nz * 8, cudaMemcpyDeviceToDevice));
  for (DevBuf* b : {&ly, &lF0, &lf0, &lf1, &lf2, &lk, &yk}) SCY_TRY(b->alloc(nv * 8));
  SCY_TRY(ltau.alloc(Nz * 8));
  SCY_TRY(lu.alloc(N * 8));
  SCY_TRY(w.alloc(N * 8));
  SCY_TRY(grad.alloc(3 * Nz * 8));
  SCY_TRY(ev.alloc((size_t)(ck + 1) * 3 * 3 * Nz * 8));
  SCY_TRY(evs.alloc((size_t)(ck + 1) * Ny * 8));
  return SCY_OK;
}

int AdjointContext::set_steps(const double* dt, long n) {
  if (n < 1) {
    set_error("at least one step");
    return SCY_ERR_ARG;
  }
  dts.assign(dt, dt + n);
  M = n;
  const long nck = M / ck + 1;
  SCY_TRY(ckpt.alloc((size_t)nck * q->nvar * 8));
  SCY_TRY(Jn.alloc(M * 8));
  SCY_TRY(obs_s.alloc((size_t)M * q->Ny * 8));
  SCY_TRY(obs_v.alloc((size_t)M * q->Nz * 8));
  have_targets = 0;
  return SCY_OK;
}

int AdjointContext::set_targets(const double* surf, const double* vel, double ws, double wv) {
  if (!M) {
    set_error("set the steps first");
    return SCY_ERR_STATE;
  }
  SCY_TRY(tgt_s.alloc((size_t)M * q->Ny * 8));
  SCY_TRY(tgt_v.alloc((size_t)M * q->Nz * 8));
  SCY_CUDA_TRY(cudaMemcpy(tgt_s.p, surf, (size_t)M * q->Ny * 8, cudaMemcpyHostToDevice));
  SCY_CUDA_TRY(cudaMemcpy(tgt_v.p, vel, (size_t)M * q->Nz * 8, cudaMemcpyHostToDevice));
  w_s = ws;
  w_v = wv;
  have_targets = 1;
  return SCY_OK;
}

int AdjointContext::set_fault_params(const double* a, const double* b, const double* Dc) {
  const size_t n = (size_t)q->Nz * 8;
  cudaStream_t s = q->sbp.stream;
  if (a) SCY_CUDA_TRY(cudaMemcpyAsync(q->fa.p, a, n, cudaMemcpyHostToDevice, s));
  if (b) SCY_CUDA_TRY(cudaMemcpyAsync(q->fb.p, b, n, cudaMemcpyHostToDevice, s));
  if (Dc) SCY_CUDA_TRY(cudaMemcpyAsync(q->fDc.p, Dc, n, cudaMemcpyHostToDevice, s));
  if (a) q->h_a.assign(a, a + q->Nz);
  if (b) q->h_b.assign(b, b + q->Nz);
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  return SCY_OK;
}

int AdjointContext::stage_combine(double* out, const double* y,
                                  std::initializer_list<std::pair<const double*, double>> terms) {
  AxCombo cb{};
  int j = 0;
  for (auto& t : terms) {
    cb.f[j] = t.first;
    cb.c[j] = t.second;
    ++j;
  }
  cb.nf = j;
  adj_combine_kernel<<<blocks(q->nvar, 256), 256, 0, q->sbp.stream>>>(out, y, cb, q->nvar);
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

// d_dt at (t, y) into f; with store, psi / V / tau (and surfDisp for e = 0)
// into evaluation slot (slot, e)
int AdjointContext::eval(double t, const double* y, double* f, long slot, int e, int store) {
  SCY_TRY(q->d_dt(t, y, f));
  if (store) {
    const int Nz = q->Nz, Ny = q->Ny;
    double* evp = ev.as<double>() + ((size_t)slot * 3 + e) * 3 * Nz;
    double* evsp = e == 0 ? evs.as<double>() + (size_t)slot * Ny : nullptr;
    adj_capture_kernel<<<blocks(std::max(Nz, Ny), 128), 128, 0, q->sbp.stream>>>(
        y, q->fp.psi_off, q->slipVel.as<double>(), q->tauQSP.as<double>(), q->u.as<double>(), Ny, Nz, evp, evsp);
    SCY_LAUNCH_CHECK();
  }
  return SCY_OK;
}

int AdjointContext::forward(double* J, int keep_checkpoints) {
  if (!M) {
    set_error("set the steps first");
    return SCY_ERR_STATE;
  }
  cudaStream_t s = q->sbp.stream;
  const long nv = q->nvar;
  const int Ny = q->Ny, Nz = q->Nz;
  double* var = q->rk[V_VAR].as<double>();
  double* f0 = q->rk[V_DVAR].as<double>();
  double* k = q->rk[V_K].as<double>();
  double* f1 = q->rk[V_F1].as<double>();
  double* f2 = q->rk[V_F2].as<double>();
  double* hi = q->rk[V_HI].as<double>();
  SCY_CUDA_TRY(cudaMemcpyAsync(var, y0.p, nv * 8, cudaMemcpyDeviceToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(q->slipVel.p, v0.p, Nz * 8, cudaMemcpyDeviceToDevice, s));
  double t = t0;
  SCY_TRY(eval(t, var, f0, 0, 0, 0));
  for (long n = 0; n < M; ++n) {
    if (keep_checkpoints && n % ck == 0)
      SCY_CUDA_TRY(cudaMemcpyAsync(ckpt.as<double>() + (size_t)(n / ck) * nv, var, nv * 8, cudaMemcpyDeviceToDevice, s));
    const double dt = dts[n];
    SCY_TRY(stage_combine(k, var, {{f0, 0.5 * dt}}));
    SCY_TRY(eval(t + 0.5 * dt, k, f1, 0, 0, 0));
    SCY_TRY(stage_combine(k, var, {{f0, -dt}, {f1, 2 * dt}}));
    SCY_TRY(eval(t + dt, k, f2, 0, 0, 0));
    SCY_TRY(stage_combine(hi, var, {{f0, dt / 6.0}, {f1, 2 * dt / 3.0}, {f2, dt / 6.0}}));
    SCY_CUDA_TRY(cudaMemcpyAsync(var, hi, nv * 8, cudaMemcpyDeviceToDevice, s));
    t = t + dt;
    SCY_TRY(eval(t, var, f0, 0, 0, 0));
    adj_misfit_kernel<<<1, 256, 0, s>>>(q->slipVel.as<double>(), q->u.as<double>(), Ny, Nz,
                                        have_targets ? tgt_s.as<double>() + (size_t)n * Ny : nullptr,
                                        have_targets ? tgt_v.as<double>() + (size_t)n * Nz : nullptr, w_s, w_v,
                                        obs_s.as<double>() + (size_t)n * Ny, obs_v.as<double>() + (size_t)n * Nz,
                                        Jn.as<double>() + n);
    SCY_LAUNCH_CHECK();
  }
  SCY_TRY(q->read_flags());
  std::vector<double> h(M);
  SCY_CUDA_TRY(cudaMemcpy(h.data(), Jn.p, M * 8, cudaMemcpyDeviceToHost));
  double sum = 0.0;
  for (long n = 0; n < M; ++n) sum += h[n];
  if (J) *J = sum;
  return SCY_OK;
}

// Recomputes steps s0 .. s1-1 from the checkpoint at s0, storing every
// evaluation (slot j = n - s0; the accepted state s1 in slot s1 - s0).
int AdjointContext::segment_forward(long s0, long s1) {
  cudaStream_t s = q->sbp.stream;
  const long nv = q->nvar;
  double* var = q->rk[V_VAR].as<double>();
  double* f0 = q->rk[V_DVAR].as<double>();
  double* k = q->rk[V_K].as<double>();
  double* f1 = q->rk[V_F1].as<double>();
  double* f2 = q->rk[V_F2].as<double>();
  double* hi = q->rk[V_HI].as<double>();
  SCY_CUDA_TRY(cudaMemcpyAsync(var, ckpt.as<double>() + (size_t)(s0 / ck) * nv, nv * 8, cudaMemcpyDeviceToDevice, s));
  double t = t0;
  for (long n = 0; n < s0; ++n) t = t + dts[n];
  SCY_TRY(eval(t, var, f0, 0, 0, 1));
  for (long n = s0; n < s1; ++n) {
    const long j = n - s0;
    const double dt = dts[n];
    SCY_TRY(stage_combine(k, var, {{f0, 0.5 * dt}}));
    SCY_TRY(eval(t + 0.5 * dt, k, f1, j, 1, 1));
    SCY_TRY(stage_combine(k, var, {{f0, -dt}, {f1, 2 * dt}}));
    SCY_TRY(eval(t + dt, k, f2, j, 2, 1));
    SCY_TRY(stage_combine(hi, var, {{f0, dt / 6.0}, {f1, 2 * dt / 3.0}, {f2, dt / 6.0}}));
    SCY_CUDA_TRY(cudaMemcpyAsync(var, hi, nv * 8, cudaMemcpyDeviceToDevice, s));
    t = t + dt;
    SCY_TRY(eval(t, var, f0, j + 1, 0, 1));
  }
  return SCY_OK;
}

// lam_y += (d d_dt / d y)^T lam_f at evaluation (slot, e), plus the misfit of
// accepted state `step` when with_misfit; the parameter part into grad.
int AdjointContext::vjp(long slot, int e, const double* lam_f, double* lam_y, int with_misfit, long step) {
  cudaStream_t s = q->sbp.stream;
  const int Nz = q->Nz, Ny = q->Ny;
  const long N = q->N;
  const LevelDev<double>& L = q->sbp.fine->dev;
  const double* evp = ev.as<double>() + ((size_t)slot * 3 + e) * 3 * Nz;
  const bool mf = with_misfit && have_targets;
  adj_fault_kernel<<<blocks(Nz, 128), 128, 0, s>>>(evp, q->fp, lam_f,
                                                   mf ? tgt_v.as<double>() + (size_t)step * Nz : nullptr, w_v, lam_y,
                                                   ltau.as<double>(), grad.as<double>());
  SCY_LAUNCH_CHECK();
  SCY_CUDA_TRY(cudaMemsetAsync(lu.p, 0, N * 8, s));
  adj_tau_scatter_kernel<<<blocks(Nz, 128), 128, 0, s>>>(L, ltau.as<double>(), lu.as<double>());
  SCY_LAUNCH_CHECK();
  if (mf) {
    adj_surf_kernel<<<blocks(Ny, 128), 128, 0, s>>>(evs.as<double>() + (size_t)slot * Ny,
                                                    tgt_s.as<double>() + (size_t)step * Ny, w_s, Ny, Nz, lu.as<double>());
    SCY_LAUNCH_CHECK();
  }
  // A w = lu (A is symmetric: the adjoint solve is a forward solve)
  scy_solve_opts o = q->solve_opts;
  o.nonzero_guess = 0;
  if (o.check_every < 1) o.check_every = 1;
  scy_solve_stats st{};
  SCY_TRY(q->sbp.solve(lu.as<double>(), w.as<double>(), o, st));
  q->n_solves += 1;
  q->n_solve_its += st.iterations;
  if (q->bcL_from_slip) {
    adj_bcl_kernel<<<blocks(Nz, 128), 128, 0, s>>>(L, w.as<double>(), 1.0 / q->fts, q->fp.slip_off, lam_y);
    SCY_LAUNCH_CHECK();
  }
  return SCY_OK;
}

int AdjointContext::gradient(double* J, double* ga, double* gb, double* gDc) {
  if (!have_targets) {
    set_error("set the targets first");
    return SCY_ERR_STATE;
  }
  SCY_TRY(forward(J, 1));
  cudaStream_t s = q->sbp.stream;
  const long nv = q->nvar;
  const int Nz = q->Nz;
  const int tb = 256, gbk = blocks(nv, tb);
  SCY_CUDA_TRY(cudaMemsetAsync(grad.p, 0, 3 * Nz * 8, s));
  SCY_CUDA_TRY(cudaMemsetAsync(ly.p, 0, nv * 8, s));
  SCY_CUDA_TRY(cudaMemsetAsync(lF0.p, 0, nv * 8, s));
  const long nseg = (M + ck - 1) / ck;
  for (long sg = nseg - 1; sg >= 0; --sg) {
    const long s0 = sg * ck, s1 = std::min(M, s0 + ck);
    SCY_TRY(segment_forward(s0, s1));
    for (long n = s1 - 1; n >= s0; --n) {
      const long j = n - s0;
      const double dt = dts[n];
      // the evaluation at the accepted state n+1: its rates feed f0 of step
      // n+1 (lF0) and its fields the misfit of state n+1
      SCY_TRY(vjp(j + 1, 0, lF0.as<double>(), ly.as<double>(), 1, n));
      // y_{n+1} = y_n + dt/6 f0 + 2dt/3 f1 + dt/6 f2
      adj_scale_kernel<<<gbk, tb, 0, s>>>(lf0.as<double>(), ly.as<double>(), dt / 6.0, nv);
      adj_scale_kernel<<<gbk, tb, 0, s>>>(lf1.as<double>(), ly.as<double>(), 2 * dt / 3.0, nv);
      adj_scale_kernel<<<gbk, tb, 0, s>>>(lf2.as<double>(), ly.as<double>(), dt / 6.0, nv);
      SCY_LAUNCH_CHECK();
      // f2 = d_dt(k2), k2 = y - dt f0 + 2 dt f1
      SCY_CUDA_TRY(cudaMemsetAsync(lk.p, 0, nv * 8, s));
      SCY_TRY(vjp(j, 2, lf2.as<double>(), lk.as<double>(), 0, 0));
      adj_axpy_kernel<<<gbk, tb, 0, s>>>(ly.as<double>(), lk.as<double>(), 1.0, nv);
      adj_axpy_kernel<<<gbk, tb, 0, s>>>(lf0.as<double>(), lk.as<double>(), -dt, nv);
      adj_axpy_kernel<<<gbk, tb, 0, s>>>(lf1.as<double>(), lk.as<double>(), 2 * dt, nv);
      SCY_LAUNCH_CHECK();
      // f1 = d_dt(k1), k1 = y + dt/2 f0
      SCY_CUDA_TRY(cudaMemsetAsync(lk.p, 0, nv * 8, s));
      SCY_TRY(vjp(j, 1, lf1.as<double>(), lk.as<double>(), 0, 0));
      adj_axpy_kernel<<<gbk, tb, 0, s>>>(ly.as<double>(), lk.as<double>(), 1.0, nv);
      adj_axpy_kernel<<<gbk, tb, 0, s>>>(lf0.as<double>(), lk.as<double>(), 0.5 * dt, nv);
      SCY_LAUNCH_CHECK();
      SCY_CUDA_TRY(cudaMemcpyAsync(lF0.p, lf0.p, nv * 8, cudaMemcpyDeviceToDevice, s));
    }
  }
  // f0 at the initial state (its state cotangent is not needed)
  SCY_TRY(segment_forward(0, 0));
  SCY_TRY(vjp(0, 0, lF0.as<double>(), ly.as<double>(), 0, 0));
  SCY_TRY(q->read_flags());
  std::vector<double> g(3 * Nz);
  SCY_CUDA_TRY(cudaMemcpy(g.data(), grad.p, 3 * Nz * 8, cudaMemcpyDeviceToHost));
  if (ga) std::memcpy(ga, g.data(), Nz * 8);
  if (gb) std::memcpy(gb, g.data() + Nz, Nz * 8);
  if (gDc) std::memcpy(gDc, g.data() + 2 * Nz, Nz * 8);
  return SCY_OK;
}

int AdjointContext::observations(double* surf, double* vel) {
  if (!M) {
    set_error("run the forward first");
    return SCY_ERR_STATE;
  }
  if (surf) SCY_CUDA_TRY(cudaMemcpy(surf, obs_s.p, (size_t)M * q->Ny * 8, cudaMemcpyDeviceToHost));
  if (vel) SCY_CUDA_TRY(cudaMemcpy(vel, obs_v.p, (size_t)M * q->Nz * 8, cudaMemcpyDeviceToHost));
  return SCY_OK;
}

}  // namespace scy

// ---------------------------------------------------------------------------
struct scy_adj {
  scy::AdjointContext ctx;
};

extern "C" {

scy_status scy_adj_create(scy_qd* q, int checkpoint_every, scy_adj** out) {
  if (!q || !out) return SCY_ERR_ARG;
  *out = nullptr;
  scy_adj* a = new (std::nothrow) scy_adj();
  if (!a) return SCY_ERR_NOMEM;
  int rc = a->ctx.create(&q->ctx, checkpoint_every);
  if (rc != SCY_OK) {
    delete a;
    return rc;
  }
  *out = a;
  return SCY_OK;
}

scy_status scy_adj_destroy(scy_adj* a) {
  delete a;
  return SCY_OK;
}

scy_status scy_adj_set_steps(scy_adj* a, const double* dts, long n) {
  if (!a || !dts) return SCY_ERR_ARG;
  return a->ctx.set_steps(dts, n);
}

scy_status scy_adj_set_targets(scy_adj* a, const double* surf, const double* vel, double w_surf, double w_vel) {
  if (!a || !surf || !vel) return SCY_ERR_ARG;
  return a->ctx.set_targets(surf, vel, w_surf, w_vel);
}

scy_status scy_adj_set_fault_params(scy_adj* a, const double* fa, const double* fb, const double* fDc) {
  if (!a) return SCY_ERR_ARG;
  return a->ctx.set_fault_params(fa, fb, fDc);
}

scy_status scy_adj_forward(scy_adj* a, double* J) {
  if (!a) return SCY_ERR_ARG;
  return a->ctx.forward(J, 0);
}

scy_status scy_adj_observations(scy_adj* a, double* surf, double* vel) {
  if (!a) return SCY_ERR_ARG;
  return a->ctx.observations(surf, vel);
}

scy_status scy_adj_gradient(scy_adj* a, double* J, double* grad_a, double* grad_b, double* grad_Dc) {
  if (!a) return SCY_ERR_ARG;
  return a->ctx.gradient(J, grad_a, grad_b, grad_Dc);
}

}  // extern "C"
