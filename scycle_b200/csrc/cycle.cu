// Quasi-dynamic / fully dynamic cycle driver (strikeSlip_linearElastic_qd_fd).
//
// Reference map (source/strikeSlip_linearElastic_qd_fd.cpp): computeTimeStep
// :356-442 and computePenaltyVectors :446-505 (CycleContext::create),
// integrate :511-581 (run), checkSwitchRegime :586-662 (check_switch and the
// last block of fd_fault_kernel), initiateIntegrands :668-744 (begin),
// prepare_fd2qd :747-804 (leave_fd), prepare_qd2fd :807-888 with
// integrate_singleQDTimeStep :891-956 (the CP_FD_BEGIN / CP_FD_SINGLE
// states and enter_fd), propagateWaves :1170-1239 (EpiWave), integrate_qd
// :1436-1508, integrate_fd :1511-1545 with OdeSolver_WaveEq::integrate
// (source/odeSolver_WaveEq.cpp:147-186), fully dynamic d_dt :1676-1757 and
// Fault_fd::d_dt / setPhi (source/fault.cpp:1436-1575) (fd_fault_kernel),
// timeMonitor :1814-1859 (qd_monitor and the fault kernel's switch test).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "cycle.hpp"
#include "cycle_host.hpp"
#include "sbp_dev.cuh"

namespace scy {

// ---------------------------------------------------------------------------
// propagateWaves as a stencil epilogue.  wc = dt^2 / rho * Hinv * Jinv per
// node, or the product of two 1D factors when rho and the metrics are
// separable; ay is nonzero only on boundary nodes (either indexing of the
// penalty vector puts it there), so interior nodes skip its load.  The fault
// row also stores d2u = (A u * Hinv) * Jinv for Fault_fd::setPhi.
struct EpiWave {
  const double* __restrict__ uPrev;
  double* __restrict__ uNext;
  const double* __restrict__ wc;
  const double* __restrict__ wcy;  // separable dt^2/rho Hinv Jinv = wcy[iy] * wcz[iz] (else null)
  const double* __restrict__ wcz;
  const double* __restrict__ ay;
  const double* __restrict__ hinvf;
  const double* __restrict__ jinvf;
  double* __restrict__ d2u;
  double dt;
  int Ny, Nz;
  // fused step: the fault tile keeps uNext rows 0..4 and the fault row's d2u
  // of its 32 columns in shared memory (null elsewhere)
  double* s_rows;
  double* s_d2u;
  static constexpr bool kReduce = false;
  __device__ __forceinline__ double operator()(long node, int iy, int iz, double Ax, double u) const {
    return apply(node, iy, iz, Ax, u, uPrev[node]);
  }
  // the same with uPrev at the node given (loaded ahead by the caller)
  __device__ __forceinline__ double apply(long node, int iy, int iz, double Ax, double u, double up) const {
    const bool edge = iy == 0 || iy == Ny - 1 || iz == 0 || iz == Nz - 1;
    const double a = edge ? ay[node] : 0.0;
    const double w = wcy ? wcy[iy] * wcz[iz] : wc[node];
    const double acc = w * Ax + 2. * u;
    double un;
    if (a == 0.0)
      un = acc - up;
    else
      un = (acc + (dt * a - 1.0) * up) / (dt * a + 1.0);
    uNext[node] = un;
    if (s_rows) {
      if (iy < 5) s_rows[iy * TZ + (iz & (TZ - 1))] = un;
      if (iy == 0) s_d2u[iz & (TZ - 1)] = (Ax * hinvf[iz]) * jinvf[iz];
    } else if (iy == 0) {
      d2u[iz] = (Ax * hinvf[iz]) * jinvf[iz];
    }
    return 0.0;
  }
};

// RPT = 0: the two-stage tile (stencil_tile); 1, 2, 4: the full-form tile
// with that many rows per thread (full_tile).
template <int RPT>
__device__ __forceinline__ void wave_tile(const LevelDev<double>& L, const LoadPlain<double>& ld, const EpiWave& ep) {
  if constexpr (RPT == 0) {
    stencil_tile<double, LoadPlain<double>, EpiWave>(L, ld, ep, nullptr, nullptr, nullptr);
  } else {
    __shared__ double xs[full_smem_values<RPT>()];
    const double* __restrict__ up = ep.uPrev;
    auto pre = [&](long node, int, int) { return up[node]; };
    auto out = [&](long node, int iy, int iz, double Ax, double u, double upv) { ep.apply(node, iy, iz, Ax, u, upv); };
    auto row = [](int) {};
    full_apply<double, RPT>(L, ld, pre, out, row, xs);
  }
}

template <int RPT>
__global__ void __launch_bounds__(256) fd_wave_kernel(LevelDev<double> L, LoadPlain<double> ld, EpiWave ep,
                                                      const CycleDevState* st) {
  if (st->stop) return;
  wave_tile<RPT>(L, ld, ep);
}

struct FDFaultArgs {
  FaultParams fp;
  const double* D0;  // Dy row 0 (band)
  const double *mu0, *qy0;
  int Ny, var_grid;
  const double *slip, *slipPrev, *psi, *psiPrev;
  double *slipNext, *psiNext;
  const double *slip0, *tau0, *alphay, *rho_f, *d2u, *u0;
  double* uNext;
  double *slipVel, *tauQSP, *tauP, *strength;
  double dt, fts, inv_fts;
  double limit_fd, trigger_fd2qd;
  double* partials;  // >= gridDim.x
  CycleDevState* st;
};

constexpr int kFaultBlock = 128;

// Fault_fd::d_dt for fault node iz (fault.cpp:1436-1575), the fault-row
// stress of uNext + u0, tauQS and tauP; returns eta V / tauQS.  d2u is the
// node's Hinv Jinv A u; un(k) returns uNext at body row k (k = 1..4).
template <class Rows>
__device__ __forceinline__ double fd_fault_node(const FDFaultArgs& A, int iz, double d2u, const Rows& un_row,
                                                unsigned* bad_out) {
  const FaultParams& fp = A.fp;
  const int Nz = fp.Nz;
  CycleDevState* st = A.st;
  const double dt = A.dt;
  const double rho = A.rho_f[iz], alphay = A.alphay[iz];
  const double a = fp.a[iz], sN = fp.sN[iz], eta = fp.eta[iz];
  const double slip0 = A.slip0[iz];
  const double uPrev = (A.slipPrev[iz] - slip0) * A.inv_fts;
  double u = (A.slip[iz] - slip0) * A.inv_fts;
  // setPhi (fault.cpp:1527-1575)
  const double an = d2u + A.tau0[iz] / alphay;
  const double Phi = 2.0 / dt * (u - uPrev) + dt * an / rho;
  const double fricPen = dt / alphay / rho;
  const double psi = A.psi[iz];
  // ComputeVel_fd::computeVel (fault.cpp:1594-1644)
  double V;
  const double lk = fp.locked[iz];
  unsigned bad = 0;
  if (lk > 0.5) {
    V = 0.0;
  } else if (lk < -0.5) {
    V = fp.vL;
  } else {
    const double right = fabs(Phi);
    if (isnan(right)) {
      bad |= FAULT_NONFINITE;
      V = 0.0;
    } else if (fabs(0.0 - right) < 1e-14) {
      V = 0.0;
    } else {
      const ResidVelFD R1{right, fricPen, sN, psi, a, fp.v0, exp(psi / a)};
      int its = 0;
      bool ok = true;
      V = bracketed_newton_f(R1, 0.0, right, fabs(A.slipVel[iz]), fp.root_tol, fp.max_its, &its, &ok);
      atomicAdd(&st->its, (unsigned long long)its);
      if (!ok) bad |= FAULT_ROOT_NOCONV;
    }
  }
  // velocity and displacement update (fault.cpp:1481-1496)
  if (!(V < 1e-14)) {
    const double fric = strength_psi(sN, psi, V, a, fp.v0);
    const double alpha = 1.0 / (rho * alphay) * fric / V;
    const double Ad = 1.0 + alpha * dt;
    V = Phi / (1. + dt * alpha);
    u = (2. * u + (an * dt * dt / rho) + (dt * alpha - 1.) * uPrev) / Ad;
  }
  A.slipVel[iz] = V;
  // ComputeAging_fd / ComputeSlipLaw_fd (fault.cpp:1702-1745, :1802-1846)
  const double psiPrev = A.psiPrev[iz];
  double psiN;
  {
    int its = 0;
    bool ok = true;
    if (fp.state_law == 0) {
      const ResidAgingFD R2{psiPrev, V, fp.b[iz], fp.f0, fp.v0, fp.Dc[iz], dt};
      psiN = bracketed_newton_f(R2, -2.0, 2.0, psi, fp.root_tol, fp.max_its, &its, &ok);
    } else {
      const ResidSlipFD R2{psiPrev, V, a, fp.b[iz], fp.f0, fp.v0, fp.Dc[iz], dt};
      psiN = bracketed_newton_f(R2, -2.0, 2.0, psi, fp.root_tol, fp.max_its, &its, &ok);
    }
    atomicAdd(&st->its, (unsigned long long)its);
    if (!ok) bad |= FAULT_ROOT_NOCONV;
  }
  A.psiNext[iz] = psiN;
  A.slipNext[iz] = A.fts * u + slip0;
  A.strength[iz] = strength_psi(sN, psiN, V, a, fp.v0);
  A.uNext[iz] = u;  // body row 0 takes the fault displacement
  // sxy = mu * Dy (uNext + u0) at the fault (LinearElastic::computeStresses)
  double d = 0.0;
#pragma unroll
  for (int j = HALF; j < BAND; ++j) {
    const int k = j - HALF;
    if (k < A.Ny) {
      const double un = k == 0 ? u : un_row(k);
      d += A.D0[j] * (un + 1.0 * A.u0[(long)k * Nz + iz]);
    }
  }
  if (A.var_grid) d *= A.qy0[iz];
  const double tq = A.mu0[iz] * d + 1.0 * fp.prestress[iz];
  A.tauQSP[iz] = tq;
  A.tauP[iz] = -1.0 * (eta * V) + tq;
  if (!isfinite(V) || !isfinite(psiN)) bad |= FAULT_NONFINITE;
  *bad_out = bad;
  return eta * V / tq;
}

// The last of the gridDim.x participating blocks finishes max(eta V / tauQS)
// and runs checkSwitchRegime for the fully dynamic phase.
__device__ __forceinline__ void fd_switch_test(const FDFaultArgs& A, double block_max) {
  CycleDevState* st = A.st;
  __shared__ bool am_last;
  if (threadIdx.x == 0) {
    A.partials[blockIdx.x] = block_max;
    __threadfence();
    const unsigned prev = atomicAdd(&st->counter, 1u);
    am_last = prev == gridDim.x - 1;
  }
  __syncthreads();
  if (am_last && threadIdx.x == 0) {
    __threadfence();
    double mx = ((volatile double*)A.partials)[0];
    for (unsigned b = 1; b < gridDim.x; ++b) {
      const double v = ((volatile double*)A.partials)[b];
      mx = v > mx ? v : mx;
    }
    st->maxR = mx;
    if (!st->allowed && mx > A.limit_fd) st->allowed = 1;
    if (st->allowed && mx < A.trigger_fd2qd) st->stop = 1;
    st->steps_done += 1;
    st->counter = 0u;
  }
}

// Fault launch of the two-launch step (used for profiling and as the
// reference the fused step is tested against).
__global__ void __launch_bounds__(kFaultBlock) fd_fault_kernel(FDFaultArgs A) {
  CycleDevState* st = A.st;
  if (st->stop) return;
  const int Nz = A.fp.Nz;
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  double R = -INFINITY;
  if (iz < Nz) {
    unsigned bad = 0;
    auto rows = [&](int k) { return A.uNext[(long)k * Nz + iz]; };
    R = fd_fault_node(A, iz, A.d2u[iz], rows, &bad);
    if (bad) atomicOr(&st->flags, bad);
  }
  __shared__ double sh[32];
  double m = warp_max(R);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  double b = sh[0];
  for (int w = 1; w < (int)(blockDim.x >> 5); ++w) b = sh[w] > b ? sh[w] : b;
  fd_switch_test(A, b);
}

// One fully dynamic step in one launch: every tile applies the wave update;
// the tiles of the fault row (blockIdx.y == 0, rows 0 .. 7 or more) then run
// the fault update of their 32 columns from the rows they just computed,
// while the rest of the grid is still stepping the body.
template <int RPT>
__global__ void __launch_bounds__(256) fd_step_kernel(LevelDev<double> L, LoadPlain<double> ld, EpiWave ep,
                                                      FDFaultArgs A) {
  CycleDevState* st = A.st;
  if (st->stop) return;
  __shared__ double s_rows[5 * TZ];
  __shared__ double s_d2u[TZ];
  const bool fault_tile = blockIdx.y == 0;
  EpiWave e = ep;
  e.s_rows = fault_tile ? s_rows : nullptr;
  e.s_d2u = fault_tile ? s_d2u : nullptr;
  wave_tile<RPT>(L, ld, e);
  if (!fault_tile) return;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  double R = -INFINITY;
  if (threadIdx.x < 32) {
    const int iz = blockIdx.x * TZ + lane;
    if (iz < A.fp.Nz) {
      unsigned bad = 0;
      auto rows = [&](int k) { return s_rows[k * TZ + lane]; };
      R = fd_fault_node(A, iz, s_d2u[lane], rows, &bad);
      if (bad) atomicOr(&st->flags, bad);
    }
    R = warp_max(R);
  }
  fd_switch_test(A, R);
}

// max over the fault of eta V / tauQS (the quasi-dynamic phase's test)
__global__ void qd_max_ratio_kernel(const double* __restrict__ eta, const double* __restrict__ V,
                                    const double* __restrict__ tq, int Nz, double* out) {
  __shared__ double sh[32];
  double m = -INFINITY;
  for (int i = threadIdx.x; i < Nz; i += blockDim.x) {
    const double r = eta[i] * V[i] / tq[i];
    m = r > m ? r : m;
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = sh[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) b = sh[w] > b ? sh[w] : b;
    *out = b;
  }
}

// enter the fully dynamic phase: du = u_n - u_{n-1} as both var and varPrev
__global__ void fd_enter_body_kernel(const double* __restrict__ u_new, const double* __restrict__ u_old,
                                     double* __restrict__ uA, double* __restrict__ uB, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double d = u_new[i] + (-1.0) * u_old[i];
    uA[i] = d;
    uB[i] = d;
  }
}

__global__ void fd_enter_fault_kernel(const double* __restrict__ var, const double* __restrict__ strength,
                                      const double* __restrict__ prestress, double* psiA, double* psiB,
                                      double* slipA, double* slipB, double* slip0, double* tau0, int Nz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Nz) return;
  const double p = var[i], s = var[Nz + i];
  psiA[i] = p;
  psiB[i] = p;
  slipA[i] = s;
  slipB[i] = s;
  slip0[i] = s;
  tau0[i] = strength[i] + 1.0 * prestress[i];
}

__global__ void add_kernel(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out,
                           long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = a[i] + 1.0 * b[i];
}

// ---------------------------------------------------------------------------
CycleContext::~CycleContext() {
  for (auto& g : graphs) cudaGraphExecDestroy(g.second);
  graphs.clear();
  if (h_state) cudaFreeHost(h_state);
}

static int upload(DevBuf& b, const std::vector<double>& v, cudaStream_t s) {
  SCY_TRY(b.alloc(std::max<size_t>(v.size(), 1) * sizeof(double)));
  if (!v.empty()) SCY_CUDA_TRY(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  return SCY_OK;
}

int CycleContext::create(const scy_qd_desc& qd, const scy_cycle_desc& cd) {
  if (!cd.rho || !cd.rho_fault) {
    set_error("cycle descriptor needs rho and rho_fault");
    return SCY_ERR_ARG;
  }
  if (qd.fault.state_law != SCY_LAW_AGING && qd.fault.state_law != SCY_LAW_SLIP) {
    set_error("the fully dynamic state update exists for the aging and slip laws only");
    return SCY_ERR_ARG;
  }
  if (!qd.bcL_from_slip) {
    set_error("the cycle driver needs a fault (symmFault / rigidFault) on the left boundary");
    return SCY_ERR_ARG;
  }
  SCY_TRY(q.create(qd));
  Ny = q.Ny;
  Nz = q.Nz;
  N = q.N;
  cudaStream_t s = q.sbp.stream;
  trigger_qd2fd = cd.trigger_qd2fd;
  trigger_fd2qd = cd.trigger_fd2qd;
  limit_qd = cd.limit_qd;
  limit_fd = cd.limit_fd;
  max_num_cycles = cd.max_num_cycles;
  ay_quirk = cd.ay_index_quirk ? 1 : 0;
  const scy_grid_desc& g = q.sbp.desc;
  const int nm[4] = {SCY_BC_NEUMANN, SCY_BC_NEUMANN, SCY_BC_NEUMANN, SCY_BC_NEUMANN};
  try {
    fd_host = build_level(g.order, Ny, Nz, g.Ly, g.Lz, g.grid_type, g.compat, q.sbp.y, q.sbp.z, q.sbp.mu, nm);
  } catch (const std::exception& e) {
    set_error("fully dynamic operator: %s", e.what());
    return SCY_ERR_ARG;
  }
  SCY_TRY(fd_level.init(fd_host, s));
  const bool var = g.grid_type == SCY_GRID_VAR;
  std::vector<double> cs(N);
  for (long i = 0; i < N; ++i) cs[i] = cd.cs ? cd.cs[i] : std::sqrt(std::fabs(q.sbp.mu[i] / cd.rho[i]));
  dt_fd = cycle_time_step(fd_host, cs, cd.deltaT_fd, cd.CFL);
  const double h11 = g.order == 2 ? 0.5 : 17.0 / 48.0;
  const double h11y = h11 * fd_host.dy, h11z = h11 * fd_host.dz;
  std::vector<double> ayv = penalty_ay(Ny, Nz, h11y, h11z, cd.fd_bcR == SCY_FD_OUTGOING, cd.fd_bcT == SCY_FD_OUTGOING,
                                       cd.fd_bcB == SCY_FD_OUTGOING, ay_quirk, cs);
  for (long i = 0; i < N; ++i) {
    const int iy = (int)(i / Nz), iz = (int)(i % Nz);
    const bool edge = iy == 0 || iy == Ny - 1 || iz == 0 || iz == Nz - 1;
    if (!edge && ayv[i] != 0.0) {
      set_error("penalty vector has an interior entry at node %ld", i);
      return SCY_ERR_STATE;
    }
  }
  SCY_TRY(upload(ay, ayv, s));
  // wc = dt^2/rho * Hinv * Jinv; fault-row Hinv, Jinv; alphay = h11y (* yq)
  std::vector<double> wcv(N), hf(Nz), jf(Nz), al(Nz), rf(cd.rho_fault, cd.rho_fault + Nz);
  // separable when rho depends on iz only and qy on iy, rz on iz only
  bool sep = true;
  for (long i = 0; i < N && sep; ++i) {
    const int iy = (int)(i / Nz), iz = (int)(i % Nz);
    if (cd.rho[i] != cd.rho[iz]) sep = false;
    if (var && (fd_host.qy[i] != fd_host.qy[(size_t)iy * Nz] || fd_host.rz[i] != fd_host.rz[iz])) sep = false;
  }
  if (sep) {
    std::vector<double> wy1(Ny), wz1(Nz);
    for (int iy = 0; iy < Ny; ++iy)
      wy1[iy] = dt_fd * dt_fd * fd_host.ty.Hinvd[iy] * (var ? fd_host.qy[(size_t)iy * Nz] : 1.0);
    for (int iz = 0; iz < Nz; ++iz) wz1[iz] = fd_host.tz.Hinvd[iz] * (var ? fd_host.rz[iz] : 1.0) / cd.rho[iz];
    SCY_TRY(upload(wcy, wy1, s));
    SCY_TRY(upload(wcz, wz1, s));
    for (long i = 0; i < N; ++i) wcv[i] = wy1[i / Nz] * wz1[i % Nz];
  } else {
    for (long i = 0; i < N; ++i) {
      const int iy = (int)(i / Nz), iz = (int)(i % Nz);
      const double hinv = fd_host.ty.Hinvd[iy] * fd_host.tz.Hinvd[iz];
      const double jinv = var ? fd_host.qy[i] * fd_host.rz[i] : 1.0;
      wcv[i] = dt_fd * dt_fd / cd.rho[i] * hinv * jinv;
    }
  }
  wc_sep = sep ? 1 : 0;
  for (int iz = 0; iz < Nz; ++iz) {
    hf[iz] = fd_host.ty.Hinvd[0] * fd_host.tz.Hinvd[iz];
    jf[iz] = var ? fd_host.qy[iz] * fd_host.rz[iz] : 1.0;
    al[iz] = var ? fd_host.yq[iz] * h11y : h11y;
  }
  SCY_TRY(upload(wc, wcv, s));
  SCY_TRY(upload(hinvf, hf, s));
  SCY_TRY(upload(jinvf, jf, s));
  SCY_TRY(upload(alphay, al, s));
  SCY_TRY(upload(rho_f, rf, s));
  for (int k = 0; k < 3; ++k) {
    SCY_TRY(u3[k].alloc(N * 8));
    SCY_TRY(psi3[k].alloc(Nz * 8));
    SCY_TRY(slip3[k].alloc(Nz * 8));
    SCY_CUDA_TRY(cudaMemsetAsync(u3[k].p, 0, N * 8, s));
  }
  SCY_TRY(u0.alloc(N * 8));
  SCY_TRY(utmp.alloc(N * 8));
  SCY_CUDA_TRY(cudaMemsetAsync(u0.p, 0, N * 8, s));
  SCY_TRY(d2u.alloc(Nz * 8));
  SCY_TRY(slip0.alloc(Nz * 8));
  SCY_TRY(tau0.alloc(Nz * 8));
  // block maxima of the switch test: one per fault-row tile (fused step) or
  // per fault block (two-launch step)
  SCY_TRY(dstate.alloc(sizeof(CycleDevState) + 8 * (size_t)((Nz + TZ - 1) / TZ + (Nz + kFaultBlock - 1) / kFaultBlock + 2)));
  SCY_CUDA_TRY(cudaMemsetAsync(dstate.p, 0, dstate.bytes, s));
  SCY_CUDA_TRY(cudaMallocHost((void**)&h_state, sizeof(CycleDevState)));
  std::memset(h_state, 0, sizeof(CycleDevState));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  q.monitor = [this](int* stop) { return qd_monitor(stop); };
  return SCY_OK;
}

// ---------------------------------------------------------------------------
int CycleContext::check_switch(double maxR, int* stop) {
  int must = 0;
  if (inDynamic && !allowed && maxR > limit_fd) allowed = 1;
  if (!inDynamic && !allowed && maxR < limit_qd) allowed = 1;
  if (inDynamic && allowed && maxR < trigger_fd2qd) must = 1;
  if (!inDynamic && allowed && maxR > trigger_qd2fd) must = 1;
  last_R = maxR;
  *stop = must;
  return SCY_OK;
}

int CycleContext::qd_max_ratio(double* out) {
  cudaStream_t s = q.sbp.stream;
  double* dst = reinterpret_cast<double*>(q.errbuf.as<double>()) + 12;
  qd_max_ratio_kernel<<<1, 1024, 0, s>>>(q.feta.as<double>(), q.slipVel.as<double>(), q.tauQSP.as<double>(), Nz,
                                         dst);
  SCY_LAUNCH_CHECK();
  SCY_CUDA_TRY(cudaMemcpyAsync(out, dst, sizeof(double), cudaMemcpyDeviceToHost, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  return SCY_OK;
}

int CycleContext::qd_monitor(int* stop) {
  // timeMonitor: the step count always advances in the RK loop, so the
  // duplicate-step early return never fires here
  currT = q.currT;
  stepCount = q.stepCount;
  ++qd_steps;
  double R = 0;
  SCY_TRY(qd_max_ratio(&R));
  SCY_TRY(check_switch(R, stop));
  if (*stop) switches.push_back({stepCount, currT, 1, R});
  return SCY_OK;
}

int CycleContext::begin(const scy_ode_opts& o, const double* var0_host) {
  cudaStream_t s = q.sbp.stream;
  ode = o;
  if (ode.n_err <= 0) {
    ode.n_err = 2;
    ode.err_keys[0] = SCY_KEY_PSI;
    ode.err_keys[1] = SCY_KEY_SLIP;
    ode.err_scale[0] = ode.err_scale[1] = 1.0;
  }
  q.ode = ode;
  SCY_CUDA_TRY(cudaMemcpyAsync(q.rk[0].p, var0_host, 2 * (size_t)Nz * 8, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemsetAsync(u0.p, 0, N * 8, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  currT = o.t0;
  stepCount = 0;
  cycleCount = 0;
  allowed = 0;
  inDynamic = 0;
  first_cycle = 1;
  rot = 0;
  qd_steps = fd_steps = 0;
  qd_ms = fd_ms = 0;
  switches.clear();
  phase = CP_QD_BEGIN;
  began = 1;
  return SCY_OK;
}

// The material displacement of the phase the driver is in (device).
int CycleContext::current_u(double* dst) {
  cudaStream_t s = q.sbp.stream;
  if (inDynamic) {
    const int cur = (rot + 1) % 3;
    add_kernel<<<grid_for(N), kBlock, 0, s>>>(u3[cur].as<double>(), u0.as<double>(), dst, N);
    SCY_LAUNCH_CHECK();
    return SCY_OK;
  }
  if (q.mode == SCY_QD_MODE_RESPONSE) SCY_TRY(q.full_solve_for_output());
  if (dst != q.u.as<double>())
    SCY_CUDA_TRY(cudaMemcpyAsync(dst, q.u.p, N * 8, cudaMemcpyDeviceToDevice, s));
  return SCY_OK;
}

int CycleContext::enter_fd() {
  cudaStream_t s = q.sbp.stream;
  // u0 holds the displacement before the single step; the one after it:
  double* unew = q.u.as<double>();
  if (q.mode == SCY_QD_MODE_RESPONSE) SCY_TRY(q.full_solve_for_output());
  rot = 0;  // prev = 0, cur = 1, next = 2
  fd_enter_body_kernel<<<grid_for(N), kBlock, 0, s>>>(unew, u0.as<double>(), u3[1].as<double>(),
                                                       u3[0].as<double>(), N);
  SCY_LAUNCH_CHECK();
  fd_enter_fault_kernel<<<(Nz + 127) / 128, 128, 0, s>>>(
      q.rk[0].as<double>(), q.strength.as<double>(), q.fprestress.as<double>(), psi3[1].as<double>(),
      psi3[0].as<double>(), slip3[1].as<double>(), slip3[0].as<double>(), slip0.as<double>(), tau0.as<double>(), Nz);
  SCY_LAUNCH_CHECK();
  CycleDevState init{};
  init.allowed = allowed;
  SCY_CUDA_TRY(cudaMemcpyAsync(dstate.p, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  fd_max_steps = stepCount + ode.max_steps;
  return SCY_OK;
}

int CycleContext::set_fd_state(double t, long step, int allow, const double* const* now, const double* u,
                               const double* const* prev, const double* uPrev, const double* u0_host,
                               const double* slip0_host, const double* tau0_host, const double* slipVel_host) {
  if (!began) {
    set_error("scy_cycle_set_fd_state called before scy_cycle_begin");
    return SCY_ERR_STATE;
  }
  cudaStream_t s = q.sbp.stream;
  rot = 0;  // prev = 0, cur = 1
  const size_t fb = (size_t)Nz * 8, bb = (size_t)N * 8;
  SCY_CUDA_TRY(cudaMemcpyAsync(psi3[1].p, now[0], fb, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(slip3[1].p, now[1], fb, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(u3[1].p, u, bb, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(psi3[0].p, prev[0], fb, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(slip3[0].p, prev[1], fb, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(u3[0].p, uPrev, bb, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(u0.p, u0_host, bb, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(slip0.p, slip0_host, fb, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(tau0.p, tau0_host, fb, cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(q.slipVel.p, slipVel_host, fb, cudaMemcpyHostToDevice, s));
  CycleDevState init{};
  init.allowed = allow ? 1 : 0;
  SCY_CUDA_TRY(cudaMemcpyAsync(dstate.p, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  currT = t;
  stepCount = step;
  allowed = allow ? 1 : 0;
  inDynamic = 1;
  fd_max_steps = stepCount + ode.max_steps;
  phase = CP_FD;
  return SCY_OK;
}

int CycleContext::leave_fd() {
  cudaStream_t s = q.sbp.stream;
  const int cur = (rot + 1) % 3;
  SCY_CUDA_TRY(cudaMemcpyAsync(q.rk[0].p, psi3[cur].p, Nz * 8, cudaMemcpyDeviceToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(q.rk[0].as<double>() + Nz, slip3[cur].p, Nz * 8, cudaMemcpyDeviceToDevice, s));
  // the fully dynamic displacement is the first guess of the next solve
  add_kernel<<<grid_for(N), kBlock, 0, s>>>(u3[cur].as<double>(), u0.as<double>(), q.u.as<double>(), N);
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

int CycleContext::fd_launch_step(int r, cudaStream_t s, int part) {
  const int prev = r % 3, cur = (r + 1) % 3, next = (r + 2) % 3;
  CycleDevState* st = dstate.as<CycleDevState>();
  const LevelDev<double>& L = fd_level.dev;
  EpiWave ep{u3[prev].as<double>(),
             u3[next].as<double>(),
             wc.as<double>(),
             wc_sep ? wcy.as<double>() : nullptr,
             wc_sep ? wcz.as<double>() : nullptr,
             ay.as<double>(),
             hinvf.as<double>(),
             jinvf.as<double>(),
             d2u.as<double>(),
             dt_fd,
             Ny,
             Nz,
             nullptr,
             nullptr};
  FDFaultArgs A{};
  A.fp = q.fp;
  A.D0 = L.y.D;  // row 0 of the band table
  A.mu0 = L.mu;
  A.qy0 = L.qy;
  A.Ny = Ny;
  A.var_grid = L.var;
  A.slip = slip3[cur].as<double>();
  A.slipPrev = slip3[prev].as<double>();
  A.psi = psi3[cur].as<double>();
  A.psiPrev = psi3[prev].as<double>();
  A.slipNext = slip3[next].as<double>();
  A.psiNext = psi3[next].as<double>();
  A.slip0 = slip0.as<double>();
  A.tau0 = tau0.as<double>();
  A.alphay = alphay.as<double>();
  A.rho_f = rho_f.as<double>();
  A.d2u = d2u.as<double>();
  A.u0 = u0.as<double>();
  A.uNext = u3[next].as<double>();
  A.slipVel = q.slipVel.as<double>();
  A.tauQSP = q.tauQSP.as<double>();
  A.tauP = q.tauP.as<double>();
  A.strength = q.strength.as<double>();
  A.dt = dt_fd;
  A.fts = q.fts;
  A.inv_fts = 1.0 / q.fts;
  A.limit_fd = limit_fd;
  A.trigger_fd2qd = trigger_fd2qd;
  A.partials = reinterpret_cast<double*>(dstate.as<char>() + sizeof(CycleDevState));
  A.st = st;
  const LoadPlain<double> ld{u3[cur].as<double>()};
  const dim3 g = apply_grid(L);
  const int rpt = L.full ? L.rpt : 0;
  if (part & FD_FUSED) {
    if (rpt == 4)
      fd_step_kernel<4><<<g, 256, 0, s>>>(L, ld, ep, A);
    else if (rpt == 2)
      fd_step_kernel<2><<<g, 256, 0, s>>>(L, ld, ep, A);
    else if (rpt == 1)
      fd_step_kernel<1><<<g, 256, 0, s>>>(L, ld, ep, A);
    else
      fd_step_kernel<0><<<g, 256, 0, s>>>(L, ld, ep, A);
    SCY_LAUNCH_CHECK();
  }
  if (part & FD_WAVE) {
    if (rpt == 4)
      fd_wave_kernel<4><<<g, 256, 0, s>>>(L, ld, ep, st);
    else if (rpt == 2)
      fd_wave_kernel<2><<<g, 256, 0, s>>>(L, ld, ep, st);
    else if (rpt == 1)
      fd_wave_kernel<1><<<g, 256, 0, s>>>(L, ld, ep, st);
    else
      fd_wave_kernel<0><<<g, 256, 0, s>>>(L, ld, ep, st);
    SCY_LAUNCH_CHECK();
  }
  if (part & FD_FAULT) {
    fd_fault_kernel<<<(Nz + kFaultBlock - 1) / kFaultBlock, kFaultBlock, 0, s>>>(A);
    SCY_LAUNCH_CHECK();
  }
  return SCY_OK;
}

int CycleContext::time_kernels(int reps, double* wave_us, double* fault_us, double* step_us) {
  if (reps < 1) reps = 1;
  cudaStream_t s = q.sbp.stream;
  CycleDevState* st = dstate.as<CycleDevState>();
  SCY_CUDA_TRY(cudaMemsetAsync(&st->stop, 0, sizeof(int), s));
  cudaEvent_t e0, e1;
  SCY_CUDA_TRY(cudaEventCreate(&e0));
  SCY_CUDA_TRY(cudaEventCreate(&e1));
  const int parts[3] = {FD_WAVE, FD_FAULT, FD_FUSED};
  float ms[3] = {0, 0, 0};
  int rc = SCY_OK;
  for (int p = 0; p < 3 && rc == SCY_OK; ++p) {
    rc = fd_launch_step(rot, s, parts[p]);  // warm-up
    if (rc != SCY_OK) break;
    cudaEventRecord(e0, s);
    for (int i = 0; i < reps && rc == SCY_OK; ++i) {
      // keep the stop flag clear: a firing switch test would make later launches no-ops
      cudaMemsetAsync(&st->stop, 0, sizeof(int), s);
      rc = fd_launch_step(rot, s, parts[p]);
    }
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms[p], e0, e1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  SCY_TRY(rc);
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  if (wave_us) *wave_us = ms[0] * 1e3 / reps;
  if (fault_us) *fault_us = ms[1] * 1e3 / reps;
  if (step_us) *step_us = ms[2] * 1e3 / reps;
  return SCY_OK;
}

// K wave-equation steps from rotation `rot` as one graph launch; the device
// stops stepping after the step whose switch test fires.
int CycleContext::fd_batch_run(int K, int* n_done, int* stopped) {
  cudaStream_t s = q.sbp.stream;
  const int r0 = rot % 3;
  auto key = std::make_pair(K, r0);
  auto it = graphs.find(key);
  if (it == graphs.end()) {
    cudaStream_t cs = nullptr;
    SCY_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    SCY_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    int rc = SCY_OK;
    for (int j = 0; j < K && rc == SCY_OK; ++j) rc = fd_launch_step(r0 + j, cs, fd_parts);
    cudaError_t ce = cudaStreamEndCapture(cs, &graph);
    cudaStreamDestroy(cs);
    if (rc != SCY_OK) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (ce != cudaSuccess) {
      set_error("capturing the wave-equation steps failed: %s", cudaGetErrorString(ce));
      return SCY_ERR_CUDA;
    }
    cudaGraphExec_t ex = nullptr;
    ce = cudaGraphInstantiate(&ex, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
      set_error("instantiating the wave-equation graph failed: %s", cudaGetErrorString(ce));
      return SCY_ERR_CUDA;
    }
    it = graphs.emplace(key, ex).first;
  }
  CycleDevState* st = dstate.as<CycleDevState>();
  SCY_CUDA_TRY(cudaMemsetAsync(&st->steps_done, 0, sizeof(int), s));
  SCY_CUDA_TRY(cudaGraphLaunch(it->second, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(h_state, st, sizeof(CycleDevState), cudaMemcpyDeviceToHost, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  if (h_state->flags) {
    if (h_state->flags & FAULT_NONFINITE) {
      set_error("non-finite value in the fully dynamic fault update");
      return SCY_ERR_NONFINITE;
    }
    set_error("rootFinder BracketedNewton did not converge within %d iterations (fully dynamic phase)",
              q.fp.max_its);
    return SCY_ERR_ROOT_NOCONV;
  }
  *n_done = h_state->steps_done;
  *stopped = h_state->stop;
  return SCY_OK;
}

// ---------------------------------------------------------------------------
int CycleContext::run(long budget, scy_cycle_stats* stats) {
  if (!began) {
    set_error("scy_cycle_run called before scy_cycle_begin");
    return SCY_ERR_STATE;
  }
  const double t1 = ode.t1;
  using clk = std::chrono::steady_clock;
  auto ms_since = [](clk::time_point a) { return std::chrono::duration<double, std::milli>(clk::now() - a).count(); };
  while (budget > 0 && phase != CP_DONE) {
    const clk::time_point t_iter = clk::now();
    if (phase == CP_QD_BEGIN) {
      // prepare_fd2qd + integrate_qd
      allowed = 0;
      inDynamic = 0;
      if (!first_cycle || cycleCount > 0) SCY_TRY(leave_fd());
      SCY_TRY(q.phase_begin(currT, t1, dt_fd, ode.min_dt, ode.max_dt, stepCount, ode.max_steps));
      phase = CP_QD;
    }
    if (phase == CP_QD) {
      scy_ode_stats os{};
      const long before = q.stepCount;
      SCY_TRY(q.integrate_steps(budget, &os));
      qd_ms += ms_since(t_iter);
      budget -= q.stepCount - before;
      currT = q.currT;
      stepCount = q.stepCount;
      const bool over = q.phase_stopped || q.stepCount >= q.ode.max_steps || !(q.currT < q.ode.t1);
      if (!over) continue;
      if (first_cycle && (currT >= t1 || stepCount >= ode.max_steps)) {
        phase = CP_DONE;
        break;
      }
      phase = CP_FD_BEGIN;
    }
    if (phase == CP_FD_BEGIN) {
      // prepare_qd2fd: _allowed = false, then integrate_singleQDTimeStep (one
      // step of size deltaT_fd, timeMonitor in quasi-dynamic mode); the
      // fields stay those of the quasi-dynamic fault until enter_fd
      allowed = 0;
      if (q.mode == SCY_QD_MODE_RESPONSE) SCY_TRY(q.full_solve_for_output());
      SCY_CUDA_TRY(cudaMemcpyAsync(u0.p, q.u.p, N * 8, cudaMemcpyDeviceToDevice, q.sbp.stream));
      SCY_TRY(q.phase_begin(currT, currT + dt_fd, dt_fd, dt_fd, dt_fd, stepCount, 1));
      phase = CP_FD_SINGLE;
      continue;
    }
    if (phase == CP_FD_SINGLE) {
      scy_ode_stats os{};
      const long before = q.stepCount;
      SCY_TRY(q.integrate_steps(1, &os));
      qd_ms += ms_since(t_iter);
      budget -= q.stepCount - before;
      currT = q.currT;
      stepCount = q.stepCount;
      SCY_TRY(enter_fd());
      inDynamic = 1;
      phase = CP_FD;
      continue;
    }
    if (phase == CP_FD) {
      // OdeSolver_WaveEq::integrate: loop while stepCount < max and t < t1
      long K = std::min<long>(fd_batch, budget);
      K = std::min(K, fd_max_steps - stepCount);
      if (K > 0 && !(currT < t1)) K = 0;
      if (K > 0) {
        double t = currT;
        for (long k = 1; k <= K; ++k) {
          t = t + dt_fd;
          if (!(t < t1)) {
            K = k;
            break;
          }
        }
      }
      int n = 0, stopped = 0;
      if (K > 0) {
        SCY_TRY(fd_batch_run((int)K, &n, &stopped));
        fd_ms += ms_since(t_iter);
        if (n <= 0 || n > K || (n < K && !stopped)) {
          set_error("wave-equation batch of %ld steps reported %d completed steps", K, n);
          return SCY_ERR_STATE;
        }
        for (int k = 0; k < n; ++k) {
          currT = currT + dt_fd;
          if (currT > t1) currT = t1;
        }
        stepCount += n;
        fd_steps += n;
        rot = (rot + n) % 3;
        budget -= n;
        last_R = h_state->maxR;
        allowed = h_state->allowed;
        if (stopped) switches.push_back({stepCount, currT, 0, h_state->maxR});
      }
      const bool over = stopped || K <= 0 || stepCount >= fd_max_steps || !(currT < t1);
      if (!over) continue;
      if (first_cycle) {
        if (currT >= t1 || stepCount >= ode.max_steps || max_num_cycles <= 1) {
          phase = CP_DONE;
          break;
        }
        first_cycle = 0;
      }
      ++cycleCount;
      if (cycleCount < max_num_cycles && stepCount <= ode.max_steps && currT <= t1)
        phase = CP_QD_BEGIN;
      else
        phase = CP_DONE;
    }
  }
  if (stats) fill_stats(stats);
  return SCY_OK;
}

void CycleContext::fill_stats(scy_cycle_stats* st) const {
  st->t = currT;
  st->dt_fd = dt_fd;
  st->step_count = stepCount;
  st->phase = phase == CP_DONE ? SCY_PHASE_DONE : (inDynamic ? SCY_PHASE_FD : SCY_PHASE_QD);
  st->cycle_count = cycleCount;
  st->allowed = allowed;
  st->done = phase == CP_DONE ? 1 : 0;
  st->qd_steps = qd_steps;
  st->fd_steps = fd_steps;
  st->switches = (long)switches.size();
  st->last_ratio = last_R;
  st->d_dt_evals = q.n_d_dt;
  st->solve_its = q.n_solve_its;
  st->solves = q.n_solves;
  st->dt = q.last_dt;
  st->new_dt = q.newDeltaT;
  st->qd_ms = qd_ms;
  st->fd_ms = fd_ms;
}

int CycleContext::get_field(int field, double* out) {
  cudaStream_t s = q.sbp.stream;
  const bool fd = inDynamic != 0;
  const int cur = (rot + 1) % 3;
  const double* src = nullptr;
  size_t n = Nz;
  long stride = 1;
  switch (field) {
    case SCY_FIELD_PSI: src = fd ? psi3[cur].as<double>() : q.rk[0].as<double>(); break;
    case SCY_FIELD_SLIP: src = fd ? slip3[cur].as<double>() : q.rk[0].as<double>() + Nz; break;
    case SCY_FIELD_SLIPVEL: src = q.slipVel.as<double>(); break;
    case SCY_FIELD_TAUP: src = q.tauP.as<double>(); break;
    case SCY_FIELD_TAUQSP: src = q.tauQSP.as<double>(); break;
    case SCY_FIELD_STRENGTH: src = q.strength.as<double>(); break;
    case SCY_FIELD_U:
    case SCY_FIELD_SURFDISP:
    case SCY_FIELD_SXY: {
      double* dst = utmp.as<double>();
      SCY_TRY(current_u(dst));
      if (field == SCY_FIELD_SXY) {
        SCY_TRY(q.sbp.apply(SCY_OP_MUXDY, dst, q.sxy.as<double>()));
        src = q.sxy.as<double>();
        n = N;
      } else {
        src = dst;
        n = field == SCY_FIELD_U ? N : Ny;
        stride = field == SCY_FIELD_U ? 1 : Nz;
      }
      break;
    }
    case SCY_FIELD_DPSI:
    case SCY_FIELD_DSLIP:
      if (fd) {
        set_error("rates are defined in the quasi-dynamic phase only");
        return SCY_ERR_STATE;
      }
      src = q.rk[1].as<double>() + (field == SCY_FIELD_DSLIP ? Nz : 0);
      break;
    default:
      set_error("unknown field %d", field);
      return SCY_ERR_ARG;
  }
  if (stride == 1) {
    SCY_CUDA_TRY(cudaMemcpyAsync(out, src, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  } else {
    SCY_CUDA_TRY(cudaMemcpy2DAsync(out, sizeof(double), src, stride * sizeof(double), sizeof(double), n,
                                   cudaMemcpyDeviceToHost, s));
  }
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  return SCY_OK;
}

}  // namespace scy
