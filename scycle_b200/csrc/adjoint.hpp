// Discrete adjoint of the quasi-dynamic RK32 integration (scy_adj_* in the
// C ABI).
//
// The forward map is the linear-elastic driver's RK32 integration over a
// fixed sequence of accepted step sizes (the sequence an adaptive run took,
// as RK32::integrate accepts them, odeSolver.cpp:567-603): per step the
// stages k1 = y + dt/2 f0, k2 = y - dt f0 + 2 dt f1 and
// y' = y + dt/6 f0 + 2 dt/3 f1 + dt/6 f2, then f0' = d_dt(t + dt, y').  The
// misfit is J = sum_n w_s |surfDisp_n - target_n|^2 + w_v |V_n - target_n|^2
// over the accepted states n = 1..M (fields of the d_dt at y_n).  The
// gradient with respect to the fault's a, b and Dc at every fault node comes
// from the reverse sweep through the same stages:
//   * the d_dt of StrikeSlip_LinearElastic_qd (strikeSlip_linearElastic_qd.cpp:756-798)
//     is differentiated node by node: the state law (fault.cpp:1984-2088) by
//     hand, the slip velocity of ComputeVel_qd (fault.cpp:954-1059) by the
//     implicit-function rule dV = -(F_psi dpsi + F_tau dtau + F_a da) / F_V
//     of its residual F = a sN asinh(V/(2 v0) e^(psi/a)) - (tau - eta V);
//   * tau = mu Dy u on the fault row and surfDisp = u on the surface feed a
//     transposed solve A w = dJ/du (A is symmetric, so the forward solver is
//     reused) and dJ/dslip = M_L^T w / faultTypeScale through setRhs;
//   * the states are checkpointed every `ck` steps; each segment is
//     recomputed forward (storing psi, V and tau at every stage) before its
//     reverse sweep.
// The initial state is taken as independent of the parameters.  Each step
// advances state and time by the same size; where the reference kept a
// larger rejected attempt's solution while advancing time by minDeltaT
// (odeSolver.cpp:580-592), the map here advances time by the attempt's size.
// The step sizes come from scy_qd_get_step_sizes of the run.
#pragma once
#include <vector>

#include "qd.hpp"

namespace scy {

struct AdjointContext {
  QDContext* q = nullptr;
  int ck = 50;
  std::vector<double> dts;      // accepted step sizes
  long M = 0;                   // steps
  double t0 = 0.0;
  DevBuf y0;                    // initial state (nvar)
  DevBuf v0;                    // slip velocity at the start (the first root guess)
  DevBuf ckpt;                  // checkpoints: (M / ck + 1) x nvar
  DevBuf tgt_s, tgt_v;          // targets: M x Ny, M x Nz (device)
  double w_s = 1.0, w_v = 1.0;
  int have_targets = 0;
  // per segment, per step (ck + 1 slots) and evaluation e (0: at y_n, 1: k1,
  // 2: k2): psi, V and tau of the stage (3 Nz each); surfDisp at y_n (Ny)
  DevBuf ev, evs;
  DevBuf Jn;                    // misfit per step (M)
  // adjoint work vectors
  DevBuf ly, lF0, lf0, lf1, lf2, lk, ltau, lu, w, grad;  // grad: [a | b | Dc]
  DevBuf yk;                    // stage state
  DevBuf obs_s, obs_v;          // observed fields of the last forward run (M x Ny, M x Nz)

  int create(QDContext* qd, int checkpoint_every);
  int set_steps(const double* dt, long n);
  int set_targets(const double* surf, const double* vel, double ws, double wv);
  int set_fault_params(const double* a, const double* b, const double* Dc);
  // fixed-step forward from y0: observations and (with targets) the misfit
  int forward(double* J, int keep_checkpoints);
  int gradient(double* J, double* ga, double* gb, double* gDc);
  int observations(double* surf, double* vel);

 private:
  int eval(double t, const double* y, double* f, long step_slot, int e, int store);
  int stage_combine(double* out, const double* y, std::initializer_list<std::pair<const double*, double>> terms);
  int vjp(long slot, int e, const double* lam_f, double* lam_y, int with_misfit, long step);
  int segment_forward(long s0, long s1);
};

}  // namespace scy
