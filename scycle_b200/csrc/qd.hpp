// Linear-elastic quasi-dynamic strike-slip driver on the device: the d_dt of
// StrikeSlip_LinearElastic_qd and the adaptive RK32 / RK43 integrators.
#pragma once
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "fault_dev.cuh"
#include "sbp_solver.hpp"
#include "writer.hpp"

namespace scy {

// RK vector slots of QDContext::rk
enum { V_VAR = 0, V_DVAR, V_K, V_F1, V_F2, V_F3, V_F4, V_F5, V_F6, V_LO, V_HI };

// RK43 tableau (odeSolver.cpp:985-1023): stage times c, stage weights a,
// solution weights b (order 4) and hb (order 3)
namespace rk43 {
constexpr double c2 = 1. / 2., c3 = 83. / 250., c4 = 31. / 50., c5 = 17. / 20., c6 = 1.;
constexpr double b1 = 82889. / 524892., b3 = 15625. / 83664., b4 = 69875. / 102672., b5 = -2260. / 8211.,
                 b6 = 1. / 4.;
constexpr double hb1 = 4586570599. / 29645900160., hb3 = 178811875. / 945068544.,
                 hb4 = 814220225. / 1159782912., hb5 = -3700637. / 11593932., hb6 = 61727. / 225920.;
constexpr double a21 = 1. / 2., a31 = 13861. / 62500., a32 = 6889. / 62500.;
constexpr double a41 = -116923316275. / 2393684061468., a42 = -2731218467317. / 15368042101831.,
                 a43 = 9408046702089. / 11113171139209.;
constexpr double a51 = -451086348788. / 2902428689909., a52 = -2682348792572. / 7519795681897.,
                 a53 = 12662868775082. / 11960479115383., a54 = 3355817975965. / 11060851509271.;
constexpr double a61 = 647845179188. / 3216320057751., a62 = 73281519250. / 8382639484533.,
                 a63 = 552539513391. / 3454668386233., a64 = 3354512671639. / 8306763924573., a65 = 4040. / 17871.;
}  // namespace rk43

struct QDProblem;
struct ThermalContext;

struct QDContext {
  SbpContext sbp;
  int Ny = 0, Nz = 0;
  long N = 0;
  FaultParams fp{};
  DevBuf fa, fb, fsN, fDc, feta, flocked, fprestress;
  DevBuf slipVel, tauQSP, tauP, strength;  // Nz
  DevBuf bcL, bcR, bcT, bcB, bcRShift;     // boundary data
  DevBuf rhs, u, sxy;                       // N
  DevBuf flags;                             // unsigned, fault status bits
  DevBuf fault_its;                         // unsigned long long, root iterations
  double vL = 1e-9, fts = 2.0;
  int bcL_from_slip = 1, bcR_remote = 1;
  scy_solve_opts solve_opts{};
  long n_d_dt = 0, n_solve_its = 0, n_solves = 0;
  double last_rnorm = 0.0;

  // RK integrator state
  scy_ode_opts ode{};
  int ode_ready = 0;
  DevBuf rk[16];  // var, dvar, k/f stage vectors, lo/hi
  DevBuf errbuf;  // 8 doubles
  double currT = 0, deltaT = 0, newDeltaT = 0, totTol = 1e-9, last_dt = 0;
  long stepCount = 0, numRejected = 0, numMin = 0, numMax = 0;
  double errA[2] = {0, 0};
  std::vector<double> forced_dt;
  std::vector<int> forced_acc;
  size_t forced_pos = 0;
  std::vector<double> log_dt;
  std::vector<int> log_acc;
  std::vector<double> log_step_dt;  // per taken step, the size of the attempt whose solution was kept
  // timeMonitor's output at the reference's strides (writer.cu); null: none
  std::unique_ptr<OutputWriter> out;
  // checkpointing (timeMonitor :448-455 with writeCheckpoint of the driver,
  // LinearElastic and Fault): every ckpt_interval steps and at the end, the
  // chkpt_* files under ckpt_dir, after which integrate_steps returns with
  // done = 2 (the reference stops the run there)
  int ckpt = 0, ckpt_number = 0, ckpt_stopped = 0;
  long ckpt_interval = 10000;
  std::string ckpt_dir;
  int write_checkpoint();
  int record = 0;

  std::vector<double> h_a, h_b, h_sN;  // host copies for the steady-state guess
  // fault-response mode: tau_qs(body) = GL bcL + c(t) g1 + gs, surface
  // displacement = SL bcL + c(t) s1 + ss (c(t) = vL t / faultTypeScale)
  int mode = 0;        // SCY_QD_MODE_*
  int green_ready = 0;
  DevBuf GL, SL, g1, gs, s1, ss;
  double green_build_ms = 0.0;
  int build_green();
  int full_solve_for_output();
  double last_t = 0.0;  // time of the last d_dt (for output fields in response mode)
  double f0 = 0.6, v0 = 1e-6;

  // integrated state: length and per-field offsets / lengths by SCY_KEY_*
  long nvar = 0;
  long key_off[4] = {0, 0, 0, 0}, key_len[4] = {0, 0, 0, 0};
  int check_err_keys(scy_ode_opts& o) const;
  // power-law viscoelastic material (StrikeSlip_PowerLaw_qd); pl = 0: linear elastic
  int pl = 0;
  double inv_visc_cap = 0.0;
  DevBuf pl_c1, pl_e1, pl_n;   // 1e3*A, exp(-B/T), n per node
  DevBuf sxz, sdev, effVisc;   // N
  int create(const scy_qd_desc& d, const scy_pl_desc* pl_desc = nullptr);
  // StrikeSlip_LinearElastic_qd::solveSS + solveSSb + Fault::guessSS: fills
  // psi (unless keep_psi) and slip, updates bcL, bcRShift, slipVel, u.
  int steady_state_guess(std::vector<double>& psi, int keep_psi, std::vector<double>& slip);
  // the power-law driver's steady-state initial guess (solveSS); fills psi,
  // slip and the viscous strains gVxy, gVxz (N each), sets bcRShift / bcR;
  // *its and *err report the effective-viscosity iteration
  int ss_its = 0;        // effective-viscosity iterations of the last pl_steady_state
  double ss_err = 0.0;   // and its last relative change
  long ss_cg_its = 0;    // and the conjugate-gradient iterations of its solves
  // per viscosity iteration: correction steps, relative residual before and
  // after them, CG iterations, relative change of the viscosity
  std::vector<double> ss_trace;
  int pl_steady_state(const QDProblem& P, std::vector<double>& psi, std::vector<double>& slip,
                      double* gVxy, double* gVxz, int* its, double* err);
  // computeMinTimeStep (strikeSlip_linearElastic_qd.cpp:262-322)
  double compute_min_dt(const std::vector<double>& cs, double Ly, double Lz) const;
  // f = d_dt(t, var) with var = [psi | slip] and f = [dpsi | dslip] (device, 2*Nz each)
  int d_dt(double t, const double* var, double* f);
  // the fault's rates alone, given the body's shear stress on the fault
  int fault_d_dt(const double* var, const double* tau_body, double* f);
  int integrate_begin(const scy_ode_opts& o);
  // A fresh integrator object of a driver that restarts the RK per phase
  // (strikeSlip_linearElastic_qd_fd.cpp:1436-1508, :891-956): time range
  // [t0, t1], first step init_dt, bounds [min_dt, max_dt], step count
  // continuing from step0 with max_rel more steps allowed, empty error
  // history; evaluates the rates at t0.
  int phase_begin(double t0, double t1, double init_dt, double min_dt, double max_dt, long step0, long max_rel);
  int integrate_steps(long nsteps, scy_ode_stats* st);
  // Called after every accepted step (timeMonitor); a nonzero *stop ends
  // the phase (integrate_steps returns with phase_stopped = 1).
  std::function<int(int* stop)> monitor;
  // RK32_WBE / RK43_WBE (odeSolverImex.cpp:352-470, :837-): a strict
  // acceptance test, and after every accepted step the implicit heat step
  // of th (thermal.cu); in coupled mode the fault's temperature is set from
  // the heat equation's at the start of that step's last d_dt
  int imex = 0;
  std::shared_ptr<ThermalContext> th;
  int phase_stopped = 0;
  double compute_step_size(double totErr);
  int compute_error(const double* lo, const double* hi, double* err);
  // computeError from the per-key sums (sum d^2, sum hi^2, max |d/hi|) at h[3*key]
  double error_from(const double* h) const;
  int attempt(double dt, double** lo, double** hi);
  int read_flags();
};

int qd_green_surf_launch(QDContext& q, double c, double* host_out);
// bcL = slip/faultTypeScale, bcR = vL t/faultTypeScale + bcRShift from the state var
int qd_bc_launch(QDContext& q, double t, const double* var);
// StrikeSlip_PowerLaw_qd::d_dt (powerlaw.cu)
int pl_d_dt(QDContext& q, double t, const double* var, double* f);

}  // namespace scy
