// Quasi-dynamic / fully dynamic earthquake cycles on the device: the
// strikeSlip_linearElastic_qd_fd driver (source/strikeSlip_linearElastic_qd_fd.cpp).
//
// Quasi-dynamic phases run the QDContext integrator (one elliptic solve per
// RK stage).  Fully dynamic phases step the wave equation with a fixed
// CFL-limited step: per step one matrix-free stencil launch computes
// uNext = (dt^2/rho Hinv Jinv A u + 2u + (dt ay - 1) uPrev)/(dt ay + 1) and the
// fault row's Hinv Jinv A u, and one fault launch (a thread per fault node)
// runs Fault_fd::d_dt, the fault-row stress and the switch test
// max(eta V / tauQS), whose last block decides on the device whether the
// phase ends.  Steps are batched into CUDA graphs; a step after the switch
// step finds the stop flag set and returns at once, so a batch never runs
// past the switch.
#pragma once
#include <map>
#include <utility>
#include <vector>

#include "qd.hpp"

namespace scy {

// Device-side state of the fully dynamic phase (one instance).
struct CycleDevState {
  unsigned counter;        // last-block detection in the fault launch
  int stop;                // set by the step whose switch test fired
  int allowed;             // checkSwitchRegime's _allowed
  int steps_done;          // steps completed since the batch started
  double maxR;             // max(eta V / tauQS) of the last step
  unsigned flags;          // FAULT_* bits of root finds that failed
  unsigned pad;
  unsigned long long its;  // root iterations
};

struct CycleSwitch {
  long step;
  double t;
  int to_fd;
  double R;
};

enum CyclePhase { CP_QD_BEGIN = 0, CP_QD, CP_FD_BEGIN, CP_FD_SINGLE, CP_FD, CP_DONE };

// launches of one fully dynamic step: the wave stencil and the fault update
// as two launches, or one fused launch
enum { FD_WAVE = 1, FD_FAULT = 2, FD_FUSED = 4 };

struct CycleContext {
  QDContext q;
  int Ny = 0, Nz = 0;
  long N = 0;
  // settings (after the reference's checkInput)
  double dt_fd = 0, trigger_qd2fd = 1e-3, trigger_fd2qd = 1e-3, limit_qd = 1e-8, limit_fd = 0.1;
  int max_num_cycles = 1000;
  int ay_quirk = 1;
  scy_ode_opts ode{};  // quasi-dynamic phases: method, control, norm, tol, bounds, time range, step budget
  // fully dynamic operator (all material boundaries Neumann) and fields
  LevelHost fd_host;
  LevelStore<double> fd_level;
  DevBuf u3[3], psi3[3], slip3[3];  // rotating n-1 / n / n+1
  DevBuf u0, wc, wcy, wcz, ay, hinvf, jinvf, d2u, slip0, tau0, alphay, rho_f, utmp;
  int wc_sep = 0;  // wc = wcy[iy] * wcz[iz]
  DevBuf dstate;
  CycleDevState* h_state = nullptr;  // pinned
  // driver state
  double currT = 0;
  long stepCount = 0;
  int cycleCount = 0, allowed = 0, inDynamic = 0, first_cycle = 1;
  int phase = CP_DONE;
  int rot = 0;          // completed fully dynamic steps modulo 3
  long fd_max_steps = 0;
  double last_R = 0;
  long qd_steps = 0, fd_steps = 0;
  double qd_ms = 0, fd_ms = 0;
  int fd_batch = 64;
  int began = 0;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  std::vector<CycleSwitch> switches;

  ~CycleContext();
  int create(const scy_qd_desc& qd, const scy_cycle_desc& cd);
  // initiateIntegrands: var0 = [psi | slip] after the optional steady-state guess
  int begin(const scy_ode_opts& o, const double* var0_host);
  // Advances up to `budget` global steps (quasi-dynamic accepted steps,
  // the single quasi-dynamic step of each switch, wave-equation steps).
  int run(long budget, scy_cycle_stats* st);
  int get_field(int field, double* host_out);
  int set_fd_state(double t, long step, int allowed, const double* const* fault_now, const double* u,
                   const double* const* fault_prev, const double* uPrev, const double* u0_host,
                   const double* slip0_host, const double* tau0_host, const double* slipVel_host);
  void fill_stats(scy_cycle_stats* st) const;

  // internals
  int check_switch(double maxR, int* stop);     // checkSwitchRegime
  int qd_monitor(int* stop);                    // timeMonitor of the quasi-dynamic phases
  int qd_max_ratio(double* out);
  int enter_fd();                               // the rest of prepare_qd2fd
  int leave_fd();                               // prepare_fd2qd's data movement
  int fd_batch_run(int K, int* n_done, int* stopped);
  int fd_launch_step(int r, cudaStream_t s, int part);  // FD_* bits
  int time_kernels(int reps, double* wave_us, double* fault_us, double* step_us);
  int fd_parts = FD_FUSED;  // what one graph step launches
  int current_u(double* dst);                   // material u of the phase (device)
};

}  // namespace scy
