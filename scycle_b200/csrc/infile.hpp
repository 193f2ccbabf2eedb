// The reference's ``.in`` input format and PETSc-binary vectors, on the host.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "../../include/scycle_b200.h"

namespace scy {

struct HeatProblem;

struct InEntry {
  std::string var, rhs, full;  // key, value up to the first space, everything after " = "
};

// Splits every line at the first " = " (source/domain.cpp:153-166 and the
// same loop in every class's loadSettings).  Throws std::runtime_error if
// the file cannot be read.
std::vector<InEntry> parse_in_file(const std::string& path);
std::vector<InEntry> parse_in_text(const std::string& text);

double c_atof(const std::string& s);
int c_atoi(const std::string& s);
// ``[v1 v2 ...]`` lists (source/genFuncs.cpp:413-440, :476-505)
std::vector<double> load_vector_double(const std::string& s);
std::vector<std::string> load_vector_string(const std::string& s);
// Piecewise-linear depth profile with extrapolation (source/genFuncs.cpp:574-617).
std::vector<double> set_vec(const std::vector<double>& coord, const std::vector<double>& vals,
                            const std::vector<double>& depths);
// Reads the first Vec record of a PETSc binary file into out.  Returns false
// if the file does not exist; throws std::runtime_error if it is malformed
// or holds a different length than n.
bool read_petsc_vec(const std::string& path, size_t n, std::vector<double>& out);
// Writes (append = 0) or appends (append = 1) one Vec record.
void write_petsc_vec(const std::string& path, const double* v, size_t n, int append);

// Everything StrikeSlip_LinearElastic_qd reads from an input file, with the
// host arrays the descriptor points into.
struct QDProblem {
  scy_qd_desc desc{};
  scy_ode_opts ode{};
  int guess_ss = 0;
  int stride1D = 1, stride2D = 1;
  std::string inputDir, outputDir, stateLaw, integrator;
  double vL = 1e-9, min_dt_user = -1.0;
  double ksp_tol = -1.0;  // kspTol (LinearElastic: KSP rtol = atol = kspTol), -1 if absent
  std::vector<double> y, z, mu, rho, cs;
  std::vector<double> a, b, sN, Dc, locked, prestress, psi, eta, mu_f, rho_f;
  std::vector<double> bcL0, bcRShift;
  int stateVals_given = 0;
  // StrikeSlip_PowerLaw_qd (bulkDeformationType powerLaw)
  int pl = 0;
  scy_pl_desc pdesc{};
  std::vector<double> plA, plB, pln, plT, gVxy0, gVxz0;
  // the steady-state iteration of guessSteadyStateICs = 1
  // (strikeSlip_powerLaw_qd.cpp:27-29, :157-163) and its optional
  // inputDir/effVisc and inputDir/tauSS (empty if absent)
  double ss_fss = 0.2, ss_gss_t = 1e-10, ss_atol = 1e-3;
  int ss_max_its = 50;
  std::vector<double> ss_effvisc, ss_tau;
  double init_time = 0.0;
  // strikeSlip_linearElastic_qd_fd only (cycle = 1)
  int cycle = 0;
  scy_cycle_desc cdesc{};
  std::vector<double> slip_file;  // inputDir/slip, empty if absent
  // checkpointing (Domain enableCheckpointing / interval, domain.cpp:17-28,
  // :187-188); a restart (ckptNumber > 0 in outputDir) starts from the
  // chkpt_* files written by the previous run
  int ckpt = 0, ckpt_number = 0;
  long ckpt_interval = 10000;
  // extension key ckptContinueSteps (not read by the reference): a restart
  // keeps the checkpoint's step count and error history instead of
  // starting both from zero as the reference's does
  int ckpt_continue = 0;
  long step0 = 0;
  double errA[2] = {0.0, 0.0};
  std::vector<double> slipVel0;  // chkpt_slipVel (first guess of the root finder), empty if none
  // RK32_WBE / RK43_WBE (strict acceptance, a heat step after each accepted
  // step) and the heat equation of thermalCoupling uncoupled / coupled
  int imex = 0;
  std::shared_ptr<HeatProblem> heat;
};

// Builds the problem like Domain + LinearElastic + Fault_qd +
// StrikeSlip_LinearElastic_qd constructors do, or (cycle = 1) like
// strikeSlip_linearElastic_qd_fd's.  Throws std::runtime_error with a
// message on invalid input.
void load_qd_problem(const std::string& path, QDProblem& P, int cycle = 0);

}  // namespace scy
