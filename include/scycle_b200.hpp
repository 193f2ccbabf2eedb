/* C++ classes over the C ABI of scycle_b200.h with the reference's class
 * interfaces, for a C++ caller that keeps SCycle's structure and hands its
 * vectors to the device (header-only; link libscycle_b200.so).
 *
 *   scycle_b200::SbpOps  the interface of SbpOps (source/sbpOps.hpp:42-104)
 *                        for device vectors: set* options, computeMatrices,
 *                        changeBCTypes, setRhs, Dy / muxDy / Dyxmu / Dz /
 *                        muxDz / Dzxmu / H / Hinv, and solve (the
 *                        KSPSolve of LinearElastic::computeU,
 *                        linearElastic.cpp:465-489);
 *   scycle_b200::QD      a whole quasi-dynamic driver from a .in file
 *                        (StrikeSlip_LinearElastic_qd or _PowerLaw_qd:
 *                        main.cpp:227-233 and integrate());
 *   scycle_b200::Fault_qd  the interface of Fault_qd (fault.hpp:138-160)
 *                        over a driver's fault: d_dt given the body's
 *                        stress on the fault, the member vectors.
 *
 * Methods return the library's status (0 = success, as PetscErrorCode 0);
 * scycle_b200::last_error() gives the message.  Vectors are device
 * pointers of Ny*Nz doubles (y-major, the reference's ordering); boundary
 * vectors have Nz (left, right) or Ny (top, bottom) values. */
#pragma once
#include <string>
#include <vector>

#include "scycle_b200.h"

namespace scycle_b200 {

inline std::string last_error() { return scy_get_last_error(); }

inline int bc_type(const std::string& t) {
  if (t == "Dirichlet") return SCY_BC_DIRICHLET;
  if (t == "Neumann") return SCY_BC_NEUMANN;
  return -1;
}

class SbpOps {
 public:
  /* SbpOps_m_constGrid(order, Ny, Nz, Ly, Lz, muVec) / SbpOps_m_varGrid:
   * mu is a host array of Ny*Nz values (GPa). */
  SbpOps(int order, int Ny, int Nz, double Ly, double Lz, const double* mu_host)
      : order_(order), Ny_(Ny), Nz_(Nz), Ly_(Ly), Lz_(Lz), mu_(mu_host, mu_host + (size_t)Ny * Nz) {}
  ~SbpOps() {
    if (s_) scy_sbp_destroy(s_);
  }
  SbpOps(const SbpOps&) = delete;
  SbpOps& operator=(const SbpOps&) = delete;

  int setBCTypes(const std::string& R, const std::string& T, const std::string& L, const std::string& B) {
    const int b[4] = {bc_type(R), bc_type(T), bc_type(L), bc_type(B)};
    for (int v : b)
      if (v < 0) return SCY_ERR_ARG;
    for (int i = 0; i < 4; ++i) bc_[i] = b[i];
    return s_ ? scy_sbp_change_bc_types(s_, bc_[0], bc_[1], bc_[2], bc_[3]) : SCY_OK;
  }
  /* setGrid(y, z): host coordinate arrays of Ny*Nz values (variable grid) */
  int setGrid(const double* y_host, const double* z_host) {
    y_.assign(y_host, y_host + (size_t)Ny_ * Nz_);
    z_.assign(z_host, z_host + (size_t)Ny_ * Nz_);
    grid_ = SCY_GRID_VAR;
    return SCY_OK;
  }
  int setCompatibilityType(const std::string& t) {
    if (t == "fullyCompatible") compat_ = SCY_COMPAT_FULLY;
    else if (t == "compatible") compat_ = SCY_COMPAT_COMPATIBLE;
    else return SCY_ERR_ARG;
    return SCY_OK;
  }
  /* the device operator is the H-multiplied "yz" form LinearElastic builds
   * (linearElastic.cpp:441-446); the other choices are not built */
  int setMultiplyByH(int m) { return m == 1 ? SCY_OK : SCY_ERR_ARG; }
  int setLaplaceType(const std::string& t) { return t == "yz" ? SCY_OK : SCY_ERR_ARG; }
  int setDeleteIntermediateFields(int) { return SCY_OK; }
  int computeMatrices() {
    if (s_) return SCY_OK;
    scy_grid_desc d{};
    d.order = order_;
    d.Ny = Ny_;
    d.Nz = Nz_;
    d.Ly = Ly_;
    d.Lz = Lz_;
    d.grid_type = grid_;
    d.compat = compat_;
    d.y = y_.empty() ? nullptr : y_.data();
    d.z = z_.empty() ? nullptr : z_.data();
    d.mu = mu_.data();
    d.bcR = bc_[0];
    d.bcT = bc_[1];
    d.bcL = bc_[2];
    d.bcB = bc_[3];
    return scy_sbp_create(&d, &s_);
  }
  int changeBCTypes(const std::string& R, const std::string& T, const std::string& L, const std::string& B) {
    return setBCTypes(R, T, L, B);
  }
  /* setRhs(rhs, bcL, bcR, bcT, bcB) */
  int setRhs(double* rhs, const double* bcL, const double* bcR, const double* bcT, const double* bcB) {
    return ready() ? scy_sbp_set_rhs(s_, bcL, bcR, bcT, bcB, rhs) : SCY_ERR_STATE;
  }
  int A(const double* in, double* out) { return op(SCY_OP_A, in, out); }
  int Dy(const double* in, double* out) { return op(SCY_OP_DY, in, out); }
  int muxDy(const double* in, double* out) { return op(SCY_OP_MUXDY, in, out); }
  int Dyxmu(const double* in, double* out) { return op(SCY_OP_DYXMU, in, out); }
  int Dz(const double* in, double* out) { return op(SCY_OP_DZ, in, out); }
  int muxDz(const double* in, double* out) { return op(SCY_OP_MUXDZ, in, out); }
  int Dzxmu(const double* in, double* out) { return op(SCY_OP_DZXMU, in, out); }
  int H(const double* in, double* out) { return op(SCY_OP_H, in, out); }
  int Hinv(const double* in, double* out) { return op(SCY_OP_HINV, in, out); }
  /* the KSPSolve of LinearElastic::computeU: A u = rhs (u also the initial
   * guess when opts.nonzero_guess = 1) */
  int solve(const double* rhs, double* u, const scy_solve_opts& opts, scy_solve_stats* stats = nullptr) {
    scy_solve_stats st{};
    const int rc = ready() ? scy_sbp_solve(s_, rhs, u, &opts, &st) : SCY_ERR_STATE;
    if (stats) *stats = st;
    return rc;
  }
  int synchronize() { return ready() ? scy_sbp_synchronize(s_) : SCY_ERR_STATE; }
  scy_sbp* handle() { return s_; }

 private:
  bool ready() const { return s_ != nullptr; }
  int op(int o, const double* in, double* out) { return ready() ? scy_sbp_apply(s_, o, in, out) : SCY_ERR_STATE; }
  int order_, Ny_, Nz_;
  double Ly_, Lz_;
  std::vector<double> mu_, y_, z_;
  int grid_ = SCY_GRID_CONST, compat_ = SCY_COMPAT_FULLY;
  int bc_[4] = {SCY_BC_DIRICHLET, SCY_BC_NEUMANN, SCY_BC_DIRICHLET, SCY_BC_NEUMANN};
  scy_sbp* s_ = nullptr;
};

class QD {
 public:
  /* the driver main.cpp builds from inputFile, with the solver options of
   * the device solve */
  explicit QD(const std::string& inputFile, const scy_solve_opts& solve) {
    status_ = scy_qd_create_from_in(inputFile.c_str(), &solve, &q_);
  }
  ~QD() {
    if (q_) scy_qd_destroy(q_);
  }
  QD(const QD&) = delete;
  QD& operator=(const QD&) = delete;
  int status() const { return status_; }
  /* initiateIntegrand (with the steady-state guess where the file asks for
   * it) and the first d_dt */
  int initiateIntegrand() { return q_ ? scy_qd_integrate_begin_from_in(q_) : status_; }
  /* nsteps accepted RK steps (the reference's integrate() loop, bounded) */
  int integrate(long nsteps, scy_ode_stats* stats) { return q_ ? scy_qd_integrate_steps(q_, nsteps, stats) : status_; }
  /* a fault or body field into a host array (SCY_FIELD_*) */
  int getField(int field, double* host) { return q_ ? scy_qd_get_field(q_, field, host) : status_; }
  scy_qd* handle() { return q_; }

 private:
  scy_qd* q_ = nullptr;
  int status_ = SCY_OK;
};

/* The interface of Fault_qd (fault.hpp:138-160) over a driver's fault:
 * d_dt with the body's shear stress on the fault supplied by the caller
 * (what StrikeSlip_LinearElastic_qd::d_dt passes after its solve), the
 * member vectors read back through getField.  The fault's parameters are
 * those of the driver's input file. */
class Fault_qd {
 public:
  explicit Fault_qd(QD& qd) : q_(qd.handle()) {}
  /* var, dvar: device, scy_qd_state_size doubles; tauBody: device, Nz */
  int d_dt(const double* var, const double* tauBody, double* dvar) {
    return q_ ? scy_qd_fault_d_dt(q_, var, tauBody, dvar) : SCY_ERR_STATE;
  }
  int slipVel(double* host) { return get(SCY_FIELD_SLIPVEL, host); }
  int tauP(double* host) { return get(SCY_FIELD_TAUP, host); }
  int tauQSP(double* host) { return get(SCY_FIELD_TAUQSP, host); }
  int strength(double* host) { return get(SCY_FIELD_STRENGTH, host); }

 private:
  int get(int f, double* host) { return q_ ? scy_qd_get_field(q_, f, host) : SCY_ERR_STATE; }
  scy_qd* q_;
};

}  // namespace scycle_b200
