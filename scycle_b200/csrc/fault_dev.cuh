// Rate-and-state fault on the device: one thread per fault node.
//
// Follows Fault_qd::d_dt / ComputeVel_qd::computeVel (reference
// source/fault.cpp:861-1059), BracketedNewton::findRoot
// (source/rootFinder.cpp:174-257) and the state laws (fault.cpp:1984-2088,
// strength :2247-2251).
#pragma once
#include <cuda_runtime.h>

namespace scy {

enum FaultFlags : unsigned {
  FAULT_ROOT_NOCONV = 1u,
  FAULT_NONFINITE = 2u,
};

struct FaultParams {
  int Nz;
  long psi_off, slip_off;  // offsets of psi and slip in the integrated state
  const double *a, *b, *sN, *Dc, *eta, *locked, *prestress;
  double f0, v0, vL, root_tol;
  int max_its;
  int state_law;  // 0 aging, 1 slip, 2 constant state, 3 flash heating
  int jacobian;   // 0 the reference's derivative expression, 1 the exact derivative
  // flash heating (state law 3; the heat equation's fields on the fault):
  // temperature Tf, rho c, k and the weakening temperature Tw per node, the
  // weakening velocity written back to Vw
  const double *Tf = nullptr, *rc_f = nullptr, *k_f = nullptr, *Tw = nullptr;
  double* Vw = nullptr;
  double fl_D = 5.0, fl_tau_c = 3.0, fl_fw = 0.64;
};

__device__ __forceinline__ double strength_psi(double sN, double psi, double V, double a, double v0) {
  return a * sN * asinh((0.5 * V / v0) * exp(psi / a));
}

// flashHeating_Vw (fault.cpp:2162-2168): the weakening velocity
__device__ __forceinline__ double flash_heating_vw(double T, double rc, double k, double D, double Tw, double tau_c) {
  const double ath = k / rc;
  const double s = rc * (Tw - T) / tau_c;
  return (M_PI * ath / D) * (s * s);
}

// flashHeating_psi (fault.cpp:2171-2196): the regularised steady-state
// friction fLV, weakened to fw + (fLV - fw) Vw / |V| above Vw
__device__ __forceinline__ double flash_heating_psi(double psi, double V, double Vw, double fw, double Dc, double a,
                                                    double b, double f0, double v0) {
  const double absV = fabs(V);
  const double fLV = (a - b) * asinh(absV / v0 / 2.0 * exp(f0 / (a - b)));
  const double fss = absV > Vw ? fw + (fLV - fw) * (Vw / absV) : fLV;
  const double f = a * asinh((absV / 2. / v0) * exp(psi / a));
  return -absV / Dc * (f - fss);
}

// Residual of tau_qs - eta V = strength(V) and its derivative.  E =
// exp(psi/a) is computed once per node by the caller.  With exact == 0 the
// derivative is the reference's expression a*sN*V/sqrt(B^2 V^2 + 1) + eta
// with B = E/(2 v0) (fault.cpp:1051); the exact derivative has B in place of
// V in the numerator.  The derivative only steers the Newton / bisection
// choice: both converge to the same root within the residual tolerance, the
// reference's expression through many more (mostly bisection) steps.
__device__ __forceinline__ void resid_qd(double V, double tauQS, double eta, double sN, double E, double a,
                                         double v0, int exact, double& f, double& J) {
  f = a * sN * asinh((0.5 * V / v0) * E) - (tauQS - eta * V);
  double A = a * sN;
  double B = E / (2.0 * v0);
  double s = sqrt(B * B * V * V + 1.0);
  J = (exact ? A * B / s : A * V / s) + eta;
}

// Safeguarded Newton on [left, right] starting from x0 for the residual
// R(x, f, f'), following BracketedNewton::findRoot (rootFinder.cpp:174-257).
// Returns the root; sets *its and *ok.  Every loop is bounded by max_its.
template <class Resid>
__device__ __forceinline__ double bracketed_newton_f(const Resid& R, double left, double right, double x0,
                                                     double atol, int max_its, int* its, bool* ok) {
  double f, fp, fl, fr, dum;
  *its = 0;
  *ok = true;
  R(x0, f, fp);
  if (fabs(f) <= atol) return x0;
  R(left, fl, dum);
  R(right, fr, dum);
  if (!isfinite(fl) || !isfinite(fr)) {
    *ok = false;
    return x0;
  }
  if (sqrt(fl * fl) <= atol) return left;
  if (sqrt(fr * fr) <= atol) return right;
  if (fl > 0) {
    double t = left;
    left = right;
    right = t;
  }
  double x = x0;
  double dxold = fabs(right - left), dx = dxold;
  R(x, f, fp);
  int n = 0;
  while (n <= max_its && fabs(f) >= atol) {
    if (((x - right) * fp - f) * ((x - left) * fp - f) > 0.0 || fabs(2.0 * f) > fabs(dxold * fp)) {
      dxold = dx;
      dx = 0.5 * (right - left);
      x = left + dx;
    } else {
      dxold = dx;
      dx = f / fp;
      x -= dx;
    }
    R(x, f, fp);
    if (f < 0.0)
      left = x;
    else
      right = x;
    ++n;
  }
  *its = n;
  if (!(fabs(f) <= atol)) *ok = false;
  if (!isfinite(f)) *ok = false;
  return x;
}

// Quasi-dynamic slip-velocity residual (ComputeVel_qd::getResid).
struct ResidQD {
  double tauQS, eta, sN, E, a, v0;
  int exact;
  __device__ __forceinline__ void operator()(double V, double& f, double& J) const {
    resid_qd(V, tauQS, eta, sN, E, a, v0, exact, f, J);
  }
};

__device__ __forceinline__ double bracketed_newton(double left, double right, double x0, double atol, int max_its,
                                                   double tauQS, double eta, double sN, double psi, double a,
                                                   double v0, int exact, int* its, bool* ok) {
  const ResidQD R{tauQS, eta, sN, exp(psi / a), a, v0, exact};
  return bracketed_newton_f(R, left, right, x0, atol, max_its, its, ok);
}

__device__ __forceinline__ double aging_law_psi(double psi, double V, double b, double f0, double v0, double Dc) {
  double A = exp((f0 - psi) / b);
  if (!isinf(A) && b > 1e-3) return (b * v0 / Dc) * (A - V / v0);
  return 0.0;
}

__device__ __forceinline__ double slip_law_psi(double psi, double V, double a, double b, double f0, double v0,
                                               double Dc) {
  if (V == 0.0) return 0.0;
  double absV = fabs(V);
  double fss = f0 + (a - b) * log(absV / v0);
  double f = a * asinh((absV / 2.0 / v0) * exp(psi / a));
  return -absV / Dc * (f - fss);
}

}  // namespace scy

namespace scy {

// Fully dynamic slip-velocity residual (ComputeVel_fd::getResid,
// fault.cpp:1649-1685): fricPen*strength(V) - (|Phi| - V), exact derivative.
struct ResidVelFD {
  double absPhi, fricPen, sN, psi, a, v0, E;
  __device__ __forceinline__ void operator()(double V, double& f, double& J) const {
    const double constraints = fricPen * (a * sN * asinh((0.5 * V / v0) * E));
    const double stress = absPhi - V;
    f = constraints - stress;
    const double A = a * sN;
    const double B = E / (2. * v0);
    J = 1 + fricPen * A * B / sqrt(1. + B * B * V * V);
  }
};

// Implicit-midpoint state residuals of the fully dynamic phase
// (ComputeAging_fd / ComputeSlipLaw_fd ::getResid, fault.cpp:1750-1763,
// :1851-1865): -2 dt G((psiPrev + state)/2, V) + (state - psiPrev).
struct ResidAgingFD {
  double psiPrev, V, b, f0, v0, Dc, dt;
  __device__ __forceinline__ void operator()(double state, double& f, double& J) const {
    const double G = aging_law_psi((psiPrev + state) / 2.0, V, b, f0, v0, Dc);
    f = -2 * dt * G + (state - psiPrev);
    J = 1 + dt * v0 / Dc * exp((f0 - (psiPrev + state) / 2.) / b);
  }
};

struct ResidSlipFD {
  double psiPrev, V, a, b, f0, v0, Dc, dt;
  __device__ __forceinline__ void operator()(double state, double& f, double& J) const {
    const double G = slip_law_psi((psiPrev + state) / 2.0, V, a, b, f0, v0, Dc);
    f = -2 * dt * G + (state - psiPrev);
    const double A = fabs(V) / 2. / v0 * exp((psiPrev + state) / 2.0 / a);
    J = 1 + dt * fabs(V) / Dc * A / sqrt(1 + A * A);
  }
};

}  // namespace scy
