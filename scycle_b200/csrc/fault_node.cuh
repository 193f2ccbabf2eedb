// Fault_qd::d_dt for one fault node (one thread per node), shared by the
// linear-elastic, response-mode and power-law drivers.
#pragma once
#include "fault_dev.cuh"

namespace scy {

// Fault_qd::d_dt for one node given its quasi-static shear stress from the
// body (fault.cpp:861-918): prestress, bracketed Newton, state law, tauP,
// strength.
__device__ __forceinline__ void fault_node_update(int iz, double tau_body, const FaultParams& fp,
                                                  const double* __restrict__ var, double* __restrict__ f,
                                                  double* __restrict__ slipVel, double* __restrict__ tauQSP,
                                                  double* __restrict__ tauP, double* __restrict__ strength,
                                                  unsigned* flags, unsigned long long* its_total) {
  const double tq = tau_body + fp.prestress[iz];
  tauQSP[iz] = tq;
  const double psi = var[fp.psi_off + iz];
  const double a = fp.a[iz], sN = fp.sN[iz], eta = fp.eta[iz];
  double V;
  const double lk = fp.locked[iz];
  if (lk > 0.5) {
    V = 0.0;
  } else if (lk < -0.5) {
    V = fp.vL;
  } else {
    double left = 0.0, right = tq / eta;
    if (isnan(right)) {
      atomicOr(flags, (unsigned)FAULT_NONFINITE);
      V = slipVel[iz];
    } else if (fabs(left - right) < 1e-14) {
      V = left;
    } else {
      int its = 0;
      bool ok = true;
      V = bracketed_newton(left, right, slipVel[iz], fp.root_tol, fp.max_its, tq, eta, sN, psi, a, fp.v0,
                           fp.jacobian, &its, &ok);
      atomicAdd(its_total, (unsigned long long)its);
      if (!ok) atomicOr(flags, (unsigned)FAULT_ROOT_NOCONV);
    }
  }
  slipVel[iz] = V;
  double dpsi;
  if (fp.state_law == 0)
    dpsi = aging_law_psi(psi, V, fp.b[iz], fp.f0, fp.v0, fp.Dc[iz]);
  else if (fp.state_law == 1)
    dpsi = slip_law_psi(psi, V, a, fp.b[iz], fp.f0, fp.v0, fp.Dc[iz]);
  else if (fp.state_law == 3) {
    // flashHeating_psi_Vec (fault.cpp:2199-2243): Vw from the fault's temperature
    const double vw = flash_heating_vw(fp.Tf[iz], fp.rc_f[iz], fp.k_f[iz], fp.fl_D, fp.Tw[iz], fp.fl_tau_c);
    fp.Vw[iz] = vw;
    dpsi = flash_heating_psi(psi, V, vw, fp.fl_fw, fp.Dc[iz], a, fp.b[iz], fp.f0, fp.v0);
  } else
    dpsi = 0.0;
  if (!isfinite(dpsi) || !isfinite(V)) atomicOr(flags, (unsigned)FAULT_NONFINITE);
  f[fp.psi_off + iz] = dpsi;
  f[fp.slip_off + iz] = V;
  tauP[iz] = tq - eta * V;
  strength[iz] = strength_psi(sN, psi, V, a, fp.v0);
}

}  // namespace scy
