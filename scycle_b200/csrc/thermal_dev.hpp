// Device state of the heat equation of a thermal quasi-dynamic driver (see
// thermal.hpp for the equations; thermal.cu).
#pragma once
#include "sbp_solver.hpp"
#include "thermal.hpp"

namespace scy {

struct QDContext;

// The device state of the heat equation of one driver.
struct ThermalContext {
  int Ny = 0, Nz = 0;
  long N = 0;
  int coupled = 0, steady = 0, fric = 1, var_grid = 0;
  double ksp_tol = 1e-11, wMax = 0.0;
  SbpContext sbp;                         // operator of k (R, T, B Dirichlet; L Neumann)
  DevBuf Tamb, T, dT, Iw, rc, diagK, Gw, Qrad;  // N
  DevBuf Tf, rc_f, k_f, Tw, Vw;           // fault (Nz): temperature the friction law reads, ...
  DevBuf bcL, zNz, zNy;                   // heat boundary data, zero vectors
  DevBuf r, z, p, q_, rhs, sc;            // CG work (N) and block partial sums
  long solves = 0, its = 0;
  int create(QDContext& q, const HeatProblem& H);
  // HeatEquation::be after an accepted step of size dt: the fault's slip
  // velocity and tauP of the accepted state from q; T, dT updated
  int step(QDContext& q, double dt);
  // updateTemperature: the fault temperature the flash-heating law reads
  int set_fault_temperature();
  // Jacobi-preconditioned CG on (rho c I - dt A_k) dT = rhs from the last dT
  int pcg(double dt);
};

}  // namespace scy
