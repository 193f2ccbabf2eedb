// Heat equation of the thermal quasi-dynamic drivers (thermalCoupling
// uncoupled / coupled with the RK32_WBE / RK43_WBE integrators) and the
// flash-heating state law's fault fields.
//
// Host side (thermal_host.cpp): HeatEquation's settings and fields
// (source/heatEquation.cpp: loadSettings :138-216, checkInput :369-407,
// setFields :316-366, loadFieldsFromFiles :217-259, constructMapV :460-523)
// and the initial steady-state geotherm (computeInitialSteadyStateTemp
// :525-683): k T'' = -Qrad in the lithosphere, the first Nz_lab nodes of
// every column, with the "z" Laplace type, whose operator couples the nodes
// of a column only, so every column is a 1D SBP problem (Dirichlet top and
// bottom values from the linear extrapolation of TVals[0..1]); the mantle
// adiabat of the last two TVals below.  The fault's flash-heating fields
// (Fault::loadSettings fault.cpp:89-97, setThermalFields :316-345).
//
// Device side (thermal.cu): the backward-Euler step of be_transient
// (:1146-1240) as conjugate gradients on the symmetrised system
//   (rho c I - dt A_k) dT = dt (setRhs_k(bcL) + [var. grid] H J Q) + rho c I dTn,
// I = (J) H, A_k the SBP operator of k with R, T, B Dirichlet and L Neumann
// (setUpTransientProblem :1627-1711), Jacobi-preconditioned; the steady step
// of be_steadyState (:1242-1318) as A_k dT = setRhs_k(bcL) - H J Q with the
// solver of the SBP context; frictional heating (computeFrictionalShearHeating
// :1543-1576) as the fault flux -tau V / 2 (zero-width shear zone) or the
// Gaussian body source; the heat flux k Dz T at the surface (computeHeatFlux
// :1713-1733).
#pragma once
#include <memory>
#include <string>
#include <vector>


namespace scy {

struct QDProblem;

struct HeatProblem {
  int coupling = 0;  // thermalCoupling: 0 no, 1 uncoupled, 2 coupled
  int steady = 0;    // heatEquationType: 0 transient, 1 steadyState
  int fric = 1, visc = 1, radio = 1;  // withFrictionalHeating, withViscShearHeating, withRadioHeatGeneration
  double ksp_tol = 1e-11;             // kspTol_heateq
  int Nz_lab = 0;
  double Lz_lab = 0.0;
  std::vector<double> TVals, TDepths;
  // fields, length Ny*Nz
  std::vector<double> k, rho, c, Tamb, T, dT, Qrad, w, Gw;
  double wMax = 0.0;
  // flash heating (stateLaw = flashHeating)
  int flash = 0;
  std::vector<double> Tw, rho_f;  // Nz
  double fw = 0.64, Vw = 0.12, D = 5.0, tau_c = 3.0;
};

// Reads the heat settings of the input file (P must be loaded already:
// grid, coordinates, fault rho); computes the initial geotherm unless
// inputDir holds Tamb.  Throws std::runtime_error on invalid input.
void load_heat_problem(const std::string& path, const QDProblem& P, HeatProblem& H);

}  // namespace scy
