// Heat-equation settings, fields and the initial geotherm (see thermal.hpp).
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "infile.hpp"
#include "sbp_host.hpp"
#include "thermal.hpp"

namespace scy {

namespace {

// dense LU with partial pivoting: solves M x = b in place (M row-major n x n)
void dense_solve(std::vector<double>& M, std::vector<double>& b, int n) {
  std::vector<int> piv(n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(M[(size_t)i * n + k]) > std::fabs(M[(size_t)p * n + k])) p = i;
    if (M[(size_t)p * n + k] == 0.0) throw std::runtime_error("singular geotherm system");
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(M[(size_t)k * n + j], M[(size_t)p * n + j]);
      std::swap(b[k], b[p]);
    }
    const double d = M[(size_t)k * n + k];
    for (int i = k + 1; i < n; ++i) {
      const double f = M[(size_t)i * n + k] / d;
      if (f == 0.0) continue;
      M[(size_t)i * n + k] = 0.0;
      for (int j = k + 1; j < n; ++j) M[(size_t)i * n + j] -= f * M[(size_t)k * n + j];
      b[i] -= f * b[k];
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    double s = b[k];
    for (int j = k + 1; j < n; ++j) s -= M[(size_t)k * n + j] * b[j];
    b[k] = s / M[(size_t)k * n + k];
  }
}

// computeInitialSteadyStateTemp (heatEquation.cpp:525-683)
void initial_geotherm(const QDProblem& P, HeatProblem& H) {
  const scy_grid_desc& g = P.desc.grid;
  const int Ny = g.Ny, Nz = g.Nz;
  const size_t N = (size_t)Ny * Nz;
  const auto& TV = H.TVals;
  const auto& TD = H.TDepths;
  if (Nz == 1) {
    H.Tamb.assign(N, TV[0]);
    H.T = H.Tamb;
    H.dT.assign(N, 0.0);
    return;
  }
  const double slope = (TV[1] - TV[0]) / (TD[1] - TD[0]);
  const double gT = slope * (0.0 - TD[0]) + TV[0];
  const double gB = slope * (H.Lz_lab - TD[0]) + TV[0];
  const int Nzl = H.Nz_lab;
  const bool var = g.grid_type == SCY_GRID_VAR;
  // the lithosphere grid: Ny x Nz_lab nodes with the full Ly, Lz (on the
  // constant grid Nz_lab points then span Lz, as in the reference),
  // Dirichlet on every side, coefficient k
  std::vector<double> kl((size_t)Ny * Nzl), yl, zl;
  if (var) {
    yl.resize(kl.size());
    zl.resize(kl.size());
  }
  for (int iy = 0; iy < Ny; ++iy)
    for (int iz = 0; iz < Nzl; ++iz) {
      const size_t a = (size_t)iy * Nzl + iz, b = (size_t)iy * Nz + iz;
      kl[a] = H.k[b];
      if (var) {
        yl[a] = P.y[b];
        zl[a] = P.z[b];
      }
    }
  const int bc[4] = {SCY_BC_DIRICHLET, SCY_BC_DIRICHLET, SCY_BC_DIRICHLET, SCY_BC_DIRICHLET};
  LevelHost L = build_level(g.order, Ny, Nzl, g.Ly, g.Lz, var ? 1 : 0, g.compat, yl, zl, kl, bc);
  // the "z" Laplace type: A = H Dzz(k) + SAT_T + SAT_B, which for column iy
  // is the z line operator (with its coefficients and Dirichlet SATs) times
  // the column's outer weight wz = Hy (yq); setRhs puts the same SAT
  // coefficients on the data, and the source is -H (J) Q, so per column
  //   C T = SAT data - H (J) Q / wz.
  std::vector<double> c1(Nzl), m31(Nzl), C, col_prev_c, col_prev_m, col_prev_r, sol_prev;
  const DirTables& t = L.tz;
  H.Tamb.resize(N);
  for (int iy = 0; iy < Ny; ++iy) {
    std::vector<double> rhs(Nzl, 0.0);
    for (int iz = 0; iz < Nzl; ++iz) {
      const size_t a = (size_t)iy * Nzl + iz;
      c1[iz] = L.cz[a];
      m31[iz] = L.m3z[a];
    }
    for (int i = 0; i < 9 && i < Nzl; ++i) rhs[i] += (t.bs0[i] + (i == 0 ? t.alphaD : 0.0)) * c1[0] * gT;
    for (int i = std::max(0, Nzl - 9); i < Nzl; ++i)
      rhs[i] += (t.bsN[i - (Nzl - 9)] + (i == Nzl - 1 ? t.alphaD : 0.0)) * c1[Nzl - 1] * gB;
    if (H.radio) {
      for (int iz = 0; iz < Nzl; ++iz) {
        const size_t a = (size_t)iy * Nzl + iz;
        const double HJ = L.ty.Hd[iy] * t.Hd[iz] * (var ? L.yq[a] * L.zr[a] : 1.0);
        rhs[iz] -= HJ * H.Qrad[(size_t)iy * Nz + iz] / L.wz[a];
      }
    }
    std::vector<double> sol;
    if (iy > 0 && c1 == col_prev_c && m31 == col_prev_m && rhs == col_prev_r) {
      sol = sol_prev;
    } else {
      compose_line(t, SCY_BC_DIRICHLET, SCY_BC_DIRICHLET, c1, m31, C);
      std::vector<double> M((size_t)Nzl * Nzl, 0.0);
      for (int i = 0; i < Nzl; ++i)
        for (int o = -8; o <= 8; ++o) {
          const int j = i + o;
          if (j >= 0 && j < Nzl) M[(size_t)i * Nzl + j] = C[(size_t)i * 17 + o + 8];
        }
      sol = rhs;
      dense_solve(M, sol, Nzl);
      col_prev_c = c1;
      col_prev_m = m31;
      col_prev_r = rhs;
      sol_prev = sol;
    }
    for (int iz = 0; iz < Nzl; ++iz) H.Tamb[(size_t)iy * Nz + iz] = sol[iz];
  }
  // the mantle adiabat below the lithosphere (four TVals)
  if (Nzl < Nz && H.Lz_lab < g.Lz && TV.size() > 3) {
    const double a = (TV[TV.size() - 1] - TV[TV.size() - 2]) / (TD[TD.size() - 1] - TD[TD.size() - 2]);
    for (size_t i = 0; i < N; ++i)
      if (P.z[i] >= H.Lz_lab) H.Tamb[i] = a * (P.z[i] - TD[TD.size() - 2]) + TV[TV.size() - 2];
  }
  H.dT.assign(N, 0.0);
  H.T = H.Tamb;
}

}  // namespace

void load_heat_problem(const std::string& path, const QDProblem& P, HeatProblem& H) {
  const scy_grid_desc& g = P.desc.grid;
  const int Ny = g.Ny, Nz = g.Nz;
  const size_t N = (size_t)Ny * Nz;
  std::string heatType = "transient", fricH = "yes", viscH = "yes", radioH = "yes", coupling = "no";
  std::vector<double> kV, kD, rhoV, rhoD, cV, cD, wV, wD, A0V, A0D, TwV, TwD;
  double Lrad = NAN;
  H.Nz_lab = Nz;
  std::string stateLaw;
  for (const auto& e : parse_in_file(path)) {
    auto add = [&](std::vector<double>& v) {
      auto x = load_vector_double(e.full);
      v.insert(v.end(), x.begin(), x.end());
    };
    if (e.var == "thermalCoupling") coupling = e.rhs;
    else if (e.var == "heatEquationType") heatType = e.rhs;
    else if (e.var == "withFrictionalHeating") fricH = e.rhs;
    else if (e.var == "withViscShearHeating") viscH = e.rhs;
    else if (e.var == "withRadioHeatGeneration") radioH = e.rhs;
    else if (e.var == "kspTol_heateq") H.ksp_tol = c_atof(e.rhs);
    else if (e.var == "Nz_lab") H.Nz_lab = c_atoi(e.rhs);
    else if (e.var == "he_Lrad") Lrad = c_atof(e.rhs);
    else if (e.var == "kVals") add(kV);
    else if (e.var == "kDepths") add(kD);
    else if (e.var == "rhoVals") add(rhoV);
    else if (e.var == "rhoDepths") add(rhoD);
    else if (e.var == "cVals") add(cV);
    else if (e.var == "cDepths") add(cD);
    else if (e.var == "TVals") add(H.TVals);
    else if (e.var == "TDepths") add(H.TDepths);
    else if (e.var == "wVals") add(wV);
    else if (e.var == "wDepths") add(wD);
    else if (e.var == "he_A0Vals") add(A0V);
    else if (e.var == "he_A0Depths") add(A0D);
    else if (e.var == "TwVals") add(TwV);
    else if (e.var == "TwDepths") add(TwD);
    else if (e.var == "stateLaw") stateLaw = e.rhs;
    else if (e.var == "fw") H.fw = c_atof(e.rhs);
    else if (e.var == "Vw") H.Vw = c_atof(e.rhs);
    else if (e.var == "D") H.D = c_atof(e.rhs);
    else if (e.var == "tau_c") H.tau_c = c_atof(e.rhs);
  }
  H.coupling = coupling == "uncoupled" ? 1 : coupling == "coupled" ? 2 : 0;
  if (coupling != "no" && !H.coupling) throw std::runtime_error("thermalCoupling must be no, uncoupled or coupled");
  if (heatType != "transient" && heatType != "steadyState")
    throw std::runtime_error("heatEquationType must be transient or steadyState");
  H.steady = heatType == "steadyState";
  H.fric = fricH == "yes";
  H.visc = viscH == "yes";
  H.radio = radioH == "yes";
  auto pair = [](const std::vector<double>& a, const std::vector<double>& b, const char* n) {
    if (a.size() != b.size()) throw std::runtime_error(std::string(n) + ": values and depths differ in length");
  };
  pair(kV, kD, "kVals");
  pair(rhoV, rhoD, "rhoVals");
  pair(cV, cD, "cVals");
  pair(H.TVals, H.TDepths, "TVals");
  pair(wV, wD, "wVals");
  if (H.TVals.size() < 2 || H.TVals.size() > 4) throw std::runtime_error("TVals needs 2 to 4 entries");
  if (H.Nz_lab > Nz) throw std::runtime_error("Nz_lab must not exceed Nz");
  H.Lz_lab = H.TDepths[1];
  if (H.Lz_lab > g.Lz) throw std::runtime_error("the LAB depth TDepths[1] must not exceed Lz");
  if (H.radio) {
    pair(A0V, A0D, "he_A0Vals");
    if (A0V.empty()) {
      A0V = {0.0};
      A0D = {0.0};
    }
  }
  // setFields (:316-366)
  H.k = set_vec(P.z, kV, kD);
  H.rho = set_vec(P.z, rhoV, rhoD);
  H.c = set_vec(P.z, cV, cD);
  H.Tamb = set_vec(P.z, H.TVals, H.TDepths);
  H.T = H.Tamb;
  H.dT.assign(N, 0.0);
  H.Qrad.assign(N, 0.0);
  if (H.radio) {
    std::vector<double> A0 = set_vec(P.z, A0V, A0D);
    if (std::isnan(Lrad)) {
      for (double v : A0)
        if (v != 0.0) throw std::runtime_error("he_Lrad is needed with a nonzero he_A0Vals");
    } else {
      for (size_t i = 0; i < N; ++i) H.Qrad[i] = A0[i] * std::exp(-P.z[i] / Lrad);
    }
  }
  // loadFieldsFromFiles (:217-259)
  read_petsc_vec(P.inputDir + "rho", N, H.rho);
  read_petsc_vec(P.inputDir + "k", N, H.k);
  read_petsc_vec(P.inputDir + "h", N, H.Qrad);
  read_petsc_vec(P.inputDir + "c", N, H.c);
  std::vector<double> Tamb, T, dT;
  const bool have_tamb = read_petsc_vec(P.inputDir + "Tamb", N, Tamb);
  const bool have_t = read_petsc_vec(P.inputDir + "T", N, T);
  const bool have_dt = read_petsc_vec(P.inputDir + "dT", N, dT);
  if (have_tamb) {
    H.Tamb = Tamb;
    H.T = have_t ? T : Tamb;
    if (have_dt) {
      H.dT = dT;
    } else {
      H.dT.resize(N);
      for (size_t i = 0; i < N; ++i) H.dT[i] = H.T[i] - H.Tamb[i];
    }
  } else {
    if (have_t) H.T = T;
    if (have_dt) H.dT = dT;
    initial_geotherm(P, H);
  }
  // constructMapV (:460-523): shear-zone width w (m -> km) and the Gaussian
  H.w.assign(N, 0.0);
  H.Gw.assign(N, 0.0);
  H.wMax = 0.0;
  if (!wV.empty()) {
    H.w = set_vec(P.z, wV, wD);
    for (size_t i = 0; i < N; ++i) {
      H.w[i] *= 1e-3;
      const double y = P.y[i], ww = H.w[i];
      H.Gw[i] = std::exp(-y * y / (2.0 * ww * ww)) / std::sqrt(2.0 * M_PI) / ww;
      H.wMax = std::max(H.wMax, ww);
    }
  }
  // the fault's flash-heating fields (fault.cpp:89-97, :316-345)
  H.flash = stateLaw == "flashHeating";
  if (H.flash) {
    std::vector<double> zf(P.z.begin(), P.z.begin() + Nz);
    if (TwV.empty()) throw std::runtime_error("flashHeating needs TwVals / TwDepths");
    pair(TwV, TwD, "TwVals");
    H.Tw = set_vec(zf, TwV, TwD);
    H.rho_f = P.rho_f;
  }
}

}  // namespace scy
