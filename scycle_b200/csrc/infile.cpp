// Host reader of the reference's ``.in`` input files, its depth
// interpolation and its PETSc-binary vectors, and assembly of a
// linear-elastic quasi-dynamic problem from them.
#include "infile.hpp"
#include "thermal.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <sys/stat.h>

namespace scy {

namespace {
const std::string kDelim = " = ";

std::vector<std::string> split_spaces(const std::string& s) {
  std::vector<std::string> out;
  size_t start = 0;
  while (true) {
    size_t sp = s.find(' ', start);
    if (sp == std::string::npos) {
      out.push_back(s.substr(start));
      break;
    }
    out.push_back(s.substr(start, sp - start));
    start = sp + 1;
  }
  return out;
}

std::string bracket_content(const std::string& s) {
  if (s.empty()) return std::string();
  size_t close = s.find(']');
  size_t n = close == std::string::npos ? std::string::npos : close - 1;
  return s.substr(1, n);
}

bool file_exists(const std::string& p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

uint32_t be32(const unsigned char* p) {
  return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | (uint32_t)p[3];
}
}  // namespace

std::vector<InEntry> parse_in_text(const std::string& text) {
  std::vector<InEntry> out;
  std::istringstream in(text);
  std::string line;
  while (std::getline(in, line)) {
    InEntry e;
    size_t pos = line.find(kDelim);
    if (pos == std::string::npos) {
      // no delimiter: the whole line is the key; the reference's index
      // arithmetic then wraps and takes the value from character 2 on
      e.var = line;
      e.full = line.size() > 2 ? line.substr(2) : std::string();
    } else {
      e.var = line.substr(0, pos);
      e.full = line.size() > pos + kDelim.size() ? line.substr(pos + kDelim.size()) : std::string();
    }
    size_t sp = e.full.find(' ');
    e.rhs = e.full.substr(0, sp);
    out.push_back(e);
  }
  return out;
}

std::vector<InEntry> parse_in_file(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open input file " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return parse_in_text(ss.str());
}

double c_atof(const std::string& s) { return std::atof(s.c_str()); }
int c_atoi(const std::string& s) { return std::atoi(s.c_str()); }

// A list with no space in it yields nothing; otherwise every space-separated
// token counts, empty ones reading as 0 (genFuncs.cpp:413-440).
std::vector<double> load_vector_double(const std::string& s) {
  std::vector<double> out;
  std::string c = bracket_content(s);
  if (c.find(' ') == std::string::npos) return out;
  for (const auto& t : split_spaces(c)) out.push_back(c_atof(t));
  return out;
}

std::vector<std::string> load_vector_string(const std::string& s) { return split_spaces(bracket_content(s)); }

std::vector<double> set_vec(const std::vector<double>& coord, const std::vector<double>& vals,
                            const std::vector<double>& depths) {
  if (vals.empty()) throw std::runtime_error("depth profile without values");
  std::vector<double> out(coord.size(), vals[0]);
  if (coord.size() == 1) return out;
  const size_t m = depths.size();
  if (vals.size() < m) throw std::runtime_error("depth profile with fewer values than depths");
  for (size_t j = 0; j < coord.size(); ++j) {
    const double z = coord[j];
    for (size_t k = 0; k + 1 < m; ++k) {
      const double z0 = depths[k], z1 = depths[k + 1], v0 = vals[k], v1 = vals[k + 1];
      const bool inside = z >= z0 && z <= z1;
      const bool beyond = z > z1 && k == m - 2;
      if (inside || beyond) out[j] = (v1 - v0) / (z1 - z0) * (z - z0) + v0;
    }
  }
  return out;
}

bool read_petsc_vec(const std::string& path, size_t n, std::vector<double>& out) {
  if (!file_exists(path)) return false;
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open " + path);
  unsigned char hdr[8];
  if (!f.read((char*)hdr, 8)) throw std::runtime_error("truncated PETSc vector file " + path);
  if (be32(hdr) != 1211214u) throw std::runtime_error("not a PETSc Vec file: " + path);
  uint32_t len = be32(hdr + 4);
  if ((size_t)len != n)
    throw std::runtime_error(path + " holds " + std::to_string(len) + " values, expected " + std::to_string(n));
  std::vector<unsigned char> buf((size_t)len * 8);
  if (!f.read((char*)buf.data(), (std::streamsize)buf.size())) throw std::runtime_error("truncated PETSc Vec " + path);
  out.resize(len);
  for (size_t i = 0; i < len; ++i) {
    uint64_t v = 0;
    for (int b = 0; b < 8; ++b) v = (v << 8) | buf[i * 8 + b];
    double d;
    std::memcpy(&d, &v, 8);
    out[i] = d;
  }
  return true;
}

void write_petsc_vec(const std::string& path, const double* v, size_t n, int append) {
  std::ofstream f(path, std::ios::binary | (append ? std::ios::app : std::ios::trunc));
  if (!f) throw std::runtime_error("cannot write " + path);
  auto put32 = [&](uint32_t x) {
    unsigned char b[4] = {(unsigned char)(x >> 24), (unsigned char)(x >> 16), (unsigned char)(x >> 8), (unsigned char)x};
    f.write((const char*)b, 4);
  };
  put32(1211214u);
  put32((uint32_t)n);
  for (size_t i = 0; i < n; ++i) {
    uint64_t u;
    std::memcpy(&u, &v[i], 8);
    unsigned char b[8];
    for (int k = 0; k < 8; ++k) b[k] = (unsigned char)(u >> (56 - 8 * k));
    f.write((const char*)b, 8);
  }
}

static int parse_bc(const std::string& t) {
  if (t == "symmFault" || t == "rigidFault" || t == "remoteLoading") return SCY_BC_DIRICHLET;
  if (t == "freeSurface" || t == "outGoingCharacteristics") return SCY_BC_NEUMANN;
  throw std::runtime_error("unknown boundary condition type '" + t + "'");
}

// First number of a PETSc ASCII value file (loadValueFromCheckpoint,
// genFuncs.cpp:889-935); `fallback` when the file is absent.
static double read_ascii_value(const std::string& path, double fallback) {
  if (!file_exists(path)) return fallback;
  std::ifstream f(path);
  double v = fallback;
  if (!(f >> v)) throw std::runtime_error("cannot read a value from " + path);
  return v;
}

void load_qd_problem(const std::string& path, QDProblem& P, int cycle) {
  const std::vector<InEntry> E = parse_in_file(path);
  // ---- Domain (domain.cpp:8-16, :133-196, :233-262)
  int order = 4, Ny = -1, Nz = -1;
  double Ly = -1, Lz = -1, bCoordTrans = -1, vL_dom = 1e-9;
  std::string gridType = "variableGridSpacing", compat = "fullyCompatible", bulk = "linearElastic",
              momBal = "quasidynamic";
  P.inputDir = "unspecified_";
  P.outputDir = "data/";
  for (const auto& e : E) {
    if (e.var == "order") order = c_atoi(e.rhs);
    else if (e.var == "Ny" && Ny < 0) Ny = c_atoi(e.rhs);
    else if (e.var == "Nz" && Nz < 0) Nz = c_atoi(e.rhs);
    else if (e.var == "Ly") Ly = c_atof(e.rhs);
    else if (e.var == "Lz") Lz = c_atof(e.rhs);
    else if (e.var == "inputDir") P.inputDir = e.rhs;
    else if (e.var == "outputDir") P.outputDir = e.rhs;
    else if (e.var == "sbpCompatibilityType") compat = e.rhs;
    else if (e.var == "gridSpacingType") gridType = e.rhs;
    else if (e.var == "bulkDeformationType") bulk = e.rhs;
    else if (e.var == "momentumBalanceType") momBal = e.rhs;
    else if (e.var == "bCoordTrans") bCoordTrans = c_atof(e.rhs);
    else if (e.var == "vL") vL_dom = c_atof(e.rhs);
    else if (e.var == "enableCheckpointing") P.ckpt = c_atoi(e.rhs);
    else if (e.var == "interval") P.ckpt_interval = (long)c_atof(e.rhs);
    else if (e.var == "ckptContinueSteps") P.ckpt_continue = c_atoi(e.rhs);
  }
  if (P.ckpt < 0 || P.ckpt_interval < 0) throw std::runtime_error("invalid enableCheckpointing / interval");
  if (bCoordTrans > 0.0) gridType = "variableGridSpacing";
  P.pl = (!cycle && bulk == "powerLaw") ? 1 : 0;
  if (bulk != "linearElastic" && !P.pl)
    throw std::runtime_error("bulkDeformationType '" + bulk + "' is not on this path");
  if (!cycle && momBal != "quasidynamic")
    throw std::runtime_error("momentumBalanceType '" + momBal + "' is not the quasi-dynamic path");
  if (cycle && momBal != "quasidynamic_and_dynamic")
    throw std::runtime_error("momentumBalanceType '" + momBal + "' is not the quasi-dynamic / fully dynamic path");
  P.cycle = cycle;
  if (order != 2 && order != 4) throw std::runtime_error("order must be 2 or 4");
  if (Ny < 2 || Nz < 2) throw std::runtime_error("Ny and Nz must both exceed 1");
  if (!(Ly > 0) || !(Lz > 0)) throw std::runtime_error("Ly and Lz must be positive");
  if (gridType != "variableGridSpacing" && gridType != "constantGridSpacing")
    throw std::runtime_error("unknown gridSpacingType '" + gridType + "'");
  if (compat != "fullyCompatible" && compat != "compatible")
    throw std::runtime_error("unknown sbpCompatibilityType '" + compat + "'");
  const size_t N = (size_t)Ny * Nz;
  const double dq = 1.0 / (Ny - 1.0), dr = 1.0 / (Nz - 1.0);
  std::vector<double> q(N), r(N);
  for (size_t i = 0; i < N; ++i) {
    q[i] = dq * (double)(i / Nz);
    r[i] = dr * (double)(i - Nz * (i / Nz));
  }
  if (!read_petsc_vec(P.inputDir + "y", N, P.y)) {
    P.y.resize(N);
    for (size_t i = 0; i < N; ++i)
      P.y[i] = bCoordTrans <= 0 ? q[i] * Ly : Ly * std::sinh(bCoordTrans * q[i]) / std::sinh(bCoordTrans);
  }
  if (!read_petsc_vec(P.inputDir + "z", N, P.z)) {
    P.z.resize(N);
    for (size_t i = 0; i < N; ++i) P.z[i] = r[i] * Lz;
  }
  // ---- LinearElastic (linearElastic.cpp:99-148, :297-323): mu against y, rho against z
  std::vector<double> muVals, muDepths, rhoVals, rhoDepths;
  for (const auto& e : E) {
    if (e.var == "muVals") { auto v = load_vector_double(e.full); muVals.insert(muVals.end(), v.begin(), v.end()); }
    else if (e.var == "muDepths") { auto v = load_vector_double(e.full); muDepths.insert(muDepths.end(), v.begin(), v.end()); }
    else if (e.var == "rhoVals") { auto v = load_vector_double(e.full); rhoVals.insert(rhoVals.end(), v.begin(), v.end()); }
    else if (e.var == "rhoDepths") { auto v = load_vector_double(e.full); rhoDepths.insert(rhoDepths.end(), v.begin(), v.end()); }
  }
  if (muVals.empty() || muVals.size() != muDepths.size()) throw std::runtime_error("muVals/muDepths missing or of different lengths");
  if (rhoVals.empty() || rhoVals.size() != rhoDepths.size()) throw std::runtime_error("rhoVals/rhoDepths missing or of different lengths");
  if (P.pl) {
    // PowerLaw::setMaterialParameters interpolates mu and rho against z and
    // loadFieldsFromFiles reads inputDir/mu, rho (powerLaw.cpp:1016-1017, :1070-1071)
    P.mu = set_vec(P.z, muVals, muDepths);
    P.rho = set_vec(P.z, rhoVals, rhoDepths);
    read_petsc_vec(P.inputDir + "mu", N, P.mu);
    read_petsc_vec(P.inputDir + "rho", N, P.rho);
  } else {
    P.mu = set_vec(P.y, muVals, muDepths);
    P.rho = set_vec(P.z, rhoVals, rhoDepths);
    read_petsc_vec(P.inputDir + "momBal_mu", N, P.mu);
    read_petsc_vec(P.inputDir + "momBal_rho", N, P.rho);
  }
  P.cs.resize(N);
  for (size_t i = 0; i < N; ++i) P.cs[i] = std::sqrt(std::fabs(P.mu[i] / P.rho[i]));
  read_petsc_vec(P.inputDir + "momBal_cs", N, P.cs);
  // ---- Fault (fault.cpp:8-16, :35-109, :200-288)
  std::string stateLaw = "agingLaw";
  double f0 = 0.6, v0 = 1e-6, sN_cap = 1e14, sN_floor = 0.0, rootTol = 1e-12;
  std::vector<double> DcV, DcD, sNV, sND, aV, aD, bV, bD, lkV, lkD, stV, stD;
  for (const auto& e : E) {
    auto app = [&](std::vector<double>& dst) { auto v = load_vector_double(e.full); dst.insert(dst.end(), v.begin(), v.end()); };
    if (e.var == "DcVals") app(DcV);
    else if (e.var == "DcDepths") app(DcD);
    else if (e.var == "sNVals") app(sNV);
    else if (e.var == "sNDepths") app(sND);
    else if (e.var == "aVals") app(aV);
    else if (e.var == "aDepths") app(aD);
    else if (e.var == "bVals") app(bV);
    else if (e.var == "bDepths") app(bD);
    else if (e.var == "lockedVals") app(lkV);
    else if (e.var == "lockedDepths") app(lkD);
    else if (e.var == "stateVals") app(stV);
    else if (e.var == "stateDepths") app(stD);
    else if (e.var == "sN_cap") sN_cap = c_atof(e.rhs);
    else if (e.var == "sN_floor") sN_floor = c_atof(e.rhs);
    else if (e.var == "stateLaw") stateLaw = e.rhs;
    else if (e.var == "rootTol") rootTol = c_atof(e.rhs);
    else if (e.var == "f0") f0 = c_atof(e.rhs);
    else if (e.var == "v0") v0 = c_atof(e.rhs);
  }
  auto need = [](const std::vector<double>& v, const std::vector<double>& d, const char* nm) {
    if (v.empty() || v.size() != d.size()) throw std::runtime_error(std::string(nm) + " values/depths missing or of different lengths");
  };
  need(DcV, DcD, "Dc");
  need(aV, aD, "a");
  need(bV, bD, "b");
  need(sNV, sND, "sN");
  if (!(rootTol >= 1e-14)) throw std::runtime_error("rootTol must be >= 1e-14");
  std::vector<double> zf(P.z.begin(), P.z.begin() + Nz);
  P.a = set_vec(zf, aV, aD);
  P.b = set_vec(zf, bV, bD);
  P.sN = set_vec(zf, sNV, sND);
  P.Dc = set_vec(zf, DcV, DcD);
  P.locked = lkV.empty() ? std::vector<double>(Nz, 0.0) : set_vec(zf, lkV, lkD);
  P.rho_f = set_vec(zf, rhoVals, rhoDepths);
  P.mu_f = set_vec(zf, muVals, muDepths);
  P.stateVals_given = stV.empty() ? 0 : 1;
  P.psi = stV.empty() ? std::vector<double>(Nz, f0) : set_vec(zf, stV, stD);
  for (auto& s : P.sN) s = std::max(std::min(s, sN_cap), sN_floor);
  read_petsc_vec(P.inputDir + "sNEff", Nz, P.sN);
  read_petsc_vec(P.inputDir + "psi", Nz, P.psi);
  read_petsc_vec(P.inputDir + "a", Nz, P.a);
  read_petsc_vec(P.inputDir + "b", Nz, P.b);
  // per-node Dc is an extension: the reference does not load inputDir/Dc
  read_petsc_vec(P.inputDir + "Dc", Nz, P.Dc);
  P.prestress.assign(Nz, 0.0);
  read_petsc_vec(P.inputDir + "prestress", Nz, P.prestress);
  // ---- StrikeSlip_LinearElastic_qd (strikeSlip_linearElastic_qd.cpp:7-20, :126-256, :326-373)
  std::string timeIntegrator = "RK43", timeControlType = "PID", normType = "L2_absolute";
  std::string bcRType = "remoteLoading", bcTType = "freeSurface", bcLType = "symmFault", bcBType = "freeSurface";
  long maxStepCount = 100000000;
  // the cycle driver's constructor sets minDeltaT = 1e-3 where the
  // quasi-dynamic driver leaves -1 for computeMinTimeStep
  // (strikeSlip_linearElastic_qd_fd.cpp:25)
  double initTime = 0, maxTime = 1e15, minDeltaT = (cycle || P.pl) ? 1e-3 : -1, maxDeltaT = 1e10,
         initDeltaT = 1e-3, timeStepTol = 1e-8;
  // strikeSlip_linearElastic_qd_fd keys and defaults (:8-33, :135-230)
  double trig_qd2fd = 1e-3, trig_fd2qd = 1e-3, limit_qd = 10 * 1e-9, limit_fd = 1e-1, limit_stride_fd = -1;
  double deltaT_fd = -1, CFL = -1;
  int maxNumCycles = 1000;
  // extension key (not read by the reference): 0 puts the outgoing-
  // characteristics damping on the boundary nodes it names instead of the
  // reference's indexing of computePenaltyVectors
  int ay_quirk = 1;
  std::string fdR = "outGoingCharacteristics", fdT = "freeSurface", fdL = "symmFault", fdB = "outGoingCharacteristics";
  double vL = 1e-9;
  std::vector<std::string> timeIntInds;
  std::vector<double> scale;
  int guess = 0;
  std::string thermal = "no", hydraulic = "no", forcing = "no", driverLaw;
  for (const auto& e : E) {
    if (e.var == "thermalCoupling") thermal = e.rhs;
    else if (e.var == "hydraulicCoupling") hydraulic = e.rhs;
    else if (e.var == "stateLaw") driverLaw = e.rhs;
    else if (e.var == "guessSteadyStateICs") guess = c_atoi(e.rhs);
    else if (e.var == "forcingType") forcing = e.rhs;
    else if (e.var == "timeIntegrator") timeIntegrator = e.rhs;
    else if (e.var == "timeControlType") timeControlType = e.rhs;
    else if (e.var == "stride1D") P.stride1D = (int)c_atof(e.rhs);
    else if (e.var == "stride2D") P.stride2D = (int)c_atof(e.rhs);
    else if (e.var == "maxStepCount") maxStepCount = (long)c_atof(e.rhs);
    else if (e.var == "initTime") initTime = c_atof(e.rhs);
    else if (e.var == "maxTime") maxTime = c_atof(e.rhs);
    else if (e.var == "minDeltaT") minDeltaT = c_atof(e.rhs);
    else if (e.var == "maxDeltaT") maxDeltaT = c_atof(e.rhs);
    else if (e.var == "initDeltaT") initDeltaT = c_atof(e.rhs);
    else if (e.var == "timeStepTol") timeStepTol = c_atof(e.rhs);
    else if (e.var == "timeIntInds") { auto v = load_vector_string(e.full); timeIntInds.insert(timeIntInds.end(), v.begin(), v.end()); }
    else if (e.var == "scale") { auto v = load_vector_double(e.full); scale.insert(scale.end(), v.begin(), v.end()); }
    else if (e.var == "normType") normType = e.rhs;
    else if (e.var == "vL") vL = c_atof(e.rhs);
    else if (e.var == "kspTol") P.ksp_tol = c_atof(e.rhs);
    else if (e.var == "momBal_bcR_qd") bcRType = e.rhs;
    else if (e.var == "momBal_bcT_qd") bcTType = e.rhs;
    else if (e.var == "momBal_bcL_qd") bcLType = e.rhs;
    else if (e.var == "momBal_bcB_qd") bcBType = e.rhs;
    else if (cycle && e.var == "trigger_qd2fd") trig_qd2fd = c_atof(e.rhs);
    else if (cycle && e.var == "trigger_fd2qd") trig_fd2qd = c_atof(e.rhs);
    else if (cycle && e.var == "limit_qd") limit_qd = c_atof(e.rhs);
    else if (cycle && e.var == "limit_fd") limit_fd = c_atof(e.rhs);
    else if (cycle && e.var == "limit_stride_fd") limit_stride_fd = c_atof(e.rhs);
    else if (cycle && e.var == "deltaT_fd") deltaT_fd = c_atof(e.rhs);
    else if (cycle && e.var == "CFL") CFL = c_atof(e.rhs);
    else if (cycle && e.var == "maxNumCycles") maxNumCycles = c_atoi(e.rhs);
    else if (cycle && e.var == "momBal_bcR_fd") fdR = e.rhs;
    else if (cycle && e.var == "momBal_bcT_fd") fdT = e.rhs;
    else if (cycle && e.var == "momBal_bcL_fd") fdL = e.rhs;
    else if (cycle && e.var == "momBal_bcB_fd") fdB = e.rhs;
    else if (cycle && e.var == "fd_ayIndexQuirk") ay_quirk = c_atoi(e.rhs);
  }
  if (hydraulic != "no") throw std::runtime_error("hydraulic coupling is outside this path");
  if (thermal != "no" && thermal != "uncoupled" && thermal != "coupled")
    throw std::runtime_error("thermalCoupling must be no, uncoupled or coupled");
  if (thermal != "no" && (cycle || P.pl))
    throw std::runtime_error("thermal coupling is built for the linear-elastic quasi-dynamic driver");
  if (forcing != "no") throw std::runtime_error("forcingType '" + forcing + "' is outside this path");
  if (stateLaw != "agingLaw" && stateLaw != "slipLaw" && stateLaw != "constantState" && stateLaw != "flashHeating")
    throw std::runtime_error("stateLaw '" + stateLaw + "' is outside this path");
  if (stateLaw == "flashHeating" && thermal == "no")
    throw std::runtime_error("stateLaw flashHeating reads the heat equation's temperature: set thermalCoupling");
  if (guess != 0 && guess != 1) throw std::runtime_error("guessSteadyStateICs must be 0 or 1");
  // RK32_WBE / RK43_WBE (odeSolverImex.cpp): the RK32 / RK43 stages with a
  // strict acceptance test, then one implicit heat step per accepted step
  P.imex = (timeIntegrator == "RK32_WBE" || timeIntegrator == "RK43_WBE") ? 1 : 0;
  if (P.imex) timeIntegrator = timeIntegrator.substr(0, 4);
  if (P.imex && thermal == "no") throw std::runtime_error("RK32_WBE / RK43_WBE integrate the heat equation: set thermalCoupling");
  if (thermal != "no" && !P.imex) throw std::runtime_error("thermalCoupling needs timeIntegrator RK32_WBE or RK43_WBE");
  if (timeIntegrator != "RK32" && timeIntegrator != "RK43")
    throw std::runtime_error("timeIntegrator '" + timeIntegrator + "' is outside this path (RK32, RK43, RK32_WBE, RK43_WBE)");
  if (timeControlType != "P" && timeControlType != "PID") throw std::runtime_error("timeControlType must be P or PID");
  if (normType != "L2_absolute" && normType != "L2_relative") throw std::runtime_error("normType must be L2_absolute or L2_relative");
  // checkInput runs before computeMinTimeStep (strikeSlip_linearElastic_qd.cpp:218-220)
  if (initDeltaT < minDeltaT || initDeltaT < 1e-14) initDeltaT = minDeltaT;
  if (!(initTime >= 0) || !(maxTime >= initTime)) throw std::runtime_error("invalid initTime / maxTime");
  if (!(timeStepTol >= 1e-14)) throw std::runtime_error("timeStepTol must be >= 1e-14");
  if (!(maxDeltaT >= 1e-14) || !(maxDeltaT >= minDeltaT)) throw std::runtime_error("invalid maxDeltaT");
  if (!(initDeltaT > 0) || initDeltaT > maxDeltaT) throw std::runtime_error("invalid initDeltaT");
  P.guess_ss = guess;
  P.stateLaw = stateLaw;
  P.integrator = timeIntegrator;
  P.vL = vL;
  P.min_dt_user = minDeltaT;
  const double fts = bcLType == "rigidFault" ? 1.0 : 2.0;
  P.eta.resize(Nz);
  for (int i = 0; i < Nz; ++i) P.eta[i] = std::sqrt(std::fabs(P.mu_f[i] * P.rho_f[i])) * (1.0 / fts);
  P.bcL0.assign(Nz, 0.0);
  P.bcRShift.assign(Nz, 0.0);
  read_petsc_vec(P.inputDir + "momBal_bcL", Nz, P.bcL0);
  read_petsc_vec(P.inputDir + "momBal_bcR", Nz, P.bcRShift);
  // a restart: the driver's, the material's and the fault's checkpoint files
  // (StrikeSlip_LinearElastic_qd ctor :33-39, LinearElastic::loadCheckpoint
  // :396-410, Fault::loadCheckpoint fault.cpp:144-166); the rate-and-state
  // parameters come from this file as for the first run
  if (P.ckpt > 0 && !cycle && !P.pl) {
    P.ckpt_number = (int)read_ascii_value(P.outputDir + "ckptNumber", 0.0);
    if (P.ckpt_number > 0) {
      initTime = read_ascii_value(P.outputDir + "chkpt_currT", initTime);
      initDeltaT = read_ascii_value(P.outputDir + "chkpt_deltaT", initDeltaT);
      P.step0 = (long)read_ascii_value(P.outputDir + "chkpt_stepCount", 0.0);
      P.errA[1] = read_ascii_value(P.outputDir + "chkpt_prevErr", 0.0);
      P.errA[0] = read_ascii_value(P.outputDir + "chkpt_currErr", 0.0);
      P.guess_ss = 0;
      const std::string c = P.outputDir + "chkpt_";
      read_petsc_vec(c + "psi", Nz, P.psi);
      if (!read_petsc_vec(c + "slip", Nz, P.slip_file)) throw std::runtime_error("checkpoint without chkpt_slip");
      if (!read_petsc_vec(c + "slipVel", Nz, P.slipVel0)) P.slipVel0.clear();
      read_petsc_vec(c + "sNEff", Nz, P.sN);
      read_petsc_vec(c + "prestress", Nz, P.prestress);
      read_petsc_vec(c + "momBal_bcRShift", Nz, P.bcRShift);
      read_petsc_vec(c + "momBal_bcL", Nz, P.bcL0);
    }
  }
  // descriptor
  scy_qd_desc& d = P.desc;
  d.grid.order = order;
  d.grid.Ny = Ny;
  d.grid.Nz = Nz;
  d.grid.Ly = Ly;
  d.grid.Lz = Lz;
  d.grid.grid_type = gridType == "constantGridSpacing" ? SCY_GRID_CONST : SCY_GRID_VAR;
  d.grid.compat = compat == "fullyCompatible" ? SCY_COMPAT_FULLY : SCY_COMPAT_COMPATIBLE;
  d.grid.y = P.y.data();
  d.grid.z = P.z.data();
  d.grid.mu = P.mu.data();
  d.grid.bcR = parse_bc(bcRType);
  d.grid.bcT = parse_bc(bcTType);
  d.grid.bcL = parse_bc(bcLType);
  d.grid.bcB = parse_bc(bcBType);
  if (bcLType != "symmFault" && bcLType != "rigidFault") throw std::runtime_error("momBal_bcL_qd must be symmFault or rigidFault");
  d.fault.Nz = Nz;
  d.fault.a = P.a.data();
  d.fault.b = P.b.data();
  d.fault.sN = P.sN.data();
  d.fault.Dc = P.Dc.data();
  d.fault.eta = P.eta.data();
  d.fault.locked = P.locked.data();
  d.fault.prestress = P.prestress.data();
  d.fault.f0 = f0;
  d.fault.v0 = v0;
  d.fault.vL = vL_dom;
  d.fault.root_tol = rootTol;
  d.fault.max_its = 10000;
  d.fault.state_law = stateLaw == "agingLaw" ? SCY_LAW_AGING : stateLaw == "slipLaw" ? SCY_LAW_SLIP
                      : stateLaw == "flashHeating" ? SCY_LAW_FLASH : SCY_LAW_CONSTANT;
  // the heat equation (thermalCoupling uncoupled / coupled)
  if (thermal != "no") {
    P.heat = std::make_shared<HeatProblem>();
    load_heat_problem(path, P, *P.heat);
  }
  d.fault.exact_jacobian = 1;
  d.fault_type_scale = fts;
  d.bcL_from_slip = 1;
  d.bcR_remote = bcRType == "remoteLoading" ? 1 : 0;
  d.vL = vL;
  d.bcL0 = P.bcL0.data();
  d.bcRShift = P.bcRShift.data();
  scy_ode_opts& o = P.ode;
  o.method = timeIntegrator == "RK32" ? SCY_RK32 : SCY_RK43;
  o.control = timeControlType == "P" ? SCY_CTRL_P : SCY_CTRL_PID;
  o.norm = normType == "L2_absolute" ? SCY_NORM_L2_ABS : SCY_NORM_L2_REL;
  o.tol = timeStepTol;
  o.min_dt = minDeltaT;
  o.max_dt = maxDeltaT;
  o.init_dt = initDeltaT;
  o.t0 = initTime;
  P.init_time = initTime;
  o.t1 = maxTime;
  o.max_steps = maxStepCount;
  if (timeIntInds.size() > (P.pl ? 4u : 2u)) throw std::runtime_error("timeIntInds names more fields than are integrated");
  o.n_err = (int)timeIntInds.size();
  for (size_t i = 0; i < timeIntInds.size(); ++i) {
    if (timeIntInds[i] == "psi") o.err_keys[i] = SCY_KEY_PSI;
    else if (timeIntInds[i] == "slip") o.err_keys[i] = SCY_KEY_SLIP;
    else if (P.pl && timeIntInds[i] == "gVxy") o.err_keys[i] = SCY_KEY_GVXY;
    else if (P.pl && timeIntInds[i] == "gVxz") o.err_keys[i] = SCY_KEY_GVXZ;
    else throw std::runtime_error("timeIntInds entry '" + timeIntInds[i] + "' is not an integrated field");
    o.err_scale[i] = scale.empty() ? 1.0 : (i < scale.size() ? scale[i] : 1.0);
  }
  if (!scale.empty() && scale.size() != timeIntInds.size()) throw std::runtime_error("scale and timeIntInds differ in length");
  if (P.pl) {
    // ---- PowerLaw + DislocationCreep settings (powerLaw.cpp:260-305, :851-915)
    std::string wDisl = "yes", wDiff = "no", wPlast = "no", wLM = "no";
    double cap = 1e30;
    std::vector<double> AV, AD, BV, BD, nV, nD, TV, TD;
    for (const auto& e : E) {
      auto app = [&](std::vector<double>& dst) { auto v = load_vector_double(e.full); dst.insert(dst.end(), v.begin(), v.end()); };
      if (e.var == "wDislCreep") wDisl = e.rhs;
      else if (e.var == "wDiffCreep") wDiff = e.rhs;
      else if (e.var == "wPlasticity") wPlast = e.rhs;
      else if (e.var == "wLinearMaxwell") wLM = e.rhs;
      else if (e.var == "maxEffVisc") cap = c_atof(e.rhs);
      else if (e.var == "disl_AVals") app(AV);
      else if (e.var == "disl_ADepths") app(AD);
      else if (e.var == "disl_BVals") app(BV);
      else if (e.var == "disl_BDepths") app(BD);
      else if (e.var == "disl_nVals") app(nV);
      else if (e.var == "disl_nDepths") app(nD);
      else if (e.var == "TVals") app(TV);
      else if (e.var == "TDepths") app(TD);
    }
    if (wDisl != "yes" || wDiff != "no" || wPlast != "no" || wLM != "no")
      throw std::runtime_error("the power-law path covers dislocation creep only (wDislCreep = yes, the others no)");
    // the steady-state iteration's settings (strikeSlip_powerLaw_qd.cpp:27-29,
    // :157-163) and optional input fields (powerLaw.cpp:2021, strikeSlip_powerLaw_qd.cpp:898)
    for (const auto& e : E) {
      if (e.var == "fss_EffVisc") P.ss_fss = c_atof(e.rhs);
      else if (e.var == "gss_t") P.ss_gss_t = c_atof(e.rhs);
      else if (e.var == "atolSS_effVisc") P.ss_atol = c_atof(e.rhs);
      else if (e.var == "maxSSIts_effVisc") P.ss_max_its = c_atoi(e.rhs);
    }
    if (guess) {
      if (!read_petsc_vec(P.inputDir + "effVisc", N, P.ss_effvisc)) P.ss_effvisc.clear();
      if (!read_petsc_vec(P.inputDir + "tauSS", Nz, P.ss_tau)) P.ss_tau.clear();
    }
    if (AV.size() < 2 || BV.size() < 2 || nV.size() < 2 || AV.size() != AD.size() || BV.size() != BD.size() ||
        nV.size() != nD.size())
      throw std::runtime_error("disl_A/B/n values and depths need at least two matching entries");
    if (TV.empty() || TV.size() != TD.size()) throw std::runtime_error("TVals/TDepths missing or of different lengths");
    P.plA = set_vec(P.z, AV, AD);
    P.plB = set_vec(P.z, BV, BD);
    P.pln = set_vec(P.z, nV, nD);
    P.plT = set_vec(P.z, TV, TD);
    read_petsc_vec(P.inputDir + "T", N, P.plT);
    P.gVxy0.assign(N, 0.0);
    P.gVxz0.assign(N, 0.0);
    read_petsc_vec(P.inputDir + "GVxy", N, P.gVxy0);
    read_petsc_vec(P.inputDir + "GVxz", N, P.gVxz0);
    if (!read_petsc_vec(P.inputDir + "slip", Nz, P.slip_file)) P.slip_file.clear();
    P.pdesc.A = P.plA.data();
    P.pdesc.B = P.plB.data();
    P.pdesc.n = P.pln.data();
    P.pdesc.T = P.plT.data();
    P.pdesc.visc_cap = cap;
    return;
  }
  if (!cycle) return;
  // ---- strikeSlip_linearElastic_qd_fd::checkInput (:232-305)
  auto fd_side = [](const std::string& t, const char* key) {
    if (t == "outGoingCharacteristics") return (int)SCY_FD_OUTGOING;
    if (t == "freeSurface") return (int)SCY_FD_FREE_SURFACE;
    throw std::runtime_error(std::string(key) + " must be freeSurface or outGoingCharacteristics");
  };
  if (fdL != "symmFault" && fdL != "rigidFault") throw std::runtime_error("momBal_bcL_fd must be symmFault or rigidFault");
  if (stateLaw != "agingLaw" && stateLaw != "slipLaw")
    throw std::runtime_error("the fully dynamic phase needs stateLaw agingLaw or slipLaw");
  if (limit_fd < trig_qd2fd) limit_fd = 10 * trig_qd2fd;
  if (limit_qd > trig_fd2qd) limit_qd = trig_qd2fd / 10.0;
  if (limit_stride_fd == -1) limit_stride_fd = limit_fd / 10.0;
  scy_cycle_desc& c = P.cdesc;
  c.rho = P.rho.data();
  c.cs = P.cs.data();
  c.rho_fault = P.rho_f.data();
  c.fd_bcR = fd_side(fdR, "momBal_bcR_fd");
  c.fd_bcT = fd_side(fdT, "momBal_bcT_fd");
  c.fd_bcB = fd_side(fdB, "momBal_bcB_fd");
  c.deltaT_fd = deltaT_fd;
  c.CFL = CFL;
  c.trigger_qd2fd = trig_qd2fd;
  c.trigger_fd2qd = trig_fd2qd;
  c.limit_qd = limit_qd;
  c.limit_fd = limit_fd;
  c.max_num_cycles = maxNumCycles;
  c.ay_index_quirk = ay_quirk ? 1 : 0;
  // initiateIntegrands reads inputDir/slip when present (:678)
  if (!read_petsc_vec(P.inputDir + "slip", Nz, P.slip_file)) P.slip_file.clear();
}

}  // namespace scy
