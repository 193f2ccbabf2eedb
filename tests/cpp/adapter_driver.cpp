// A compiled C++ caller of the library through include/scycle_b200.hpp (the
// reference's SbpOps interface and a whole driver), built and run by
// tests/test_cpp_caller_gpu.py.
//
//   adapter_driver sbp <Ny> <Nz> <out.bin>
//     SbpOps on an Ny x Nz constant grid (mu = 32.04 + 0.01 iy, so muxDy
//     differs from Dy): muxDy, Dz, A and H of x = sin(0.1 i) and the solve
//     of A u = setRhs(bcL = 1, bcR = 0.5, 0, 0); writes the five vectors.
//   adapter_driver qd <input.in> <steps> <out.bin>
//     the driver of the input file for that many accepted steps; writes
//     slip, slip velocity and state.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "scycle_b200.hpp"

namespace {

int fail(const char* what, int rc) {
  std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, scycle_b200::last_error().c_str());
  return 1;
}

void put(FILE* f, const std::vector<double>& v) { std::fwrite(v.data(), sizeof(double), v.size(), f); }

std::vector<double> down(const double* d, size_t n) {
  std::vector<double> h(n);
  cudaMemcpy(h.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost);
  return h;
}

int run_sbp(int Ny, int Nz, const char* out) {
  const size_t N = (size_t)Ny * Nz;
  std::vector<double> mu(N), x(N);
  for (int iy = 0; iy < Ny; ++iy)
    for (int iz = 0; iz < Nz; ++iz) mu[(size_t)iy * Nz + iz] = 32.04 + 0.01 * iy;
  for (size_t i = 0; i < N; ++i) x[i] = std::sin(0.1 * (double)i);
  // as LinearElastic sets it up (linearElastic.cpp:436-449)
  scycle_b200::SbpOps sbp(4, Ny, Nz, 30.0, 30.0, mu.data());
  int rc;
  if ((rc = sbp.setCompatibilityType("fullyCompatible"))) return fail("setCompatibilityType", rc);
  if ((rc = sbp.setBCTypes("Dirichlet", "Neumann", "Dirichlet", "Neumann"))) return fail("setBCTypes", rc);
  if ((rc = sbp.setMultiplyByH(1))) return fail("setMultiplyByH", rc);
  if ((rc = sbp.setLaplaceType("yz"))) return fail("setLaplaceType", rc);
  if ((rc = sbp.computeMatrices())) return fail("computeMatrices", rc);
  double *dx, *dy, *dz, *dA, *dH, *drhs, *du, *dbl, *dbr, *dbt, *dbb;
  cudaMalloc(&dx, N * 8);
  cudaMalloc(&dy, N * 8);
  cudaMalloc(&dz, N * 8);
  cudaMalloc(&dA, N * 8);
  cudaMalloc(&dH, N * 8);
  cudaMalloc(&drhs, N * 8);
  cudaMalloc(&du, N * 8);
  cudaMalloc(&dbl, Nz * 8);
  cudaMalloc(&dbr, Nz * 8);
  cudaMalloc(&dbt, Ny * 8);
  cudaMalloc(&dbb, Ny * 8);
  cudaMemcpy(dx, x.data(), N * 8, cudaMemcpyHostToDevice);
  std::vector<double> bl(Nz, 1.0), br(Nz, 0.5), bt(Ny, 0.0);
  cudaMemcpy(dbl, bl.data(), Nz * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(dbr, br.data(), Nz * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(dbt, bt.data(), Ny * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(dbb, bt.data(), Ny * 8, cudaMemcpyHostToDevice);
  cudaMemset(du, 0, N * 8);
  if ((rc = sbp.muxDy(dx, dy))) return fail("muxDy", rc);
  if ((rc = sbp.Dz(dx, dz))) return fail("Dz", rc);
  if ((rc = sbp.A(dx, dA))) return fail("A", rc);
  if ((rc = sbp.H(dx, dH))) return fail("H", rc);
  if ((rc = sbp.setRhs(drhs, dbl, dbr, dbt, dbb))) return fail("setRhs", rc);
  scy_solve_opts o{};
  o.rtol = 1e-13;
  o.max_its = 500;
  o.precision = SCY_PREC_FP64;
  o.check_every = 1;
  o.precond = SCY_PC_AUTO;
  o.verify = 1;
  scy_solve_stats st{};
  if ((rc = sbp.solve(drhs, du, o, &st))) return fail("solve", rc);
  if ((rc = sbp.synchronize())) return fail("synchronize", rc);
  FILE* f = std::fopen(out, "wb");
  if (!f) return 1;
  put(f, down(dy, N));
  put(f, down(dz, N));
  put(f, down(dA, N));
  put(f, down(dH, N));
  put(f, down(du, N));
  std::fclose(f);
  std::printf("sbp ok: %d CG iterations, |r| %.3e of |b| %.3e\n", st.iterations, st.rnorm, st.bnorm);
  for (double* p : {dx, dy, dz, dA, dH, drhs, du, dbl, dbr, dbt, dbb}) cudaFree(p);
  return 0;
}

int run_qd(const char* path, long steps, const char* out) {
  // the solver options of the whole-driver example in INTEGRATION.md: warm
  // starts from the previous stage's solution, the residual read back every
  // iteration
  scy_solve_opts o{};
  o.rtol = 1e-12;
  o.max_its = 300;
  o.precision = SCY_PREC_FP64;
  o.nonzero_guess = 1;
  o.check_every = 1;
  o.precond = SCY_PC_AUTO;
  o.verify = 0;
  scycle_b200::QD qd(path, o);
  int rc;
  if ((rc = qd.status())) return fail("QD", rc);
  if ((rc = qd.initiateIntegrand())) return fail("initiateIntegrand", rc);
  scy_ode_stats st{};
  if ((rc = qd.integrate(steps, &st))) return fail("integrate", rc);
  long n = 0;
  if ((rc = scy_qd_state_size(qd.handle(), &n))) return fail("scy_qd_state_size", rc);
  const long nz = n / 2;  // linear elastic: [psi | slip]
  std::vector<double> buf((size_t)nz);
  FILE* f = std::fopen(out, "wb");
  if (!f) return 1;
  for (int field : {SCY_FIELD_SLIP, SCY_FIELD_SLIPVEL, SCY_FIELD_PSI}) {
    if ((rc = qd.getField(field, buf.data()))) return fail("getField", rc);
    std::fwrite(buf.data(), sizeof(double), (size_t)nz, f);
  }
  std::fclose(f);
  std::printf("qd ok: %ld steps to t = %.9e s\n", st.step_count, st.t);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc == 5 && std::string(argv[1]) == "sbp") return run_sbp(std::atoi(argv[2]), std::atoi(argv[3]), argv[4]);
  if (argc == 5 && std::string(argv[1]) == "qd") return run_qd(argv[2], std::atol(argv[3]), argv[4]);
  std::fprintf(stderr, "usage: adapter_driver sbp <Ny> <Nz> <out> | qd <input.in> <steps> <out>\n");
  return 2;
}
