// Device-side SbpOps context and the multigrid-preconditioned CG solver.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <type_traits>
#include <vector>

#include "sbp_dev.cuh"
#include "sbp_host.hpp"

namespace scy {

const char* last_error();
long long launch_count();
void profile_enable(int on);
int profile_collect(int level, int width, double* ms, long long* launches, double* bytes);

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) {
    o.p = nullptr;
    o.bytes = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      bytes = o.bytes;
      o.p = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DevBuf();
  int alloc(size_t b);
  void release();
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Partial sums for the deterministic grid reductions.
struct Reducer {
  DevBuf partials, counter;
  int init(int max_blocks);
};

template <typename T>
struct LevelStore {
  int Ny = 0, Nz = 0;
  DevBuf tab[2][10];  // per direction: D, R3, R4, Q, R3T, R4T, w3, w4, Hd, Hinvd
  DevBuf fld[10];     // cy, cz, m3y, m3z, wy, wz, mu, qy, rz, dinv
  DevBuf sep1[6];     // cy1, m3y1, wz1 (Ny), cz1, m3z1, wy1 (Nz) when separable
  DevBuf comp[2];     // composed interior stencils Cy (Ny x 9) and CzT (9 x Nz)
  DevBuf comp17[2];   // composed whole-operator stencils Cy17 (classes x Ny x 17), CzT17 (classes x 17 x Nz)
  DevBuf cls[2];      // line classes of the full form: ycls (Nz), zcls (Ny)
  DevBuf fullw[2];    // the full form's outer weights wy1 (Nz), wz1 (Ny) when the interior is not separable
  LevelDev<T> dev{};
  int init(const LevelHost& h, cudaStream_t s);
};

struct Transfer {
  Interp1D iy, iz;
  std::vector<int> ylo, yhi, zlo, zhi;  // fine index range feeding each coarse index
};

struct TransferDev {
  DevBuf jy, wy0, wy1, jz, wz0, wz1, ylo, yhi, zlo, zhi;
};

struct ChebCoef {
  double c1, c2;
};

template <typename T>
struct Multigrid {
  struct Work {
    DevBuf v[5];  // x ping, x pong, d, b, r
  };
  int nlev = 0, nu = 2, ncoarse = 0;
  std::vector<std::unique_ptr<LevelStore<T>>> lev;
  std::vector<Work> work;
  std::vector<TransferDev> tr;
  std::vector<std::vector<ChebCoef>> cheb;
  std::vector<double> lambda;
  DevBuf coarse_inv;
  int init(const std::vector<LevelHost>& hosts, const std::vector<Transfer>& xfer, cudaStream_t s);
  int setup_smoothers(const std::vector<LevelHost>& hosts, Reducer& red, double* dscal, cudaStream_t s);
  template <typename Tin>
  int vcycle(int l, const Tin* b_in, T** x_out, cudaStream_t s);
};

int build_hierarchy(const scy_grid_desc& g, const std::vector<double>& y, const std::vector<double>& z,
                    const std::vector<double>& mu, const int bc[4], std::vector<LevelHost>& hosts,
                    std::vector<Transfer>& xfer);

struct FDPrecond;

struct SbpContext {
  SbpContext();
  ~SbpContext();
  scy_grid_desc desc{};
  std::vector<double> y, z, mu;
  int bc[4] = {0, 1, 0, 1};  // R, T, L, B
  cudaStream_t stream = nullptr;
  std::vector<LevelHost> hosts;
  std::vector<Transfer> xfer;
  std::unique_ptr<LevelStore<double>> fine;
  std::unique_ptr<Multigrid<double>> mg64;
  std::unique_ptr<Multigrid<float>> mg32;
  std::shared_ptr<FDPrecond> fd;  // shared by the instances of a batch with one operator
  int separable = 0;  // metrics and mu separable: fast diagonalisation is exact up to the mu3 column
  Reducer red;
  DevBuf scal;
  DevBuf cg_r, cg_p[2], cg_q, cg_z, cg_z32;

  int create(const scy_grid_desc& g);
  int rebuild();
  int apply(int op, const double* in, double* out);
  int set_rhs(const double* bcL, const double* bcR, const double* bcT, const double* bcB, double* rhs);
  int solve(const double* rhs, double* u, const scy_solve_opts& o, scy_solve_stats& st);
  int solve_noalloc(const double* rhs, double* u, const scy_solve_opts& o, scy_solve_stats& st);
  int change_bc(int R, int T, int L, int B);
  // r = rhs - A u with A u summed in double-double arithmetic (error-free
  // products and sums over the 33-point cross form) and rounded once, so r
  // is the true residual to rounding even where ||A|| ||u|| >> ||rhs||;
  // *rnorm2 (device or host pointer, may be NULL) gets ||r||^2 through the
  // context's reducer.  For defect correction of ill-conditioned solves.
  int residual_dd(const double* rhs, const double* u, double* r, double* rnorm2_host);
  DevBuf cross;  // cross-form planes of the fine level (built on first use)
  template <typename T>
  int ensure_mg(std::unique_ptr<Multigrid<T>>& mg);
  int ensure_fd();
  template <typename Tz, class PC>
  int pcg(PC&& pc, const double* rhs, double* u, const scy_solve_opts& o, scy_solve_stats& st);
};

}  // namespace scy
