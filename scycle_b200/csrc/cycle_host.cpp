#include "cycle_host.hpp"

#include <algorithm>
#include <cmath>

namespace scy {

double cycle_time_step(const LevelHost& h, const std::vector<double>& cs, double deltaT_fd, double CFL) {
  const int Ny = h.Ny, Nz = h.Nz;
  const long N = (long)Ny * Nz;
  const bool var = h.grid_type == SCY_GRID_VAR;
  double gcfl = 0.7071;  // order 2
  if (h.order == 4) gcfl = 0.7071 / std::sqrt(1.4498);
  double min_ts_dy = INFINITY, min_ts_dz = INFINITY;
  for (long i = 0; i < N; ++i) {
    const double dy = var ? h.yq[i] * (1.0 / (Ny - 1)) : h.Ly / (Ny - 1.0);
    const double dz = var ? h.zr[i] * (1.0 / (Nz - 1)) : h.Lz / (Nz - 1.0);
    min_ts_dy = std::min(min_ts_dy, dy / cs[i]);
    min_ts_dz = std::min(min_ts_dz, dz / cs[i]);
  }
  const double max_deltaT = gcfl * std::min(std::fabs(min_ts_dy), std::fabs(min_ts_dz));
  const double cfl_deltaT = CFL * gcfl * max_deltaT;
  const double req = deltaT_fd;
  if (req <= 0. && cfl_deltaT <= 0.) return max_deltaT;
  if (req > 0. && cfl_deltaT <= 0.) return req;
  if (req <= 0. && cfl_deltaT > 0.) return cfl_deltaT;
  return req;
}

std::vector<double> penalty_ay(int Ny, int Nz, double h11y, double h11z, int outR, int outT, int outB, int quirk,
                               const std::vector<double>& cs) {
  const long N = (long)Ny * Nz;
  std::vector<double> ay(N, 0.0);
  if (quirk) {
    long Jj = 0;
    for (long Ii = 0; Ii < N; ++Ii) {
      ay[Jj] = 0;
      if (Ii / Nz == Ny - 1 && outR) ay[Jj] += 0.5 / h11y;
      if (Ii % Nz == 0 && outT) ay[Jj] += 0.5 / h11z;
      if ((Ii + 1) % Nz == 0 && outB) ay[Jj] += 0.5 / h11z;
      if (Ii / Nz == 0) Jj++;  // the left boundary is a fault (symmFault / rigidFault)
    }
  } else {
    for (long Ii = 0; Ii < N; ++Ii) {
      if (Ii / Nz == Ny - 1 && outR) ay[Ii] += 0.5 / h11y;
      if (Ii % Nz == 0 && outT) ay[Ii] += 0.5 / h11z;
      if ((Ii + 1) % Nz == 0 && outB) ay[Ii] += 0.5 / h11z;
    }
  }
  for (long i = 0; i < N; ++i) ay[i] *= cs[i];
  return ay;
}

}  // namespace scy
