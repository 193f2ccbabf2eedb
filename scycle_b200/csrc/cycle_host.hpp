// Host-side set-up of the fully dynamic phase: the CFL step and the
// outgoing-characteristics penalty vector (strikeSlip_linearElastic_qd_fd.cpp
// computeTimeStep :356-442, computePenaltyVectors :446-505).
#pragma once
#include <vector>

#include "../../include/scycle_b200.h"
#include "sbp_host.hpp"

namespace scy {

// computeTimeStep: gcfl * min over nodes of (dy/cs, dz/cs), then the
// user's deltaT_fd / CFL choice (a CFL request scales by gcfl once more).
double cycle_time_step(const LevelHost& h, const std::vector<double>& cs, double deltaT_fd, double CFL);

// computePenaltyVectors' ay (times cs).  quirk = 1 reproduces the
// reference's indexing: its output index advances only while the fault-side
// test holds (iy = 0), so rows iy >= 1 all land on entry Nz.
std::vector<double> penalty_ay(int Ny, int Nz, double h11y, double h11z, int outR, int outT, int outB, int quirk,
                               const std::vector<double>& cs);

}  // namespace scy
