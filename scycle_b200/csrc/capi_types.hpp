// The opaque handle types of the C ABI (include/scycle_b200.h).
#pragma once
#include <memory>

#include "cycle.hpp"
#include "infile.hpp"
#include "qd.hpp"
#include "sbp_solver.hpp"

struct scy_sbp {
  scy::SbpContext ctx;
};

struct scy_qd {
  scy::QDContext ctx;
  std::unique_ptr<scy::QDProblem> prob;  // set by scy_qd_create_from_in
};

struct scy_cycle {
  scy::CycleContext ctx;
  std::unique_ptr<scy::QDProblem> prob;  // set by scy_cycle_create_from_in
};
