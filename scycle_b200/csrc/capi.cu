// extern "C" entry points of libscycle_b200 (declared in include/scycle_b200.h).
#include <new>
#include <stdexcept>
#include <vector>

#include "common.cuh"
#include "sbp_solver.hpp"

struct scy_sbp {
  scy::SbpContext ctx;
};

extern "C" {

const char* scy_get_last_error(void) { return scy::last_error(); }

const char* scy_version(void) { return "scycle_b200 0.1 (sm_100a)"; }

scy_status scy_sbp_create(const scy_grid_desc* desc, scy_sbp** out) {
  if (!desc || !out) {
    scy::set_error("scy_sbp_create: NULL argument");
    return SCY_ERR_ARG;
  }
  *out = nullptr;
  scy_sbp* s = new (std::nothrow) scy_sbp();
  if (!s) return SCY_ERR_NOMEM;
  int st = s->ctx.create(*desc);
  if (st != SCY_OK) {
    delete s;
    return st;
  }
  *out = s;
  return SCY_OK;
}

scy_status scy_sbp_destroy(scy_sbp* s) {
  delete s;
  return SCY_OK;
}

scy_status scy_sbp_set_stream(scy_sbp* s, void* stream) {
  if (!s) return SCY_ERR_ARG;
  s->ctx.stream = (cudaStream_t)stream;
  return SCY_OK;
}

scy_status scy_sbp_synchronize(scy_sbp* s) {
  if (!s) return SCY_ERR_ARG;
  SCY_CUDA_TRY(cudaStreamSynchronize(s->ctx.stream));
  return SCY_OK;
}

scy_status scy_sbp_change_bc_types(scy_sbp* s, int bcR, int bcT, int bcL, int bcB) {
  if (!s) return SCY_ERR_ARG;
  for (int b : {bcR, bcT, bcL, bcB})
    if (b != SCY_BC_DIRICHLET && b != SCY_BC_NEUMANN) {
      scy::set_error("boundary types must be SCY_BC_DIRICHLET or SCY_BC_NEUMANN");
      return SCY_ERR_ARG;
    }
  return s->ctx.change_bc(bcR, bcT, bcL, bcB);
}

scy_status scy_sbp_apply(scy_sbp* s, int op, const double* in, double* out) {
  if (!s || !in || !out) {
    scy::set_error("scy_sbp_apply: NULL argument");
    return SCY_ERR_ARG;
  }
  if (in == out) {
    scy::set_error("scy_sbp_apply: in and out must not alias");
    return SCY_ERR_ARG;
  }
  return s->ctx.apply(op, in, out);
}

scy_status scy_sbp_set_rhs(scy_sbp* s, const double* bcL, const double* bcR, const double* bcT, const double* bcB,
                           double* rhs) {
  if (!s || !bcL || !bcR || !bcT || !bcB || !rhs) {
    scy::set_error("scy_sbp_set_rhs: NULL argument");
    return SCY_ERR_ARG;
  }
  return s->ctx.set_rhs(bcL, bcR, bcT, bcB, rhs);
}

scy_status scy_sbp_solve(scy_sbp* s, const double* rhs, double* u, const scy_solve_opts* opts,
                         scy_solve_stats* stats) {
  if (!s || !rhs || !u || !opts) {
    scy::set_error("scy_sbp_solve: NULL argument");
    return SCY_ERR_ARG;
  }
  if (opts->max_its < 1 || !(opts->rtol >= 0.0) || !(opts->atol >= 0.0)) {
    scy::set_error("scy_sbp_solve: invalid options");
    return SCY_ERR_ARG;
  }
  scy_solve_stats tmp{};
  int st = s->ctx.solve(rhs, u, *opts, tmp);
  if (stats) *stats = tmp;
  return st;
}

scy_status scy_sbp_info(scy_sbp* s, int* Ny, int* Nz, int* n_levels) {
  if (!s) return SCY_ERR_ARG;
  if (Ny) *Ny = s->ctx.desc.Ny;
  if (Nz) *Nz = s->ctx.desc.Nz;
  if (n_levels) *n_levels = (int)s->ctx.hosts.size();
  return SCY_OK;
}

scy_status scy_grid_host_apply(const scy_grid_desc* g, const double* in, double* out) {
  if (!g || !in || !out || !g->mu) {
    scy::set_error("scy_grid_host_apply: NULL argument");
    return SCY_ERR_ARG;
  }
  try {
    const size_t N = (size_t)g->Ny * g->Nz;
    std::vector<double> y, z, mu(g->mu, g->mu + N);
    if (g->grid_type == SCY_GRID_VAR) {
      if (g->y) y.assign(g->y, g->y + N);
      if (g->z) z.assign(g->z, g->z + N);
    }
    int bc[4] = {g->bcR, g->bcT, g->bcL, g->bcB};
    scy::LevelHost L = scy::build_level(g->order, g->Ny, g->Nz, g->Ly, g->Lz, g->grid_type, g->compat, y, z, mu, bc);
    L.apply_A(in, out);
  } catch (const std::exception& e) {
    scy::set_error("scy_grid_host_apply: %s", e.what());
    return SCY_ERR_ARG;
  }
  return SCY_OK;
}

}  // extern "C"
