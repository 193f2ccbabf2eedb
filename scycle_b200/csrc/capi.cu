// extern "C" entry points of libscycle_b200 (declared in include/scycle_b200.h).
#include <new>
#include <stdexcept>
#include <vector>

#include <memory>

#include "common.cuh"
#include "cycle.hpp"
#include "cycle_host.hpp"
#include "infile.hpp"
#include "thermal.hpp"
#include "thermal_dev.hpp"
#include "qd.hpp"
#include "sbp_solver.hpp"

#include "capi_types.hpp"

namespace {
void default_solve(scy_solve_opts& o) {
  o.rtol = 1e-12;
  o.atol = 0.0;
  o.max_its = 300;
  o.precision = SCY_PREC_FP64;
  o.nonzero_guess = 1;
  o.check_every = 1;
}
}  // namespace

extern "C" {

const char* scy_get_last_error(void) { return scy::last_error(); }

const char* scy_version(void) { return "scycle_b200 0.1 (sm_100a)"; }

long long scy_launch_count(void) { return scy::launch_count(); }

scy_status scy_profile_enable(int on) {
  scy::profile_enable(on);
  return SCY_OK;
}

scy_status scy_profile_collect(int level, int width, double* ms, long long* launches, double* bytes) {
  if (!ms || !launches || !bytes) return SCY_ERR_ARG;
  return scy::profile_collect(level, width, ms, launches, bytes);
}

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

scy_status scy_sbp_solve_noalloc(scy_sbp* s, const double* rhs, double* u, const scy_solve_opts* opts,
                                 scy_solve_stats* stats) {
  if (!s || !rhs || !u || !opts) {
    scy::set_error("scy_sbp_solve_noalloc: NULL argument");
    return SCY_ERR_ARG;
  }
  if (opts->max_its < 1 || !(opts->rtol >= 0.0) || !(opts->atol >= 0.0)) {
    scy::set_error("scy_sbp_solve_noalloc: invalid options");
    return SCY_ERR_ARG;
  }
  scy_solve_stats tmp{};
  int st = s->ctx.solve_noalloc(rhs, u, *opts, tmp);
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

scy_status scy_grid_host_apply_cross(const scy_grid_desc* g, const double* in, double* out) {
  if (!g || !in || !out || !g->mu) {
    scy::set_error("scy_grid_host_apply_cross: NULL argument");
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
    std::vector<double> C;
    scy::build_cross_planes(L, C);
    scy::apply_cross_planes(C, g->Ny, g->Nz, in, out);
  } catch (const std::exception& e) {
    scy::set_error("scy_grid_host_apply_cross: %s", e.what());
    return SCY_ERR_ARG;
  }
  return SCY_OK;
}

scy_status scy_grid_host_apply_full(const scy_grid_desc* g, const double* in, double* out) {
  if (!g || !in || !out || !g->mu) {
    scy::set_error("scy_grid_host_apply_full: NULL argument");
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
    scy::FullForm F;
    if (!scy::build_full_form(L, F)) {
      scy::set_error("scy_grid_host_apply_full: the operator has no full form (order 2, fewer than 17 points in a "
                     "direction, non-separable weights or more than %d exceptional lines)",
                     scy::kMaxLineClasses);
      return SCY_ERR_ARG;
    }
    scy::apply_full_form(F, g->Ny, g->Nz, in, out);
  } catch (const std::exception& e) {
    scy::set_error("scy_grid_host_apply_full: %s", e.what());
    return SCY_ERR_ARG;
  }
  return SCY_OK;
}

scy_status scy_qd_create(const scy_qd_desc* d, scy_qd** out) {
  if (!d || !out) {
    scy::set_error("scy_qd_create: NULL argument");
    return SCY_ERR_ARG;
  }
  *out = nullptr;
  scy_qd* q = new (std::nothrow) scy_qd();
  if (!q) return SCY_ERR_NOMEM;
  int st = q->ctx.create(*d);
  if (st != SCY_OK) {
    delete q;
    return st;
  }
  *out = q;
  return SCY_OK;
}

scy_status scy_pl_create(const scy_qd_desc* d, const scy_pl_desc* pl, scy_qd** out) {
  if (!d || !pl || !out) {
    scy::set_error("scy_pl_create: NULL argument");
    return SCY_ERR_ARG;
  }
  *out = nullptr;
  scy_qd* q = new (std::nothrow) scy_qd();
  if (!q) return SCY_ERR_NOMEM;
  int st = q->ctx.create(*d, pl);
  if (st != SCY_OK) {
    delete q;
    return st;
  }
  *out = q;
  return SCY_OK;
}

scy_status scy_qd_state_size(scy_qd* q, long* n) {
  if (!q || !n) return SCY_ERR_ARG;
  *n = q->ctx.nvar;
  return SCY_OK;
}

scy_status scy_qd_destroy(scy_qd* q) {
  delete q;
  return SCY_OK;
}

scy_status scy_qd_set_stream(scy_qd* q, void* stream) {
  if (!q) return SCY_ERR_ARG;
  q->ctx.sbp.stream = (cudaStream_t)stream;
  return SCY_OK;
}

scy_status scy_qd_d_dt(scy_qd* q, double t, const double* var, double* dvar) {
  if (!q || !var || !dvar) {
    scy::set_error("scy_qd_d_dt: NULL argument");
    return SCY_ERR_ARG;
  }
  SCY_TRY(q->ctx.d_dt(t, var, dvar));
  return q->ctx.read_flags();
}

scy_status scy_qd_fault_d_dt(scy_qd* q, const double* var, const double* tau_body, double* dvar) {
  if (!q || !var || !tau_body || !dvar) {
    scy::set_error("scy_qd_fault_d_dt: NULL argument");
    return SCY_ERR_ARG;
  }
  SCY_TRY(q->ctx.fault_d_dt(var, tau_body, dvar));
  return q->ctx.read_flags();
}

scy_status scy_qd_integrate_begin(scy_qd* q, const scy_ode_opts* o, const double* var0) {
  if (!q || !o || !var0) {
    scy::set_error("scy_qd_integrate_begin: NULL argument");
    return SCY_ERR_ARG;
  }
  if (!(o->tol > 0) || !(o->max_dt >= o->min_dt) || !(o->t1 >= o->t0) || o->max_steps < 0 || o->n_err > 4) {
    scy::set_error("scy_qd_integrate_begin: invalid options");
    return SCY_ERR_ARG;
  }
  scy::QDContext& c = q->ctx;
  SCY_CUDA_TRY(cudaMemcpyAsync(c.rk[0].p, var0, (size_t)c.nvar * sizeof(double), cudaMemcpyHostToDevice,
                               c.sbp.stream));
  return c.integrate_begin(*o);
}

scy_status scy_qd_integrate_steps(scy_qd* q, long nsteps, scy_ode_stats* st) {
  if (!q || nsteps < 0) {
    scy::set_error("scy_qd_integrate_steps: invalid argument");
    return SCY_ERR_ARG;
  }
  return q->ctx.integrate_steps(nsteps, st);
}

scy_status scy_qd_force_attempts(scy_qd* q, const double* dts, const int* acc, long n) {
  if (!q || n < 0 || (n > 0 && (!dts || !acc))) return SCY_ERR_ARG;
  q->ctx.forced_dt.assign(dts, dts + n);
  q->ctx.forced_acc.assign(acc, acc + n);
  q->ctx.forced_pos = 0;
  return SCY_OK;
}

scy_status scy_qd_record_attempts(scy_qd* q, int on) {
  if (!q) return SCY_ERR_ARG;
  q->ctx.record = on ? 1 : 0;
  if (on) {
    q->ctx.log_dt.clear();
    q->ctx.log_acc.clear();
    q->ctx.log_step_dt.clear();
  }
  return SCY_OK;
}

scy_status scy_qd_get_attempts(scy_qd* q, double* dts, int* acc, long cap, long* n) {
  if (!q || !n) return SCY_ERR_ARG;
  long m = (long)q->ctx.log_dt.size();
  *n = m;
  for (long i = 0; i < m && i < cap; ++i) {
    if (dts) dts[i] = q->ctx.log_dt[i];
    if (acc) acc[i] = q->ctx.log_acc[i];
  }
  return SCY_OK;
}

scy_status scy_qd_get_step_sizes(scy_qd* q, double* dts, long cap, long* n) {
  if (!q || !n) return SCY_ERR_ARG;
  const long m = (long)q->ctx.log_step_dt.size();
  *n = m;
  for (long i = 0; i < m && i < cap; ++i)
    if (dts) dts[i] = q->ctx.log_step_dt[i];
  return SCY_OK;
}

scy_status scy_qd_get_field(scy_qd* q, int field, double* out) {
  if (!q || !out) return SCY_ERR_ARG;
  scy::QDContext& c = q->ctx;
  cudaStream_t s = c.sbp.stream;
  const double* src = nullptr;
  size_t n = c.Nz;
  long stride = 1;
  if (c.mode == SCY_QD_MODE_RESPONSE && c.green_ready &&
      (field == SCY_FIELD_U || field == SCY_FIELD_SXY || field == SCY_FIELD_SURFDISP)) {
    const double cc = c.bcR_remote ? c.vL * c.last_t * (1.0 / c.fts) : 0.0;
    if (field == SCY_FIELD_SURFDISP) return scy::qd_green_surf_launch(c, cc, out);
    SCY_TRY(c.full_solve_for_output());
  }
  const long op = c.key_off[SCY_KEY_PSI], os = c.key_off[SCY_KEY_SLIP];
  switch (field) {
    case SCY_FIELD_PSI: src = c.rk[0].as<double>() + op; break;
    case SCY_FIELD_SLIP: src = c.rk[0].as<double>() + os; break;
    case SCY_FIELD_DPSI: src = c.rk[1].as<double>() + op; break;
    case SCY_FIELD_DSLIP: src = c.rk[1].as<double>() + os; break;
    case SCY_FIELD_GVXY:
    case SCY_FIELD_GVXZ:
    case SCY_FIELD_SXZ:
    case SCY_FIELD_SDEV:
    case SCY_FIELD_EFFVISC:
      if (!c.pl) {
        scy::set_error("field %d exists for the power-law driver only", field);
        return SCY_ERR_ARG;
      }
      n = c.N;
      src = field == SCY_FIELD_GVXY   ? c.rk[0].as<double>() + c.key_off[SCY_KEY_GVXY]
            : field == SCY_FIELD_GVXZ ? c.rk[0].as<double>() + c.key_off[SCY_KEY_GVXZ]
            : field == SCY_FIELD_SXZ  ? c.sxz.as<double>()
            : field == SCY_FIELD_SDEV ? c.sdev.as<double>()
                                      : c.effVisc.as<double>();
      break;
    case SCY_FIELD_TEMPERATURE:
    case SCY_FIELD_DTEMP:
    case SCY_FIELD_VW:
      if (!c.th || (field == SCY_FIELD_VW && c.fp.state_law != SCY_LAW_FLASH)) {
        scy::set_error("field %d needs a thermal driver%s", field, field == SCY_FIELD_VW ? " with flash heating" : "");
        return SCY_ERR_ARG;
      }
      if (field == SCY_FIELD_TEMPERATURE || field == SCY_FIELD_DTEMP) {
        src = field == SCY_FIELD_TEMPERATURE ? c.th->T.as<double>() : c.th->dT.as<double>();
        n = c.N;
      } else {
        src = c.th->Vw.as<double>();
      }
      break;
    case SCY_FIELD_SLIPVEL: src = c.slipVel.as<double>(); break;
    case SCY_FIELD_TAUP: src = c.tauP.as<double>(); break;
    case SCY_FIELD_TAUQSP: src = c.tauQSP.as<double>(); break;
    case SCY_FIELD_STRENGTH: src = c.strength.as<double>(); break;
    case SCY_FIELD_U: src = c.u.as<double>(); n = c.N; break;
    case SCY_FIELD_SURFDISP: src = c.u.as<double>(); n = c.Ny; stride = c.Nz; break;
    case SCY_FIELD_SXY:
      // the power-law material keeps sxy = mu (Dy u - gVxy) from its last d_dt
      if (!c.pl) SCY_TRY(c.sbp.apply(SCY_OP_MUXDY, c.u.as<double>(), c.sxy.as<double>()));
      src = c.sxy.as<double>();
      n = c.N;
      break;
    default:
      scy::set_error("unknown field %d", field);
      return SCY_ERR_ARG;
  }
  if (stride == 1) {
    SCY_CUDA_TRY(cudaMemcpyAsync(out, src, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  } else {
    SCY_CUDA_TRY(cudaMemcpy2DAsync(out, sizeof(double), src, stride * sizeof(double), sizeof(double), n,
                                   cudaMemcpyDeviceToHost, s));
  }
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  return SCY_OK;
}

scy_status scy_qd_create_from_in(const char* path, const scy_solve_opts* solve, scy_qd** out) {
  if (!path || !out) {
    scy::set_error("scy_qd_create_from_in: NULL argument");
    return SCY_ERR_ARG;
  }
  *out = nullptr;
  std::unique_ptr<scy::QDProblem> P(new (std::nothrow) scy::QDProblem());
  if (!P) return SCY_ERR_NOMEM;
  try {
    scy::load_qd_problem(path, *P);
  } catch (const std::exception& e) {
    scy::set_error("%s", e.what());
    return SCY_ERR_IO;
  }
  if (solve) {
    P->desc.solve = *solve;
  } else {
    P->desc.solve.rtol = 1e-12;
    P->desc.solve.atol = 0.0;
    P->desc.solve.max_its = 300;
    P->desc.solve.precision = SCY_PREC_FP64;
    P->desc.solve.nonzero_guess = 1;
    P->desc.solve.check_every = 1;
    // LinearElastic / PowerLaw: KSPSetTolerances(ksp, kspTol, kspTol, ...)
    if (P->ksp_tol > 0) P->desc.solve.rtol = P->desc.solve.atol = P->ksp_tol;
  }
  scy_qd* q = new (std::nothrow) scy_qd();
  if (!q) return SCY_ERR_NOMEM;
  int st = q->ctx.create(P->desc, P->pl ? &P->pdesc : nullptr);
  if (st != SCY_OK) {
    delete q;
    return st;
  }
  if (P->min_dt_user == -1.0) P->ode.min_dt = q->ctx.compute_min_dt(P->cs, P->desc.grid.Ly, P->desc.grid.Lz);
  // the thermal driver: the heat equation on the device and the IMEX
  // integrator (RK32_WBE / RK43_WBE)
  q->ctx.imex = P->imex;
  if (P->heat) {
    q->ctx.th = std::make_shared<scy::ThermalContext>();
    st = q->ctx.th->create(q->ctx, *P->heat);
    if (st != SCY_OK) {
      delete q;
      return st;
    }
  }
  q->prob = std::move(P);
  *out = q;
  return SCY_OK;
}

scy_status scy_qd_get_problem(scy_qd* q, int* Ny, int* Nz, scy_ode_opts* ode) {
  if (!q) return SCY_ERR_ARG;
  if (Ny) *Ny = q->ctx.Ny;
  if (Nz) *Nz = q->ctx.Nz;
  if (ode) {
    if (!q->prob) {
      scy::set_error("driver was not created from an input file");
      return SCY_ERR_STATE;
    }
    *ode = q->prob->ode;
  }
  return SCY_OK;
}

scy_status scy_qd_integrate_begin_from_in(scy_qd* q) {
  if (!q || !q->prob) {
    scy::set_error("scy_qd_integrate_begin_from_in: driver was not created from an input file");
    return SCY_ERR_STATE;
  }
  scy::QDProblem& P = *q->prob;
  scy::QDContext& c = q->ctx;
  const int Nz = c.Nz;
  std::vector<double> psi = P.psi, slip(Nz);
  std::vector<double> var0((size_t)c.nvar);
  if (P.pl) {
    // StrikeSlip_PowerLaw_qd::initiateIntegrand (:305-350): slip = 2 bcL or
    // inputDir/slip; the viscous strains of the material
    for (int i = 0; i < Nz; ++i) slip[i] = P.bcL0[i] * 2.0;
    if (!P.slip_file.empty()) slip = P.slip_file;
    std::copy(P.gVxy0.begin(), P.gVxy0.end(), var0.begin() + c.key_off[SCY_KEY_GVXY]);
    std::copy(P.gVxz0.begin(), P.gVxz0.end(), var0.begin() + c.key_off[SCY_KEY_GVXZ]);
    // guessSteadyStateICs = 1: the steady-state iteration first (:320-324)
    if (P.guess_ss)
      SCY_TRY(c.pl_steady_state(P, psi, slip, var0.data() + c.key_off[SCY_KEY_GVXY],
                                var0.data() + c.key_off[SCY_KEY_GVXZ], &c.ss_its, &c.ss_err));
  } else if (P.ckpt_number > 0) {
    slip = P.slip_file;  // a restart: the checkpoint's state
    if (!P.slipVel0.empty())
      SCY_CUDA_TRY(cudaMemcpy(c.slipVel.p, P.slipVel0.data(), Nz * sizeof(double), cudaMemcpyHostToDevice));
  } else {
    for (int i = 0; i < Nz; ++i) slip[i] = P.bcL0[i] * P.desc.fault_type_scale;
    if (P.guess_ss) SCY_TRY(c.steady_state_guess(psi, P.stateVals_given, slip));
  }
  std::copy(psi.begin(), psi.end(), var0.begin() + c.key_off[SCY_KEY_PSI]);
  std::copy(slip.begin(), slip.end(), var0.begin() + c.key_off[SCY_KEY_SLIP]);
  SCY_CUDA_TRY(cudaMemcpyAsync(c.rk[0].p, var0.data(), var0.size() * sizeof(double), cudaMemcpyHostToDevice,
                               c.sbp.stream));
  SCY_CUDA_TRY(cudaStreamSynchronize(c.sbp.stream));
  // the file's output settings (stride1D / stride2D under outputDir), as the
  // reference's timeMonitor writes them
  if (!P.pl && !c.out && (P.stride1D > 0 || P.stride2D > 0))
    SCY_TRY(scy_qd_set_output(q, P.outputDir.c_str(), P.stride1D, P.stride2D, P.ckpt_number > 0 ? 1 : 0));
  if (!P.pl && P.ckpt > 0) {
    c.ckpt = P.ckpt;
    c.ckpt_interval = P.ckpt_interval;
    c.ckpt_number = P.ckpt_number;
    c.ckpt_dir = P.outputDir;
  }
  SCY_TRY(c.integrate_begin(P.ode));
  // A restart in the reference (strikeSlip_linearElastic_qd.cpp:727-738):
  // timeMonitor(initTime, initDeltaT, 0) first sets the driver's step count
  // to 0 and rewrites the checkpoint with the fresh integrator's error
  // history (zeros); the step count and errors then read back are those,
  // so the restarted run counts its steps from 0 (P control for its first
  // three steps) with an empty error history, as integrate_begin leaves it.
  // With the extension key ckptContinueSteps = 1 the run instead continues
  // the checkpoint's step count and error history.
  if (P.ckpt_number > 0 && P.ckpt_continue) {
    c.stepCount = P.step0;
    c.errA[0] = P.errA[0];
    c.errA[1] = P.errA[1];
  }
  return SCY_OK;
}

scy_status scy_qd_set_output(scy_qd* q, const char* output_dir, int stride1D, int stride2D, int append) {
  if (!q) return SCY_ERR_ARG;
  scy::QDContext& c = q->ctx;
  if (c.out) SCY_TRY(c.out->flush());
  c.out.reset();
  if (!output_dir || (stride1D <= 0 && stride2D <= 0)) return SCY_OK;
  std::unique_ptr<scy::OutputWriter> w(new (std::nothrow) scy::OutputWriter());
  if (!w) return SCY_ERR_NOMEM;
  const double tmax = q->prob ? q->prob->ode.t1 : c.ode.t1;
  SCY_TRY(w->open(output_dir, stride1D, stride2D, tmax, append ? 1 : 0, c));
  c.out = std::move(w);
  return SCY_OK;
}

scy_status scy_qd_flush_output(scy_qd* q) {
  if (!q) return SCY_ERR_ARG;
  return q->ctx.out ? q->ctx.out->flush() : SCY_OK;
}

scy_status scy_qd_set_mode(scy_qd* q, int mode) {
  if (!q || (mode != SCY_QD_MODE_SOLVE && mode != SCY_QD_MODE_RESPONSE)) {
    scy::set_error("scy_qd_set_mode: unknown mode");
    return SCY_ERR_ARG;
  }
  q->ctx.mode = mode;
  q->ctx.green_ready = 0;
  return SCY_OK;
}

scy_status scy_qd_set_jacobian(scy_qd* q, int exact) {
  if (!q) return SCY_ERR_ARG;
  q->ctx.fp.jacobian = exact ? 1 : 0;
  return SCY_OK;
}

scy_status scy_qd_steady_state_info(scy_qd* q, int* ss_its, double* ss_err, long* cg_its) {
  if (!q) return SCY_ERR_ARG;
  if (ss_its) *ss_its = q->ctx.ss_its;
  if (ss_err) *ss_err = q->ctx.ss_err;
  if (cg_its) *cg_its = q->ctx.ss_cg_its;
  return SCY_OK;
}

scy_status scy_qd_steady_state_trace(scy_qd* q, double* out, long cap, long* n) {
  if (!q || !n) return SCY_ERR_ARG;
  const std::vector<double>& t = q->ctx.ss_trace;
  *n = (long)t.size() / 5;
  if (out)
    for (long i = 0; i < std::min<long>((long)t.size(), cap * 5); ++i) out[i] = t[i];
  return SCY_OK;
}

scy_status scy_qd_set_state(scy_qd* q, const double* var, int recompute) {
  if (!q || !var) return SCY_ERR_ARG;
  scy::QDContext& c = q->ctx;
  if (!c.ode_ready) {
    scy::set_error("scy_qd_set_state: integration not started");
    return SCY_ERR_STATE;
  }
  SCY_CUDA_TRY(cudaMemcpyAsync(c.rk[0].p, var, (size_t)c.nvar * sizeof(double), cudaMemcpyHostToDevice,
                               c.sbp.stream));
  if (!recompute) return SCY_OK;
  SCY_TRY(c.d_dt(c.currT, c.rk[0].as<double>(), c.rk[1].as<double>()));
  return c.read_flags();
}

scy_status scy_in_problem_field(const char* path, const char* name, double* out, long cap, long* n) {
  if (!path || !name || !n) return SCY_ERR_ARG;
  scy::QDProblem P;
  try {
    scy::load_qd_problem(path, P);
  } catch (const std::exception& e) {
    scy::set_error("%s", e.what());
    return SCY_ERR_IO;
  }
  const std::string nm(name);
  const std::vector<double>* v = nullptr;
  if (nm == "y") v = &P.y;
  else if (nm == "z") v = &P.z;
  else if (nm == "mu") v = &P.mu;
  else if (nm == "rho") v = &P.rho;
  else if (nm == "cs") v = &P.cs;
  else if (nm == "a") v = &P.a;
  else if (nm == "b") v = &P.b;
  else if (nm == "sN") v = &P.sN;
  else if (nm == "Dc") v = &P.Dc;
  else if (nm == "psi") v = &P.psi;
  else if (nm == "locked") v = &P.locked;
  else if (nm == "prestress") v = &P.prestress;
  else if (nm == "eta") v = &P.eta;
  else if (nm == "bcL") v = &P.bcL0;
  else if (nm == "bcRShift") v = &P.bcRShift;
  else if (P.heat) {
    // the heat equation's fields (thermalCoupling set)
    const scy::HeatProblem& H = *P.heat;
    if (nm == "Tamb") v = &H.Tamb;
    else if (nm == "T") v = &H.T;
    else if (nm == "heat_k") v = &H.k;
    else if (nm == "heat_rho") v = &H.rho;
    else if (nm == "heat_c") v = &H.c;
    else if (nm == "Qrad") v = &H.Qrad;
    else if (nm == "Gw") v = &H.Gw;
    else if (nm == "Tw") v = &H.Tw;
  }
  if (!v) {
    scy::set_error("unknown problem field '%s'", name);
    return SCY_ERR_ARG;
  }
  *n = (long)v->size();
  if (out)
    for (long i = 0; i < *n && i < cap; ++i) out[i] = (*v)[i];
  return SCY_OK;
}

scy_status scy_in_problem_info(const char* path, scy_grid_desc* grid, scy_ode_opts* ode, int* state_law,
                               int* guess_ss, double* fault_type_scale) {
  if (!path) return SCY_ERR_ARG;
  scy::QDProblem P;
  try {
    scy::load_qd_problem(path, P);
  } catch (const std::exception& e) {
    scy::set_error("%s", e.what());
    return SCY_ERR_IO;
  }
  if (grid) {
    *grid = P.desc.grid;
    grid->y = grid->z = grid->mu = nullptr;
  }
  if (ode) *ode = P.ode;
  if (state_law) *state_law = P.desc.fault.state_law;
  if (guess_ss) *guess_ss = P.guess_ss;
  if (fault_type_scale) *fault_type_scale = P.desc.fault_type_scale;
  return SCY_OK;
}

// ---------------------------------------------------------------------------
// quasi-dynamic / fully dynamic cycles

scy_status scy_in_cycle_info(const char* path, scy_cycle_desc* cd, double* dt_fd, double* ay, long cap, long* n) {
  if (!path) return SCY_ERR_ARG;
  scy::QDProblem P;
  try {
    scy::load_qd_problem(path, P, 1);
    const scy_grid_desc& g = P.desc.grid;
    const int nm[4] = {SCY_BC_NEUMANN, SCY_BC_NEUMANN, SCY_BC_NEUMANN, SCY_BC_NEUMANN};
    scy::LevelHost h = scy::build_level(g.order, g.Ny, g.Nz, g.Ly, g.Lz, g.grid_type, g.compat, P.y, P.z, P.mu, nm);
    if (cd) {
      *cd = P.cdesc;
      cd->rho = cd->cs = cd->rho_fault = nullptr;
    }
    if (dt_fd) *dt_fd = scy::cycle_time_step(h, P.cs, P.cdesc.deltaT_fd, P.cdesc.CFL);
    if (n) {
      const double h11 = g.order == 2 ? 0.5 : 17.0 / 48.0;
      std::vector<double> a = scy::penalty_ay(g.Ny, g.Nz, h11 * h.dy, h11 * h.dz, P.cdesc.fd_bcR == SCY_FD_OUTGOING,
                                              P.cdesc.fd_bcT == SCY_FD_OUTGOING, P.cdesc.fd_bcB == SCY_FD_OUTGOING,
                                              P.cdesc.ay_index_quirk, P.cs);
      *n = (long)a.size();
      if (ay)
        for (long i = 0; i < *n && i < cap; ++i) ay[i] = a[i];
    }
  } catch (const std::exception& e) {
    scy::set_error("%s", e.what());
    return SCY_ERR_IO;
  }
  return SCY_OK;
}

scy_status scy_cycle_create(const scy_qd_desc* qd, const scy_cycle_desc* cd, scy_cycle** out) {
  if (!qd || !cd || !out) {
    scy::set_error("scy_cycle_create: NULL argument");
    return SCY_ERR_ARG;
  }
  *out = nullptr;
  scy_cycle* c = new (std::nothrow) scy_cycle();
  if (!c) return SCY_ERR_NOMEM;
  int st = c->ctx.create(*qd, *cd);
  if (st != SCY_OK) {
    delete c;
    return st;
  }
  *out = c;
  return SCY_OK;
}

scy_status scy_cycle_create_from_in(const char* path, const scy_solve_opts* solve, scy_cycle** out) {
  if (!path || !out) {
    scy::set_error("scy_cycle_create_from_in: NULL argument");
    return SCY_ERR_ARG;
  }
  *out = nullptr;
  std::unique_ptr<scy::QDProblem> P(new (std::nothrow) scy::QDProblem());
  if (!P) return SCY_ERR_NOMEM;
  try {
    scy::load_qd_problem(path, *P, 1);
  } catch (const std::exception& e) {
    scy::set_error("%s", e.what());
    return SCY_ERR_IO;
  }
  if (solve) {
    P->desc.solve = *solve;
  } else {
    default_solve(P->desc.solve);
    if (P->ksp_tol > 0) P->desc.solve.rtol = P->desc.solve.atol = P->ksp_tol;
  }
  scy_cycle* c = new (std::nothrow) scy_cycle();
  if (!c) return SCY_ERR_NOMEM;
  int st = c->ctx.create(P->desc, P->cdesc);
  if (st != SCY_OK) {
    delete c;
    return st;
  }
  c->prob = std::move(P);
  *out = c;
  return SCY_OK;
}

scy_status scy_cycle_destroy(scy_cycle* c) {
  delete c;
  return SCY_OK;
}

scy_status scy_cycle_get_problem(scy_cycle* c, int* Ny, int* Nz, double* dt_fd, scy_ode_opts* ode) {
  if (!c) return SCY_ERR_ARG;
  if (Ny) *Ny = c->ctx.Ny;
  if (Nz) *Nz = c->ctx.Nz;
  if (dt_fd) *dt_fd = c->ctx.dt_fd;
  if (ode) {
    if (!c->prob) {
      scy::set_error("driver was not created from an input file");
      return SCY_ERR_STATE;
    }
    *ode = c->prob->ode;
  }
  return SCY_OK;
}

scy_status scy_cycle_begin(scy_cycle* c, const scy_ode_opts* o, const double* var0) {
  if (!c || !o || !var0) {
    scy::set_error("scy_cycle_begin: NULL argument");
    return SCY_ERR_ARG;
  }
  if (!(o->tol > 0) || !(o->max_dt >= o->min_dt) || !(o->t1 >= o->t0) || o->max_steps < 0 || o->n_err > 2 ||
      (o->method != SCY_RK32 && o->method != SCY_RK43)) {
    scy::set_error("scy_cycle_begin: invalid options");
    return SCY_ERR_ARG;
  }
  return c->ctx.begin(*o, var0);
}

scy_status scy_cycle_begin_from_in(scy_cycle* c) {
  if (!c || !c->prob) {
    scy::set_error("scy_cycle_begin_from_in: driver was not created from an input file");
    return SCY_ERR_STATE;
  }
  scy::QDProblem& P = *c->prob;
  scy::QDContext& q = c->ctx.q;
  const int Nz = q.Nz;
  std::vector<double> psi = P.psi, slip(Nz);
  for (int i = 0; i < Nz; ++i) slip[i] = P.bcL0[i] * P.desc.fault_type_scale;
  if (!P.slip_file.empty()) slip = P.slip_file;
  if (P.guess_ss) SCY_TRY(q.steady_state_guess(psi, P.stateVals_given, slip));
  std::vector<double> var0(2 * (size_t)Nz);
  std::copy(psi.begin(), psi.end(), var0.begin());
  std::copy(slip.begin(), slip.end(), var0.begin() + Nz);
  return c->ctx.begin(P.ode, var0.data());
}

scy_status scy_cycle_run(scy_cycle* c, long max_steps, scy_cycle_stats* st) {
  if (!c || max_steps < 0) {
    scy::set_error("scy_cycle_run: invalid argument");
    return SCY_ERR_ARG;
  }
  int rc = c->ctx.run(max_steps, st);
  if (rc != SCY_OK && st) c->ctx.fill_stats(st);
  return rc;
}

scy_status scy_cycle_get_field(scy_cycle* c, int field, double* out) {
  if (!c || !out) return SCY_ERR_ARG;
  return c->ctx.get_field(field, out);
}

scy_status scy_cycle_get_switches(scy_cycle* c, long* steps, double* times, int* to_fd, long cap, long* n) {
  if (!c || !n) return SCY_ERR_ARG;
  const auto& sw = c->ctx.switches;
  *n = (long)sw.size();
  for (long i = 0; i < (long)sw.size() && i < cap; ++i) {
    if (steps) steps[i] = sw[i].step;
    if (times) times[i] = sw[i].t;
    if (to_fd) to_fd[i] = sw[i].to_fd;
  }
  return SCY_OK;
}

scy_status scy_cycle_set_fd_state(scy_cycle* c, double t, long step, int allowed, const double* psi,
                                  const double* slip, const double* u, const double* psiPrev,
                                  const double* slipPrev, const double* uPrev, const double* u0,
                                  const double* slip0, const double* tau0, const double* slipVel) {
  if (!c || !psi || !slip || !u || !psiPrev || !slipPrev || !uPrev || !u0 || !slip0 || !tau0 || !slipVel) {
    scy::set_error("scy_cycle_set_fd_state: NULL argument");
    return SCY_ERR_ARG;
  }
  const double* now[2] = {psi, slip};
  const double* prev[2] = {psiPrev, slipPrev};
  return c->ctx.set_fd_state(t, step, allowed, now, u, prev, uPrev, u0, slip0, tau0, slipVel);
}

scy_status scy_cycle_time_kernels(scy_cycle* c, int reps, double* wave_us, double* fault_us, double* step_us) {
  if (!c) return SCY_ERR_ARG;
  return c->ctx.time_kernels(reps, wave_us, fault_us, step_us);
}

scy_status scy_cycle_set_fd_fused(scy_cycle* c, int fused) {
  if (!c) return SCY_ERR_ARG;
  const int parts = fused ? scy::FD_FUSED : (scy::FD_WAVE | scy::FD_FAULT);
  if (parts != c->ctx.fd_parts) {
    for (auto& g : c->ctx.graphs) cudaGraphExecDestroy(g.second);
    c->ctx.graphs.clear();
    c->ctx.fd_parts = parts;
  }
  return SCY_OK;
}

scy_status scy_cycle_force_attempts(scy_cycle* c, const double* dts, const int* acc, long n) {
  if (!c || n < 0 || (n > 0 && (!dts || !acc))) return SCY_ERR_ARG;
  scy::QDContext& q = c->ctx.q;
  q.forced_dt.assign(dts, dts + n);
  q.forced_acc.assign(acc, acc + n);
  q.forced_pos = 0;
  return SCY_OK;
}

scy_status scy_cycle_record_attempts(scy_cycle* c, int on) {
  if (!c) return SCY_ERR_ARG;
  scy::QDContext& q = c->ctx.q;
  q.record = on ? 1 : 0;
  if (on) {
    q.log_dt.clear();
    q.log_acc.clear();
    q.log_step_dt.clear();
  }
  return SCY_OK;
}

scy_status scy_cycle_get_attempts(scy_cycle* c, double* dts, int* acc, long cap, long* n) {
  if (!c || !n) return SCY_ERR_ARG;
  const scy::QDContext& q = c->ctx.q;
  long m = (long)q.log_dt.size();
  *n = m;
  for (long i = 0; i < m && i < cap; ++i) {
    if (dts) dts[i] = q.log_dt[i];
    if (acc) acc[i] = q.log_acc[i];
  }
  return SCY_OK;
}

scy_status scy_cycle_set_mode(scy_cycle* c, int mode) {
  if (!c || (mode != SCY_QD_MODE_SOLVE && mode != SCY_QD_MODE_RESPONSE)) {
    scy::set_error("scy_cycle_set_mode: unknown mode");
    return SCY_ERR_ARG;
  }
  c->ctx.q.mode = mode;
  c->ctx.q.green_ready = 0;
  return SCY_OK;
}

scy_status scy_cycle_set_jacobian(scy_cycle* c, int exact) {
  if (!c) return SCY_ERR_ARG;
  c->ctx.q.fp.jacobian = exact ? 1 : 0;
  return SCY_OK;
}

scy_status scy_cycle_set_fd_batch(scy_cycle* c, int steps) {
  if (!c || steps < 1 || steps > 4096) {
    scy::set_error("scy_cycle_set_fd_batch: steps must be in 1..4096");
    return SCY_ERR_ARG;
  }
  c->ctx.fd_batch = steps;
  return SCY_OK;
}

}  // extern "C"
