/*
 * scycle_b200 -- C ABI of the B200 implementation of SCycle's per-time-step
 * quasi-dynamic path.
 *
 * Every entry point takes plain pointers and sizes.  Pointers documented as
 * "device" are CUDA device memory of length N = Ny*Nz (body) or Nz (fault),
 * laid out like the reference's PETSc Vecs: flattened index Ii = iy*Nz + iz,
 * z fastest (reference source/domain.cpp:380-381).  Pointers documented as
 * "host" are read during the call and copied.  All work is ordered on the
 * context's CUDA stream (scy_*_set_stream).  Every call returns a scy_status;
 * scy_get_last_error() returns the message of the last failure on the
 * calling thread.  No call traps or asserts on the device: conditions the
 * reference asserts on (root non-convergence, non-finite values, solver
 * failure) come back as status codes.
 */
#ifndef SCYCLE_B200_H
#define SCYCLE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int scy_status;

enum {
  SCY_OK = 0,
  SCY_ERR_ARG = 1,          /* invalid argument (size, type, NULL)          */
  SCY_ERR_CUDA = 2,         /* CUDA runtime error                           */
  SCY_ERR_NOMEM = 3,        /* device allocation failed                     */
  SCY_ERR_ROOT_NOCONV = 4,  /* fault root finder hit its iteration cap      */
  SCY_ERR_NONFINITE = 5,    /* NaN/Inf in a root bracket or residual        */
  SCY_ERR_CG_NOCONV = 6,    /* elliptic solve did not reach its tolerance   */
  SCY_ERR_DT_UNDERFLOW = 7, /* step size fell to the minimum                */
  SCY_ERR_STATE = 8,        /* call out of order                            */
  SCY_ERR_IO = 9,           /* file read/write failed                       */
  SCY_ERR_TIMEOUT = 10      /* a bounded device wait ran out                */
};

enum { SCY_BC_DIRICHLET = 0, SCY_BC_NEUMANN = 1 };
enum { SCY_GRID_CONST = 0, SCY_GRID_VAR = 1 };
enum { SCY_COMPAT_FULLY = 0, SCY_COMPAT_COMPATIBLE = 1 };

/* Number of kernels this library has launched in the process so far. */
long long scy_launch_count(void);
/* Brackets every launch of the SBP stencil kernel with CUDA events while on
 * (adds host overhead: use it in a separate measurement pass). */
scy_status scy_profile_enable(int on);
/* Sums the recorded stencil launches of multigrid level `level` (-1: all)
 * and value width `width` (4, 8; 0: both): total milliseconds, launch
 * count and algorithmic bytes (operand + mu read, result written); clears
 * the record. */
scy_status scy_profile_collect(int level, int width, double* ms, long long* launches, double* bytes);

/* Returns the message of the last failed call on this thread. */
const char* scy_get_last_error(void);
/* Library version string. */
const char* scy_version(void);

/* ------------------------------------------------------------------------
 * SbpOps + elliptic solver.
 *
 * Replaces SbpOps_m_constGrid / SbpOps_m_varGrid (reference
 * source/sbpOps.hpp:42-104, constructors sbpOps_m_constGrid.cpp:9-50 and
 * sbpOps_m_varGrid.cpp:5-45, computeMatrices :261-286 / :280-302) with
 * setMultiplyByH(1) and setLaplaceType("yz") as LinearElastic configures it
 * (source/linearElastic.cpp:426-461), and the KSP that LinearElastic solves
 * with (source/linearElastic.cpp:211-292, :465-489).
 * ---------------------------------------------------------------------- */
typedef struct scy_grid_desc {
  int order;          /* 2 or 4 */
  int Ny, Nz;         /* grid points; order 4 needs > 8, order 2 needs > 2 */
  double Ly, Lz;      /* domain size (km) */
  int grid_type;      /* SCY_GRID_CONST or SCY_GRID_VAR */
  int compat;         /* SCY_COMPAT_FULLY or SCY_COMPAT_COMPATIBLE */
  const double* y;    /* host, Ny*Nz coordinates (var grid; NULL -> q*Ly) */
  const double* z;    /* host, Ny*Nz coordinates (var grid; NULL -> r*Lz) */
  const double* mu;   /* host, Ny*Nz shear modulus (GPa) */
  int bcR, bcT, bcL, bcB; /* SCY_BC_DIRICHLET / SCY_BC_NEUMANN */
} scy_grid_desc;

typedef struct scy_sbp scy_sbp;

/* SbpOps constructor + computeMatrices (sbpOps_m_constGrid.cpp:9, :261). */
scy_status scy_sbp_create(const scy_grid_desc* desc, scy_sbp** out);
scy_status scy_sbp_destroy(scy_sbp* s);
/* Orders subsequent work on the given cudaStream_t (NULL = legacy default). */
scy_status scy_sbp_set_stream(scy_sbp* s, void* cuda_stream);
scy_status scy_sbp_synchronize(scy_sbp* s);
/* SbpOps::changeBCTypes (sbpOps_m_constGrid.cpp:163-195) + the KSP reset of
 * LinearElastic::changeBCTypes (linearElastic.cpp:513-534). */
scy_status scy_sbp_change_bc_types(scy_sbp* s, int bcR, int bcT, int bcL, int bcB);

enum {
  SCY_OP_A = 0,     /* getA + MatMult                      (constGrid.cpp:652-701) */
  SCY_OP_DY = 1,    /* SbpOps::Dy                          (constGrid.cpp:1460)    */
  SCY_OP_DZ = 2,    /* SbpOps::Dz                                                   */
  SCY_OP_MUXDY = 3, /* SbpOps::muxDy = mu*Dy*in            (constGrid.cpp:1466)    */
  SCY_OP_MUXDZ = 4, /* SbpOps::muxDz                                                */
  SCY_OP_H = 5,     /* SbpOps::H                                                    */
  SCY_OP_HINV = 6,  /* SbpOps::Hinv                                                 */
  SCY_OP_DYXMU = 7, /* SbpOps::Dyxmu = Dy*mu*in                                     */
  SCY_OP_DZXMU = 8  /* SbpOps::Dzxmu                                                */
};
/* out = op(in); in/out are device, length Ny*Nz, and must not alias. */
scy_status scy_sbp_apply(scy_sbp* s, int op, const double* in, double* out);

/* SbpOps::setRhs (sbpOps_m_constGrid.cpp:877-914):
 * rhs = rhsL*bcL + rhsR*bcR + rhsT*bcT + rhsB*bcB.
 * bcL, bcR: device, Nz;  bcT, bcB: device, Ny;  rhs: device, Ny*Nz. */
scy_status scy_sbp_set_rhs(scy_sbp* s, const double* bcL, const double* bcR,
                           const double* bcT, const double* bcB, double* rhs);

enum { SCY_PREC_FP64 = 0, SCY_PREC_MIXED = 1, SCY_PREC_TF32 = 2 };
enum {
  SCY_PC_AUTO = 0, /* fast diagonalisation when the grid metrics and mu are
                      separable (y depends only on iy, z only on iz, mu
                      constant), multigrid otherwise */
  SCY_PC_MG = 1,   /* geometric-multigrid V-cycle */
  SCY_PC_FD = 2    /* fast diagonalisation of the separable part: four dense
                      GEMMs per application (tensor cores) */
};

typedef struct scy_solve_opts {
  double rtol;       /* stop when ||A u - rhs||_2 <= max(rtol*||rhs||_2, atol) */
  double atol;
  int max_its;       /* PCG iteration cap */
  int precision;     /* SCY_PREC_FP64: FP64 preconditioner; SCY_PREC_MIXED:
                        FP32 preconditioner inside FP64 CG with an FP64
                        true-residual check */
  int nonzero_guess; /* 1: start from the incoming u (KSPSetInitialGuessNonzero) */
  int check_every;   /* residual read-back interval in iterations (>= 1) */
  int precond;       /* SCY_PC_* */
  int verify;        /* 1: recompute the true residual A u - rhs after the
                        last iteration (one more operator application);
                        0: trust the CG recurrence residual */
} scy_solve_opts;

typedef struct scy_solve_stats {
  int iterations;
  int converged;
  double rnorm0;     /* ||rhs - A u0|| */
  double rnorm;      /* final residual norm (true residual when verify = 1) */
  double bnorm;      /* ||rhs|| */
} scy_solve_stats;

/* LinearElastic::computeU's KSPSolve: solve A u = rhs.  rhs, u: device N. */
scy_status scy_sbp_solve(scy_sbp* s, const double* rhs, double* u,
                         const scy_solve_opts* opts, scy_solve_stats* stats);

/* The same solve for callers that cannot allocate device memory.  No
 * counterpart in the reference.  cudaMalloc/cudaFree can synchronise the
 * device and fail when another allocator (a framework's caching pool, a
 * memory manager that reserved the device up front) holds the free memory;
 * callers in that position, or that cannot afford an implicit device
 * synchronisation between stages, use this entry point: it allocates
 * nothing.  Its work vectors live in one fixed device array inside the
 * library (about 2.6 MB, held by every GPU that loads the library until the
 * process exits), so it accepts grids of at most 65,536 nodes (e.g.
 * 256 x 256) and returns SCY_ERR_ARG beyond that.  It preconditions CG with
 * point Jacobi instead of multigrid, so it needs more iterations; opts and
 * stats mean what they mean for scy_sbp_solve (opts->precision is ignored:
 * FP64).  All calls share the array: calls that overlap on the GPU race.
 * The first call on each device looks up the array's address with that
 * device current; with lazy module loading (the CUDA default) that first
 * call also loads the library's module on the device, which is when the
 * array's memory is reserved, so make it before another allocator reserves
 * the device.  A zero rhs with atol = 0 returns u = 0, as scy_sbp_solve
 * does. */
scy_status scy_sbp_solve_noalloc(scy_sbp* s, const double* rhs, double* u,
                                 const scy_solve_opts* opts, scy_solve_stats* stats);

/* FP64-accurate dense product on the integer tensor cores: D[r][c] =
 * sum_k X[r][k] W[c][k] for r < rows, c < cols, with each row of X and W
 * written as S = 3..7 signed 8-bit digit planes scaled by a power of two,
 * the S(S+1)/2 digit products accumulated exactly in 32-bit integers
 * (tcgen05.mma kind::i8) and combined in FP64; relative error per row about
 * 100^-S.  X and D are device arrays (row strides ldx, ldd), W a host array
 * (row stride ldw), K <= 1024.  ctas_per_sm: 1; 2 for S <= 5 (narrower
 * column tiles, one CTA's epilogue overlapping the other's products); 0 for
 * S <= 5, the persistent shape (one CTA per SM walking the narrower tiles
 * with two accumulator sets in tensor memory, one tile's epilogue under the
 * next tile's products); the same result in every shape.  bf16_digits = 1 holds the same digits in bf16 and
 * multiplies them with FP32 accumulation (tcgen05.mma kind::f16), exact and
 * so bit-identical while S * 64 * 64 * K' < 2^24 (K' = K rounded up to 32;
 * SCY_ERR_ARG beyond).  No counterpart in the reference: it is the z
 * transform of the fast-diagonalisation preconditioner that stands in for
 * the reference's direct solve, exported so it can be checked on its own. */
scy_status scy_ozaki_matmul(const double* X, long ldx, int rows, int K, const double* W, long ldw, int cols, int S,
                            double* D, long ldd, int ctas_per_sm, int bf16_digits);

/* Grid facts for callers (levels of the multigrid hierarchy, sizes). */
scy_status scy_sbp_info(scy_sbp* s, int* Ny, int* Nz, int* n_levels);

/* Host-side evaluation of A*in from the same operator tables the device
 * stencil reads (the routine that assembles the coarsest multigrid matrix).
 * Needs no GPU; exported so the table construction can be checked on any
 * machine.  in/out are host arrays of length Ny*Nz.  The solver never uses
 * it on the hot path. */
scy_status scy_grid_host_apply(const scy_grid_desc* desc, const double* in, double* out);
/* Host reference of the operator in the per-node form the batched ensemble
 * applies (A as a 33-point cross stencil per node: every column's y
 * operator and every row's z operator composed with that line's
 * coefficients and SAT terms).  Same arguments as scy_grid_host_apply. */
scy_status scy_grid_host_apply_cross(const scy_grid_desc* desc, const double* in, double* out);
/* Host reference of the operator in the full form the single-instance
 * operator kernels and the batched ensemble apply when it exists: outer
 * weights separable over every node, every column's y operator and every
 * row's z operator composed into 17-point stencils, one table per class of
 * lines (the lines equal to the middle column / row, plus at most eight
 * exceptional lines per direction such as the grid's corner lines), 9-point
 * on the interior box.  Same arguments as scy_grid_host_apply; SCY_ERR_ARG
 * when the operator has no full form. */
scy_status scy_grid_host_apply_full(const scy_grid_desc* desc, const double* in, double* out);

/* ------------------------------------------------------------------------
 * Fault_qd + StrikeSlip_LinearElastic_qd (linear-elastic quasi-dynamic).
 *
 * scy_qd_d_dt replaces StrikeSlip_LinearElastic_qd::d_dt
 * (source/strikeSlip_linearElastic_qd.cpp:756-798): boundary data from slip
 * and time, setRHS + KSPSolve + muxDy (solveMomentumBalance :874-891), the
 * body-to-fault scatter and Fault_qd::d_dt (source/fault.cpp:861-918) with
 * ComputeVel_qd's bracketed Newton (fault.cpp:954-1059,
 * rootFinder.cpp:174-257) and the aging / slip laws (fault.cpp:1984-2088).
 * scy_qd_integrate_* replace RK32::integrate / RK43::integrate
 * (source/odeSolver.cpp:505-627, :973-1175) with P / PID step control
 * (:395-445, :846-898).
 * ---------------------------------------------------------------------- */
/* SCY_LAW_FLASH: flashHeating_psi (fault.cpp:2171-2196) with the weakening
 * velocity of the fault temperature (flashHeating_Vw :2162-2168); drivers
 * created from an input file with thermalCoupling set only. */
enum { SCY_LAW_AGING = 0, SCY_LAW_SLIP = 1, SCY_LAW_CONSTANT = 2, SCY_LAW_FLASH = 3 };

typedef struct scy_fault_desc {
  int Nz;
  const double* a;         /* host, Nz: direct-effect parameter */
  const double* b;         /* host, Nz: evolution-effect parameter */
  const double* sN;        /* host, Nz: effective normal stress (MPa) */
  const double* Dc;        /* host, Nz: state evolution distance (m) */
  const double* eta;       /* host, Nz: radiation damping sqrt(mu rho)/faultTypeScale */
  const double* locked;    /* host, Nz or NULL: >0.5 held at 0, <-0.5 creeps at vL */
  const double* prestress; /* host, Nz or NULL */
  double f0, v0, vL;
  double root_tol;         /* absolute residual tolerance (MPa), reference default 1e-12 */
  int max_its;             /* root iteration cap, reference default 1e4 */
  int state_law;           /* SCY_LAW_* */
  int exact_jacobian;      /* 0: Newton steps use the reference's derivative
                              expression (fault.cpp:1051), reproducing its
                              iteration path; 1: the exact derivative (same
                              root within root_tol, far fewer iterations) */
} scy_fault_desc;

typedef struct scy_qd_desc {
  scy_grid_desc grid;
  scy_fault_desc fault;
  double fault_type_scale; /* 2 for symmFault, 1 for rigidFault */
  int bcL_from_slip;       /* 1: bcL = slip/fault_type_scale (symmFault, rigidFault) */
  int bcR_remote;          /* 1: bcR = vL*t/fault_type_scale + bcRShift (remoteLoading) */
  double vL;               /* loading rate of the driver (m/s) */
  const double* bcL0;      /* host, Nz or NULL: initial bcL (momBal_bcL) */
  const double* bcRShift;  /* host, Nz or NULL (momBal_bcR) */
  scy_solve_opts solve;    /* elliptic solve settings for every stage */
} scy_qd_desc;

typedef struct scy_qd scy_qd;

scy_status scy_qd_create(const scy_qd_desc* desc, scy_qd** out);
scy_status scy_qd_destroy(scy_qd* q);
scy_status scy_qd_set_stream(scy_qd* q, void* cuda_stream);

/* dvar = d_dt(t, var).  var = [psi | slip], dvar = [dpsi | dslip]: device,
 * 2*Nz doubles each (psi first: the reference integrates a std::map, whose
 * keys iterate in sorted order).  Updates the fault fields (slipVel, tauQS,
 * tauP, strength) and the body displacement like the reference. */
scy_status scy_qd_d_dt(scy_qd* q, double t, const double* var, double* dvar);

enum { SCY_RK32 = 0, SCY_RK43 = 1 };
enum { SCY_CTRL_P = 0, SCY_CTRL_PID = 1 };
enum { SCY_NORM_L2_ABS = 0, SCY_NORM_L2_REL = 1 };
/* Integrated fields.  The state vector holds them in the std::map's key
 * order: [psi | slip] (Nz each) for the linear-elastic drivers, [gVxy |
 * gVxz | psi | slip] (Ny*Nz, Ny*Nz, Nz, Nz) for the power-law driver. */
enum { SCY_KEY_PSI = 0, SCY_KEY_SLIP = 1, SCY_KEY_GVXY = 2, SCY_KEY_GVXZ = 3 };

typedef struct scy_ode_opts {
  int method;           /* SCY_RK32 / SCY_RK43 */
  int control;          /* SCY_CTRL_P / SCY_CTRL_PID */
  int norm;             /* SCY_NORM_L2_ABS / SCY_NORM_L2_REL */
  double tol;           /* timeStepTol */
  double min_dt, max_dt, init_dt;
  double t0, t1;        /* initTime, maxTime */
  long max_steps;       /* maxStepCount */
  int n_err;            /* 0: all keys in sorted order with scale 1 */
  int err_keys[4];      /* SCY_KEY_* in timeIntInds order */
  double err_scale[4];  /* scale per key */
} scy_ode_opts;

typedef struct scy_ode_stats {
  double t, dt, new_dt;
  long step_count, rejected, d_dt_evals, solve_its, solves;
  double errA[2];       /* errA[0] newest accepted error */
  int done;             /* 1: reached t1 or max_steps; 2: stopped after writing a checkpoint
                           (enableCheckpointing, as the reference's run ends there) */
} scy_ode_stats;

/* Fault_qd::d_dt (fault.cpp:861-918) on its own: with tau_body the body's
 * shear stress on the fault (device, Nz: the fault-row mu Dy u a driver
 * takes from its solve, LinearElastic::computeStresses), every fault node's
 * tauQS = tau_body + prestress, its slip velocity from the bracketed Newton
 * root of the friction law (ComputeVel_qd, fault.cpp:954-1059, starting from
 * the current slip velocity), the state rate of the driver's state law,
 * tauP and strength.  var, dvar: device arrays laid out as for scy_qd_d_dt
 * (scy_qd_state_size doubles; only the fault entries of dvar are written).
 * The fault fields (SCY_FIELD_SLIPVEL, TAUP, TAUQSP, ...) are updated as
 * the member vectors of Fault_qd are. */
scy_status scy_qd_fault_d_dt(scy_qd* q, const double* var, const double* tau_body, double* dvar);

/* OdeSolver setInitialConds + the first d_dt.  var0 = [psi | slip] host. */
scy_status scy_qd_integrate_begin(scy_qd* q, const scy_ode_opts* opts, const double* var0_host);
/* Advances up to nsteps accepted steps (fewer at t1 / max_steps). */
scy_status scy_qd_integrate_steps(scy_qd* q, long nsteps, scy_ode_stats* stats);
/* Forces the step size and accept decision of the next n attempts. */
scy_status scy_qd_force_attempts(scy_qd* q, const double* dts, const int* accept, long n);
/* Starts (1) / stops (0) recording (dt, accept) of every attempt. */
scy_status scy_qd_record_attempts(scy_qd* q, int on);
/* Copies the recorded attempts; *n receives their number. */
scy_status scy_qd_get_attempts(scy_qd* q, double* dts, int* accept, long cap, long* n);
/* While recording: per step taken, the size of the attempt whose solution
 * was kept (the accepted attempt, or the last one when the step fell to the
 * minimum size or the attempt cap); *n receives their number. */
scy_status scy_qd_get_step_sizes(scy_qd* q, double* dts, long cap, long* n);

enum {
  SCY_FIELD_PSI = 0, SCY_FIELD_SLIP = 1, SCY_FIELD_SLIPVEL = 2, SCY_FIELD_TAUP = 3,
  SCY_FIELD_TAUQSP = 4, SCY_FIELD_STRENGTH = 5, SCY_FIELD_U = 6, SCY_FIELD_SURFDISP = 7,
  SCY_FIELD_SXY = 8, SCY_FIELD_DPSI = 9, SCY_FIELD_DSLIP = 10
};
/* Copies a field to host memory (Nz, Ny or Ny*Nz doubles; see SCY_FIELD_*). */
scy_status scy_qd_get_field(scy_qd* q, int field, double* host_out);

/* Reads a StrikeSlip_LinearElastic_qd input file (the reference's .in
 * format: Domain, LinearElastic, Fault and driver keys, inputDir
 * PETSc-binary fields) and creates the driver (the reference's
 * Domain(file) + StrikeSlip_LinearElastic_qd(D), source/main.cpp:227-233).
 * `solve` sets the elliptic solver (NULL: FP64, rtol 1e-12 and atol 0, or rtol = atol =
 * kspTol when the file sets it, as LinearElastic passes it to KSPSetTolerances). */
scy_status scy_qd_create_from_in(const char* path, const scy_solve_opts* solve, scy_qd** out);
/* Sizes and the integrator settings read from the input file (min_dt is the
 * computeMinTimeStep value unless the file set minDeltaT). */
scy_status scy_qd_get_problem(scy_qd* q, int* Ny, int* Nz, scy_ode_opts* ode);
/* integrate()'s set-up for a driver made by scy_qd_create_from_in:
 * initiateIntegrand (with the steady-state guess when the file asks for it,
 * strikeSlip_linearElastic_qd.cpp:377-413; for the power-law driver the
 * effective-viscosity iteration of solveSS, strikeSlip_powerLaw_qd.cpp:922-955
 * and :1018-1107, each iteration a GPU solve with mu = effVisc) and the
 * first d_dt.  With
 * enableCheckpointing > 0 and a checkpoint in outputDir (ckptNumber > 0) the
 * run restarts from its chkpt_* files (time, step size, step count, error
 * history, state, slip velocity, stresses, boundary data) and appends to the
 * output files; checkpoints are written at step 0, every `interval` steps
 * and at the end, after which scy_qd_integrate_steps returns with done = 2. */
scy_status scy_qd_integrate_begin_from_in(scy_qd* q);
/* Output at the reference's strides (timeMonitor with writeStep1D/2D of the
 * driver, LinearElastic and Fault, strikeSlip_linearElastic_qd.cpp:417-495,
 * linearElastic.cpp:623-686, fault.cpp:512-557): PETSc-binary Vec records
 * appended to files named output_dir + field (surfDisp, momBal_bcR/T/L/B,
 * momBal_bcRShift, slip, slipVel, tauP, tauQSP, strength, psi, sNEff; with
 * stride2D momBal_u, momBal_sxy) and med_time1D/2D.txt, med_dt1D/2D.txt, at
 * step 0 (before the first rates) and every stride-th accepted step.  The
 * copies are queued on the driver's stream and written by a worker thread.
 * stride1D = stride2D = 0 or output_dir = NULL: no output.  append = 1
 * continues existing files.  scy_qd_integrate_begin_from_in turns it on from
 * the file's outputDir / stride1D / stride2D (linear-elastic driver). */
scy_status scy_qd_set_output(scy_qd* q, const char* output_dir, int stride1D, int stride2D, int append);
/* Waits until every queued output step is in its files. */
scy_status scy_qd_flush_output(scy_qd* q);
/* Host-only inspection of an input file (no GPU needed): the derived array
 * `name` ("y", "z", "mu", "rho", "cs", "a", "b", "sN", "Dc", "psi",
 * "locked", "prestress", "eta", "bcL", "bcRShift") is copied to out (cap
 * doubles); *n receives its length. */
scy_status scy_in_problem_field(const char* path, const char* name, double* out, long cap, long* n);
/* Host-only: grid descriptor scalars and integrator settings of an input
 * file (pointer members of *grid are set to NULL). */
scy_status scy_in_problem_info(const char* path, scy_grid_desc* grid, scy_ode_opts* ode, int* state_law,
                               int* guess_ss, double* fault_type_scale);

enum {
  SCY_QD_MODE_SOLVE = 0,    /* every d_dt solves the momentum balance (default) */
  SCY_QD_MODE_RESPONSE = 1  /* every d_dt evaluates the fault stress from the
                               discrete response of the fault to its boundary
                               data: tau = GL*(slip/faultTypeScale) + c(t)*g1 + gs,
                               GL (Nz x Nz) and g1, gs built once from Nz + 2
                               solves with the same solver; exact to the solve
                               tolerance because the momentum balance is linear
                               and its right-hand side depends only on bcL, bcR */
};
/* Selects how d_dt gets the fault stress (SCY_QD_MODE_*).  The response
 * matrices are built at the first d_dt after the switch (after the
 * steady-state guess, which changes bcRShift). */
scy_status scy_qd_set_mode(scy_qd* q, int mode);

/* Selects the root finder's derivative: 0 the reference's expression, 1 the
 * exact derivative (see scy_fault_desc.exact_jacobian).  Drivers made by
 * scy_qd_create_from_in start with the exact derivative. */
scy_status scy_qd_set_jacobian(scy_qd* q, int exact);

/* The power-law steady-state initial guess (guessSteadyStateICs = 1, run by
 * scy_qd_integrate_begin_from_in; StrikeSlip_PowerLaw_qd::solveSS,
 * strikeSlip_powerLaw_qd.cpp:922-955): effective-viscosity iterations, the
 * last relative change of the viscosity (computeNormDiff_L2_scaleL2) and
 * the conjugate-gradient iterations of all its elliptic solves.  Zeros when
 * no guess was made.  Any pointer may be NULL. */
scy_status scy_qd_steady_state_info(scy_qd* q, int* ss_its, double* ss_err, long* cg_its);
/* Per effective-viscosity iteration of that guess, five doubles: defect-
 * correction steps of its solve, relative residual ||rhs - A v|| / ||rhs||
 * (double-double) before and after them, CG iterations, relative change of
 * the viscosity.  *n gets the number of iterations; at most cap records are
 * written to out (may be NULL). */
scy_status scy_qd_steady_state_trace(scy_qd* q, double* out, long cap, long* n);

/* Overwrites the integrated state [psi | slip] (host, 2*Nz) between steps.
 * recompute = 1 re-evaluates the rates from it (one d_dt); recompute = 0
 * only uploads it (for a host round trip of the state the device holds). */
scy_status scy_qd_set_state(scy_qd* q, const double* var_host, int recompute);

/* ---------------------------------------------------------------------------
 * Power-law viscoelastic quasi-dynamic driver: StrikeSlip_PowerLaw_qd
 * (source/strikeSlip_powerLaw_qd.cpp) with PowerLaw's dislocation creep
 * (source/powerLaw.cpp).  The driver is an scy_qd whose integrated state is
 * [gVxy | gVxz | psi | slip]; every scy_qd_* entry point applies to it.
 * d_dt adds the viscous source B*gVxy + C*gVxz to the momentum balance
 * (computeViscStrainSourceTerms :1651-1671), forms the total strains and
 * the stresses sxy = mu (Dy u - gVxy), sxz = mu (Dz u - gVxz), the effective
 * viscosity 1/eta = 1/maxEffVisc + 1e3 A sdev^(n-1) exp(-B/T)
 * (DislocationCreep::computeInvEffVisc :438-474) and the viscous strain
 * rates with their boundary SAT term (computeViscStrainRates :1707-1743),
 * and feeds sxy on the fault to the rate-and-state fault.
 * ------------------------------------------------------------------------- */
typedef struct scy_pl_desc {
  const double* A;         /* host, Ny*Nz: dislocation-creep prefactor (disl_AVals) */
  const double* B;         /* host, Ny*Nz: activation temperature Q/R in K (disl_BVals) */
  const double* n;         /* host, Ny*Nz: stress exponent (disl_nVals) */
  const double* T;         /* host, Ny*Nz: temperature in K (TVals) */
  double visc_cap;         /* maxEffVisc (reference default 1e30) */
} scy_pl_desc;

/* A power-law driver; desc->grid.mu is PowerLaw's mu (interpolated against
 * z, powerLaw.cpp:1016). */
scy_status scy_pl_create(const scy_qd_desc* desc, const scy_pl_desc* pl, scy_qd** out);
/* Length of the integrated state of a driver (2*Nz, or 2*Ny*Nz + 2*Nz). */
scy_status scy_qd_state_size(scy_qd* q, long* n);

enum {
  SCY_FIELD_GVXY = 11, SCY_FIELD_GVXZ = 12, SCY_FIELD_SXZ = 13, SCY_FIELD_SDEV = 14, SCY_FIELD_EFFVISC = 15,
  /* thermal drivers (thermalCoupling uncoupled / coupled): the heat
   * equation's temperature (Ny*Nz) and the flash-heating law's weakening
   * velocity (Nz) */
  SCY_FIELD_TEMPERATURE = 16, SCY_FIELD_VW = 17, SCY_FIELD_DTEMP = 18 /* T - Tamb (Ny*Nz) */
};

/* ---------------------------------------------------------------------------
 * Quasi-dynamic / fully dynamic earthquake cycles: the
 * strikeSlip_linearElastic_qd_fd driver (source/strikeSlip_linearElastic_qd_fd.cpp,
 * selected by momentumBalanceType = quasidynamic_and_dynamic, main.cpp:266-274).
 * Quasi-dynamic phases run the scy_qd integrator, restarted per phase
 * (integrate_qd :1436-1508); fully dynamic phases step the wave equation with
 * a fixed CFL-limited step (computeTimeStep :356-442, propagateWaves
 * :1170-1239, Fault_fd::d_dt fault.cpp:1436-1523, OdeSolver_WaveEq::integrate
 * odeSolver_WaveEq.cpp:147-186).  The phases switch on R = max(eta V / tauQS)
 * (checkSwitchRegime :586-662).
 * ------------------------------------------------------------------------- */
enum { SCY_FD_FREE_SURFACE = 0, SCY_FD_OUTGOING = 1 };

typedef struct scy_cycle_desc {
  const double* rho;        /* host, Ny*Nz: body density (LinearElastic::_rho) */
  const double* cs;         /* host, Ny*Nz or NULL (sqrt(mu/rho)): shear-wave speed (LinearElastic::_cs) */
  const double* rho_fault;  /* host, Nz: fault density (Fault::_rho) */
  int fd_bcR, fd_bcT, fd_bcB; /* SCY_FD_*: momBal_bcR_fd, momBal_bcT_fd, momBal_bcB_fd; the
                                 left boundary is the fault (symmFault / rigidFault) */
  double deltaT_fd;         /* requested wave-equation step (s), <= 0: not given */
  double CFL;               /* requested CFL number, <= 0: not given */
  double trigger_qd2fd, trigger_fd2qd, limit_qd, limit_fd; /* after checkInput (:292-303) */
  int max_num_cycles;       /* maxNumCycles */
  int ay_index_quirk;       /* 1: the outgoing-characteristics damping ay indexed as
                               computePenaltyVectors does (its index advances only in
                               the last test, :493-495, so the damping lands on body
                               entries 0..Nz); 0: on the boundary nodes it names */
} scy_cycle_desc;

typedef struct scy_cycle scy_cycle;

enum { SCY_PHASE_QD = 0, SCY_PHASE_FD = 1, SCY_PHASE_DONE = 2 };

typedef struct scy_cycle_stats {
  double t;                 /* _currTime */
  double dt;                /* last quasi-dynamic step size */
  double new_dt;            /* the quasi-dynamic integrator's next step size (_newDeltaT) */
  double dt_fd;             /* wave-equation step (_deltaT_fd) */
  long step_count;          /* _stepCount: quasi-dynamic and wave-equation steps */
  int phase;                /* SCY_PHASE_* */
  int cycle_count;          /* _cycleCount */
  int allowed;              /* _allowed */
  int done;                 /* 1: integrate() has returned */
  long qd_steps, fd_steps;  /* quasi-dynamic steps (with the single step at each switch), wave steps */
  long switches;            /* phase switches so far */
  double last_ratio;        /* max(eta V / tauQS) at the last switch test */
  long d_dt_evals, solve_its, solves;
  double qd_ms, fd_ms;      /* host time spent in quasi-dynamic phases (with the single
                               steps) and in wave-equation batches */
} scy_cycle_stats;

scy_status scy_cycle_create(const scy_qd_desc* qd, const scy_cycle_desc* cd, scy_cycle** out);
/* Reads a strikeSlip_linearElastic_qd_fd input file (.in format; the
 * quasi-dynamic keys of scy_qd_create_from_in plus trigger_qd2fd,
 * trigger_fd2qd, limit_qd, limit_fd, deltaT_fd, CFL, maxNumCycles and
 * momBal_bc*_fd, loadSettings :135-230, with the defaults of :8-33). */
scy_status scy_cycle_create_from_in(const char* path, const scy_solve_opts* solve, scy_cycle** out);
scy_status scy_cycle_destroy(scy_cycle* c);
/* Sizes, the wave-equation step and the quasi-dynamic integrator settings
 * (a driver made from an input file). */
scy_status scy_cycle_get_problem(scy_cycle* c, int* Ny, int* Nz, double* dt_fd, scy_ode_opts* ode);
/* initiateIntegrands (:668-744) from var0 = [psi | slip] (host, 2*Nz). */
scy_status scy_cycle_begin(scy_cycle* c, const scy_ode_opts* ode, const double* var0_host);
/* initiateIntegrands for a driver made from an input file, with the
 * steady-state guess when the file asks for it (solveSS :1243-1340). */
scy_status scy_cycle_begin_from_in(scy_cycle* c);
/* integrate() (:511-581), advanced by at most max_steps steps; call again to
 * continue.  Returns with stats->done = 1 once the reference would return. */
scy_status scy_cycle_run(scy_cycle* c, long max_steps, scy_cycle_stats* stats);
/* Fields of the current phase (SCY_FIELD_*; U and SURFDISP are the material
 * displacement, u + u0 in a fully dynamic phase). */
scy_status scy_cycle_get_field(scy_cycle* c, int field, double* host_out);
/* Phase switches so far: the step and time of each, and to_fd = 1 for a
 * quasi-dynamic to fully dynamic switch. */
scy_status scy_cycle_get_switches(scy_cycle* c, long* steps, double* times, int* to_fd, long cap, long* n);
/* Forced / recorded attempts of the quasi-dynamic integrator, across all
 * quasi-dynamic phases and single steps (see scy_qd_force_attempts). */
scy_status scy_cycle_force_attempts(scy_cycle* c, const double* dts, const int* accept, long n);
scy_status scy_cycle_record_attempts(scy_cycle* c, int on);
scy_status scy_cycle_get_attempts(scy_cycle* c, double* dts, int* accept, long cap, long* n);
/* Quasi-dynamic phase mode (SCY_QD_MODE_*) and root-finder derivative. */
scy_status scy_cycle_set_mode(scy_cycle* c, int mode);
scy_status scy_cycle_set_jacobian(scy_cycle* c, int exact);
/* Wave-equation steps per graph launch (default 64; 1..4096). */
scy_status scy_cycle_set_fd_batch(scy_cycle* c, int steps);
/* Restart hook: puts the driver at the start of a fully dynamic step at time
 * t after global step `step`, with the wave-equation state of steps n
 * (psi, slip, u) and n-1 (psiPrev, slipPrev, uPrev), the displacement offset
 * u0 (material u = u + u0), the fault's slip0 and tau0 (strength + prestress
 * at the switch), its slip velocity and the switch test's _allowed (host
 * arrays: Nz for fault fields, Ny*Nz for u, uPrev, u0).  A driver made by
 * scy_cycle_create_from_in must have been begun first. */
scy_status scy_cycle_set_fd_state(scy_cycle* c, double t, long step, int allowed, const double* psi,
                                  const double* slip, const double* u, const double* psiPrev,
                                  const double* slipPrev, const double* uPrev, const double* u0,
                                  const double* slip0, const double* tau0, const double* slipVel);
/* Profiling hook: average device time (CUDA events, `reps` back-to-back
 * launches each) of one fully dynamic step as the fused launch (step_us) and
 * of the two-launch form's wave stencil and fault update, on the driver's
 * current wave state.  The launches rewrite the step-n+1 buffers and the
 * fault's slip velocity, so call it only when the run is over or about to be
 * restarted. */
scy_status scy_cycle_time_kernels(scy_cycle* c, int reps, double* wave_us, double* fault_us, double* step_us);
/* 1: one fused launch per wave step (default); 0: the two-launch form. */
scy_status scy_cycle_set_fd_fused(scy_cycle* c, int fused);
/* Host-only (no GPU needed): the cycle settings of an input file after
 * checkInput (pointer members set to NULL), the wave-equation step of
 * computeTimeStep and the penalty vector ay of computePenaltyVectors (Ny*Nz
 * doubles into ay when cap allows; *n receives the length). */
scy_status scy_in_cycle_info(const char* path, scy_cycle_desc* cd, double* dt_fd, double* ay, long cap, long* n);

/* ---------------------------------------------------------------------------
 * Batched ensemble of quasi-dynamic instances (linear elastic or power law).
 *
 * The reference runs one StrikeSlip_*_qd per process
 * (strikeSlip_linearElastic_qd.cpp:475-505 integrate(), power law
 * strikeSlip_powerLaw_qd.cpp:521-560); an ensemble is many such runs.  Here
 * the instances of one batch share every launch: instances whose operators
 * are identical (grid size, coordinates, mu, boundary types) form a group,
 * and each RK attempt of every instance is one round of batched launches
 * per group, captured once as a CUDA graph with the groups on concurrent
 * streams.  Every instance keeps its own adaptive RK32/RK43 step control
 * (odeSolver.cpp:505-627, :973-1175), decided on the host from one read-back
 * per round, and so takes the same steps as the same instance run alone.
 * The stage solves run a fixed number of preconditioned CG iterations
 * (fast diagonalisation of the group's operator, FP64 or FP32) with the
 * convergence test on the device; a round in which an instance misses the
 * tolerance is repeated for that instance with more iterations, and later
 * rounds use one more.  Instances must all use the same driver (linear
 * elastic or power law) and integrator. */
typedef struct scy_batch scy_batch;
typedef struct scy_batch_opts {
  int precision;  /* preconditioner of the FP64 CG: SCY_PREC_FP64 (FP64 data, FP64-accurate z
                     transforms), SCY_PREC_MIXED (FP32 data and sweeps, z transforms of FP32
                     accuracy), SCY_PREC_TF32 (FP32 data, coarser z transforms) */
  int cg_its;     /* CG iterations per stage solve at the start (0: 1 for FP64, 2 otherwise); the
                     batch raises it after a missed tolerance and tries one fewer after a run of
                     rounds without one */
  int graphs;     /* 1: one CUDA graph launch per round (default); 0: the same launches issued directly */
  int concurrent; /* 1: groups on concurrent streams (default); 0: one stream */
  int exact_jacobian; /* root-finder derivative of every instance (see scy_qd_set_jacobian) */
  int fd_dense;   /* 1: the preconditioner as four cuBLAS GEMMs (y and z transforms) even where the
                     y part is banded, a reference form for tests; 0 (default): z transforms on the
                     integer tensor cores (see scy_ozaki_matmul) and banded Cholesky solves along y */
  int transform_planes; /* digit planes of those z transforms, 3..7 (0: 5 with the FP64
                           preconditioner, 4 with SCY_PREC_MIXED, 3 with SCY_PREC_TF32); the CG
                           and its residuals stay FP64 whatever the planes, so they change the
                           iteration count, not the converged solution */
} scy_batch_opts;
typedef struct scy_batch_stats {
  long rounds;          /* rounds of batched attempts so far */
  long redo_rounds;     /* rounds repeated after a missed solve tolerance */
  long graph_launches;  /* CUDA graph launches so far */
  long instance_steps;  /* accepted steps summed over the instances */
  long stage_solves;    /* d_dt evaluations summed over the instances */
  int cg_its;           /* CG iterations per stage solve now */
  int groups;           /* groups of instances with one operator */
  int done;             /* 1: every instance reached its t1 or max_steps */
} scy_batch_stats;
/* Creates every instance from its input file (as scy_qd_create_from_in)
 * and begins it (as scy_qd_integrate_begin_from_in); `solve` as there
 * (its rtol / atol are the batched solves' tolerance).  opts may be NULL. */
scy_status scy_batch_create_from_in(int n, const char* const* paths, const scy_solve_opts* solve,
                                    const scy_batch_opts* opts, scy_batch** out);
/* Destroys the batch and its instances. */
scy_status scy_batch_destroy(scy_batch* b);
/* Number of instances and of groups; group_of (n ints, may be NULL) gets
 * each instance's group. */
scy_status scy_batch_info(scy_batch* b, int* n, int* groups, int* group_of);
/* The driver handle of instance i, owned by the batch: for scy_qd_get_field,
 * scy_qd_force_attempts, scy_qd_record_attempts, scy_qd_get_attempts and
 * scy_qd_integrate_steps(q, 0, stats) (its counters).  Advancing it on its
 * own between batched runs is allowed. */
scy_status scy_batch_instance(scy_batch* b, int i, scy_qd** q);
/* Advances every instance by up to nsteps accepted steps (fewer at its t1 /
 * max_steps); returns once all are done and their rates are evaluated at
 * the accepted states. */
scy_status scy_batch_run(scy_batch* b, long nsteps, scy_batch_stats* stats);
/* Total length of the instances' integrated states (scy_qd_state_size
 * each), concatenated in the caller's instance order. */
scy_status scy_batch_state_size(scy_batch* b, long* total);
/* Replaces every instance's integrated state from one host array of that
 * length (the rates are not recomputed: give states the instances hold,
 * e.g. read back after a run, or restart the instances on their own). */
scy_status scy_batch_set_states(scy_batch* b, const double* host);
/* A fault field (SCY_FIELD_PSI, SLIP, DPSI, DSLIP, SLIPVEL, TAUP, TAUQSP,
 * STRENGTH) of every instance into one host array, Nz values per instance
 * in the caller's instance order. */
scy_status scy_batch_get_fault_field(scy_batch* b, int field, double* host);
/* 1: each round is one CUDA graph launch; 0: its launches issued directly. */
scy_status scy_batch_set_graphs(scy_batch* b, int on);
/* Per-launch timing of the batch's main kernels while on (takes effect in
 * rounds launched directly, see scy_batch_set_graphs): CUDA events on the
 * launching stream around each launch, for measurement passes. */
scy_status scy_batch_profile(scy_batch* b, int on);
enum { SCY_BATCH_KERNEL_YSOLVE = 0, SCY_BATCH_KERNEL_RESIDUAL = 1, SCY_BATCH_KERNEL_MATVEC = 2,
       SCY_BATCH_KERNEL_ZTRANSFORM = 3, SCY_BATCH_KERNEL_ZSPLIT = 4 };
/* Sums the timed launches of one kernel (SCY_BATCH_KERNEL_*): milliseconds,
 * launch count and algorithmic bytes (the banded sweeps: factor once plus
 * read and write of the transform twice; the operator kernels: coefficient
 * planes once plus the per-node operands and results of the active
 * instances; a z transform of the preconditioner on the tensor cores: the
 * digit planes and exponents of the operand and of the weights read, the
 * result written; the digit split: the operand read, its planes and
 * exponents written). */
scy_status scy_batch_profile_collect(scy_batch* b, int kernel, double* ms, long long* launches, double* bytes);
/* Drops the recorded launches. */
scy_status scy_batch_profile_clear(scy_batch* b);
/* Test hook (no counterpart in the reference) for the banded sweeps'
 * bounded data waits: polls bounds the waits (default 2^18; every poll is an
 * mbarrier.try_wait, which itself waits a while), and drop_first_copy = 1
 * withholds each block's first chunk copy, so that wait runs out as a copy
 * that never arrives would make it.  A wait that runs out marks its
 * instances (status bit 4) and the round is repeated; after three repeats
 * scy_batch_run returns SCY_ERR_TIMEOUT.  Nothing is left in flight: a
 * block awaits the copies it did issue (at the full limit) before it exits.
 * (polls, 0) with the default restores normal operation. */
scy_status scy_batch_set_sweep_test(scy_batch* b, int polls, int drop_first_copy);

/* The autotuner's choices for group g (no counterpart in the reference): at
 * set-up every group times, on its own buffers, the CG operator kernel in
 * the cross form (33 coefficient planes) with 1, 2, 4 and 8 instances per
 * block and, when the operator is separable over every node, in the
 * separable form (1D coefficient tables) with 1, 2 and 4 rows per thread,
 * the banded sweeps in six launch shapes (chains per lane x warps per block:
 * 2 x 2, 1 x 4, 4 x 1 serving 8 instances per block, 1 x 2 and 2 x 1
 * serving 4, 1 x 1 serving 2) and the z-transform product in three shapes
 * (one CTA per tile, two CTAs per SM, persistent: one CTA per SM with two
 * accumulator sets) with 8-bit or bf16 digits (identical results), and keeps
 * the fastest.  kpb / sweep_variant / ztransform get the choices (kpb: the
 * cross form's, see scy_batch_operator_form for the form in use; ztransform
 * bit 0: two CTAs per SM, bit 1: bf16 digits, bit 2: persistent), us (22
 * doubles, may be NULL) the timings in microseconds per launch (cross form
 * at kpb 1, 2, 4, 8; sweep shapes 0-5; product with 8-bit digits, one and
 * two CTAs per SM; with bf16 digits, one and two CTAs per SM; separable form
 * at 1, 2, 4 rows per thread with the compiler's register count, then with
 * registers fitted to four blocks per SM; persistent product with 8-bit and
 * with bf16 digits; 0 where not tried).  The separable form is used
 * whenever the operator has it (its results do not depend on its launch
 * shape; they differ from the cross form's by rounding). */
scy_status scy_batch_tuning(scy_batch* b, int g, int* kpb, int* sweep_variant, int* ztransform, double* us);
/* The operator kernels group g runs: *rows_per_thread = 0 for the cross
 * form, else the separable form's rows per thread (1, 2 or 4), and
 * *min_blocks_per_sm (may be NULL) the blocks per SM its registers are
 * fitted to (1: the compiler's choice; 0 for the cross form). */
scy_status scy_batch_operator_form(scy_batch* b, int g, int* rows_per_thread, int* min_blocks_per_sm);

/* ---------------------------------------------------------------------------
 * Discrete adjoint of the linear-elastic quasi-dynamic RK32 integration.
 * No counterpart in the reference (it has no adjoint); the forward map is
 * RK32::integrate (odeSolver.cpp:505-627) over a fixed sequence of accepted
 * step sizes with StrikeSlip_LinearElastic_qd::d_dt (solve mode).  The misfit
 * is J = sum_n w_surf |surfDisp_n - target_surf_n|^2 + w_vel |V_n - target_vel_n|^2
 * over the accepted states n = 1..M; the gradient is with respect to a, b
 * and Dc at every fault node (the initial state is held fixed).  States are
 * checkpointed every `checkpoint_every` steps and each segment recomputed
 * before its reverse sweep; one reverse stage costs one elliptic solve. */
typedef struct scy_adj scy_adj;
/* On a driver that has been begun with RK32 (its current state and time are
 * the initial state and time of every forward run). */
scy_status scy_adj_create(scy_qd* q, int checkpoint_every, scy_adj** out);
scy_status scy_adj_destroy(scy_adj* a);
/* The accepted step sizes (e.g. the accepted entries of scy_qd_get_attempts). */
scy_status scy_adj_set_steps(scy_adj* a, const double* dts, long n);
/* Targets (host, n x Ny surface displacement and n x Nz slip velocity,
 * state-major) and the misfit weights. */
scy_status scy_adj_set_targets(scy_adj* a, const double* target_surf, const double* target_vel, double w_surf,
                               double w_vel);
/* Replaces the fault's a, b and / or Dc (host, Nz each; NULL keeps a field). */
scy_status scy_adj_set_fault_params(scy_adj* a, const double* fa, const double* fb, const double* fDc);
/* Runs the forward map from the initial state; J = the misfit (0 without targets). */
scy_status scy_adj_forward(scy_adj* a, double* J);
/* Surface displacement and slip velocity of the accepted states of the last
 * forward run (host, n x Ny and n x Nz). */
scy_status scy_adj_observations(scy_adj* a, double* surf, double* vel);
/* Forward run, then the reverse sweep: J and dJ/da, dJ/db, dJ/dDc (host, Nz each). */
scy_status scy_adj_gradient(scy_adj* a, double* J, double* grad_a, double* grad_b, double* grad_Dc);

#ifdef __cplusplus
}
#endif

#endif /* SCYCLE_B200_H */
