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

enum { SCY_PREC_FP64 = 0, SCY_PREC_MIXED = 1 };

typedef struct scy_solve_opts {
  double rtol;       /* stop when ||A u - rhs||_2 <= max(rtol*||rhs||_2, atol) */
  double atol;
  int max_its;       /* PCG iteration cap */
  int precision;     /* SCY_PREC_FP64: FP64 multigrid; SCY_PREC_MIXED: FP32
                        multigrid preconditioner inside FP64 CG with FP64
                        true-residual refinement */
  int nonzero_guess; /* 1: start from the incoming u (KSPSetInitialGuessNonzero) */
  int check_every;   /* residual read-back interval in iterations (>= 1) */
} scy_solve_opts;

typedef struct scy_solve_stats {
  int iterations;
  int converged;
  double rnorm0;     /* ||rhs - A u0|| */
  double rnorm;      /* final true residual norm */
  double bnorm;      /* ||rhs|| */
} scy_solve_stats;

/* LinearElastic::computeU's KSPSolve: solve A u = rhs.  rhs, u: device N. */
scy_status scy_sbp_solve(scy_sbp* s, const double* rhs, double* u,
                         const scy_solve_opts* opts, scy_solve_stats* stats);

/* Grid facts for callers (levels of the multigrid hierarchy, sizes). */
scy_status scy_sbp_info(scy_sbp* s, int* Ny, int* Nz, int* n_levels);

/* Host-side evaluation of A*in from the same operator tables the device
 * stencil reads (the routine that assembles the coarsest multigrid matrix).
 * Needs no GPU; exported so the table construction can be checked on any
 * machine.  in/out are host arrays of length Ny*Nz.  The solver never uses
 * it on the hot path. */
scy_status scy_grid_host_apply(const scy_grid_desc* desc, const double* in, double* out);

#ifdef __cplusplus
}
#endif

#endif /* SCYCLE_B200_H */
