// Batched ensemble of quasi-dynamic instances (scy_batch_* in the C ABI).
//
// Each instance is a complete single-instance driver (QDContext, made from
// its own input file); the batch only adds launches that act on many
// instances at once.  Instances whose operators are identical form a group;
// a group's work vectors for the CG solve are contiguous (instance k at
// k*N), so the fast-diagonalisation preconditioner of a whole group is four
// large GEMMs, and every other kernel takes the instance from blockIdx.z and
// reads that instance's pointers from a device table.
#pragma once
#include <cublas_v2.h>
#include <cuda.h>

#include <map>
#include <memory>
#include <vector>

#include "fdiag.hpp"
#include "ozaki.hpp"
#include "qd.hpp"

struct scy_qd;

namespace scy {

// Device view of one instance: pointers into its QDContext.
struct BatchInst {
  double* rk[11];  // V_VAR .. V_HI
  double *u, *rhs, *bcL, *bcR, *bcT, *bcB, *bcRShift, *sxy;
  double *slipVel, *tauQSP, *tauP, *strength;
  unsigned* flags;
  unsigned long long* fault_its;
  FaultParams fp;
  double vL, inv_fts;
  int bcL_from_slip, bcR_remote;
  long nvar;
  long key_off[4], key_len[4];
  // power law (c1 == nullptr for the linear-elastic driver)
  const double *c1, *e1, *n;
  double *sxz, *sdev, *effVisc;
  double inv_cap;
};

// Work arrays of a group (K instances of N nodes): CG vectors, the
// preconditioner's temporaries, CG scalars, reduction partials and counters,
// and the device-verified solve status.
struct BatchWork {
  int K, PB;
  long N;
  double *r, *p0, *p1, *q, *z, *t1, *t2;
  float *r32, *z32, *t1f, *t2f;
  double* sc;          // K * 16: [0] |rhs|^2, [1] r.r, [2] rz, [3] rz old, [4] p.q, [5] |r0|^2
  double* partials;    // K * PB
  double* partials2;   // K * PB (r.z of the first CG iteration)
  unsigned* counters;  // K * 4
  unsigned* status;    // K
};

// tags of the timed kernels (scy_batch_profile_collect)
enum { PROF_YSOLVE = 0, PROF_RESIDUAL = 1, PROF_MATVEC = 2, PROF_ZTRANSFORM = 3, PROF_ZSPLIT = 4 };

struct BatchGroup {
  int K = 0, base = 0;  // instances base .. base + K - 1 of the batch
  int Ny = 0, Nz = 0;
  long N = 0;
  LevelDev<double> L{};
  std::shared_ptr<FDPrecond> fd;
  DevBuf tab;     // BatchInst[K]
  DevBuf t1p, t1pf;  // the z transform, rows padded to the factor tables' Nzp (FP64, FP32)
  CUtensorMap mLcol, mLrow, mT, mLcol32, mLrow32, mT32;  // tile maps of the TMA-fed banded sweeps
  CUtensorMap mT4, mT2, mT4_32, mT2_32;                 // the transform for 4 and 2 instances per block
  DevBuf planes;  // the operator's 33 cross-stencil coefficient planes (build_cross_planes)
  int kpb = 1;    // instances per block of the operator kernels (autotuned at set-up)
  int ys_variant = 0;  // chains per lane x warps per block of the banded sweeps (autotuned)
  int zt_pair = 0;  // z-transform products: 0 one CTA per tile, 1 two CTAs per SM, 2 persistent (autotuned)
  int zt_bf16 = 0;  // z-transform digits in bf16 (kind::f16) instead of 8-bit integers (autotuned)
  int full_shape = -1;  // >= 0: the operator kernels in the separable form, in this launch shape (autotuned)
  // the autotuner's timings: kpb 1, 2, 4, 8; sweep variants 0..5;
  // z-transform product with 8-bit digits in the one- and two-CTAs-per-SM
  // shapes, with bf16 digits in the two shapes; the separable form at 1, 2
  // and 4 rows per thread, registers by the compiler's choice and then
  // fitted to four blocks per SM; the persistent z-transform product with
  // 8-bit and with bf16 digits
  double tune_us[22] = {0};
  DevBuf vec[7], vecf[4], sc, partials, counters, status;
  BatchWork w{};
  cudaStream_t stream = nullptr;
  cudaEvent_t join = nullptr;
  cublasHandle_t blas = nullptr;
  // the z transforms of the banded preconditioner on the integer tensor
  // cores: the digit planes of the operand (residual, then the swept
  // transform; K*Ny rows of Nz values) and of the two weight matrices
  // (rows of Vz^T for the forward transform, rows of Vz for the inverse)
  OzkOperand zx, zw1, zw2;
  OzkOperand zx16, zw1_16, zw2_16;  // the same digits in bf16 while the autotuner compares (then freed)
  DevBuf blas_ws;
  ~BatchGroup();
};

// One instance's slice of the host array of scy_batch_set_states or
// scy_batch_get_fault_field: n values of device vector p, at offset off of
// the array.
struct IoSeg {
  double* p;
  long n, off;
};
constexpr int kIoFields = 11;  // SCY_FIELD_PSI .. SCY_FIELD_DSLIP

struct BatchContext {
  std::vector<scy_qd*> inst;  // owned, in slot order (group by group)
  std::vector<int> group_of;  // by the caller's numbering
  std::vector<int> slot_of, user_of;
  std::vector<std::unique_ptr<BatchGroup>> groups;
  int n = 0, pl = 0, method = 0, precision = 0, its = 1, graphs = 1, concurrent = 1, fd_dense = 0;
  int zt_planes = 7;  // digit planes of the tensor-core z transforms
  double rtol = 1e-12, atol = 0.0;
  int max_its = 300;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  // per-round control block (device + pinned host mirror):
  // t[n], dt[n] (doubles), then copy[n], acc[n], run[n] (ints)
  DevBuf ctl;
  void* ctl_host = nullptr;
  size_t ctl_bytes = 0;
  // per-round results: 16 doubles per instance (key sums, fault flags, solve status)
  DevBuf err;
  double* err_host = nullptr;
  std::map<int, cudaGraphExec_t> graph_of_its;  // by 4 * its + phases
  std::map<int, long long> kernels_of_its;      // kernels per replay
  long calm_rounds = 0, probe_period = 64;      // iteration-count tuning
  // host step control per instance
  struct Ctl {
    int running = 0, copy = 0, acc = 0;
    int attemptCount = 0, forced = 0, forced_accept = 0;
    long done_steps = 0, target = 0;
  };
  std::vector<Ctl> hc;
  // the states and fault fields move between the caller's array and the
  // instances as one transfer through a staging buffer, scattered or
  // gathered by a kernel (IoSeg tables: the states, then one per field)
  DevBuf io, io_seg;
  long io_states = 0, io_fault = 0;
  long io_maxn = 0;
  int set_states(const double* host);
  int get_fault_field(int field, double* host);
  long rounds = 0, redo_rounds = 0, graph_launches = 0, inst_steps = 0, stage_solves = 0;
  // optional per-launch timing of the main kernels (rounds launched directly
  // while on): CUDA events on the launching stream around each launch
  struct ProfRec {
    cudaEvent_t a, b;
    int tag;
    double bytes;  // algorithmic bytes of the launch
  };
  int prof = 0;
  int sweep_polls = 1 << 18;  // polls of the banded sweeps' data waits (lowered only by a test hook)
  int sweep_drop = 0;         // test hook: the sweeps' first copy is withheld
  std::vector<ProfRec> precs;
  int active_in(const BatchGroup& g, const int* mask) const;  // instances of g the mask selects this round
  int prof_begin(cudaStream_t s, cudaEvent_t* a);
  int prof_end(cudaStream_t s, cudaEvent_t a, int tag, double bytes);
  int prof_collect(int tag, double* ms, long long* launches, double* bytes);

  ~BatchContext();
  int create(int n, const char* const* paths, const scy_solve_opts* solve, const scy_batch_opts* o);
  int run(long nsteps, scy_batch_stats* st);
  void stats(scy_batch_stats* st) const;

 private:
  QDContext& q(int i) const;
  int setup_group(int base, int K);
  // the autotuner: times the candidate launch shapes of the group's main
  // kernels on its own buffers and keeps the fastest
  int autotune(BatchGroup& g);
  int launch_ysolve(BatchGroup& g, int variant);
  // phases: 1 = copy + rates at accepted states, 2 = an attempt (graphs keyed by its and phases)
  int enqueue_round(int its_now, int phases);
  int launch_round(int its_now, int phases);
  int enqueue_group(BatchGroup& g, int its_now, int phases);
  int d_dt(BatchGroup& g, const int* mask, double c, int in_slot, int out_slot, int its_now);
  int solve(BatchGroup& g, const int* mask, int its_now);
  int fd_apply(BatchGroup& g);
  int combine(BatchGroup& g, const int* mask, int out_slot, std::initializer_list<int> slots,
              std::initializer_list<double> num, std::initializer_list<double> den);
  int check_fault_flags() const;
  void begin_step(int i);
  void begin_attempt(int i);
  void consume(int i, double totErr);
  void finish_step(int i, double totErr, double used_dt);
  const int* d_copy(const BatchGroup& g) const;
  const int* d_acc(const BatchGroup& g) const;
  const int* d_run(const BatchGroup& g) const;
  const double* d_t() const;
  const double* d_dt_() const;
};

}  // namespace scy
