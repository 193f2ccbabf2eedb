// scy_sbp_solve_noalloc: the elliptic solve for callers that cannot allocate
// device memory.
//
// cudaMalloc / cudaFree may synchronise the whole device and can fail when
// another allocator (a framework's caching pool, a memory manager that
// reserved the device up front) already holds the free memory.  A caller
// that runs its time-step loop under such an allocator, or cannot afford an
// implicit device synchronisation between stages, gets this variant: it
// allocates nothing.  Its CG work vectors and reduction partials live in one
// file-scope __device__ array of fixed size, held by every GPU that loads
// the library until the process exits.
//
// Limits and sharing:
// * at most kNoAllocMaxNodes = 65,536 grid nodes (e.g. 256 x 256); larger
//   grids are rejected with SCY_ERR_ARG;
// * the preconditioner is point Jacobi (the multigrid hierarchy of
//   scy_sbp_solve would need allocations), so it takes more iterations;
// * every call uses the same array and leaves its contents behind: the call
//   clears what must start at zero itself, and calls that overlap on the GPU
//   (different streams, threads or contexts at the same time) race on it.
// * the address of the array is looked up once per device, on the first call
//   made with that device current (cudaGetSymbolAddress).  With lazy module
//   loading (CUDA_MODULE_LOADING=LAZY, the default) that first call is also
//   when the module is loaded on the device and the array's memory is
//   reserved, so it may itself need about 2.6 MB of free device memory:
//   make the first call on each device before another allocator reserves
//   the device, and outside any code that forbids runtime set-up calls.
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "sbp_dev.cuh"
#include "sbp_solver.hpp"

namespace scy {

constexpr long kNoAllocMaxNodes = 65536;
constexpr int kNoAllocPartials = 2048;  // >= blocks of any reduction below
// layout (doubles): r | z | p0 | p1 | q | partials | scalars(16) | counter(2 doubles wide)
constexpr long kNoAllocDoubles = 5 * kNoAllocMaxNodes + kNoAllocPartials + 16 + 2;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

namespace {
std::mutex g_addr_mu;
double* g_addr[64] = {nullptr};

int scratch_address(double** out) {
  int dev = 0;
  SCY_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("device ordinal %d out of range for the no-alloc scratch table", dev);
    return SCY_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      set_error("cudaGetSymbolAddress of the no-alloc scratch failed: %s", cudaGetErrorString(e));
      return SCY_ERR_CUDA;
    }
    g_addr[dev] = static_cast<double*>(p);
  }
  *out = g_addr[dev];
  return SCY_OK;
}

__global__ void na_jacobi_dot_kernel(const double* __restrict__ r, const double* __restrict__ dinv,
                                     double* __restrict__ z, long n, double* partials, unsigned* counter,
                                     double* out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double zv = dinv[i] * r[i];
    z[i] = zv;
    acc += r[i] * zv;
  }
  double t = block_sum(acc, sh);
  grid_reduce_finish(t, partials, counter, out, sh);
}

__global__ void na_dot_kernel(const double* __restrict__ a, const double* __restrict__ b, long n, double* partials,
                              unsigned* counter, double* out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    acc += a[i] * b[i];
  double t = block_sum(acc, sh);
  grid_reduce_finish(t, partials, counter, out, sh);
}

__global__ void na_update_kernel(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                                 const double* __restrict__ q, const double* __restrict__ rz,
                                 const double* __restrict__ pq, long n, double* partials, unsigned* counter,
                                 double* out) {
  __shared__ double sh[32];
  const double pqv = *pq;
  const double alpha = pqv != 0.0 ? *rz / pqv : 0.0;
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    double rv = r[i] - alpha * q[i];
    r[i] = rv;
    acc += rv * rv;
  }
  double t = block_sum(acc, sh);
  grid_reduce_finish(t, partials, counter, out, sh);
}

__global__ void na_copy_scalar(double* dst, const double* src) { *dst = *src; }

template <class Ld, class Ep>
int na_stencil(const LevelDev<double>& L, Ld ld, Ep ep, double* partials, unsigned* counter, double* out,
               cudaStream_t s) {
  const dim3 g = apply_grid(L);
  if ((long)g.x * g.y > kNoAllocPartials) {
    set_error("grid of %u tiles exceeds the no-alloc partial-sum slots", g.x * g.y);
    return SCY_ERR_ARG;
  }
  launch_apply<double, Ld, Ep>(L, ld, ep, partials, counter, out, s);
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}
}  // namespace

int SbpContext::solve_noalloc(const double* rhs, double* u, const scy_solve_opts& o, scy_solve_stats& st) {
  const LevelDev<double>& L = fine->dev;
  const long n = (long)L.Ny * L.Nz;
  if (n > kNoAllocMaxNodes) {
    set_error("scy_sbp_solve_noalloc handles at most %ld grid nodes; this grid has %ld", kNoAllocMaxNodes, n);
    return SCY_ERR_ARG;
  }
  double* base = nullptr;
  SCY_TRY(scratch_address(&base));
  double* r = base;
  double* z = base + kNoAllocMaxNodes;
  double* p[2] = {base + 2 * kNoAllocMaxNodes, base + 3 * kNoAllocMaxNodes};
  double* q = base + 4 * kNoAllocMaxNodes;
  double* parts = base + 5 * kNoAllocMaxNodes;
  double* sc = parts + kNoAllocPartials;  // 0 ||rhs||^2, 1 r.r, 2 rz_new, 3 rz_old, 4 p.q
  unsigned* cnt = reinterpret_cast<unsigned*>(sc + 16);
  cudaStream_t s = stream;
  // the array keeps the previous call's contents: clear what must start at zero
  SCY_CUDA_TRY(cudaMemsetAsync(sc, 0, 18 * sizeof(double), s));
  SCY_CUDA_TRY(cudaMemsetAsync(p[0], 0, n * sizeof(double), s));
  const int rb = grid_for(n, 256, 1024);
  na_dot_kernel<<<rb, 256, 0, s>>>(rhs, rhs, n, parts, cnt, sc + 0);
  SCY_LAUNCH_CHECK();
  if (!o.nonzero_guess) SCY_CUDA_TRY(cudaMemsetAsync(u, 0, n * sizeof(double), s));
  SCY_TRY(na_stencil(L, LoadPlain<double>{u}, EpiResidual<double, double>{rhs, r, -1.0}, parts, cnt, sc + 1, s));
  double h2[2];
  SCY_CUDA_TRY(cudaMemcpyAsync(h2, sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  st.bnorm = std::sqrt(h2[0]);
  st.rnorm0 = std::sqrt(h2[1]);
  st.rnorm = st.rnorm0;
  st.iterations = 0;
  st.converged = 0;
  const double tol = std::max(o.rtol * st.bnorm, o.atol);
  if (h2[0] == 0.0 && tol == 0.0) {
    // zero right-hand side: the solution is zero (as in scy_sbp_solve; a
    // warm start would otherwise never reach ||r|| <= 0)
    SCY_CUDA_TRY(cudaMemsetAsync(u, 0, n * sizeof(double), s));
    st.rnorm = 0.0;
    st.converged = 1;
    return SCY_OK;
  }
  if (st.rnorm0 <= tol) {
    st.converged = 1;
    return SCY_OK;
  }
  const int check = o.check_every > 0 ? o.check_every : 1;
  int pi = 0;
  for (int it = 1; it <= o.max_its; ++it) {
    if (it > 1) na_copy_scalar<<<1, 1, 0, s>>>(sc + 3, sc + 2);
    na_jacobi_dot_kernel<<<rb, 256, 0, s>>>(r, L.dinv, z, n, parts, cnt, sc + 2);
    SCY_LAUNCH_CHECK();
    LoadPUpdate<double> lp{z, p[pi], sc + 2, sc + 3, it == 1 ? 1 : 0};
    SCY_TRY(na_stencil(L, lp, EpiCGMatvec{p[pi ^ 1], q}, parts, cnt, sc + 4, s));
    na_update_kernel<<<rb, 256, 0, s>>>(u, r, p[pi ^ 1], q, sc + 2, sc + 4, n, parts, cnt, sc + 1);
    SCY_LAUNCH_CHECK();
    pi ^= 1;
    st.iterations = it;
    if (it % check == 0 || it == o.max_its) {
      double rr = 0.0;
      SCY_CUDA_TRY(cudaMemcpyAsync(&rr, sc + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
      SCY_CUDA_TRY(cudaStreamSynchronize(s));
      st.rnorm = std::sqrt(rr);
      if (!std::isfinite(rr)) {
        set_error("non-finite residual in the elliptic solve");
        return SCY_ERR_NONFINITE;
      }
      if (st.rnorm <= tol) {
        st.converged = 1;
        break;
      }
    }
  }
  SCY_TRY(na_stencil(L, LoadPlain<double>{u}, EpiResidual<double, double>{rhs, r, -1.0}, parts, cnt, sc + 1, s));
  double rr = 0.0;
  SCY_CUDA_TRY(cudaMemcpyAsync(&rr, sc + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  st.rnorm = std::sqrt(rr);
  if (!std::isfinite(rr)) {
    set_error("non-finite residual in the elliptic solve");
    return SCY_ERR_NONFINITE;
  }
  // the recursive residual may have met the target while the true one
  // does not: the true residual decides
  st.converged = st.rnorm <= tol * 1.0000001 + 1e-300 ? 1 : 0;
  if (!st.converged) {
    set_error("elliptic solve stopped at ||r|| = %g after %d iterations (target %g)", st.rnorm, st.iterations, tol);
    return SCY_ERR_CG_NOCONV;
  }
  return SCY_OK;
}

}  // namespace scy
