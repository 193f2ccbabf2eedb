// SbpOps + elliptic solve on the device: context, multigrid hierarchy,
// preconditioned CG, and the SbpOps operator entry points of the C ABI.
//
// The reference solves A u = rhs with a MUMPS Cholesky factorisation
// (source/linearElastic.cpp:251-260, :475).  Here K = -A (symmetric positive
// definite) is solved with conjugate gradients in FP64, preconditioned by one
// geometric-multigrid V-cycle (rediscretised SBP-SAT operators on coarsened
// grids, Chebyshev-Jacobi smoothing, bilinear transfer, dense coarsest solve)
// run in FP64 or FP32.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

#include "common.cuh"
#include "sbp_dev.cuh"
#include "sbp_host.hpp"
#include "sbp_solver.hpp"
#include "fdiag.hpp"

namespace scy {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
const char* last_error() { return g_err; }

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(); }

// Optional per-launch timing of the stencil kernel (CUDA events around each
// launch); off unless scy_profile_enable(1) was called.
struct ProfRec {
  cudaEvent_t a, b;
  long long bytes;  // algorithmic bytes: read the operand and mu, write the result
  int level;
  int width;        // bytes per value (4 or 8)
};
static bool g_prof = false;
static std::vector<ProfRec> g_recs;
void profile_enable(int on) { g_prof = on != 0; }
int profile_collect(int level, int width, double* ms, long long* launches, double* bytes) {
  double tms = 0, tb = 0;
  long long nl = 0;
  for (auto& r : g_recs) {
    if (cudaEventSynchronize(r.b) != cudaSuccess) {
      set_error("profile event failed");
      return SCY_ERR_CUDA;
    }
    float m = 0;
    cudaEventElapsedTime(&m, r.a, r.b);
    if ((level < 0 || r.level == level) && (width == 0 || r.width == width)) {
      tms += m;
      tb += (double)r.bytes;
      ++nl;
    }
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  g_recs.clear();
  *ms = tms;
  *launches = nl;
  *bytes = tb;
  return SCY_OK;
}

// ------------------------------------------------------------------------
// device buffers
DevBuf::~DevBuf() { release(); }
void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}
int DevBuf::alloc(size_t b) {
  release();
  if (b == 0) b = 16;
  if (cudaMalloc(&p, b) != cudaSuccess) {
    cudaGetLastError();
    p = nullptr;
    set_error("cudaMalloc of %zu bytes failed", b);
    return SCY_ERR_NOMEM;
  }
  bytes = b;
  return SCY_OK;
}

template <typename T>
static int upload(DevBuf& buf, const std::vector<double>& v, cudaStream_t s) {
  std::vector<T> tmp(v.begin(), v.end());
  SCY_TRY(buf.alloc(tmp.size() * sizeof(T)));
  SCY_CUDA_TRY(cudaMemcpyAsync(buf.p, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  return SCY_OK;
}

template <typename T>
static int upload_ints(DevBuf& buf, const std::vector<int>& v, cudaStream_t s) {
  SCY_TRY(buf.alloc(v.size() * sizeof(int)));
  SCY_CUDA_TRY(cudaMemcpyAsync(buf.p, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  return SCY_OK;
}

template <typename T>
int LevelStore<T>::init(const LevelHost& h, cudaStream_t s) {
  Ny = h.Ny;
  Nz = h.Nz;
  const DirTables* td[2] = {&h.ty, &h.tz};
  for (int d = 0; d < 2; ++d) {
    const DirTables& t = *td[d];
    SCY_TRY(upload<T>(tab[d][0], t.D, s));
    SCY_TRY(upload<T>(tab[d][1], t.R3, s));
    SCY_TRY(upload<T>(tab[d][2], t.R4, s));
    SCY_TRY(upload<T>(tab[d][3], t.Q, s));
    SCY_TRY(upload<T>(tab[d][4], t.R3T, s));
    SCY_TRY(upload<T>(tab[d][5], t.R4T, s));
    SCY_TRY(upload<T>(tab[d][6], t.w3, s));
    SCY_TRY(upload<T>(tab[d][7], t.w4, s));
    SCY_TRY(upload<T>(tab[d][8], t.Hd, s));
    SCY_TRY(upload<T>(tab[d][9], t.Hinvd, s));
  }
  const std::vector<double>* f[10] = {&h.cy, &h.cz, &h.m3y, &h.m3z, &h.wy, &h.wz, &h.mu, &h.qy, &h.rz, nullptr};
  for (int i = 0; i < 9; ++i) SCY_TRY(upload<T>(fld[i], *f[i], s));
  std::vector<double> dinv(h.diagK.size());
  for (size_t i = 0; i < dinv.size(); ++i) dinv[i] = 1.0 / h.diagK[i];
  SCY_TRY(upload<T>(fld[9], dinv, s));
  dev.Ny = Ny;
  dev.Nz = Nz;
  dev.var = h.grid_type;
  for (int d = 0; d < 2; ++d) {
    DirDev<T>& D = d == 0 ? dev.y : dev.z;
    const DirTables& t = *td[d];
    D.n = t.n;
    D.D = tab[d][0].template as<T>();
    D.R3 = tab[d][1].template as<T>();
    D.R4 = t.nterms == 3 ? tab[d][2].template as<T>() : nullptr;
    D.Q = tab[d][3].template as<T>();
    D.R3T = tab[d][4].template as<T>();
    D.R4T = t.nterms == 3 ? tab[d][5].template as<T>() : nullptr;
    D.w3 = tab[d][6].template as<T>();
    D.w4 = tab[d][7].template as<T>();
    D.Hd = tab[d][8].template as<T>();
    D.Hinvd = tab[d][9].template as<T>();
    for (int j = 0; j < BAND; ++j) {
      D.bs0[j] = (T)t.bs0[j];
      D.bsN[j] = (T)t.bsN[j];
    }
    D.alphaD = (T)t.alphaD;
    D.bc_lo = d == 0 ? h.bc[2] : h.bc[1];
    D.bc_hi = d == 0 ? h.bc[0] : h.bc[3];
    D.fast = (h.order == 4 && t.n >= 17) ? 1 : 0;
    if (D.fast) {
      const int m = t.n / 2;
      auto c = [&](const std::vector<double>& b, int off) { return (T)b[(size_t)m * BAND + off + HALF]; };
      const int od[4] = {-2, -1, 1, 2};
      for (int j = 0; j < 4; ++j) {
        D.cD[j] = c(t.D, od[j]);
        D.cQ[j] = c(t.Q, od[j]);
        D.cR3[j] = c(t.R3, j - 1);
        D.cR3T[j] = c(t.R3T, j - 2);
      }
      for (int j = 0; j < 5; ++j) {
        D.cR4[j] = c(t.R4, j - 2);
        D.cR4T[j] = c(t.R4T, j - 2);
      }
      D.cw3 = (T)t.w3[m];
      D.cw4 = (T)t.w4[m];
    }
  }
  dev.cy = fld[0].template as<T>();
  dev.cz = fld[1].template as<T>();
  dev.m3y = fld[2].template as<T>();
  dev.m3z = fld[3].template as<T>();
  dev.wy = fld[4].template as<T>();
  dev.wz = fld[5].template as<T>();
  dev.mu = fld[6].template as<T>();
  dev.qy = fld[7].template as<T>();
  dev.rz = fld[8].template as<T>();
  dev.dinv = fld[9].template as<T>();
  // separable interior (see LevelDev::sep): verified bitwise over the box
  // of nodes the interior fast path can read
  dev.sep = 0;
  if (dev.y.fast && dev.z.fast) {
    const int iy_ref = Ny / 2, iz_ref = Nz / 2;
    std::vector<double> cy1(Ny), m3y1(Ny), wz1(Ny), cz1(Nz), m3z1(Nz), wy1(Nz);
    for (int iy = 0; iy < Ny; ++iy) {
      const size_t i = (size_t)iy * Nz + iz_ref;
      cy1[iy] = h.cy[i];
      m3y1[iy] = h.m3y[i];
      wz1[iy] = h.wz[i];
    }
    for (int iz = 0; iz < Nz; ++iz) {
      const size_t i = (size_t)iy_ref * Nz + iz;
      cz1[iz] = h.cz[i];
      m3z1[iz] = h.m3z[i];
      wy1[iz] = h.wy[i];
    }
    bool ok = true;
    for (int iy = 4; ok && iy <= Ny - 6; ++iy)
      for (int iz = 4; iz <= Nz - 6; ++iz) {
        const size_t i = (size_t)iy * Nz + iz;
        if (h.cy[i] != cy1[iy] || h.m3y[i] != m3y1[iy] || h.wz[i] != wz1[iy] || h.cz[i] != cz1[iz] ||
            h.m3z[i] != m3z1[iz] || h.wy[i] != wy1[iz]) {
          ok = false;
          break;
        }
      }
    if (ok) {
      const std::vector<double>* v[6] = {&cy1, &m3y1, &wz1, &cz1, &m3z1, &wy1};
      for (int k = 0; k < 6; ++k) SCY_TRY(upload<T>(sep1[k], *v[k], s));
      // compose stage 2 (Q, D3^T, D4^T at offsets -2..2) with stage 1 (D, D3,
      // D4 at offsets -2..2, scaled per row by c, w3*m3, w4*c) into one
      // 9-point stencil per interior row; rows whose stage-1 rows leave the
      // interior band stay zero (the fast path never reaches them)
      auto compose = [](const DirDev<T>& d, int n, const std::vector<double>& c1, const std::vector<double>& m31,
                        std::vector<double>& C) {
        C.assign((size_t)n * BAND, 0.0);
        const int oQ[4] = {-2, -1, 1, 2}, oD[4] = {-2, -1, 1, 2};
        for (int i = 6; i <= n - 8; ++i) {
          double row[17] = {0};  // offsets -8..8
          for (int a = 0; a < 4; ++a) {  // Q * c * D
            const int k = i + oQ[a];
            for (int b = 0; b < 4; ++b) row[oQ[a] + oD[b] + 8] += (double)d.cQ[a] * c1[k] * (double)d.cD[b];
          }
          for (int a = 0; a < 4; ++a) {  // - D3^T * (w3 m3) * D3: D3^T at -2..1, D3 at -1..2
            const int k = i + a - 2;
            for (int b = 0; b < 4; ++b)
              row[(a - 2) + (b - 1) + 8] -= (double)d.cR3T[a] * (double)d.cw3 * m31[k] * (double)d.cR3[b];
          }
          for (int a = 0; a < 5; ++a) {  // - D4^T * (w4 c) * D4: both at -2..2
            const int k = i + a - 2;
            for (int b = 0; b < 5; ++b)
              row[(a - 2) + (b - 2) + 8] -= (double)d.cR4T[a] * (double)d.cw4 * c1[k] * (double)d.cR4[b];
          }
          for (int o = -4; o <= 4; ++o) C[(size_t)i * BAND + o + HALF] = row[o + 8];
        }
      };
      std::vector<double> Cy, Cz, CzT((size_t)BAND * Nz);
      compose(dev.y, Ny, cy1, m3y1, Cy);
      compose(dev.z, Nz, cz1, m3z1, Cz);
      for (int iz = 0; iz < Nz; ++iz)
        for (int o = 0; o < BAND; ++o) CzT[(size_t)o * Nz + iz] = Cz[(size_t)iz * BAND + o];
      SCY_TRY(upload<T>(comp[0], Cy, s));
      SCY_TRY(upload<T>(comp[1], CzT, s));
      dev.Cy = comp[0].template as<T>();
      dev.CzT = comp[1].template as<T>();
      dev.cy1 = sep1[0].template as<T>();
      dev.m3y1 = sep1[1].template as<T>();
      dev.wz1 = sep1[2].template as<T>();
      dev.cz1 = sep1[3].template as<T>();
      dev.m3z1 = sep1[4].template as<T>();
      dev.wy1 = sep1[5].template as<T>();
      dev.sep = 1;
    }
    // the full form (LevelDev::full, build_full_form); its outer weights
    // are the separable interior's where that exists
    FullForm F;
    if (build_full_form(h, F)) {
      SCY_TRY(upload<T>(comp17[0], F.Cy17, s));
      SCY_TRY(upload<T>(comp17[1], F.CzT17, s));
      SCY_TRY(upload_ints<T>(cls[0], F.ycls, s));
      SCY_TRY(upload_ints<T>(cls[1], F.zcls, s));
      dev.Cy17 = comp17[0].template as<T>();
      dev.CzT17 = comp17[1].template as<T>();
      dev.ycls = cls[0].template as<int>();
      dev.zcls = cls[1].template as<int>();
      dev.full = 1;
      if (!dev.sep) {
        SCY_TRY(upload<T>(fullw[0], F.wy1, s));
        SCY_TRY(upload<T>(fullw[1], F.wz1, s));
        dev.wy1 = fullw[0].template as<T>();
        dev.wz1 = fullw[1].template as<T>();
      }
      dev.ylo = F.ylo;
      dev.yhi = F.yhi;
      dev.zlo = F.zlo;
      dev.zhi = F.zhi;
      // whether the interior box's rows (columns) all carry the same 9
      // entries in the stored precision (a constant grid)
      auto same9 = [](int lo, int hi, auto entry, int& same, T* c9) {
        same = lo <= hi ? 1 : 0;
        for (int i = lo; same && i <= hi; ++i)
          for (int o = 0; o < BAND; ++o)
            if ((T)entry(i, o) != (T)entry(lo, o)) same = 0;
        for (int o = 0; o < BAND; ++o) c9[o] = same ? (T)entry(lo, o) : T(0);
      };
      same9(F.ylo, F.yhi, [&](int i, int o) { return F.Cy17[(size_t)i * 17 + 8 - HALF + o]; }, dev.crow, dev.cyc);
      same9(F.zlo, F.zhi, [&](int i, int o) { return F.CzT17[(size_t)(8 - HALF + o) * Nz + i]; }, dev.ccol,
            dev.czc);
      // rows per thread: the tallest tile that still gives about six
      // blocks per SM (SCY_FULL_RPT = 1, 2 or 4 overrides)
      const long cols = (Nz + TZ - 1) / TZ;
      dev.rpt = 1;
      for (int r : {4, 2})
        if (cols * ((Ny + 8 * r - 1) / (8 * r)) >= 6L * kNumSMs) {
          dev.rpt = r;
          break;
        }
      if (const char* e = getenv("SCY_FULL_RPT")) {
        const int r = atoi(e);
        if (r == 1 || r == 2 || r == 4) dev.rpt = r;
      }
    }
  }
  return SCY_OK;
}

template struct LevelStore<double>;
template struct LevelStore<float>;

template <typename T, class Ld, class Ep>
static int launch_stencil(const LevelDev<T>& L, Ld ld, Ep ep, Reducer* red, double* out, cudaStream_t s,
                          int level = 0) {
  double* parts = red ? red->partials.template as<double>() : nullptr;
  unsigned* cnt = red ? red->counter.template as<unsigned>() : nullptr;
  ProfRec rec{};
  if (g_prof) {
    cudaEventCreate(&rec.a);
    cudaEventCreate(&rec.b);
    cudaEventRecord(rec.a, s);
  }
  launch_apply<T, Ld, Ep>(L, ld, ep, parts, cnt, out, s);
  SCY_LAUNCH_CHECK();
  if (g_prof) {
    cudaEventRecord(rec.b, s);
    rec.bytes = 3LL * (long long)sizeof(T) * (long long)L.Ny * L.Nz;
    rec.level = level;
    rec.width = (int)sizeof(T);
    g_recs.push_back(rec);
  }
  return SCY_OK;
}

// ------------------------------------------------------------------------
// elementwise kernels
template <typename T, typename Tin>
__global__ void cheb_first_kernel(const Tin* __restrict__ b_in, T* __restrict__ b_keep, const T* __restrict__ dinv,
                                  T* __restrict__ d, T* __restrict__ x, T c2, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    T bv = (T)b_in[i];
    if (b_keep) b_keep[i] = bv;
    T dv = c2 * dinv[i] * bv;
    d[i] = dv;
    x[i] = dv;
  }
}

template <typename T>
__global__ void restrict_kernel(const T* __restrict__ rf, T* __restrict__ bc, int Nfz, int Ncy, int Ncz,
                                const int* __restrict__ ylo, const int* __restrict__ yhi,
                                const int* __restrict__ zlo, const int* __restrict__ zhi,
                                const int* __restrict__ jy, const T* __restrict__ wy0, const T* __restrict__ wy1,
                                const int* __restrict__ jz, const T* __restrict__ wz0, const T* __restrict__ wz1) {
  long n = (long)Ncy * Ncz;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
    int a = (int)(c / Ncz), bb = (int)(c % Ncz);
    T acc = T(0);
    for (int iy = ylo[a]; iy <= yhi[a]; ++iy) {
      T wy = (jy[iy] == a ? wy0[iy] : T(0)) + (jy[iy] + 1 == a ? wy1[iy] : T(0));
      if (wy == T(0)) continue;
      T accz = T(0);
      for (int iz = zlo[bb]; iz <= zhi[bb]; ++iz) {
        T wz = (jz[iz] == bb ? wz0[iz] : T(0)) + (jz[iz] + 1 == bb ? wz1[iz] : T(0));
        accz += wz * rf[(long)iy * Nfz + iz];
      }
      acc += wy * accz;
    }
    bc[c] = acc;
  }
}

// out = M b with a dense n x n matrix; one warp per row.
template <typename T>
__global__ void dense_matvec_kernel(const T* __restrict__ M, const T* __restrict__ b, T* __restrict__ out, int n) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  const T* row = M + (long)warp * n;
  T acc = T(0);
  for (int j = lane; j < n; j += 32) acc += row[j] * b[j];
  acc = warp_sum(acc);
  if (lane == 0) out[warp] = acc;
}

// w = dinv .* v ; returns ||w||^2 and w.v through the reducer
template <typename T>
__global__ void power_step_kernel(const T* __restrict__ Kv, const T* __restrict__ dinv, T* __restrict__ w, long n,
                                  double* partials, unsigned* counter, double* out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    T v = dinv[i] * Kv[i];
    w[i] = v;
    acc += (double)v * (double)v;
  }
  double t = block_sum(acc, sh);
  grid_reduce_finish(t, partials, counter, out, sh);
}

template <typename T>
__global__ void scale_kernel(T* __restrict__ v, const double* __restrict__ nrm2, long n) {
  double s = 1.0 / sqrt(*nrm2);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) v[i] = (T)(v[i] * s);
}

// dot(a, b) for a in double and b in T
template <typename Ta, typename Tb>
__global__ void dot_kernel(const Ta* __restrict__ a, const Tb* __restrict__ b, long n, double* partials,
                           unsigned* counter, double* out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    acc += (double)a[i] * (double)b[i];
  double t = block_sum(acc, sh);
  grid_reduce_finish(t, partials, counter, out, sh);
}

// Error-free transformation of a sum (Knuth's TwoSum): a + b = s + e
// exactly.  The _rn intrinsics keep the compiler from contracting or
// reordering the operations.
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}

// r = rhs - A x over the cross form (C: 33 planes of N, offsets -8..8 along
// y, then -8..-1 and 1..8 along z), with every product split exactly by an
// FMA (c x = p + pe) and the sum carried as hi + lo: the rounding of A x
// does not enter r.
__global__ void residual_dd_kernel(const double* __restrict__ C, const double* __restrict__ x,
                                   const double* __restrict__ rhs, double* __restrict__ r, int Ny, int Nz) {
  const long N = (long)Ny * Nz;
  for (long node = blockIdx.x * (long)blockDim.x + threadIdx.x; node < N; node += (long)gridDim.x * blockDim.x) {
    const int iy = (int)(node / Nz), iz = (int)(node % Nz);
    double hi = 0.0, lo = 0.0;
    auto add = [&](double c, double v) {
      const double p = __dmul_rn(c, v);
      const double pe = fma(c, v, -p);
      double s, e;
      two_sum(hi, p, s, e);
      hi = s;
      lo = __dadd_rn(lo, __dadd_rn(e, pe));
    };
    for (int o = -8; o <= 8; ++o) {
      const int jy = iy + o;
      if (jy >= 0 && jy < Ny) add(C[(long)(o + 8) * N + node], x[(long)jy * Nz + iz]);
    }
    for (int o = -8; o <= 8; ++o) {
      const int jz = iz + o;
      if (o != 0 && jz >= 0 && jz < Nz) add(C[(long)(o < 0 ? 25 + o : 24 + o) * N + node], x[(long)iy * Nz + jz]);
    }
    double s, e;
    two_sum(rhs[node], -hi, s, e);
    r[node] = __dadd_rn(s, __dsub_rn(e, lo));
  }
}

// x += alpha p ; r -= alpha q ; returns r.r   (alpha = rz/pq)
__global__ void cg_update_kernel(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                                 const double* __restrict__ q, const double* __restrict__ rz,
                                 const double* __restrict__ pq, long n, double* partials, unsigned* counter,
                                 double* out) {
  __shared__ double sh[32];
  const double pqv = *pq;
  const double alpha = pqv != 0.0 ? *rz / pqv : 0.0;  // zero search direction: nothing to add
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

__global__ void copy_scalar_kernel(double* dst, const double* src) { *dst = *src; }

// ------------------------------------------------------------------------
int Reducer::init(int max_blocks) {
  SCY_TRY(partials.alloc(sizeof(double) * max_blocks));
  SCY_TRY(counter.alloc(sizeof(unsigned) * 4));
  SCY_CUDA_TRY(cudaMemset(counter.p, 0, sizeof(unsigned) * 4));
  return SCY_OK;
}

static int red_blocks(long n) { return grid_for(n, 256, 1024); }

// ------------------------------------------------------------------------
template <typename T>
int Multigrid<T>::init(const std::vector<LevelHost>& hosts, const std::vector<Transfer>& xfer, cudaStream_t s) {
  nlev = (int)hosts.size();
  lev.resize(nlev);
  work.resize(nlev);
  for (int l = 0; l < nlev; ++l) {
    lev[l].reset(new LevelStore<T>());
    SCY_TRY(lev[l]->init(hosts[l], s));
    long n = (long)hosts[l].Ny * hosts[l].Nz;
    for (int k = 0; k < 5; ++k) SCY_TRY(work[l].v[k].alloc(n * sizeof(T)));
  }
  tr.resize(nlev > 0 ? nlev - 1 : 0);
  for (int l = 0; l + 1 < nlev; ++l) {
    const Transfer& t = xfer[l];
    TransferDev& d = tr[l];
    SCY_TRY(upload_ints<T>(d.jy, t.iy.j0, s));
    SCY_TRY(upload<T>(d.wy0, t.iy.w0, s));
    SCY_TRY(upload<T>(d.wy1, t.iy.w1, s));
    SCY_TRY(upload_ints<T>(d.jz, t.iz.j0, s));
    SCY_TRY(upload<T>(d.wz0, t.iz.w0, s));
    SCY_TRY(upload<T>(d.wz1, t.iz.w1, s));
    SCY_TRY(upload_ints<T>(d.ylo, t.ylo, s));
    SCY_TRY(upload_ints<T>(d.yhi, t.yhi, s));
    SCY_TRY(upload_ints<T>(d.zlo, t.zlo, s));
    SCY_TRY(upload_ints<T>(d.zhi, t.zhi, s));
  }
  return SCY_OK;
}

template struct Multigrid<double>;
template struct Multigrid<float>;

// ------------------------------------------------------------------------
// Builds the hierarchy of grids, the transfers between them, the spectral
// bounds for the Chebyshev smoother and the dense inverse at the coarsest grid.
static std::vector<double> sample_field(const std::vector<double>& f, int Nfy, int Nfz, int Ncy, int Ncz) {
  std::vector<double> out((size_t)Ncy * Ncz);
  for (int a = 0; a < Ncy; ++a) {
    double sy = Ncy > 1 ? (double)a * (Nfy - 1) / (Ncy - 1) : 0.0;
    int i0 = std::min((int)std::floor(sy), Nfy - 2);
    double wy = sy - i0;
    for (int b = 0; b < Ncz; ++b) {
      double sz = Ncz > 1 ? (double)b * (Nfz - 1) / (Ncz - 1) : 0.0;
      int k0 = std::min((int)std::floor(sz), Nfz - 2);
      double wz = sz - k0;
      auto F = [&](int i, int k) { return f[(size_t)i * Nfz + k]; };
      out[(size_t)a * Ncz + b] = (1 - wy) * ((1 - wz) * F(i0, k0) + wz * F(i0, k0 + 1)) +
                                 wy * ((1 - wz) * F(i0 + 1, k0) + wz * F(i0 + 1, k0 + 1));
    }
  }
  return out;
}

static Transfer make_transfer(int Nfy, int Nfz, int Ncy, int Ncz) {
  Transfer t;
  t.iy = make_interp(Nfy, Ncy);
  t.iz = make_interp(Nfz, Ncz);
  auto ranges = [](const Interp1D& I, std::vector<int>& lo, std::vector<int>& hi) {
    lo.assign(I.nc, I.nf);
    hi.assign(I.nc, -1);
    for (int i = 0; i < I.nf; ++i) {
      for (int j : {I.j0[i], I.j0[i] + 1}) {
        if (j < 0 || j >= I.nc) continue;
        lo[j] = std::min(lo[j], i);
        hi[j] = std::max(hi[j], i);
      }
    }
  };
  ranges(t.iy, t.ylo, t.yhi);
  ranges(t.iz, t.zlo, t.zhi);
  return t;
}

int build_hierarchy(const scy_grid_desc& g, const std::vector<double>& y, const std::vector<double>& z,
                    const std::vector<double>& mu, const int bc[4], std::vector<LevelHost>& hosts,
                    std::vector<Transfer>& xfer) {
  hosts.clear();
  xfer.clear();
  try {
    hosts.push_back(build_level(g.order, g.Ny, g.Nz, g.Ly, g.Lz, g.grid_type, g.compat, y, z, mu, bc));
    const int nmin = g.order == 4 ? 9 : 3;
    std::vector<double> cy_y = y, cy_z = z, cmu = mu;
    while (true) {
      const LevelHost& f = hosts.back();
      long N = (long)f.Ny * f.Nz;
      if (N <= 400) break;
      int ny = f.Ny >= 2 * nmin - 1 ? (f.Ny + 1) / 2 : f.Ny;
      int nz = f.Nz >= 2 * nmin - 1 ? (f.Nz + 1) / 2 : f.Nz;
      if (ny == f.Ny && nz == f.Nz) break;
      std::vector<double> ny_y, ny_z;
      if (g.grid_type == 1) {
        std::vector<double> fy = cy_y, fz = cy_z;
        if (fy.empty()) {
          fy.resize((size_t)N);
          for (long i = 0; i < N; ++i) fy[i] = g.Ly * (double)(i / f.Nz) / (f.Ny - 1.0);
        }
        if (fz.empty()) {
          fz.resize((size_t)N);
          for (long i = 0; i < N; ++i) fz[i] = g.Lz * (double)(i % f.Nz) / (f.Nz - 1.0);
        }
        ny_y = sample_field(fy, f.Ny, f.Nz, ny, nz);
        ny_z = sample_field(fz, f.Ny, f.Nz, ny, nz);
      }
      std::vector<double> nmu = sample_field(cmu, f.Ny, f.Nz, ny, nz);
      xfer.push_back(make_transfer(f.Ny, f.Nz, ny, nz));
      hosts.push_back(build_level(g.order, ny, nz, g.Ly, g.Lz, g.grid_type, g.compat, ny_y, ny_z, nmu, bc));
      cy_y = ny_y;
      cy_z = ny_z;
      cmu = nmu;
    }
  } catch (const std::exception& e) {
    set_error("grid set-up failed: %s", e.what());
    return SCY_ERR_ARG;
  }
  return SCY_OK;
}

// Dense inverse of K at the coarsest grid (Cholesky on the host).
static int dense_inverse(const LevelHost& h, std::vector<double>& inv) {
  const int n = h.Ny * h.Nz;
  std::vector<double> K((size_t)n * n), e(n, 0.0), col(n);
  for (int j = 0; j < n; ++j) {
    e[j] = 1.0;
    h.apply_A(e.data(), col.data());
    e[j] = 0.0;
    for (int i = 0; i < n; ++i) K[(size_t)i * n + j] = -col[i];
  }
  // symmetrise (the operator is symmetric up to round-off)
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      double a = 0.5 * (K[(size_t)i * n + j] + K[(size_t)j * n + i]);
      K[(size_t)i * n + j] = K[(size_t)j * n + i] = a;
    }
  std::vector<double> Lm((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    double s = K[(size_t)j * n + j];
    for (int k = 0; k < j; ++k) s -= Lm[(size_t)j * n + k] * Lm[(size_t)j * n + k];
    if (!(s > 0.0)) {
      set_error("coarse operator is not positive definite (pivot %d = %g)", j, s);
      return SCY_ERR_ARG;
    }
    double d = std::sqrt(s);
    Lm[(size_t)j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double t = K[(size_t)i * n + j];
      for (int k = 0; k < j; ++k) t -= Lm[(size_t)i * n + k] * Lm[(size_t)j * n + k];
      Lm[(size_t)i * n + j] = t / d;
    }
  }
  inv.assign((size_t)n * n, 0.0);
  std::vector<double> v(n);
  for (int c = 0; c < n; ++c) {
    for (int i = 0; i < n; ++i) {
      double t = (i == c) ? 1.0 : 0.0;
      for (int k = 0; k < i; ++k) t -= Lm[(size_t)i * n + k] * v[k];
      v[i] = t / Lm[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
      double t = v[i];
      for (int k = i + 1; k < n; ++k) t -= Lm[(size_t)k * n + i] * v[k];
      v[i] = t / Lm[(size_t)i * n + i];
    }
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + c] = v[i];
  }
  return SCY_OK;
}

// ------------------------------------------------------------------------
template <typename T>
int Multigrid<T>::setup_smoothers(const std::vector<LevelHost>& hosts, Reducer& red, double* dscal,
                                  cudaStream_t s) {
  cheb.assign(nlev, {});
  for (int l = 0; l + 1 < nlev; ++l) {
    // power iteration on diag(K)^-1 K at this level
    long n = (long)hosts[l].Ny * hosts[l].Nz;
    std::vector<T> v0(n);
    uint64_t st = 0x9E3779B97F4A7C15ull;
    for (long i = 0; i < n; ++i) {
      st ^= st << 13; st ^= st >> 7; st ^= st << 17;
      v0[i] = (T)(0.5 + (double)(st % 1000003) / 1000003.0);
    }
    T* v = work[l].v[0].template as<T>();
    T* Kv = work[l].v[1].template as<T>();
    SCY_CUDA_TRY(cudaMemcpyAsync(v, v0.data(), n * sizeof(T), cudaMemcpyHostToDevice, s));
    double lam = 0.0;
    for (int it = 0; it < 20; ++it) {
      SCY_TRY(launch_stencil<T>(lev[l]->dev, LoadPlain<T>{v}, EpiStore<T>{Kv, T(-1)}, nullptr, nullptr, s));
      power_step_kernel<T><<<red_blocks(n), 256, 0, s>>>(Kv, lev[l]->dev.dinv, v, n,
                                                          red.partials.template as<double>(),
                                                          red.counter.template as<unsigned>(), dscal);
      SCY_LAUNCH_CHECK();
      double nrm2 = 0.0;
      SCY_CUDA_TRY(cudaMemcpyAsync(&nrm2, dscal, sizeof(double), cudaMemcpyDeviceToHost, s));
      SCY_CUDA_TRY(cudaStreamSynchronize(s));
      lam = std::sqrt(nrm2);  // v had unit norm after the first normalisation
      scale_kernel<T><<<red_blocks(n), 256, 0, s>>>(v, dscal, n);
      SCY_LAUNCH_CHECK();
      if (it == 0) lam = 0.0;
    }
    if (!(lam > 0.0) || !std::isfinite(lam)) {
      set_error("smoother spectral estimate failed on level %d", l);
      return SCY_ERR_ARG;
    }
    double lmax = 1.1 * lam, lmin = lmax / 8.0;
    double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin), sigma = theta / delta;
    double rho = 1.0 / sigma;
    cheb[l].resize(nu);
    cheb[l][0] = {0.0, 1.0 / theta};
    for (int k = 1; k < nu; ++k) {
      double rn = 1.0 / (2.0 * sigma - rho);
      cheb[l][k] = {rn * rho, 2.0 * rn / delta};
      rho = rn;
    }
    lambda.push_back(lam);
  }
  // dense inverse at the coarsest level
  std::vector<double> inv;
  SCY_TRY(dense_inverse(hosts[nlev - 1], inv));
  SCY_TRY(upload<T>(coarse_inv, inv, s));
  ncoarse = hosts[nlev - 1].Ny * hosts[nlev - 1].Nz;
  return SCY_OK;
}

// z = V-cycle(b) at level l.  b_in is the level-0 right-hand side (any
// precision); the result is left in work[0] x buffer (returned pointer).
template <typename T>
template <typename Tin>
int Multigrid<T>::vcycle(int l, const Tin* b_in, T** x_out, cudaStream_t s) {
  const LevelDev<T>& L = lev[l]->dev;
  long n = (long)L.Ny * L.Nz;
  T* xa = work[l].v[0].template as<T>();
  T* xb = work[l].v[1].template as<T>();
  T* d = work[l].v[2].template as<T>();
  T* b = work[l].v[3].template as<T>();
  T* r = work[l].v[4].template as<T>();
  if (l == nlev - 1) {
    const T* bb = (const T*)b_in;
    if (!std::is_same<Tin, T>::value) {
      cheb_first_kernel<T, Tin><<<grid_for(n), 256, 0, s>>>(b_in, b, L.dinv, d, xa, T(0), n);
      SCY_LAUNCH_CHECK();
      bb = b;
    }
    int warps_per_block = 8;
    dense_matvec_kernel<T><<<(ncoarse + warps_per_block - 1) / warps_per_block, 256, 0, s>>>(
        coarse_inv.template as<T>(), bb, xa, ncoarse);
    SCY_LAUNCH_CHECK();
    *x_out = xa;
    return SCY_OK;
  }
  // pre-smoothing (x starts at zero)
  const T* bl = std::is_same<Tin, T>::value ? (const T*)b_in : b;
  cheb_first_kernel<T, Tin><<<grid_for(n), 256, 0, s>>>(b_in, std::is_same<Tin, T>::value ? nullptr : b, L.dinv,
                                                       d, xa, (T)cheb[l][0].c2, n);
  SCY_LAUNCH_CHECK();
  T* x = xa;
  T* xo = xb;
  for (int k = 1; k < nu; ++k) {
    SCY_TRY(launch_stencil<T>(L, LoadPlain<T>{x}, EpiCheb<T>{bl, L.dinv, d, xo, (T)cheb[l][k].c1, (T)cheb[l][k].c2},
                              nullptr, nullptr, s, l));
    std::swap(x, xo);
  }
  // residual and restriction
  SCY_TRY(launch_stencil<T>(L, LoadPlain<T>{x}, EpiResidual<T, T>{bl, r, T(1)}, nullptr, nullptr, s, l));
  const LevelDev<T>& C = lev[l + 1]->dev;
  long nc = (long)C.Ny * C.Nz;
  T* bcoarse = work[l + 1].v[3].template as<T>();
  const TransferDev& t = tr[l];
  restrict_kernel<T><<<grid_for(nc), 256, 0, s>>>(r, bcoarse, L.Nz, C.Ny, C.Nz, t.ylo.template as<int>(),
                                                  t.yhi.template as<int>(), t.zlo.template as<int>(),
                                                  t.zhi.template as<int>(), t.jy.template as<int>(),
                                                  t.wy0.template as<T>(), t.wy1.template as<T>(),
                                                  t.jz.template as<int>(), t.wz0.template as<T>(),
                                                  t.wz1.template as<T>());
  SCY_LAUNCH_CHECK();
  T* xc = nullptr;
  SCY_TRY(vcycle<T>(l + 1, bcoarse, &xc, s));
  // post-smoothing: the first step folds in the coarse-grid correction
  LoadProlong<T> lp{x, xc, C.Nz, t.jy.template as<int>(), t.jz.template as<int>(), t.wy0.template as<T>(),
                    t.wy1.template as<T>(), t.wz0.template as<T>(), t.wz1.template as<T>()};
  SCY_TRY(launch_stencil<T>(L, lp, EpiCheb<T>{bl, L.dinv, d, xo, T(0), (T)cheb[l][0].c2}, nullptr, nullptr, s, l));
  std::swap(x, xo);
  for (int k = 1; k < nu; ++k) {
    SCY_TRY(launch_stencil<T>(L, LoadPlain<T>{x}, EpiCheb<T>{bl, L.dinv, d, xo, (T)cheb[l][k].c1, (T)cheb[l][k].c2},
                              nullptr, nullptr, s, l));
    std::swap(x, xo);
  }
  *x_out = x;
  return SCY_OK;
}

template int Multigrid<double>::vcycle<double>(int, const double*, double**, cudaStream_t);
template int Multigrid<float>::vcycle<double>(int, const double*, float**, cudaStream_t);

// ------------------------------------------------------------------------
// operator kernels of the SbpOps interface
enum class Dir { Y, Z };

template <Dir d, int kind>  // kind 0: D, 1: mu*D, 2: D*mu
__global__ void deriv_kernel(LevelDev<double> L, const double* __restrict__ in, double* __restrict__ out) {
  const int Ny = L.Ny, Nz = L.Nz;
  long n = (long)Ny * Nz;
  for (long node = blockIdx.x * (long)blockDim.x + threadIdx.x; node < n; node += (long)gridDim.x * blockDim.x) {
    int iy = (int)(node / Nz), iz = (int)(node % Nz);
    double acc = 0.0;
    if (d == Dir::Y) {
      const double* row = L.y.D + (long)iy * BAND;
#pragma unroll
      for (int j = 0; j < BAND; ++j) {
        int k = iy + j - HALF;
        if (k >= 0 && k < Ny) {
          long kn = (long)k * Nz + iz;
          double v = in[kn];
          if (kind == 2) v *= L.mu[kn];
          acc += row[j] * v;
        }
      }
      if (L.var) acc *= L.qy[node];
    } else {
      const double* row = L.z.D + (long)iz * BAND;
#pragma unroll
      for (int j = 0; j < BAND; ++j) {
        int k = iz + j - HALF;
        if (k >= 0 && k < Nz) {
          long kn = (long)iy * Nz + k;
          double v = in[kn];
          if (kind == 2) v *= L.mu[kn];
          acc += row[j] * v;
        }
      }
      if (L.var) acc *= L.rz[node];
    }
    if (kind == 1) acc *= L.mu[node];
    out[node] = acc;
  }
}

__global__ void hmul_kernel(LevelDev<double> L, const double* __restrict__ in, double* __restrict__ out, int inv) {
  const int Nz = L.Nz;
  long n = (long)L.Ny * Nz;
  for (long node = blockIdx.x * (long)blockDim.x + threadIdx.x; node < n; node += (long)gridDim.x * blockDim.x) {
    int iy = (int)(node / Nz), iz = (int)(node % Nz);
    double h = inv ? L.y.Hinvd[iy] * L.z.Hinvd[iz] : L.y.Hd[iy] * L.z.Hd[iz];
    out[node] = h * in[node];
  }
}

// rhs = rhsL*bcL + rhsR*bcR + rhsT*bcT + rhsB*bcB (one output per node).
__global__ void set_rhs_kernel(LevelDev<double> L, const double* __restrict__ bcL, const double* __restrict__ bcR,
                               const double* __restrict__ bcT, const double* __restrict__ bcB,
                               double* __restrict__ rhs) {
  long n = (long)L.Ny * L.Nz;
  for (long node = blockIdx.x * (long)blockDim.x + threadIdx.x; node < n; node += (long)gridDim.x * blockDim.x)
    rhs[node] = set_rhs_node(L, bcL, bcR, bcT, bcB, node);
}

// ------------------------------------------------------------------------
SbpContext::SbpContext() = default;
SbpContext::~SbpContext() = default;

int SbpContext::create(const scy_grid_desc& g) {
  desc = g;
  if (g.order != 2 && g.order != 4) {
    set_error("order must be 2 or 4 (got %d)", g.order);
    return SCY_ERR_ARG;
  }
  if (g.Ny < 2 || g.Nz < 2) {
    set_error("Ny and Nz must both exceed 1 (got %d x %d)", g.Ny, g.Nz);
    return SCY_ERR_ARG;
  }
  if (!(g.Ly > 0) || !(g.Lz > 0)) {
    set_error("Ly and Lz must be positive");
    return SCY_ERR_ARG;
  }
  const long N = (long)g.Ny * g.Nz;
  if (!g.mu) {
    set_error("mu must be given");
    return SCY_ERR_ARG;
  }
  mu.assign(g.mu, g.mu + N);
  if (g.grid_type == SCY_GRID_VAR) {
    if (g.y) y.assign(g.y, g.y + N);
    if (g.z) z.assign(g.z, g.z + N);
  }
  bc[0] = g.bcR; bc[1] = g.bcT; bc[2] = g.bcL; bc[3] = g.bcB;
  for (int i = 0; i < 4; ++i)
    if (bc[i] != 0 && bc[i] != 1) {
      set_error("boundary types must be SCY_BC_DIRICHLET or SCY_BC_NEUMANN");
      return SCY_ERR_ARG;
    }
  const int tiles = ((g.Nz + TZ - 1) / TZ) * ((g.Ny + TY - 1) / TY);
  SCY_TRY(red.init(1024 + tiles));
  SCY_TRY(scal.alloc(sizeof(double) * 16));
  SCY_CUDA_TRY(cudaMemset(scal.p, 0, sizeof(double) * 16));
  long n = N;
  SCY_TRY(cg_r.alloc(n * 8));
  SCY_TRY(cg_p[0].alloc(n * 8));
  SCY_TRY(cg_p[1].alloc(n * 8));
  SCY_TRY(cg_q.alloc(n * 8));
  SCY_TRY(cg_z.alloc(n * 8));
  SCY_TRY(cg_z32.alloc(n * 4));
  SCY_CUDA_TRY(cudaMemset(cg_p[0].p, 0, n * 8));
  SCY_CUDA_TRY(cudaMemset(cg_p[1].p, 0, n * 8));
  return rebuild();
}

int SbpContext::rebuild() {
  SCY_TRY(build_hierarchy(desc, y, z, mu, bc, hosts, xfer));
  {
    // separable: yq depends only on iy, zr only on iz, mu constant
    const LevelHost& h = hosts[0];
    bool sep = true;
    const double tol = 1e-12;
    for (int iy = 0; iy < h.Ny && sep; ++iy)
      for (int iz = 0; iz < h.Nz && sep; ++iz) {
        size_t i = (size_t)iy * h.Nz + iz;
        if (std::fabs(h.yq[i] - h.yq[(size_t)iy * h.Nz]) > tol * std::fabs(h.yq[(size_t)iy * h.Nz])) sep = false;
        if (std::fabs(h.zr[i] - h.zr[iz]) > tol * std::fabs(h.zr[iz])) sep = false;
        if (std::fabs(h.mu[i] - h.mu[0]) > tol * std::fabs(h.mu[0])) sep = false;
      }
    separable = sep ? 1 : 0;
  }
  cross.release();
  fd.reset();
  fine.reset(new LevelStore<double>());
  SCY_TRY(fine->init(hosts[0], stream));
  mg64.reset();
  mg32.reset();
  return SCY_OK;
}

template <typename T>
int SbpContext::ensure_mg(std::unique_ptr<Multigrid<T>>& mg) {
  if (mg) return SCY_OK;
  mg.reset(new Multigrid<T>());
  SCY_TRY(mg->init(hosts, xfer, stream));
  SCY_TRY(mg->setup_smoothers(hosts, red, scal.as<double>() + 8, stream));
  return SCY_OK;
}

int SbpContext::apply(int op, const double* in, double* out) {
  const LevelDev<double>& L = fine->dev;
  long n = (long)L.Ny * L.Nz;
  int g = grid_for(n);
  switch (op) {
    case SCY_OP_A:
      return launch_stencil<double>(L, LoadPlain<double>{in}, EpiStore<double>{out, 1.0}, nullptr, nullptr, stream);
    case SCY_OP_DY: deriv_kernel<Dir::Y, 0><<<g, 256, 0, stream>>>(L, in, out); break;
    case SCY_OP_DZ: deriv_kernel<Dir::Z, 0><<<g, 256, 0, stream>>>(L, in, out); break;
    case SCY_OP_MUXDY: deriv_kernel<Dir::Y, 1><<<g, 256, 0, stream>>>(L, in, out); break;
    case SCY_OP_MUXDZ: deriv_kernel<Dir::Z, 1><<<g, 256, 0, stream>>>(L, in, out); break;
    case SCY_OP_DYXMU: deriv_kernel<Dir::Y, 2><<<g, 256, 0, stream>>>(L, in, out); break;
    case SCY_OP_DZXMU: deriv_kernel<Dir::Z, 2><<<g, 256, 0, stream>>>(L, in, out); break;
    case SCY_OP_H: hmul_kernel<<<g, 256, 0, stream>>>(L, in, out, 0); break;
    case SCY_OP_HINV: hmul_kernel<<<g, 256, 0, stream>>>(L, in, out, 1); break;
    default:
      set_error("unknown operator %d", op);
      return SCY_ERR_ARG;
  }
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

int SbpContext::set_rhs(const double* bcL, const double* bcR, const double* bcT, const double* bcB, double* rhs) {
  const LevelDev<double>& L = fine->dev;
  long n = (long)L.Ny * L.Nz;
  set_rhs_kernel<<<grid_for(n), 256, 0, stream>>>(L, bcL, bcR, bcT, bcB, rhs);
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

template <typename Tz, class PC>
int SbpContext::pcg(PC&& pc, const double* rhs, double* u, const scy_solve_opts& o, scy_solve_stats& st) {
  const LevelDev<double>& L = fine->dev;
  const long n = (long)L.Ny * L.Nz;
  double* sc = scal.as<double>();
  // sc[0]=||rhs||^2, sc[1]=r.r, sc[2]=rz_new, sc[3]=rz_old, sc[4]=p.q, sc[5]=||r0||^2
  double* parts = red.partials.as<double>();
  unsigned* cnt = red.counter.as<unsigned>();
  double* r = cg_r.as<double>();
  double* q = cg_q.as<double>();
  const int rb = red_blocks(n);
  dot_kernel<double, double><<<rb, 256, 0, stream>>>(rhs, rhs, n, parts, cnt, sc + 0);
  SCY_LAUNCH_CHECK();
  if (!o.nonzero_guess) SCY_CUDA_TRY(cudaMemsetAsync(u, 0, n * sizeof(double), stream));
  // r = f - K u with f = -rhs, K = -A  ->  r = -rhs + A u
  SCY_TRY(launch_stencil<double>(L, LoadPlain<double>{u}, EpiResidual<double, double>{rhs, r, -1.0}, &red, sc + 5,
                                 stream));
  st.iterations = 0;
  st.converged = 0;
  const int check = o.check_every > 0 ? o.check_every : 1;
  double tol = -1.0;
  int pi = 0;
  // The first read-back happens after the first batch of `check` iterations
  // (a warm-started stage solve is never converged on entry); iterations
  // past convergence are harmless no-ops (alpha = 0).
  for (int it = 1; it <= o.max_its; ++it) {
    Tz* z = nullptr;
    SCY_TRY(pc((const double*)r, &z));
    if (it > 1) {
      copy_scalar_kernel<<<1, 1, 0, stream>>>(sc + 3, sc + 2);
      SCY_LAUNCH_CHECK();
    }
    dot_kernel<double, Tz><<<rb, 256, 0, stream>>>(r, z, n, parts, cnt, sc + 2);
    SCY_LAUNCH_CHECK();
    double* pold = cg_p[pi].as<double>();
    double* pnew = cg_p[pi ^ 1].as<double>();
    LoadPUpdate<Tz> lp{z, pold, sc + 2, sc + 3, it == 1 ? 1 : 0};
    SCY_TRY(launch_stencil<double>(L, lp, EpiCGMatvec{pnew, q}, &red, sc + 4, stream));
    cg_update_kernel<<<rb, 256, 0, stream>>>(u, r, pnew, q, sc + 2, sc + 4, n, parts, cnt, sc + 1);
    SCY_LAUNCH_CHECK();
    pi ^= 1;
    st.iterations = it;
    if (it % check == 0 || it == o.max_its) {
      double h[6];
      SCY_CUDA_TRY(cudaMemcpyAsync(h, sc, 6 * sizeof(double), cudaMemcpyDeviceToHost, stream));
      SCY_CUDA_TRY(cudaStreamSynchronize(stream));
      if (tol < 0) {
        st.bnorm = std::sqrt(h[0]);
        st.rnorm0 = std::sqrt(h[5]);
        tol = std::max(o.rtol * st.bnorm, o.atol);
        if (h[0] == 0.0 && tol == 0.0) {
          // zero right-hand side: the solution is zero (a warm start from
          // an earlier solve would otherwise never reach ||r|| <= 0)
          SCY_CUDA_TRY(cudaMemsetAsync(u, 0, n * sizeof(double), stream));
          st.rnorm = 0.0;
          st.converged = 1;
          return SCY_OK;
        }
      }
      st.rnorm = std::sqrt(h[1]);
      if (!std::isfinite(h[1])) {
        set_error("non-finite residual in the elliptic solve");
        return SCY_ERR_NONFINITE;
      }
      if (st.rnorm <= tol || st.rnorm0 <= tol) {
        st.converged = 1;
        break;
      }
    }
  }
  if (o.verify) {
    SCY_TRY(launch_stencil<double>(L, LoadPlain<double>{u}, EpiResidual<double, double>{rhs, r, -1.0}, &red, sc + 1,
                                   stream));
    double rr = 0.0;
    SCY_CUDA_TRY(cudaMemcpyAsync(&rr, sc + 1, sizeof(double), cudaMemcpyDeviceToHost, stream));
    SCY_CUDA_TRY(cudaStreamSynchronize(stream));
    st.rnorm = std::sqrt(rr);
    if (!std::isfinite(rr)) {
      set_error("non-finite residual in the elliptic solve");
      return SCY_ERR_NONFINITE;
    }
    st.converged = st.rnorm <= tol * 1.0000001 + 1e-300 ? 1 : 0;
  }
  if (!st.converged) {
    set_error("elliptic solve stopped at ||r|| = %g after %d iterations (target %g)", st.rnorm, st.iterations, tol);
    return SCY_ERR_CG_NOCONV;
  }
  return SCY_OK;
}

int SbpContext::ensure_fd() {
  if (fd && fd->ready) return SCY_OK;
  fd.reset(new FDPrecond());
  return fd->build(hosts[0], stream);
}

int SbpContext::solve(const double* rhs, double* u, const scy_solve_opts& o, scy_solve_stats& st) {
  const bool use_fd = o.precond == SCY_PC_FD || (o.precond == SCY_PC_AUTO && separable);
  if (use_fd) {
    SCY_TRY(ensure_fd());
    if (o.precision == SCY_PREC_MIXED) {
      float* z = cg_z32.as<float>();
      auto pc = [&](const double* r, float** zo) -> int {
        SCY_TRY(fd->apply32(r, z, stream));
        *zo = z;
        return SCY_OK;
      };
      return pcg<float>(pc, rhs, u, o, st);
    }
    double* z = cg_z.as<double>();
    auto pc = [&](const double* r, double** zo) -> int {
      SCY_TRY(fd->apply(r, z, stream));
      *zo = z;
      return SCY_OK;
    };
    return pcg<double>(pc, rhs, u, o, st);
  }
  if (o.precision == SCY_PREC_MIXED) {
    SCY_TRY(ensure_mg(mg32));
    auto pc = [&](const double* r, float** zo) -> int { return mg32->vcycle(0, r, zo, stream); };
    return pcg<float>(pc, rhs, u, o, st);
  }
  SCY_TRY(ensure_mg(mg64));
  auto pc = [&](const double* r, double** zo) -> int { return mg64->vcycle(0, r, zo, stream); };
  return pcg<double>(pc, rhs, u, o, st);
}

int SbpContext::residual_dd(const double* rhs, const double* u, double* r, double* rnorm2_host) {
  const LevelHost& h = hosts[0];
  const long n = (long)h.Ny * h.Nz;
  if (!cross.p) {
    std::vector<double> planes;
    build_cross_planes(h, planes);
    SCY_TRY(cross.alloc(planes.size() * sizeof(double)));
    SCY_CUDA_TRY(cudaMemcpyAsync(cross.p, planes.data(), planes.size() * sizeof(double), cudaMemcpyHostToDevice,
                                 stream));
    SCY_CUDA_TRY(cudaStreamSynchronize(stream));
  }
  residual_dd_kernel<<<grid_for(n, 256, 4096), 256, 0, stream>>>(cross.as<double>(), u, rhs, r, h.Ny, h.Nz);
  SCY_LAUNCH_CHECK();
  if (rnorm2_host) {
    double* sc = scal.as<double>();
    dot_kernel<double, double><<<red_blocks(n), 256, 0, stream>>>(r, r, n, red.partials.as<double>(),
                                                                 red.counter.as<unsigned>(), sc + 6);
    SCY_LAUNCH_CHECK();
    SCY_CUDA_TRY(cudaMemcpyAsync(rnorm2_host, sc + 6, sizeof(double), cudaMemcpyDeviceToHost, stream));
    SCY_CUDA_TRY(cudaStreamSynchronize(stream));
    if (!std::isfinite(*rnorm2_host)) {
      set_error("non-finite residual in the elliptic solve");
      return SCY_ERR_NONFINITE;
    }
  }
  return SCY_OK;
}

int SbpContext::change_bc(int R, int T, int Lb, int B) {
  desc.bcR = R; desc.bcT = T; desc.bcL = Lb; desc.bcB = B;
  bc[0] = R; bc[1] = T; bc[2] = Lb; bc[3] = B;
  return rebuild();
}

}  // namespace scy
