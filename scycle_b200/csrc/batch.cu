// Batched ensemble of quasi-dynamic instances (see batch.hpp).
//
// One round = for every instance: (copy) var = the accepted solution and
// (acc) the rates at the accepted state, as RK32/RK43::integrate do after an
// accepted attempt (odeSolver.cpp:599-603, :1148-1152); then (run) one RK
// attempt (:567-592, :1080-1140) and its error sums (:449-501, :902-969).
// The host reads the sums of all instances once per round and takes each
// instance's accept / step-size decision with the single-instance
// QDContext's own step control, so an instance takes the steps it would
// take alone.
//
// A stage d_dt of a group: boundary data and rhs (with its norm), the
// residual of the warm start, `its` preconditioned CG iterations, the
// device convergence test, and the fault update (linear elastic) or the
// viscous rates and fault update (power law), following
// StrikeSlip_LinearElastic_qd::d_dt (strikeSlip_linearElastic_qd.cpp:756-798)
// and StrikeSlip_PowerLaw_qd::d_dt (strikeSlip_powerLaw_qd.cpp:633-690).
#include <cmath>
#include <cstring>
#include <string>

#include "batch.hpp"
#include "capi_types.hpp"
#include "common.cuh"
#include "fault_node.cuh"
#include "powerlaw_dev.cuh"
#include "tma.cuh"
#include "ysolve.cuh"

namespace scy {

#define SCY_BLAS_TRY(call)                                                 \
  do {                                                                     \
    cublasStatus_t b_ = (call);                                            \
    if (b_ != CUBLAS_STATUS_SUCCESS) {                                     \
      ::scy::set_error("%s:%d: %s failed (%d)", __FILE__, __LINE__, #call, \
                       (int)b_);                                           \
      return SCY_ERR_CUDA;                                                 \
    }                                                                      \
  } while (0)

namespace {

constexpr int TB = 256;

// blocks per instance for the node loops: about four nodes per thread
int node_blocks(long N) {
  long b = (N + 4L * TB - 1) / (4L * TB);
  return (int)std::max(1L, std::min(b, 1024L));
}

__device__ __forceinline__ double stage_time(const double* t, const double* dt, int g, double c) {
  return __dadd_rn(t[g], __dmul_rn(c, dt[g]));
}

// bcL = slip / faultTypeScale, bcR = vL t / faultTypeScale + bcRShift
__global__ void b_bc_kernel(const BatchInst* __restrict__ tab, const int* __restrict__ mask,
                            const double* __restrict__ t, const double* __restrict__ dt, int base, double c,
                            int in_slot) {
  const int k = blockIdx.z;
  if (!mask[k]) return;
  const BatchInst& I = tab[k];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= I.fp.Nz) return;
  const double te = stage_time(t, dt, base + k, c);
  if (I.bcL_from_slip) I.bcL[i] = I.rk[in_slot][I.fp.slip_off + i] * I.inv_fts;
  if (I.bcR_remote) I.bcR[i] = I.vL * te * I.inv_fts + I.bcRShift[i];
}

// rhs = setRhs(bc) (+ B gVxy + C gVxz for the power law); |rhs|^2 -> sc[0]
__global__ void b_rhs_kernel(LevelDev<double> L, const BatchInst* __restrict__ tab, const int* __restrict__ mask,
                             int in_slot, BatchWork w) {
  __shared__ double sh[32];
  const int k = blockIdx.z;
  if (!mask[k]) return;
  const BatchInst& I = tab[k];
  const double* gxy = I.c1 ? I.rk[in_slot] + I.key_off[SCY_KEY_GVXY] : nullptr;
  const double* gxz = I.c1 ? I.rk[in_slot] + I.key_off[SCY_KEY_GVXZ] : nullptr;
  double acc = 0.0;
  for (long node = blockIdx.x * (long)blockDim.x + threadIdx.x; node < w.N; node += (long)gridDim.x * blockDim.x) {
    double v = set_rhs_node(L, I.bcL, I.bcR, I.bcT, I.bcB, node);
    if (gxy) v = v + 1.0 * pl_source_node(L, gxy, gxz, node);
    I.rhs[node] = v;
    acc += v * v;
  }
  double s = block_sum(acc, sh);
  grid_reduce_finish(s, w.partials + (long)k * w.PB, w.counters + 4 * k, w.sc + 16 * k + 0, sh);
}

// Linear-elastic rhs: setRhs is nonzero only within BAND nodes of the
// boundary (SAT columns of the Dirichlet sides, boundary values of the
// Neumann sides), and the interior of every instance's rhs was written with
// zeros by its first (single-instance) d_dt, so only that frame is
// rewritten.  Frame index f < 2 * BAND * Nz: rows 0..BAND-1 and Ny-BAND..Ny-1;
// after that, columns 0..BAND-1 and Nz-BAND..Nz-1 of the rows in between.
__global__ void b_rhs_frame_kernel(LevelDev<double> L, const BatchInst* __restrict__ tab,
                                   const int* __restrict__ mask, BatchWork w, int nframe) {
  __shared__ double sh[32];
  const int k = blockIdx.z;
  if (!mask[k]) return;
  const BatchInst& I = tab[k];
  const int Ny = L.Ny, Nz = L.Nz;
  double acc = 0.0;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nframe; f += gridDim.x * blockDim.x) {
    int iy, iz;
    if (f < 2 * BAND * Nz) {
      const int r = f / Nz;
      iz = f - r * Nz;
      iy = r < BAND ? r : Ny - 2 * BAND + r;
    } else {
      const int e = f - 2 * BAND * Nz, r = e / (2 * BAND), c = e - r * (2 * BAND);
      iy = BAND + r;
      iz = c < BAND ? c : Nz - 2 * BAND + c;
    }
    const long node = (long)iy * Nz + iz;
    const double v = set_rhs_node(L, I.bcL, I.bcR, I.bcT, I.bcB, node);
    I.rhs[node] = v;
    acc += v * v;
  }
  double s = block_sum(acc, sh);
  grid_reduce_finish(s, w.partials + (long)k * w.PB, w.counters + 4 * k, w.sc + 16 * k + 0, sh);
}

// rz = r.z -> sc[2] (the previous value moves to sc[3])
template <typename Tz>
__global__ void b_dot_rz_kernel(const int* __restrict__ mask, BatchWork w, const Tz* __restrict__ z) {
  __shared__ double sh[32];
  const int k = blockIdx.z;
  if (!mask[k]) return;
  const long off = (long)k * w.N;
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < w.N; i += (long)gridDim.x * blockDim.x)
    acc += w.r[off + i] * (double)z[off + i];
  double t = block_sum(acc, sh);
  __shared__ bool am_last;
  const unsigned nb = gridDim.x;
  double* partials = w.partials + (long)k * w.PB;
  unsigned* counter = w.counters + 4 * k;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = t;
    __threadfence();
    am_last = atomicAdd(counter, 1u) == nb - 1;
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)nb; i += blockDim.x) s += ((volatile double*)partials)[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) {
      double* sc = w.sc + 16 * k;
      sc[3] = sc[2];
      sc[2] = s;
      *counter = 0u;
    }
  }
}

// A applied in its per-node cross form (33 coefficient planes shared by
// the group, see build_cross_planes): a block owns one XTY x 32 tile of
// nodes, keeps its nodes' coefficients in registers and applies them to its
// (up to XKPB) instances in turn.  Each instance's operand (the tile plus an
// 8-node halo in y and in z) is staged in shared memory by asynchronous
// copies (cp.async, zero-filled outside the grid) in an XS-stage ring, so
// the copies of the next two instances are in flight while one is computed.
//   MODE 0: r = -rhs + A u (0 where rhs = 0), r.r -> sc[5]
//   MODE 1: p = z + beta p_old (beta = rz / rz_old; p = z on the first
//           iteration), q = -A p, p stored (unless store_p = 0), p.q ->
//           partials; on the first iteration also r.z -> partials2
constexpr int XTY = 8, XTZ = 32, XH = 8, XS = 3, XKPB = 8;
constexpr int XT = XTY * XTZ, XW = XT / 32;  // threads and warps of a block
constexpr int XNY = (XTY + 2 * XH) * XTZ, XNZ = XTY * (XTZ + 2 * XH), XNS = XNY + XNZ;

__device__ __forceinline__ void cp_async4(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// dynamic shared memory of b_cross_kernel: MODE 0 stages the operand and
// the rhs of the tile; MODE 1 stages z (zsize bytes a value), p_old and the
// tile's r, and forms p in one more buffer
constexpr int xs_smem_bytes(int mode, int zsize) {
  return mode == 0 ? XS * (XNS + XT) * 8 : (XS * XNS * zsize + 15) / 16 * 16 + XS * XNS * 8 + XNS * 8 + XS * XT * 8;
}

template <int MODE, typename Tz>
__global__ void __launch_bounds__(XT) b_cross_kernel(const double* __restrict__ C, int Ny, int Nz,
                                                      const BatchInst* __restrict__ tab, const int* __restrict__ mask,
                                                      BatchWork w, const Tz* __restrict__ zv, int first, int pi,
                                                      int mixed, int kpb, int store_p = 1) {
  constexpr int NV = (XNS + XT - 1) / XT;  // staged values per thread
  extern __shared__ __align__(16) unsigned char xsm[];
  __shared__ double red[XKPB][XW];  // warp sums by instance
  __shared__ double red2[MODE == 1 ? XKPB : 1][XW];
  __shared__ int act[XKPB];                // the block's active instances
  __shared__ double sck[XKPB];             // MODE 0: |rhs|^2 (0: rhs = 0); MODE 1: beta
  __shared__ const double* srck[XKPB][2];  // MODE 0: u, rhs
  __shared__ int nact;
  const long N = (long)Ny * Nz;
  const int tid = threadIdx.x, ty = tid / XTZ, tz = tid % XTZ;
  const int y0 = blockIdx.y * XTY, z0 = blockIdx.x * XTZ;
  const int iy = y0 + ty, iz = z0 + tz;
  const bool valid = iy < Ny && iz < Nz;
  const long node = (long)iy * Nz + iz;
  const int tile = blockIdx.x + gridDim.x * blockIdx.y;
  const int kb = blockIdx.z * kpb, ke = min(w.K, kb + kpb);
  if (tid == 0) {
    int n = 0;
    for (int k = kb; k < ke; ++k) {
      if (!mask[k]) continue;
      act[n] = k;
      if (MODE == 0) {
        sck[n] = w.sc[16 * k];
        srck[n][0] = tab[k].u;
        srck[n][1] = tab[k].rhs;
      } else {
        double beta = 0.0;
        if (!first) {
          const double ro = w.sc[16 * k + 3];
          beta = ro != 0.0 ? w.sc[16 * k + 2] / ro : 0.0;
        }
        sck[n] = beta;
      }
      ++n;
    }
    nact = n;
  }
  // y arm: c[0..16] for rows iy-8..iy+8.  z arm: read as 16-byte pairs
  // from the even column at or below iz-8 (nine pairs, columns
  // (iz & ~1) - 8 .. + 17), so its coefficients are held shifted by the
  // lane's parity e: c[17 + o] multiplies column (iz & ~1) - 8 + o, zero at
  // the centre and outside the arm
  const int e = tz & 1;
  double c[35];
#pragma unroll
  for (int o = 0; o < 17; ++o) c[o] = valid ? C[(long)o * N + node] : 0.0;
  {
    double cz[18];  // by z offset + 8, with the centre 0 and cz[17] = 0
#pragma unroll
    for (int o = 0; o < 18; ++o)
      cz[o] = (valid && o != 8 && o < 17) ? C[(long)(o < 8 ? 17 + o : 16 + o) * N + node] : 0.0;
    c[17] = e ? 0.0 : cz[0];
#pragma unroll
    for (int o = 1; o < 18; ++o) c[17 + o] = e ? cz[o - 1] : cz[o];
  }
  // the staged positions do not depend on the instance: their node offsets
  // (0 outside the grid, where bit a of inb is clear and nothing is read)
  // are worked out once
  int src[NV];
  unsigned inb = 0;
#pragma unroll
  for (int a = 0; a < NV; ++a) {
    const int i = tid + XT * a;
    int jy = -1, jz = -1;
    if (i < XNY) {
      jy = y0 - XH + i / XTZ;
      jz = z0 + i % XTZ;
    } else if (i < XNS) {
      const int e = i - XNY;
      jy = y0 + e / (XTZ + 2 * XH);
      jz = z0 - XH + e % (XTZ + 2 * XH);
    }
    const bool in = jy >= 0 && jy < Ny && jz >= 0 && jz < Nz;
    src[a] = in ? jy * Nz + jz : 0;
    inb |= (in ? 1u : 0u) << a;
  }
  __syncthreads();
  const int na = nact;
  double* us = reinterpret_cast<double*>(xsm);  // MODE 0: [XS][XNS] operand, then [XS][XT] rhs
  double* rs = us + XS * XNS;
  Tz* zs = reinterpret_cast<Tz*>(xsm);  // MODE 1: [XS][XNS] z, [XS][XNS] p_old, [XNS] p
  double* ps = reinterpret_cast<double*>(xsm + (XS * XNS * sizeof(Tz) + 15) / 16 * 16);
  double* xd = ps + XS * XNS;
  double* rr = xd + XNS;  // MODE 1: [XS][XT] r of the tile (first iteration)
  // copies of the q-th active instance into stage q % XS (one commit group
  // per call, empty past the last instance)
  auto issue = [&](int q) {
    if (q < na) {
      const int st = q % XS;
      if (MODE == 0) {
        const double* x = srck[q][0];
        double* d = us + st * XNS + tid;
#pragma unroll
        for (int a = 0; a < NV; ++a)
          if (tid + XT * a < XNS) cp_async8(d + XT * a, x + src[a], (inb >> a & 1u) * 8);
        const double* rh = srck[q][1];
        const bool rv = valid && sck[q] != 0.0;
        cp_async8(rs + st * XT + tid, rv ? rh + node : rh, rv ? 8 : 0);
      } else {
        const long off = (long)act[q] * N;
        const Tz* zz = zv + off;
        const double* pold = (pi ? w.p1 : w.p0) + off;
#pragma unroll
        for (int a = 0; a < NV; ++a) {
          const int i = tid + XT * a;
          if (i >= XNS) continue;
          const unsigned in = inb >> a & 1u;
          if (sizeof(Tz) == 4)
            cp_async4(zs + st * XNS + i, zz + src[a], in * 4);
          else
            cp_async8(zs + st * XNS + i, zz + src[a], in * 8);
          if (!first) cp_async8(ps + st * XNS + i, pold + src[a], in * 8);
        }
        if (first) cp_async8(rr + st * XT + tid, w.r + off + (valid ? node : 0), valid ? 8 : 0);
      }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int q = 0; q < XS - 1; ++q) issue(q);
  for (int q = 0; q < na; ++q) {
    const int st = q % XS, k = act[q];
    cp_async_wait<XS - 2>();  // this instance's group has landed (the next may not have)
    __syncthreads();          // ... for every thread, and stage (q - 1) % XS is free
    issue(q + XS - 1);
    const double* X = us + st * XNS;
    if (MODE == 1) {
      bool direct = false;  // p = z in FP64: read the staged z as it is
      if constexpr (sizeof(Tz) == 8) {
        if (first) {
          X = reinterpret_cast<const double*>(zs + st * XNS);
          direct = true;
        }
      }
      if (!direct) {
        const double beta = sck[q];
#pragma unroll
        for (int a = 0; a < NV; ++a) {
          const int i = tid + XT * a;
          if (i < XNS)
            xd[i] = first ? (double)zs[st * XNS + i] : (double)zs[st * XNS + i] + beta * ps[st * XNS + i];
        }
        __syncthreads();
        X = xd;
      }
    }
    const long off = (long)k * N;
    double contrib = 0.0, rz = 0.0;
    if (valid) {
      const double* ay = X + ty * XTZ + tz;                   // row iy - 8
      const double2* az = reinterpret_cast<const double2*>(X + XNY + ty * (XTZ + 2 * XH) + (tz - e));
      // four partial sums (even / odd offsets of each arm), so the FMA
      // chains are short
      double Ay0 = 0.0, Ay1 = 0.0, Az0 = 0.0, Az1 = 0.0;
#pragma unroll
      for (int o = 0; o < 17; o += 2) Ay0 += c[o] * ay[o * XTZ];
#pragma unroll
      for (int o = 1; o < 17; o += 2) Ay1 += c[o] * ay[o * XTZ];
#pragma unroll
      for (int m = 0; m < 9; ++m) {
        const double2 v = az[m];
        Az0 += c[17 + 2 * m] * v.x;
        Az1 += c[18 + 2 * m] * v.y;
      }
      const double Ax = (Ay0 + Ay1) + (Az0 + Az1);
      if (MODE == 0) {
        const double vv = sck[q] == 0.0 ? 0.0 : -1.0 * rs[st * XT + tid] + Ax;
        w.r[off + node] = vv;
        if (mixed) w.r32[off + node] = (float)vv;
        contrib = vv * vv;
      } else {
        const double p = ay[XH * XTZ];
        const double qv = -Ax;
        if (store_p) (pi ? w.p0 : w.p1)[off + node] = p;
        w.q[off + node] = qv;
        contrib = p * qv;
        if (first) rz = rr[st * XT + tid] * p;
      }
    }
    // warp sums of this instance; the block partials are formed at the end
    contrib = warp_sum(contrib);
    if ((tid & 31) == 0) red[q][tid >> 5] = contrib;
    if (MODE == 1 && first) {
      rz = warp_sum(rz);
      if ((tid & 31) == 0) red2[q][tid >> 5] = rz;
    }
  }
  cp_async_wait<0>();
  // block partial of every instance (warp 0 adds the XW warp sums in order);
  // b_partials_kernel adds the tiles up
  __syncthreads();
  if (tid < 32) {
    for (int q = 0; q < na; ++q) {
      double t = tid < XW ? red[q][tid] : 0.0;
      t = warp_sum(t);
      if (tid == 0) w.partials[(long)act[q] * w.PB + tile] = t;
      if (MODE == 1 && first) {
        t = tid < XW ? red2[q][tid] : 0.0;
        t = warp_sum(t);
        if (tid == 0) w.partials2[(long)act[q] * w.PB + tile] = t;
      }
    }
  }
}

// The same two products when the group's operator is separable over every
// node (L.full: one 17-point stencil per row and per column from 1D tables
// shared by the group, L1/L2-resident): one instance per block
// (blockIdx.z), its 8*RPT x 32 tile staged once and applied by full_apply
// (register window along y, 9-point interior), so per node only the
// instance's own fields move.  The partial sums do not depend on RPT: the
// contributions go to shared memory by node, then for every band of 8 rows
// (a tile of the 8 x 32 layout, index blockIdx.x + gridDim.x * band) each
// column adds its 8 rows in order and one warp sum adds the 32 columns.
template <int MODE, typename Tz, int RPT, int MINB>
__global__ void __launch_bounds__(256, MINB) b_full_kernel(LevelDev<double> L, const BatchInst* __restrict__ tab,
                                                     const int* __restrict__ mask, BatchWork w,
                                                     const Tz* __restrict__ zv, int first, int pi, int mixed,
                                                     int store_p) {
  __shared__ double xs[full_smem_values<RPT>()];
  __shared__ double cs[2][8 * RPT][TZ];  // contributions by node of the tile
  const int k = blockIdx.z;
  if (!mask[k]) return;
  const int tid = threadIdx.x, lane = tid & 31, r0 = (tid >> 5) * RPT;
  const long off = (long)k * w.N;
  const double* sc = w.sc + 16 * k;
  double a1 = 0.0, a2 = 0.0;  // the current row's contributions
  auto row = [&](int j) {
    cs[0][r0 + j][lane] = a1;
    if (MODE == 1 && first) cs[1][r0 + j][lane] = a2;
    a1 = a2 = 0.0;
  };
  if (MODE == 0) {
    const double* u = tab[k].u;
    const double* rhs = tab[k].rhs;
    const bool zero = sc[0] == 0.0;
    auto ld = [&](long node, int, int) { return u[node]; };
    auto pre = [&](long node, int, int) { return zero ? 0.0 : rhs[node]; };
    auto out = [&](long node, int, int, double Ax, double, double b) {
      const double v = zero ? 0.0 : -1.0 * b + Ax;
      w.r[off + node] = v;
      if (mixed) w.r32[off + node] = (float)v;
      a1 = v * v;
    };
    full_apply<double, RPT>(L, ld, pre, out, row, xs);
  } else {
    double beta = 0.0;
    if (!first) {
      const double ro = sc[3];
      beta = ro != 0.0 ? sc[2] / ro : 0.0;
    }
    const Tz* z = zv + off;
    const double* pold = (pi ? w.p1 : w.p0) + off;
    double* pnew = (pi ? w.p0 : w.p1) + off;
    const double* r = w.r + off;
    double* q = w.q + off;
    auto ld = [&](long node, int, int) {
      return first ? (double)z[node] : (double)z[node] + beta * pold[node];
    };
    auto pre = [&](long node, int, int) { return first ? r[node] : 0.0; };
    auto out = [&](long node, int, int, double Ax, double p, double rv) {
      const double qv = -Ax;
      if (store_p) pnew[node] = p;
      q[node] = qv;
      a1 = p * qv;
      if (first) a2 = rv * p;
    };
    full_apply<double, RPT>(L, ld, pre, out, row, xs);
  }
  __syncthreads();
  const int wv = tid >> 5, band = blockIdx.y * RPT + wv;
  if (wv < RPT && band * 8 < L.Ny) {
    const long slot = (long)k * w.PB + blockIdx.x + (long)gridDim.x * band;
    double t = 0.0;
#pragma unroll
    for (int r = 0; r < 8; ++r) t += cs[0][wv * 8 + r][lane];
    t = warp_sum(t);
    if (lane == 0) w.partials[slot] = t;
    if (MODE == 1 && first) {
      t = 0.0;
#pragma unroll
      for (int r = 0; r < 8; ++r) t += cs[1][wv * 8 + r][lane];
      t = warp_sum(t);
      if (lane == 0) w.partials2[slot] = t;
    }
  }
}

// grid of b_full_kernel: column tiles, row tiles of 8*rpt, instances
static dim3 full_grid(const BatchGroup& g, int rpt) {
  return dim3((g.Nz + TZ - 1) / TZ, (g.Ny + 8 * rpt - 1) / (8 * rpt), g.K);
}

// the separable form's launch shapes: rows per thread x minimum blocks per
// SM the compiler fits its registers to (1: its own choice)
constexpr int kFullShapes = 6;
constexpr int kFullRpt[kFullShapes] = {1, 2, 4, 1, 2, 4}, kFullMinb[kFullShapes] = {1, 1, 1, 4, 4, 4};

template <int MODE, typename Tz>
static void launch_full(const BatchGroup& g, int shape, const BatchInst* tab, const int* mask, const Tz* zv,
                        int first, int pi, int mixed, int store_p) {
  const dim3 grid = full_grid(g, kFullRpt[shape]);
#define SCY_FULL_LAUNCH(R, M) \
  b_full_kernel<MODE, Tz, R, M><<<grid, 256, 0, g.stream>>>(g.L, tab, mask, g.w, zv, first, pi, mixed, store_p)
  switch (shape) {
    case 0: SCY_FULL_LAUNCH(1, 1); break;
    case 1: SCY_FULL_LAUNCH(2, 1); break;
    case 2: SCY_FULL_LAUNCH(4, 1); break;
    case 3: SCY_FULL_LAUNCH(1, 4); break;
    case 4: SCY_FULL_LAUNCH(2, 4); break;
    default: SCY_FULL_LAUNCH(4, 4); break;
  }
#undef SCY_FULL_LAUNCH
}

// sc[16 k + slot] = sum of the instance's first n partials (of w.partials,
// or of w.partials2 when second is set), in tile order
__global__ void b_partials_kernel(const int* __restrict__ mask, BatchWork w, int n, int slot, int second = 0) {
  __shared__ double sh[32];
  const int k = blockIdx.x;
  if (!mask[k]) return;
  const double* p = (second ? w.partials2 : w.partials) + (long)k * w.PB;
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += p[i];
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) w.sc[16 * k + slot] = acc;
}

// u += alpha p ; r -= alpha q ; r.r -> sc[1]   (alpha = rz / pq).  pz: p
// was not stored and is z (the first iteration); last: r is only summed
__global__ void b_update_kernel(const BatchInst* __restrict__ tab, const int* __restrict__ mask, BatchWork w, int pi,
                                int mixed, int pz, int last) {
  __shared__ double sh[32];
  const int k = blockIdx.z;
  if (!mask[k]) return;
  const long off = (long)k * w.N;
  double* sc = w.sc + 16 * k;
  const double pqv = sc[4];
  const double alpha = pqv != 0.0 ? sc[2] / pqv : 0.0;
  const bool zero = sc[0] == 0.0;
  const double* p = (pi ? w.p0 : w.p1) + off;  // the p_new of b_matvec_kernel
  double* x = tab[k].u;
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < w.N; i += (long)gridDim.x * blockDim.x) {
    if (zero) {
      x[i] = 0.0;
    } else {
      const double pv = !pz ? p[i] : mixed ? (double)w.z32[off + i] : w.z[off + i];
      x[i] += alpha * pv;
    }
    double rv = w.r[off + i] - alpha * w.q[off + i];
    if (!last) {
      w.r[off + i] = rv;
      if (mixed) w.r32[off + i] = (float)rv;
    }
    acc += rv * rv;
  }
  double t = block_sum(acc, sh);
  grid_reduce_finish(t, w.partials + (long)k * w.PB, w.counters + 4 * k, sc + 1, sh);
}

// status bit 1: residual above max(rtol |rhs|, atol); bit 2: non-finite
__global__ void b_verify_kernel(const int* __restrict__ mask, BatchWork w, double rtol, double atol) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= w.K || !mask[k]) return;
  const double* sc = w.sc + 16 * k;
  const double tol = fmax(rtol * sqrt(sc[0]), atol);
  const double rr = sc[1];
  if (!isfinite(rr)) atomicOr(w.status + k, 2u);
  else if (!(sqrt(rr) <= tol) && !(sqrt(sc[5]) <= tol)) atomicOr(w.status + k, 1u);
}

template <typename T>
__global__ void b_scale_kernel(T* __restrict__ x, const T* __restrict__ s, long N) {
  const long off = (long)blockIdx.z * N;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
    x[off + i] *= s[i];
}

// the caller's array <-> the instances' vectors, one segment per instance
// (blockIdx.y): scatter into the instances, or gather from them
__global__ void b_io_kernel(const IoSeg* __restrict__ seg, double* __restrict__ stage, int gather) {
  const IoSeg g = seg[blockIdx.y];
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < g.n; i += (long)gridDim.x * blockDim.x) {
    if (gather)
      stage[g.off + i] = g.p[i];
    else
      g.p[i] = stage[g.off + i];
  }
}


// Fault_qd::d_dt with tauQS = mu Dy u on the fault row (linear elastic) or
// the material's sxy there (power law)
__global__ void b_fault_kernel(LevelDev<double> L, const BatchInst* __restrict__ tab, const int* __restrict__ mask,
                               int in_slot, int out_slot) {
  const int k = blockIdx.z;
  if (!mask[k]) return;
  const BatchInst& I = tab[k];
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  if (iz >= I.fp.Nz) return;
  const double sxy = I.c1 ? I.sxy[iz] : fault_row_sxy(L, I.u, iz);
  fault_node_update(iz, sxy, I.fp, I.rk[in_slot], I.rk[out_slot], I.slipVel, I.tauQSP, I.tauP, I.strength, I.flags,
                    I.fault_its);
}

// power law: strains, stresses, viscosity and viscous strain rates per node
__global__ void b_pl_rates_kernel(LevelDev<double> L, const BatchInst* __restrict__ tab, const int* __restrict__ mask,
                                  int in_slot, int out_slot, long N) {
  const int k = blockIdx.z;
  if (!mask[k]) return;
  const BatchInst& I = tab[k];
  PLRatesArgs a;
  a.u = I.u;
  a.gxy = I.rk[in_slot] + I.key_off[SCY_KEY_GVXY];
  a.gxz = I.rk[in_slot] + I.key_off[SCY_KEY_GVXZ];
  a.bcL = I.bcL;
  a.bcR = I.bcR;
  a.c1 = I.c1;
  a.e1 = I.e1;
  a.n = I.n;
  a.inv_cap = I.inv_cap;
  a.dgxy = I.rk[out_slot] + I.key_off[SCY_KEY_GVXY];
  a.dgxz = I.rk[out_slot] + I.key_off[SCY_KEY_GVXZ];
  a.sxy = I.sxy;
  a.sxz = I.sxz;
  a.sdev = I.sdev;
  a.effVisc = I.effVisc;
  for (long node = blockIdx.x * (long)blockDim.x + threadIdx.x; node < N; node += (long)gridDim.x * blockDim.x)
    pl_rates_node(L, a, node);
}

// out = var + sum_j c_j f_j with c_j = (num_j dt) / den_j, in the order of
// the single-instance combine (first term, then var, then the others)
struct BCombo {
  int slot[5];
  double num[5], den[5];
  int nf;
};

__global__ void b_combine_kernel(const BatchInst* __restrict__ tab, const int* __restrict__ mask,
                                 const double* __restrict__ dt, int base, int out_slot, BCombo cb) {
  const int k = blockIdx.z;
  if (!mask[k]) return;
  const BatchInst& I = tab[k];
  const double h = dt[base + k];
  double c[5];
  const double* f[5];
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    if (j < cb.nf) {
      const double nd = __dmul_rn(cb.num[j], h);
      c[j] = cb.den[j] == 1.0 ? nd : __ddiv_rn(nd, cb.den[j]);
      f[j] = I.rk[cb.slot[j]];
    }
  }
  const double* var = I.rk[V_VAR];
  double* out = I.rk[out_slot];
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < I.nvar; i += (long)gridDim.x * blockDim.x) {
    double v = c[0] * f[0][i] + var[i];
    for (int j = 1; j < cb.nf; ++j) v = v + c[j] * f[j][i];
    out[i] = v;
  }
}

__global__ void b_copy_kernel(const BatchInst* __restrict__ tab, const int* __restrict__ mask) {
  const int k = blockIdx.z;
  if (!mask[k]) return;
  const BatchInst& I = tab[k];
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < I.nvar; i += (long)gridDim.x * blockDim.x)
    I.rk[V_VAR][i] = I.rk[V_HI][i];
}

// per (key, instance): sum (lo-hi)^2, sum hi^2, max |lo-hi|/hi -> err[16 g + 3 key ..]
__global__ void b_error_kernel(const BatchInst* __restrict__ tab, const int* __restrict__ mask, int base,
                               double* __restrict__ err) {
  __shared__ double sh[32];
  const int k = blockIdx.z, key = blockIdx.x;
  if (!mask[k]) return;
  const BatchInst& I = tab[k];
  const long off = I.key_off[key], len = I.key_len[key];
  if (len == 0) return;
  const double* lo = I.rk[V_LO];
  const double* hi = I.rk[V_HI];
  double ss = 0.0, sh2 = 0.0, mx = -INFINITY;
  for (long i = threadIdx.x; i < len; i += blockDim.x) {
    double h = hi[off + i];
    double d = lo[off + i] - h;
    ss += d * d;
    sh2 += h * h;
    double r = fabs(d) / h;
    mx = fmax(mx, r);
  }
  ss = block_sum(ss, sh);
  sh2 = block_sum(sh2, sh);
  double m = warp_max(mx);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < (blockDim.x + 31) / 32 ? sh[threadIdx.x] : -INFINITY;
    t = warp_max(t);
    if (threadIdx.x == 0) {
      double* o = err + 16L * (base + k) + 3 * key;
      o[0] = ss;
      o[1] = sh2;
      o[2] = t;
    }
  }
}

// fault flags and solve status of every instance of the group -> err[16 g + 14, 15], cleared
__global__ void b_status_kernel(const BatchInst* __restrict__ tab, BatchWork w, int base, double* __restrict__ err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= w.K) return;
  err[16L * (base + k) + 14] = (double)atomicExch(tab[k].flags, 0u);
  err[16L * (base + k) + 15] = (double)atomicExch(w.status + k, 0u);
}

}  // namespace

// ---------------------------------------------------------------------------
namespace {
typedef CUresult (*TmaEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// a tile map of `rank` dimensions (dims[0] innermost; strides in bytes of
// dimensions 1..rank-1) without swizzle, reads outside the array give zeros
int tma_encode(CUtensorMap* map, const void* base, CUtensorMapDataType type, int rank, const cuuint64_t* dims,
               const cuuint64_t* strides, const cuuint32_t* box,
               CUtensorMapSwizzle swizzle = CU_TENSOR_MAP_SWIZZLE_NONE) {
  static TmaEncodeFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess || !p ||
        q != cudaDriverEntryPointSuccess) {
      set_error("cuTensorMapEncodeTiled is not available");
      return SCY_ERR_CUDA;
    }
    fn = reinterpret_cast<TmaEncodeFn>(p);
  }
  const cuuint32_t es[3] = {1, 1, 1};
  const CUresult r = fn(map, type, (cuuint32_t)rank, const_cast<void*>(base), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return SCY_ERR_CUDA;
  }
  return SCY_OK;
}
}  // namespace

int tma_map_2d(CUtensorMap* map, const void* base, CUtensorMapDataType type, int esize, long cols, long rows,
               long stride_bytes, int box_cols, int box_rows) {
  (void)esize;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)stride_bytes};
  const cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  return tma_encode(map, base, type, 2, dims, strides, box);
}

int tma_map_3d(CUtensorMap* map, const void* base, CUtensorMapDataType type, long d0, long d1, long d2,
               long stride1_bytes, long stride2_bytes, int box0, int box1, int box2) {
  const cuuint64_t dims[3] = {(cuuint64_t)d0, (cuuint64_t)d1, (cuuint64_t)d2};
  const cuuint64_t strides[2] = {(cuuint64_t)stride1_bytes, (cuuint64_t)stride2_bytes};
  const cuuint32_t box[3] = {(cuuint32_t)box0, (cuuint32_t)box1, (cuuint32_t)box2};
  return tma_encode(map, base, type, 3, dims, strides, box);
}

int tma_map_3d_sw64(CUtensorMap* map, const void* base, CUtensorMapDataType type, long d0, long d1, long d2,
                    long stride1_bytes, long stride2_bytes, int box0, int box1, int box2) {
  const cuuint64_t dims[3] = {(cuuint64_t)d0, (cuuint64_t)d1, (cuuint64_t)d2};
  const cuuint64_t strides[2] = {(cuuint64_t)stride1_bytes, (cuuint64_t)stride2_bytes};
  const cuuint32_t box[3] = {(cuuint32_t)box0, (cuuint32_t)box1, (cuuint32_t)box2};
  return tma_encode(map, base, type, 3, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_64B);
}

BatchGroup::~BatchGroup() {
  if (blas) cublasDestroy(blas);
  if (join) cudaEventDestroy(join);
  if (stream) cudaStreamDestroy(stream);
}

BatchContext::~BatchContext() {
  for (auto& r : precs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto& kv : graph_of_its) cudaGraphExecDestroy(kv.second);
  graph_of_its.clear();
  groups.clear();
  if (ctl_host) cudaFreeHost(ctl_host);
  if (err_host) cudaFreeHost(err_host);
  if (fork) cudaEventDestroy(fork);
  if (stream) cudaStreamDestroy(stream);
  for (scy_qd* p : inst) delete p;
}

QDContext& BatchContext::q(int i) const { return inst[i]->ctx; }

const double* BatchContext::d_t() const { return ctl.as<double>(); }
const double* BatchContext::d_dt_() const { return ctl.as<double>() + n; }
const int* BatchContext::d_copy(const BatchGroup& g) const {
  return reinterpret_cast<const int*>(ctl.as<double>() + 2 * n) + g.base;
}
const int* BatchContext::d_acc(const BatchGroup& g) const { return d_copy(g) + n; }
const int* BatchContext::d_run(const BatchGroup& g) const { return d_copy(g) + 2 * n; }

static bool same_operator(const SbpContext& a, const SbpContext& b) {
  const scy_grid_desc &x = a.desc, &y = b.desc;
  if (x.order != y.order || x.Ny != y.Ny || x.Nz != y.Nz || x.grid_type != y.grid_type || x.compat != y.compat)
    return false;
  if (x.Ly != y.Ly || x.Lz != y.Lz) return false;
  for (int i = 0; i < 4; ++i)
    if (a.bc[i] != b.bc[i]) return false;
  return a.y == b.y && a.z == b.z && a.mu == b.mu;
}

int BatchContext::create(int n_inst, const char* const* paths, const scy_solve_opts* solve,
                         const scy_batch_opts* o) {
  n = n_inst;
  if (o) {
    precision = o->precision;
    its = o->cg_its;
    graphs = o->graphs;
    concurrent = o->concurrent;
    fd_dense = o->fd_dense;
  }
  if (precision != SCY_PREC_FP64 && precision != SCY_PREC_MIXED && precision != SCY_PREC_TF32) {
    set_error("unknown batch precision %d", precision);
    return SCY_ERR_ARG;
  }
  zt_planes = precision == SCY_PREC_FP64 ? 5 : precision == SCY_PREC_MIXED ? 4 : 3;
  if (o && o->transform_planes) zt_planes = o->transform_planes;
  if (zt_planes < 3 || zt_planes > 7) {
    set_error("transform_planes must be 3..7 (got %d)", zt_planes);
    return SCY_ERR_ARG;
  }
  if (its <= 0) its = precision == SCY_PREC_FP64 ? 1 : 2;
  std::vector<scy_qd*> made(n, nullptr);
  for (int i = 0; i < n; ++i) {
    int rc = scy_qd_create_from_in(paths[i], solve, &made[i]);
    if (rc != SCY_OK) {
      std::string e = last_error();
      for (scy_qd* h : made) delete h;
      set_error("instance %d (%s): %s", i, paths[i], e.c_str());
      return rc;
    }
  }
  if (o)
    for (scy_qd* h : made) h->ctx.fp.jacobian = o->exact_jacobian ? 1 : 0;
  // groups of instances with one operator; the batch addresses instances
  // group by group (slots), the caller by its own numbering
  std::vector<std::vector<int>> members;
  std::vector<int> gof(n);
  for (int i = 0; i < n; ++i) {
    int gi = -1;
    for (size_t g = 0; g < members.size() && gi < 0; ++g)
      if (same_operator(made[members[g][0]]->ctx.sbp, made[i]->ctx.sbp)) gi = (int)g;
    if (gi < 0) {
      gi = (int)members.size();
      members.emplace_back();
    }
    members[gi].push_back(i);
    gof[i] = gi;
  }
  slot_of.assign(n, 0);
  user_of.clear();
  inst.clear();
  group_of = gof;
  for (auto& m : members)
    for (int i : m) {
      slot_of[i] = (int)inst.size();
      user_of.push_back(i);
      inst.push_back(made[i]);
    }
  const QDContext& q0 = q(0);
  pl = q0.pl;
  rtol = q0.solve_opts.rtol;
  atol = q0.solve_opts.atol;
  max_its = q0.solve_opts.max_its;
  method = inst[0]->prob->ode.method;
  for (int s = 1; s < n; ++s) {
    if (q(s).pl != pl || inst[s]->prob->ode.method != method) {
      set_error("instance %d: every instance of a batch needs the same driver and integrator", user_of[s]);
      return SCY_ERR_ARG;
    }
  }
  // one fast-diagonalisation preconditioner per operator, shared by the
  // members' own solves as well
  int base = 0;
  for (auto& m : members) {
    SCY_TRY(q(base).sbp.ensure_fd());
    for (size_t k = 1; k < m.size(); ++k) q(base + (int)k).sbp.fd = q(base).sbp.fd;
    base += (int)m.size();
  }
  // begin every instance (initial state and first rates on its own solver);
  // the batch writes no stride output (fields come through scy_qd_get_field
  // and scy_batch_get_fault_field)
  for (int s = 0; s < n; ++s) {
    inst[s]->prob->stride1D = inst[s]->prob->stride2D = 0;
    if (inst[s]->prob->ckpt) {
      set_error("instance %d: checkpointing (enableCheckpointing) is not available in a batch", user_of[s]);
      return SCY_ERR_ARG;
    }
  }
  for (int s = 0; s < n; ++s) {
    int rc = scy_qd_integrate_begin_from_in(inst[s]);
    if (rc != SCY_OK) {
      std::string e = last_error();
      set_error("instance %d: %s", user_of[s], e.c_str());
      return rc;
    }
  }
  SCY_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  SCY_CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  base = 0;
  for (auto& m : members) {
    SCY_TRY(setup_group(base, (int)m.size()));
    base += (int)m.size();
  }
  ctl_bytes = (size_t)n * (2 * sizeof(double) + 3 * sizeof(int));
  SCY_TRY(ctl.alloc(ctl_bytes));
  SCY_CUDA_TRY(cudaMallocHost(&ctl_host, ctl_bytes));
  std::memset(ctl_host, 0, ctl_bytes);
  SCY_TRY(err.alloc((size_t)n * 16 * sizeof(double)));
  SCY_CUDA_TRY(cudaMemset(err.p, 0, (size_t)n * 16 * sizeof(double)));
  SCY_CUDA_TRY(cudaMallocHost((void**)&err_host, (size_t)n * 16 * sizeof(double)));
  hc.assign(n, Ctl());
  // segment tables of the state and fault-field transfers, in the caller's
  // numbering
  {
    std::vector<IoSeg> segs((size_t)(1 + kIoFields) * n, IoSeg{nullptr, 0, 0});
    long os = 0, of = 0;
    for (int i = 0; i < n; ++i) {
      QDContext& c = q(slot_of[i]);
      segs[i] = IoSeg{c.rk[V_VAR].as<double>(), c.nvar, os};
      os += c.nvar;
      double* var = c.rk[V_VAR].as<double>();
      double* dvar = c.rk[V_DVAR].as<double>();
      double* src[kIoFields] = {var + c.key_off[SCY_KEY_PSI], var + c.key_off[SCY_KEY_SLIP], c.slipVel.as<double>(),
                                c.tauP.as<double>(), c.tauQSP.as<double>(), c.strength.as<double>(), nullptr,
                                nullptr, nullptr, dvar + c.key_off[SCY_KEY_PSI], dvar + c.key_off[SCY_KEY_SLIP]};
      for (int f = 0; f < kIoFields; ++f) segs[(size_t)(1 + f) * n + i] = IoSeg{src[f], src[f] ? c.Nz : 0, of};
      of += c.Nz;
      io_maxn = std::max(io_maxn, std::max(c.nvar, (long)c.Nz));
    }
    io_states = os;
    io_fault = of;
    SCY_TRY(io.alloc((size_t)std::max(os, of) * sizeof(double)));
    SCY_TRY(io_seg.alloc(segs.size() * sizeof(IoSeg)));
    SCY_CUDA_TRY(cudaMemcpy(io_seg.p, segs.data(), segs.size() * sizeof(IoSeg), cudaMemcpyHostToDevice));
  }
  return SCY_OK;
}

int BatchContext::set_states(const double* host) {
  SCY_CUDA_TRY(cudaMemcpyAsync(io.p, host, (size_t)io_states * sizeof(double), cudaMemcpyHostToDevice, stream));
  const dim3 gr((unsigned)std::min((io_maxn + 255) / 256, 64L), (unsigned)n);
  b_io_kernel<<<gr, 256, 0, stream>>>(io_seg.as<IoSeg>(), io.as<double>(), 0);
  SCY_LAUNCH_CHECK();
  SCY_CUDA_TRY(cudaStreamSynchronize(stream));
  return SCY_OK;
}

int BatchContext::get_fault_field(int field, double* host) {
  if (field < 0 || field >= kIoFields || field == SCY_FIELD_U || field == SCY_FIELD_SURFDISP ||
      field == SCY_FIELD_SXY) {
    set_error("scy_batch_get_fault_field: field %d is not a fault field", field);
    return SCY_ERR_ARG;
  }
  const dim3 gr((unsigned)std::min((io_maxn + 255) / 256, 64L), (unsigned)n);
  b_io_kernel<<<gr, 256, 0, stream>>>(io_seg.as<IoSeg>() + (size_t)(1 + field) * n, io.as<double>(), 1);
  SCY_LAUNCH_CHECK();
  SCY_CUDA_TRY(cudaMemcpyAsync(host, io.p, (size_t)io_fault * sizeof(double), cudaMemcpyDeviceToHost, stream));
  SCY_CUDA_TRY(cudaStreamSynchronize(stream));
  return SCY_OK;
}

int BatchContext::setup_group(int base, int K) {
  std::unique_ptr<BatchGroup> G(new BatchGroup());
  BatchGroup& g = *G;
  g.K = K;
  g.base = base;
  QDContext& q0 = q(base);
  g.Ny = q0.Ny;
  g.Nz = q0.Nz;
  g.N = q0.N;
  // a steady-state guess changes the boundary types and back, which rebuilds
  // the members' operators: take the representative's current ones
  SCY_TRY(q0.sbp.ensure_fd());
  g.fd = q0.sbp.fd;
  g.L = q0.sbp.fine->dev;
  const long KN = (long)g.K * g.N;
  for (auto& v : g.vec) {
    SCY_TRY(v.alloc((size_t)KN * 8));
    SCY_CUDA_TRY(cudaMemset(v.p, 0, (size_t)KN * 8));
  }
  for (auto& v : g.vecf) {
    SCY_TRY(v.alloc((size_t)KN * 4));
    SCY_CUDA_TRY(cudaMemset(v.p, 0, (size_t)KN * 4));
  }
  const int tiles = ((g.Nz + XTZ - 1) / XTZ) * ((g.Ny + XTY - 1) / XTY);
  g.w.PB = std::max(tiles, node_blocks(g.N));
  // instances per block of the operator kernels: enough blocks for about
  // four per SM, at most eight instances each
  g.kpb = (int)std::max(1L, std::min((long)XKPB, (long)g.K * tiles / (148L * 4)));
  SCY_CUDA_TRY(cudaFuncSetAttribute(b_cross_kernel<0, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    xs_smem_bytes(0, 8)));
  SCY_CUDA_TRY(cudaFuncSetAttribute(b_cross_kernel<1, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    xs_smem_bytes(1, 8)));
  SCY_CUDA_TRY(cudaFuncSetAttribute(b_cross_kernel<1, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    xs_smem_bytes(1, 4)));
  {
    std::vector<double> planes;
    build_cross_planes(q0.sbp.hosts[0], planes);
    SCY_TRY(g.planes.alloc(planes.size() * sizeof(double)));
    SCY_CUDA_TRY(cudaMemcpy(g.planes.p, planes.data(), planes.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  SCY_TRY(g.sc.alloc((size_t)g.K * 16 * 8));
  SCY_CUDA_TRY(cudaMemset(g.sc.p, 0, (size_t)g.K * 16 * 8));
  SCY_TRY(g.partials.alloc((size_t)g.K * g.w.PB * 8 * 2));
  SCY_TRY(g.counters.alloc((size_t)g.K * 4 * 4));
  SCY_CUDA_TRY(cudaMemset(g.counters.p, 0, (size_t)g.K * 16));
  SCY_TRY(g.status.alloc((size_t)g.K * 4));
  SCY_CUDA_TRY(cudaMemset(g.status.p, 0, (size_t)g.K * 4));
  g.w.K = g.K;
  g.w.N = g.N;
  g.w.r = g.vec[0].as<double>();
  g.w.p0 = g.vec[1].as<double>();
  g.w.p1 = g.vec[2].as<double>();
  g.w.q = g.vec[3].as<double>();
  g.w.z = g.vec[4].as<double>();
  g.w.t1 = g.vec[5].as<double>();
  g.w.t2 = g.vec[6].as<double>();
  g.w.r32 = g.vecf[0].as<float>();
  g.w.z32 = g.vecf[1].as<float>();
  g.w.t1f = g.vecf[2].as<float>();
  g.w.t2f = g.vecf[3].as<float>();
  g.w.sc = g.sc.as<double>();
  g.w.partials = g.partials.as<double>();
  g.w.partials2 = g.w.partials + (long)g.K * g.w.PB;
  g.w.counters = g.counters.as<unsigned>();
  g.w.status = g.status.as<unsigned>();
  std::vector<BatchInst> tab(g.K);
  for (int k = 0; k < g.K; ++k) {
    QDContext& c = q(g.base + k);
    BatchInst& I = tab[k];
    std::memset(&I, 0, sizeof(I));
    for (int j = 0; j < 11; ++j) I.rk[j] = c.rk[j].as<double>();
    I.u = c.u.as<double>();
    I.rhs = c.rhs.as<double>();
    I.bcL = c.bcL.as<double>();
    I.bcR = c.bcR.as<double>();
    I.bcT = c.bcT.as<double>();
    I.bcB = c.bcB.as<double>();
    I.bcRShift = c.bcRShift.as<double>();
    I.sxy = c.sxy.as<double>();
    I.slipVel = c.slipVel.as<double>();
    I.tauQSP = c.tauQSP.as<double>();
    I.tauP = c.tauP.as<double>();
    I.strength = c.strength.as<double>();
    I.flags = c.flags.as<unsigned>();
    I.fault_its = c.fault_its.as<unsigned long long>();
    I.fp = c.fp;
    I.vL = c.vL;
    I.inv_fts = 1.0 / c.fts;
    I.bcL_from_slip = c.bcL_from_slip;
    I.bcR_remote = c.bcR_remote;
    I.nvar = c.nvar;
    for (int j = 0; j < 4; ++j) {
      I.key_off[j] = c.key_off[j];
      I.key_len[j] = c.key_len[j];
    }
    if (c.pl) {
      I.c1 = c.pl_c1.as<double>();
      I.e1 = c.pl_e1.as<double>();
      I.n = c.pl_n.as<double>();
      I.sxz = c.sxz.as<double>();
      I.sdev = c.sdev.as<double>();
      I.effVisc = c.effVisc.as<double>();
      I.inv_cap = c.inv_visc_cap;
    }
  }
  if (g.fd->ybanded) {
    // the z transform with rows padded to Nzp values (TMA strides are
    // multiples of 16 bytes), and the tile maps of the TMA-fed sweeps
    const int Nzp = g.fd->Nzp;
    const long rowsT = (long)g.K * g.Ny;
    SCY_TRY(g.t1p.alloc((size_t)rowsT * Nzp * 8));
    SCY_TRY(g.t1pf.alloc((size_t)rowsT * Nzp * 4));
    SCY_CUDA_TRY(cudaMemset(g.t1p.p, 0, (size_t)rowsT * Nzp * 8));
    SCY_CUDA_TRY(cudaMemset(g.t1pf.p, 0, (size_t)rowsT * Nzp * 4));
    const CUtensorMapDataType d64 = CU_TENSOR_MAP_DATA_TYPE_FLOAT64, d32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    SCY_TRY(tma_map_2d(&g.mLcol, g.fd->Lcol.p, d64, 8, g.Nz, (long)g.Ny * 9, (long)Nzp * 8, YS_C, YS_R * 9));
    SCY_TRY(tma_map_2d(&g.mLrow, g.fd->Lrow.p, d64, 8, g.Nz, (long)(g.Ny + 8) * 9, (long)Nzp * 8, YS_C, YS_R * 9));
    SCY_TRY(tma_map_3d(&g.mT, g.t1p.p, d64, g.Nz, g.Ny, g.K, (long)Nzp * 8, (long)g.Ny * Nzp * 8, YS_C, YS_R, YS_B));
    SCY_TRY(tma_map_2d(&g.mLcol32, g.fd->Lcol32.p, d32, 4, g.Nz, (long)g.Ny * 9, (long)Nzp * 4, YS_C, YS_R * 9));
    SCY_TRY(tma_map_2d(&g.mLrow32, g.fd->Lrow32.p, d32, 4, g.Nz, (long)(g.Ny + 8) * 9, (long)Nzp * 4, YS_C, YS_R * 9));
    SCY_TRY(tma_map_3d(&g.mT32, g.t1pf.p, d32, g.Nz, g.Ny, g.K, (long)Nzp * 4, (long)g.Ny * Nzp * 4, YS_C, YS_R,
                       YS_B));
    SCY_TRY(tma_map_3d(&g.mT4, g.t1p.p, d64, g.Nz, g.Ny, g.K, (long)Nzp * 8, (long)g.Ny * Nzp * 8, YS_C, YS_R, 4));
    SCY_TRY(tma_map_3d(&g.mT2, g.t1p.p, d64, g.Nz, g.Ny, g.K, (long)Nzp * 8, (long)g.Ny * Nzp * 8, YS_C, YS_R, 2));
    SCY_TRY(tma_map_3d(&g.mT4_32, g.t1pf.p, d32, g.Nz, g.Ny, g.K, (long)Nzp * 4, (long)g.Ny * Nzp * 4, YS_C, YS_R, 4));
    SCY_TRY(tma_map_3d(&g.mT2_32, g.t1pf.p, d32, g.Nz, g.Ny, g.K, (long)Nzp * 4, (long)g.Ny * Nzp * 4, YS_C, YS_R, 2));
    // digit planes of the z transforms: the operand (K*Ny rows of Nz) and
    // the weights, rows of Vz^T (forward) and of Vz (inverse); Vz is
    // column-major, so its columns are the forward weights' rows
    {
      const int S = zt_planes, Nz = g.Nz;
      SCY_TRY(g.zx.alloc(S, (int)rowsT, Nz, 128));
      SCY_TRY(g.zw1.alloc_weights(S, Nz, Nz));
      SCY_TRY(g.zw2.alloc_weights(S, Nz, Nz));
      std::vector<double> vz((size_t)Nz * Nz), vzt((size_t)Nz * Nz);
      SCY_CUDA_TRY(cudaMemcpy(vz.data(), g.fd->Vz.p, vz.size() * 8, cudaMemcpyDeviceToHost));
      for (int k = 0; k < Nz; ++k)
        for (int m = 0; m < Nz; ++m) vzt[(size_t)k * Nz + m] = vz[(size_t)m * Nz + k];
      SCY_TRY(ozk_set_host(g.zw1, vz.data(), Nz, 0));
      SCY_TRY(ozk_set_host(g.zw2, vzt.data(), Nz, 0));
      if (ozk_bf16_exact(S, Nz)) {
        SCY_TRY(g.zx16.alloc(S, (int)rowsT, Nz, 128, 2));
        SCY_TRY(g.zw1_16.alloc_weights(S, Nz, Nz, 2));
        SCY_TRY(g.zw2_16.alloc_weights(S, Nz, Nz, 2));
        SCY_TRY(ozk_set_host(g.zw1_16, vz.data(), Nz, 0));
        SCY_TRY(ozk_set_host(g.zw2_16, vzt.data(), Nz, 0));
      }
      SCY_TRY(ozk_prepare(S));
    }
    // every launch shape of launch_ysolve gets the shared memory of the
    // eight-instance layout (the smaller shapes use part of it)
#define SCY_YS_ATTR(I, W)                                                                                    \
  do {                                                                                                      \
    SCY_CUDA_TRY(cudaFuncSetAttribute(b_ysolve_tma_kernel<double, I, W>,                                    \
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, ys_smem_bytes(8)));      \
    SCY_CUDA_TRY(cudaFuncSetAttribute(b_ysolve_tma_kernel<float, I, W>,                                     \
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, ys_smem_bytes(4)));      \
  } while (0)
    SCY_YS_ATTR(2, 2);
    SCY_YS_ATTR(1, 4);
    SCY_YS_ATTR(4, 1);
    SCY_YS_ATTR(1, 2);
    SCY_YS_ATTR(2, 1);
    SCY_YS_ATTR(1, 1);
#undef SCY_YS_ATTR
  }
  SCY_TRY(g.tab.alloc(sizeof(BatchInst) * g.K));
  SCY_CUDA_TRY(cudaMemcpy(g.tab.p, tab.data(), sizeof(BatchInst) * g.K, cudaMemcpyHostToDevice));
  SCY_CUDA_TRY(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
  SCY_CUDA_TRY(cudaEventCreateWithFlags(&g.join, cudaEventDisableTiming));
  SCY_BLAS_TRY(cublasCreate(&g.blas));
  const size_t ws = 32u << 20;
  SCY_TRY(g.blas_ws.alloc(ws));
  SCY_BLAS_TRY(cublasSetWorkspace(g.blas, g.blas_ws.p, ws));
  SCY_BLAS_TRY(cublasSetMathMode(g.blas, CUBLAS_DEFAULT_MATH));
  SCY_TRY(autotune(g));
  groups.push_back(std::move(G));
  return SCY_OK;
}

// The banded sweeps in one of their launch shapes: variant 0 two chains per
// lane and two warps per block, 1 one chain and four warps, 2 four chains
// and one warp (a block serves eight instances in each)
int BatchContext::launch_ysolve(BatchGroup& g, int variant) {
  FDPrecond& F = *g.fd;
  const int Ny = g.Ny, Nz = g.Nz, K = g.K;
  const bool f32 = precision != SCY_PREC_FP64;
  const int sm = ys_smem_bytes(f32 ? 4 : 8);
  // B = 2 I W instances per block: the transform map whose box holds B of them
#define SCY_YS_LAUNCH(I, W, M64, M32)                                                                             \
  do {                                                                                                              \
    constexpr int B = 2 * (I) * (W);                                                                                \
    const dim3 grid((Nz + YS_C - 1) / YS_C, (K + B - 1) / B);                                                      \
    if (f32)                                                                                                        \
      b_ysolve_tma_kernel<float, I, W><<<grid, 32 * W, sm, g.stream>>>(g.mLcol32, g.mLrow32, M32,                  \
                                                                       g.t1pf.as<float>(), Ny, Nz, F.Nzp, K,        \
                                                                       g.w.status, sweep_polls, sweep_drop);        \
    else                                                                                                            \
      b_ysolve_tma_kernel<double, I, W><<<grid, 32 * W, sm, g.stream>>>(g.mLcol, g.mLrow, M64, g.t1p.as<double>(),  \
                                                                        Ny, Nz, F.Nzp, K, g.w.status, sweep_polls,  \
                                                                        sweep_drop);                                \
  } while (0)
  static_assert(2 * 2 * 2 == YS_B && 2 * 4 * 1 == YS_B && 2 * 1 * 4 == YS_B, "sweep variants 0-2 serve YS_B instances");
  if (variant == 1)
    SCY_YS_LAUNCH(1, 4, g.mT, g.mT32);
  else if (variant == 2)
    SCY_YS_LAUNCH(4, 1, g.mT, g.mT32);
  else if (variant == 3)
    SCY_YS_LAUNCH(1, 2, g.mT4, g.mT4_32);
  else if (variant == 4)
    SCY_YS_LAUNCH(2, 1, g.mT4, g.mT4_32);
  else if (variant == 5)
    SCY_YS_LAUNCH(1, 1, g.mT2, g.mT2_32);
  else
    SCY_YS_LAUNCH(2, 2, g.mT, g.mT32);
#undef SCY_YS_LAUNCH
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

// Times, on the group's own buffers (their contents do not matter here),
// the CG operator kernel with 1, 2, 4 and 8 instances per block and the
// banded sweeps in their three launch shapes; keeps the fastest of each.
// The sweep's status words are cleared afterwards.
int BatchContext::autotune(BatchGroup& g) {
  DevBuf ones;
  SCY_TRY(ones.alloc((size_t)g.K * sizeof(int)));
  std::vector<int> h(g.K, 1);
  SCY_CUDA_TRY(cudaMemcpy(ones.p, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice));
  const int* mask = ones.as<int>();
  cudaEvent_t e0, e1;
  SCY_CUDA_TRY(cudaEventCreate(&e0));
  SCY_CUDA_TRY(cudaEventCreate(&e1));
  auto timed = [&](auto&& launch, double* us) -> int {
    SCY_TRY(launch());  // warm-up
    SCY_CUDA_TRY(cudaEventRecord(e0, g.stream));
    for (int r = 0; r < 3; ++r) SCY_TRY(launch());
    SCY_CUDA_TRY(cudaEventRecord(e1, g.stream));
    SCY_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.0f;
    SCY_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    *us = ms * 1e3 / 3.0;
    return SCY_OK;
  };
  const BatchInst* tab = g.tab.as<BatchInst>();
  const double* C = g.planes.as<double>();
  const int mixed = precision != SCY_PREC_FP64 ? 1 : 0;
  int best = g.kpb;
  double best_us = 1e300;
  const int cands[4] = {1, 2, 4, 8};
  for (int c = 0; c < 4; ++c) {
    const int kpb = cands[c];
    if (kpb > XKPB || (kpb > 1 && kpb > g.K)) continue;
    const dim3 tg((g.Nz + XTZ - 1) / XTZ, (g.Ny + XTY - 1) / XTY, (g.K + kpb - 1) / kpb);
    double us = 0.0;
    int rc = timed(
        [&]() -> int {
          if (mixed)
            b_cross_kernel<1, float><<<tg, XT, xs_smem_bytes(1, 4), g.stream>>>(C, g.Ny, g.Nz, tab, mask, g.w, g.w.z32,
                                                                                1, 0, mixed, kpb, 1);
          else
            b_cross_kernel<1, double><<<tg, XT, xs_smem_bytes(1, 8), g.stream>>>(C, g.Ny, g.Nz, tab, mask, g.w, g.w.z,
                                                                                 1, 0, mixed, kpb, 1);
          SCY_LAUNCH_CHECK();
          return SCY_OK;
        },
        &us);
    if (rc != SCY_OK) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return rc;
    }
    g.tune_us[c] = us;
    if (us < best_us) {
      best_us = us;
      best = kpb;
    }
  }
  g.kpb = best;
  // the separable form (when the operator is separable over every node) at
  // 1, 2 and 4 rows per thread: used whenever it exists, so that a group's
  // results do not depend on timings (its arithmetic differs from the cross
  // form's by rounding; its rows per thread change nothing, see
  // b_full_kernel); the cross form's timings stay for comparison
  g.full_shape = -1;
  if (g.L.full) {
    best_us = 1e300;
    for (int c = 0; c < kFullShapes; ++c) {
      double us = 0.0;
      int rc = timed(
          [&]() -> int {
            if (mixed)
              launch_full<1, float>(g, c, tab, mask, g.w.z32, 1, 0, mixed, 1);
            else
              launch_full<1, double>(g, c, tab, mask, g.w.z, 1, 0, mixed, 1);
            SCY_LAUNCH_CHECK();
            return SCY_OK;
          },
          &us);
      if (rc != SCY_OK) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return rc;
      }
      g.tune_us[14 + c] = us;
      if (us < best_us) {
        best_us = us;
        g.full_shape = c;
      }
    }
  }
  if (g.fd->ybanded && !fd_dense) {
    double best_ys = 1e300;
    for (int v = 0; v < 6; ++v) {
      double us = 0.0;
      int rc = timed([&]() -> int { return launch_ysolve(g, v); }, &us);
      if (rc != SCY_OK) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return rc;
      }
      g.tune_us[4 + v] = us;
      if (us < best_ys) {
        best_ys = us;
        g.ys_variant = v;
      }
    }
    // the forward z-transform product in its three shapes (one CTA per
    // tile, two CTAs per SM, persistent) and both digit formats (identical
    // results)
    {
      double zbest = 1e300;
      for (int bf = 0; bf < 2; ++bf) {
        if (bf && !g.zx16.dig.p) continue;
        for (int pr = 0; pr < 3; ++pr) {
          if (pr && ozk_cols_per_tile_pair(zt_planes) == 0) continue;
          const OzkOperand& X = bf ? g.zx16 : g.zx;
          const OzkOperand& W = bf ? g.zw1_16 : g.zw1;
          double us = 0.0;
          int rc = timed(
              [&]() -> int {
                if (precision != SCY_PREC_FP64)
                  return ozk_gemm(X, W, g.t1pf.as<float>(), g.fd->Nzp, g.Nz, g.stream, nullptr, g.Ny, 4u, pr);
                return ozk_gemm(X, W, g.t1p.as<double>(), g.fd->Nzp, g.Nz, g.stream, nullptr, g.Ny, 4u, pr);
              },
              &us);
          if (rc != SCY_OK) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return rc;
          }
          g.tune_us[pr == 2 ? 20 + bf : 10 + 2 * bf + pr] = us;
          if (us < zbest) {
            zbest = us;
            g.zt_pair = pr;
            g.zt_bf16 = bf;
          }
        }
      }
      if (g.zt_bf16) {
        g.zx = std::move(g.zx16);
        g.zw1 = std::move(g.zw1_16);
        g.zw2 = std::move(g.zw2_16);
      } else {
        g.zx16 = OzkOperand();
        g.zw1_16 = OzkOperand();
        g.zw2_16 = OzkOperand();
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  SCY_CUDA_TRY(cudaStreamSynchronize(g.stream));
  SCY_CUDA_TRY(cudaMemset(g.status.p, 0, (size_t)g.K * 4));
  return SCY_OK;
}

int BatchContext::active_in(const BatchGroup& g, const int* mask) const {
  const int* h = reinterpret_cast<const int*>(static_cast<const double*>(ctl_host) + 2 * n);
  if (mask == d_acc(g)) h += n;
  else if (mask == d_run(g)) h += 2 * n;
  int c = 0;
  for (int k = 0; k < g.K; ++k) c += h[g.base + k] ? 1 : 0;
  return c;
}

int BatchContext::prof_begin(cudaStream_t s, cudaEvent_t* a) {
  *a = nullptr;
  if (!prof || graphs) return SCY_OK;
  SCY_CUDA_TRY(cudaEventCreate(a));
  SCY_CUDA_TRY(cudaEventRecord(*a, s));
  return SCY_OK;
}

int BatchContext::prof_end(cudaStream_t s, cudaEvent_t a, int tag, double bytes) {
  if (!a) return SCY_OK;
  ProfRec r{a, nullptr, tag, bytes};
  SCY_CUDA_TRY(cudaEventCreate(&r.b));
  SCY_CUDA_TRY(cudaEventRecord(r.b, s));
  precs.push_back(r);
  return SCY_OK;
}

int BatchContext::prof_collect(int tag, double* ms, long long* launches, double* bytes) {
  double tms = 0.0, tb = 0.0;
  long long nl = 0;
  for (auto& r : precs) {
    if (r.tag == tag) {
      SCY_CUDA_TRY(cudaEventSynchronize(r.b));
      float m = 0.0f;
      SCY_CUDA_TRY(cudaEventElapsedTime(&m, r.a, r.b));
      tms += m;
      tb += r.bytes;
      ++nl;
    }
  }
  *ms = tms;
  *launches = nl;
  *bytes = tb;
  return SCY_OK;
}

// z = K_sep^-1 r for every instance of the group (instance k's r at k*N):
// Z = Vz [ (Vz^T R Vy) ./ (lz + ly) ] Vy^T with R the Nz x Ny column-major
// view of an instance; the outer products act on all instances at once
// (Nz x Ny*K), the inner ones as strided batches.
int BatchContext::fd_apply(BatchGroup& g) {
  FDPrecond& F = *g.fd;
  const int Ny = g.Ny, Nz = g.Nz, K = g.K;
  const long N = g.N;
  SCY_BLAS_TRY(cublasSetStream(g.blas, g.stream));
  dim3 sg(node_blocks(N), 1, K);
  if (F.ybanded && !fd_dense) {
    // Z = Vz [ per z mode: (Ky + lz_j My)^-1 along y ] (Vz^T R): the z
    // transforms on the integer tensor cores (digit planes of the operand,
    // then the product), the banded sweeps in between; a pipeline wait that
    // runs out marks the instances of its tile (status bit 4) for a repeat
    const double rowsT = (double)Ny * K;
    const int S = zt_planes;
    const double split_b = rowsT * ((precision != SCY_PREC_FP64 ? 4.0 : 8.0) * Nz + S * (double)g.zx.Kp + 4.0);
    const double gemm_b = rowsT * (S * (double)g.zx.Kp + 4.0) + 2.0 * S * Nz * (double)g.zx.Kp +
                          rowsT * Nz * (precision != SCY_PREC_FP64 ? 4.0 : 8.0);
    cudaEvent_t pa;
    if (precision != SCY_PREC_FP64) {
      float* t1 = g.t1pf.as<float>();
      SCY_TRY(prof_begin(g.stream, &pa));
      SCY_TRY(ozk_split(g.zx, g.w.r, Nz, g.stream));
      SCY_TRY(prof_end(g.stream, pa, PROF_ZSPLIT, split_b));
      SCY_TRY(prof_begin(g.stream, &pa));
      SCY_TRY(ozk_gemm(g.zx, g.zw1, t1, F.Nzp, Nz, g.stream, g.w.status, Ny, 4u, g.zt_pair));
      SCY_TRY(prof_end(g.stream, pa, PROF_ZTRANSFORM, gemm_b));
      SCY_TRY(prof_begin(g.stream, &pa));
      SCY_TRY(launch_ysolve(g, g.ys_variant));
      SCY_TRY(prof_end(g.stream, pa, PROF_YSOLVE, 4.0 * (9.0 * Ny * Nz + 4.0 * N * K)));
      SCY_TRY(prof_begin(g.stream, &pa));
      SCY_TRY(ozk_split(g.zx, (const float*)t1, F.Nzp, g.stream));
      SCY_TRY(prof_end(g.stream, pa, PROF_ZSPLIT, split_b));
      SCY_TRY(prof_begin(g.stream, &pa));
      SCY_TRY(ozk_gemm(g.zx, g.zw2, g.w.z32, Nz, Nz, g.stream, g.w.status, Ny, 4u, g.zt_pair));
      SCY_TRY(prof_end(g.stream, pa, PROF_ZTRANSFORM, gemm_b));
    } else {
      double* t1 = g.t1p.as<double>();
      SCY_TRY(prof_begin(g.stream, &pa));
      SCY_TRY(ozk_split(g.zx, g.w.r, Nz, g.stream));
      SCY_TRY(prof_end(g.stream, pa, PROF_ZSPLIT, split_b));
      SCY_TRY(prof_begin(g.stream, &pa));
      SCY_TRY(ozk_gemm(g.zx, g.zw1, t1, F.Nzp, Nz, g.stream, g.w.status, Ny, 4u, g.zt_pair));
      SCY_TRY(prof_end(g.stream, pa, PROF_ZTRANSFORM, gemm_b));
      SCY_TRY(prof_begin(g.stream, &pa));
      SCY_TRY(launch_ysolve(g, g.ys_variant));
      SCY_TRY(prof_end(g.stream, pa, PROF_YSOLVE, 8.0 * (9.0 * Ny * Nz + 4.0 * N * K)));
      SCY_TRY(prof_begin(g.stream, &pa));
      SCY_TRY(ozk_split(g.zx, (const double*)t1, F.Nzp, g.stream));
      SCY_TRY(prof_end(g.stream, pa, PROF_ZSPLIT, split_b));
      SCY_TRY(prof_begin(g.stream, &pa));
      SCY_TRY(ozk_gemm(g.zx, g.zw2, g.w.z, Nz, Nz, g.stream, g.w.status, Ny, 4u, g.zt_pair));
      SCY_TRY(prof_end(g.stream, pa, PROF_ZTRANSFORM, gemm_b));
    }
    return SCY_OK;
  }
  if (precision != SCY_PREC_FP64) {
    SCY_BLAS_TRY(cublasSetMathMode(g.blas, precision == SCY_PREC_TF32 ? CUBLAS_TF32_TENSOR_OP_MATH
                                                                     : CUBLAS_DEFAULT_MATH));
    const float one = 1.0f, zero = 0.0f;
    const float* vy = F.Vy32.as<float>();
    const float* vz = F.Vz32.as<float>();
    SCY_BLAS_TRY(cublasSgemm(g.blas, CUBLAS_OP_T, CUBLAS_OP_N, Nz, Ny * K, Nz, &one, vz, Nz, g.w.r32, Nz, &zero,
                             g.w.t1f, Nz));
    SCY_BLAS_TRY(cublasSgemmStridedBatched(g.blas, CUBLAS_OP_N, CUBLAS_OP_N, Nz, Ny, Ny, &one, g.w.t1f, Nz, N, vy,
                                           Ny, 0, &zero, g.w.t2f, Nz, N, K));
    b_scale_kernel<float><<<sg, TB, 0, g.stream>>>(g.w.t2f, F.inv_lam32.as<float>(), N);
    SCY_LAUNCH_CHECK();
    SCY_BLAS_TRY(cublasSgemmStridedBatched(g.blas, CUBLAS_OP_N, CUBLAS_OP_T, Nz, Ny, Ny, &one, g.w.t2f, Nz, N, vy,
                                           Ny, 0, &zero, g.w.t1f, Nz, N, K));
    SCY_BLAS_TRY(cublasSgemm(g.blas, CUBLAS_OP_N, CUBLAS_OP_N, Nz, Ny * K, Nz, &one, vz, Nz, g.w.t1f, Nz, &zero,
                             g.w.z32, Nz));
  } else {
    SCY_BLAS_TRY(cublasSetMathMode(g.blas, CUBLAS_DEFAULT_MATH));
    const double one = 1.0, zero = 0.0;
    const double* vy = F.Vy.as<double>();
    const double* vz = F.Vz.as<double>();
    SCY_BLAS_TRY(cublasDgemm(g.blas, CUBLAS_OP_T, CUBLAS_OP_N, Nz, Ny * K, Nz, &one, vz, Nz, g.w.r, Nz, &zero,
                             g.w.t1, Nz));
    SCY_BLAS_TRY(cublasDgemmStridedBatched(g.blas, CUBLAS_OP_N, CUBLAS_OP_N, Nz, Ny, Ny, &one, g.w.t1, Nz, N, vy, Ny,
                                           0, &zero, g.w.t2, Nz, N, K));
    b_scale_kernel<double><<<sg, TB, 0, g.stream>>>(g.w.t2, F.inv_lam.as<double>(), N);
    SCY_LAUNCH_CHECK();
    SCY_BLAS_TRY(cublasDgemmStridedBatched(g.blas, CUBLAS_OP_N, CUBLAS_OP_T, Nz, Ny, Ny, &one, g.w.t2, Nz, N, vy, Ny,
                                           0, &zero, g.w.t1, Nz, N, K));
    SCY_BLAS_TRY(cublasDgemm(g.blas, CUBLAS_OP_N, CUBLAS_OP_N, Nz, Ny * K, Nz, &one, vz, Nz, g.w.t1, Nz, &zero,
                             g.w.z, Nz));
  }
  for (int i = 0; i < 4; ++i) count_launch();
  return SCY_OK;
}

int BatchContext::solve(BatchGroup& g, const int* mask, int its_now) {
  const int mixed = precision != SCY_PREC_FP64 ? 1 : 0;
  const int shape = g.full_shape, rpt = shape >= 0 ? kFullRpt[shape] : 0;  // rpt > 0: the separable form
  const dim3 tg = rpt ? full_grid(g, rpt)
                      : dim3((g.Nz + XTZ - 1) / XTZ, (g.Ny + XTY - 1) / XTY, (g.K + g.kpb - 1) / g.kpb);
  const dim3 ng(node_blocks(g.N), 1, g.K);
  const BatchInst* tab = g.tab.as<BatchInst>();
  const double* C = g.planes.as<double>();
  const int ntiles = (int)(((g.Nz + XTZ - 1) / XTZ) * ((g.Ny + XTY - 1) / XTY));  // partials of either form
  // algorithmic bytes: the coefficient planes once (the cross form), per
  // node and active instance the operand, rhs and result (residual) or z,
  // p_old, p and q
  const double nact = (double)active_in(g, mask);
  const double coef_b = rpt ? 0.0 : 33.0 * 8 * g.N;
  cudaEvent_t pa;
  SCY_TRY(prof_begin(g.stream, &pa));
  if (rpt)
    launch_full<0, double>(g, shape, tab, mask, (const double*)nullptr, 0, 0, mixed, 0);
  else
    b_cross_kernel<0, double><<<tg, XT, xs_smem_bytes(0, 8), g.stream>>>(C, g.Ny, g.Nz, tab, mask, g.w, nullptr, 0,
                                                                         0, mixed, g.kpb);
  SCY_LAUNCH_CHECK();
  SCY_TRY(prof_end(g.stream, pa, PROF_RESIDUAL, coef_b + nact * g.N * (24.0 + (mixed ? 4 : 0))));
  b_partials_kernel<<<g.K, 256, 0, g.stream>>>(mask, g.w, ntiles, 5);
  SCY_LAUNCH_CHECK();
  int pi = 0;
  for (int it = 1; it <= its_now; ++it) {
    // the first iteration has p = z: r.z comes with the operator kernel, p
    // is stored only for a later iteration, and the update reads z for it
    const int first = it == 1, last = it == its_now, store_p = !(first && last);
    SCY_TRY(fd_apply(g));
    if (!first) {
      if (mixed)
        b_dot_rz_kernel<float><<<ng, TB, 0, g.stream>>>(mask, g.w, g.w.z32);
      else
        b_dot_rz_kernel<double><<<ng, TB, 0, g.stream>>>(mask, g.w, g.w.z);
      SCY_LAUNCH_CHECK();
    }
    SCY_TRY(prof_begin(g.stream, &pa));
    if (rpt && mixed)
      launch_full<1, float>(g, shape, tab, mask, g.w.z32, first, pi, mixed, store_p);
    else if (rpt)
      launch_full<1, double>(g, shape, tab, mask, g.w.z, first, pi, mixed, store_p);
    else if (mixed)
      b_cross_kernel<1, float><<<tg, XT, xs_smem_bytes(1, 4), g.stream>>>(C, g.Ny, g.Nz, tab, mask, g.w, g.w.z32, first,
                                                                           pi, mixed, g.kpb, store_p);
    else
      b_cross_kernel<1, double><<<tg, XT, xs_smem_bytes(1, 8), g.stream>>>(C, g.Ny, g.Nz, tab, mask, g.w, g.w.z, first,
                                                                            pi, mixed, g.kpb, store_p);
    SCY_LAUNCH_CHECK();
    // z, q, p when stored, and r (first iteration) or p_old (later ones)
    SCY_TRY(prof_end(g.stream, pa, PROF_MATVEC,
                     coef_b + nact * g.N * ((mixed ? 4.0 : 8.0) + 8.0 + (store_p ? 8.0 : 0.0) + 8.0)));
    b_partials_kernel<<<g.K, 256, 0, g.stream>>>(mask, g.w, ntiles, 4);
    SCY_LAUNCH_CHECK();
    if (first) {
      b_partials_kernel<<<g.K, 256, 0, g.stream>>>(mask, g.w, ntiles, 2, 1);
      SCY_LAUNCH_CHECK();
    }
    b_update_kernel<<<ng, TB, 0, g.stream>>>(tab, mask, g.w, pi, mixed, store_p ? 0 : 1, last);
    SCY_LAUNCH_CHECK();
    pi ^= 1;
  }
  b_verify_kernel<<<(g.K + 127) / 128, 128, 0, g.stream>>>(mask, g.w, rtol, atol);
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

int BatchContext::d_dt(BatchGroup& g, const int* mask, double c, int in_slot, int out_slot, int its_now) {
  const BatchInst* tab = g.tab.as<BatchInst>();
  const dim3 fg((g.Nz + 63) / 64, 1, g.K);
  const dim3 ng(node_blocks(g.N), 1, g.K);
  b_bc_kernel<<<fg, 64, 0, g.stream>>>(tab, mask, d_t(), d_dt_(), g.base, c, in_slot);
  SCY_LAUNCH_CHECK();
  if (!pl && g.Ny > 2 * BAND && g.Nz > 2 * BAND) {
    const int nframe = 2 * BAND * g.Nz + (g.Ny - 2 * BAND) * 2 * BAND;
    const dim3 rg((nframe + TB - 1) / TB < 64 ? (nframe + TB - 1) / TB : 64, 1, g.K);
    b_rhs_frame_kernel<<<rg, TB, 0, g.stream>>>(g.L, tab, mask, g.w, nframe);
  } else {
    b_rhs_kernel<<<ng, TB, 0, g.stream>>>(g.L, tab, mask, in_slot, g.w);
  }
  SCY_LAUNCH_CHECK();
  SCY_TRY(solve(g, mask, its_now));
  if (pl) {
    b_pl_rates_kernel<<<ng, TB, 0, g.stream>>>(g.L, tab, mask, in_slot, out_slot, g.N);
    SCY_LAUNCH_CHECK();
  }
  b_fault_kernel<<<fg, 64, 0, g.stream>>>(g.L, tab, mask, in_slot, out_slot);
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

int BatchContext::combine(BatchGroup& g, const int* mask, int out_slot, std::initializer_list<int> slots,
                          std::initializer_list<double> num, std::initializer_list<double> den) {
  BCombo cb{};
  int j = 0;
  for (int s : slots) cb.slot[j++] = s;
  cb.nf = j;
  j = 0;
  for (double v : num) cb.num[j++] = v;
  j = 0;
  for (double v : den) cb.den[j++] = v;
  long nv = q(g.base).nvar;
  const dim3 gr(node_blocks(nv), 1, g.K);
  b_combine_kernel<<<gr, TB, 0, g.stream>>>(g.tab.as<BatchInst>(), mask, d_dt_(), g.base, out_slot, cb);
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

// One round of one group: copy + rates at accepted states, one attempt,
// its error sums and the status words.
int BatchContext::enqueue_group(BatchGroup& g, int its_now, int phases) {
  const BatchInst* tab = g.tab.as<BatchInst>();
  const int* mc = d_copy(g);
  const int* ma = d_acc(g);
  const int* mr = d_run(g);
  const long nv = q(g.base).nvar;
  if (phases & 1) {
    b_copy_kernel<<<dim3(node_blocks(nv), 1, g.K), TB, 0, g.stream>>>(tab, mc);
    SCY_LAUNCH_CHECK();
    SCY_TRY(d_dt(g, ma, 0.0, V_VAR, V_DVAR, its_now));
  }
  if (!(phases & 2)) {
    // no attempt this round: only the status words
  } else if (method == SCY_RK32) {
    SCY_TRY(combine(g, mr, V_K, {V_DVAR}, {0.5}, {1.0}));
    SCY_TRY(d_dt(g, mr, 0.5, V_K, V_F1, its_now));
    SCY_TRY(combine(g, mr, V_K, {V_DVAR, V_F1}, {-1.0, 2.0}, {1.0, 1.0}));
    SCY_TRY(d_dt(g, mr, 1.0, V_K, V_F2, its_now));
    SCY_TRY(combine(g, mr, V_LO, {V_DVAR, V_F2}, {0.5, 0.5}, {1.0, 1.0}));
    SCY_TRY(combine(g, mr, V_HI, {V_DVAR, V_F1, V_F2}, {1.0, 2.0, 1.0}, {6.0, 3.0, 6.0}));
  } else {
    using namespace rk43;
    SCY_TRY(combine(g, mr, V_K, {V_DVAR}, {a21}, {1.0}));
    SCY_TRY(d_dt(g, mr, c2, V_K, V_F2, its_now));
    SCY_TRY(combine(g, mr, V_K, {V_DVAR, V_F2}, {a31, a32}, {1.0, 1.0}));
    SCY_TRY(d_dt(g, mr, c3, V_K, V_F3, its_now));
    SCY_TRY(combine(g, mr, V_K, {V_DVAR, V_F2, V_F3}, {a41, a42, a43}, {1.0, 1.0, 1.0}));
    SCY_TRY(d_dt(g, mr, c4, V_K, V_F4, its_now));
    SCY_TRY(combine(g, mr, V_K, {V_DVAR, V_F2, V_F3, V_F4}, {a51, a52, a53, a54}, {1.0, 1.0, 1.0, 1.0}));
    SCY_TRY(d_dt(g, mr, c5, V_K, V_F5, its_now));
    SCY_TRY(combine(g, mr, V_K, {V_DVAR, V_F2, V_F3, V_F4, V_F5}, {a61, a62, a63, a64, a65},
                    {1.0, 1.0, 1.0, 1.0, 1.0}));
    SCY_TRY(d_dt(g, mr, c6, V_K, V_F6, its_now));
    SCY_TRY(combine(g, mr, V_LO, {V_DVAR, V_F3, V_F4, V_F5, V_F6}, {hb1, hb3, hb4, hb5, hb6},
                    {1.0, 1.0, 1.0, 1.0, 1.0}));
    SCY_TRY(combine(g, mr, V_HI, {V_DVAR, V_F3, V_F4, V_F5, V_F6}, {b1, b3, b4, b5, b6}, {1.0, 1.0, 1.0, 1.0, 1.0}));
  }
  if (phases & 2) {
    b_error_kernel<<<dim3(4, 1, g.K), 1024, 0, g.stream>>>(tab, mr, g.base, err.as<double>());
    SCY_LAUNCH_CHECK();
  }
  b_status_kernel<<<(g.K + 127) / 128, 128, 0, g.stream>>>(tab, g.w, g.base, err.as<double>());
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

int BatchContext::enqueue_round(int its_now, int phases) {
  SCY_CUDA_TRY(cudaEventRecord(fork, stream));
  for (auto& G : groups) {
    BatchGroup& g = *G;
    // concurrent: every group waits for the fork only; otherwise each waits
    // for the group before it (the fork event is re-recorded behind it)
    SCY_CUDA_TRY(cudaStreamWaitEvent(g.stream, fork, 0));
    SCY_TRY(enqueue_group(g, its_now, phases));
    SCY_CUDA_TRY(cudaEventRecord(g.join, g.stream));
    if (!concurrent) SCY_CUDA_TRY(cudaEventRecord(fork, g.stream));
  }
  for (auto& G : groups) SCY_CUDA_TRY(cudaStreamWaitEvent(stream, G->join, 0));
  return SCY_OK;
}

int BatchContext::launch_round(int its_now, int phases) {
  const int key = its_now * 4 + phases;
  SCY_CUDA_TRY(cudaMemcpyAsync(ctl.p, ctl_host, ctl_bytes, cudaMemcpyHostToDevice, stream));
  if (graphs) {
    auto it = graph_of_its.find(key);
    if (it == graph_of_its.end()) {
      cudaGraph_t graph = nullptr;
      SCY_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      const long long l0 = launch_count();
      int rc = enqueue_round(its_now, phases);
      cudaError_t ce = cudaStreamEndCapture(stream, &graph);
      if (rc != SCY_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (ce != cudaSuccess) {
        set_error("capturing a batched round failed: %s", cudaGetErrorString(ce));
        return SCY_ERR_CUDA;
      }
      cudaGraphExec_t exec = nullptr;
      ce = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) {
        set_error("instantiating a batched round failed: %s", cudaGetErrorString(ce));
        return SCY_ERR_CUDA;
      }
      // the kernels recorded while capturing run again at every replay
      kernels_of_its[key] = launch_count() - l0;
      count_launches(-kernels_of_its[key]);  // recorded, not run
      it = graph_of_its.emplace(key, exec).first;
    }
    SCY_CUDA_TRY(cudaGraphLaunch(it->second, stream));
    count_launches(kernels_of_its[key]);
    ++graph_launches;
  } else {
    SCY_TRY(enqueue_round(its_now, phases));
  }
  SCY_CUDA_TRY(cudaMemcpyAsync(err_host, err.p, (size_t)n * 16 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  SCY_CUDA_TRY(cudaStreamSynchronize(stream));
  return SCY_OK;
}

// --- host step control (QDContext::integrate_steps, one attempt at a time)
void BatchContext::begin_step(int i) {
  Ctl& h = hc[i];
  QDContext& c = q(i);
  h.running = 0;
  if (h.done_steps >= h.target || c.stepCount >= c.ode.max_steps || c.currT >= c.ode.t1) return;
  ++c.stepCount;
  h.attemptCount = 0;
  h.running = 1;
  begin_attempt(i);
}

void BatchContext::begin_attempt(int i) {
  Ctl& h = hc[i];
  QDContext& c = q(i);
  ++h.attemptCount;
  if (c.currT + c.deltaT > c.ode.t1) c.deltaT = c.ode.t1 - c.currT;
  h.forced = c.forced_pos < c.forced_dt.size() ? 1 : 0;
  h.forced_accept = 0;
  if (h.forced) {
    c.deltaT = c.forced_dt[c.forced_pos];
    h.forced_accept = c.forced_acc[c.forced_pos];
    ++c.forced_pos;
  }
}

void BatchContext::consume(int i, double totErr) {
  Ctl& h = hc[i];
  QDContext& c = q(i);
  bool acc = c.ode.method == SCY_RK32 ? (totErr <= c.totTol) : (totErr < c.totTol);
  if (h.forced) acc = h.forced_accept != 0;
  const double used = c.deltaT;
  if (c.record) {
    c.log_dt.push_back(c.deltaT);
    c.log_acc.push_back(acc ? 1 : 0);
  }
  if (acc) return finish_step(i, totErr, used);
  double nd = c.compute_step_size(totErr);
  if (!h.forced) c.deltaT = nd;
  if (c.ode.min_dt == c.deltaT) return finish_step(i, totErr, used);
  ++c.numRejected;
  if (h.attemptCount >= 100) return finish_step(i, totErr, used);
  begin_attempt(i);
}

void BatchContext::finish_step(int i, double totErr, double used_dt) {
  Ctl& h = hc[i];
  QDContext& c = q(i);
  if (c.record) c.log_step_dt.push_back(used_dt);
  c.currT = c.currT + c.deltaT;
  h.copy = h.acc = 1;  // var = hi and the rates there, at the start of the next round
  if (totErr != 0.0) c.newDeltaT = c.compute_step_size(totErr);
  c.errA[1] = c.errA[0];
  c.errA[0] = totErr;
  c.last_dt = c.deltaT;
  ++h.done_steps;
  ++inst_steps;
  c.deltaT = c.newDeltaT;
  begin_step(i);
}

int BatchContext::check_fault_flags() const {
  for (int i = 0; i < n; ++i) {
    const unsigned fb = (unsigned)err_host[16 * i + 14];
    if (fb) {
      set_error("instance %d: %s", user_of[i],
                (fb & FAULT_NONFINITE) ? "non-finite value in the fault root bracket or state rate"
                                       : "rootFinder BracketedNewton did not converge");
      return (fb & FAULT_NONFINITE) ? SCY_ERR_NONFINITE : SCY_ERR_ROOT_NOCONV;
    }
  }
  return SCY_OK;
}

int BatchContext::run(long nsteps, scy_batch_stats* st) {
  // work the caller queued on an instance's own stream comes first
  for (int i = 0; i < n; ++i) SCY_CUDA_TRY(cudaStreamSynchronize(q(i).sbp.stream));
  for (int i = 0; i < n; ++i) {
    if (!q(i).ode_ready) {
      set_error("instance %d has not been begun", i);
      return SCY_ERR_STATE;
    }
    hc[i].done_steps = 0;
    hc[i].target = nsteps;
    hc[i].copy = hc[i].acc = 0;
    begin_step(i);
  }
  const int stages = method == SCY_RK32 ? 2 : 5;
  double* t = static_cast<double*>(ctl_host);
  double* dt = t + n;
  int* mcopy = reinterpret_cast<int*>(dt + n);
  int* macc = mcopy + n;
  int* mrun = macc + n;
  auto phases_of = [&]() {
    int ph = 0;
    for (int i = 0; i < n; ++i) {
      if (macc[i]) ph |= 1;
      if (mrun[i]) ph |= 2;
    }
    return ph;
  };
  while (true) {
    for (int i = 0; i < n; ++i) {
      const QDContext& c = q(i);
      t[i] = c.currT;
      dt[i] = c.deltaT;
      mcopy[i] = hc[i].copy;
      macc[i] = hc[i].acc;
      mrun[i] = hc[i].running;
    }
    const int phases = phases_of();
    if (!phases) break;
    const int its_round = its;
    SCY_TRY(launch_round(its_round, phases));
    ++rounds;
    // a missed solve tolerance: repeat the round's work for those instances
    // (the copy is done) with more iterations; later rounds use one more
    bool missed = false;
    for (int attempt = 0; attempt < 3; ++attempt) {
      bool miss = false;
      for (int i = 0; i < n; ++i) {
        const unsigned sv = (unsigned)err_host[16 * i + 15];
        if (sv && (macc[i] || mrun[i])) {
          miss = true;
        } else {
          macc[i] = mrun[i] = 0;
        }
        mcopy[i] = 0;
      }
      if (!miss) break;
      missed = true;
      SCY_TRY(check_fault_flags());
      const int redo_its = std::min(max_its, (attempt == 0 ? 2 : 8) * its_round);
      if (attempt == 2 || redo_its <= its_round) {
        unsigned bits = 0;
        for (int i = 0; i < n; ++i) bits |= (unsigned)err_host[16 * i + 15];
        if (bits & 4u) {
          set_error("batched stage solve: a bounded pipeline wait in a kernel ran out in three repeated rounds");
          return SCY_ERR_TIMEOUT;
        }
        set_error("batched stage solve missed its tolerance after %d CG iterations", redo_its);
        return SCY_ERR_CG_NOCONV;
      }
      SCY_TRY(launch_round(redo_its, phases_of()));
      ++redo_rounds;
      for (int i = 0; i < n; ++i) {
        QDContext& c = q(i);
        const long e = macc[i] + (mrun[i] ? stages : 0);
        c.n_d_dt += e;
        c.n_solves += e;
        c.n_solve_its += e * redo_its;
        stage_solves += e;
      }
    }
    // iteration-count tuning: one more after a miss; after a run of rounds
    // without one, try one fewer (a miss costs one repeated round)
    if (missed) {
      its = std::min(max_its, its_round + 1);
      probe_period = std::min(probe_period * 2, 1L << 14);
      calm_rounds = 0;
    } else if (++calm_rounds >= probe_period && its > 1) {
      --its;
      calm_rounds = 0;
    }
    SCY_TRY(check_fault_flags());
    for (int i = 0; i < n; ++i) {
      QDContext& c = q(i);
      Ctl& h = hc[i];
      const long e = h.acc + (h.running ? stages : 0);
      c.n_d_dt += e;
      c.n_solves += e;
      c.n_solve_its += e * its_round;
      stage_solves += e;
      if (h.acc) c.last_t = c.currT;
      h.copy = h.acc = 0;
      if (h.running) consume(i, c.error_from(err_host + 16 * i));
    }
  }
  stats(st);
  return SCY_OK;
}

void BatchContext::stats(scy_batch_stats* st) const {
  if (!st) return;
  st->rounds = rounds;
  st->redo_rounds = redo_rounds;
  st->graph_launches = graph_launches;
  st->instance_steps = inst_steps;
  st->stage_solves = stage_solves;
  st->cg_its = its;
  st->groups = (int)groups.size();
  int done = 1;
  for (int i = 0; i < n; ++i) {
    const QDContext& c = q(i);
    if (!(c.stepCount >= c.ode.max_steps || c.currT >= c.ode.t1)) done = 0;
  }
  st->done = done;
}

}  // namespace scy

// ---------------------------------------------------------------------------
struct scy_batch {
  scy::BatchContext ctx;
};

extern "C" {

scy_status scy_batch_create_from_in(int n, const char* const* paths, const scy_solve_opts* solve,
                                    const scy_batch_opts* opts, scy_batch** out) {
  if (!out || n < 1 || !paths) {
    scy::set_error("scy_batch_create_from_in: invalid argument");
    return SCY_ERR_ARG;
  }
  *out = nullptr;
  for (int i = 0; i < n; ++i)
    if (!paths[i]) {
      scy::set_error("scy_batch_create_from_in: path %d is NULL", i);
      return SCY_ERR_ARG;
    }
  scy_batch* b = new (std::nothrow) scy_batch();
  if (!b) return SCY_ERR_NOMEM;
  int rc = b->ctx.create(n, paths, solve, opts);
  if (rc != SCY_OK) {
    delete b;
    return rc;
  }
  *out = b;
  return SCY_OK;
}

scy_status scy_batch_destroy(scy_batch* b) {
  delete b;
  return SCY_OK;
}

scy_status scy_batch_info(scy_batch* b, int* n, int* groups, int* group_of) {
  if (!b) return SCY_ERR_ARG;
  if (n) *n = b->ctx.n;
  if (groups) *groups = (int)b->ctx.groups.size();
  if (group_of)
    for (int i = 0; i < b->ctx.n; ++i) group_of[i] = b->ctx.group_of[i];
  return SCY_OK;
}

scy_status scy_batch_instance(scy_batch* b, int i, scy_qd** q) {
  if (!b || !q || i < 0 || i >= b->ctx.n) {
    scy::set_error("scy_batch_instance: invalid argument");
    return SCY_ERR_ARG;
  }
  *q = b->ctx.inst[b->ctx.slot_of[i]];
  return SCY_OK;
}

scy_status scy_batch_state_size(scy_batch* b, long* total) {
  if (!b || !total) return SCY_ERR_ARG;
  long t = 0;
  for (int i = 0; i < b->ctx.n; ++i) t += b->ctx.inst[b->ctx.slot_of[i]]->ctx.nvar;
  *total = t;
  return SCY_OK;
}

scy_status scy_batch_set_states(scy_batch* b, const double* host) {
  if (!b || !host) return SCY_ERR_ARG;
  return b->ctx.set_states(host);
}

scy_status scy_batch_get_fault_field(scy_batch* b, int field, double* host) {
  if (!b || !host) return SCY_ERR_ARG;
  return b->ctx.get_fault_field(field, host);
}

scy_status scy_batch_set_sweep_test(scy_batch* b, int polls, int drop_first_copy) {
  if (!b || polls < 1) return SCY_ERR_ARG;
  b->ctx.sweep_polls = polls;
  b->ctx.sweep_drop = drop_first_copy ? 1 : 0;
  // captured rounds hold the old limit
  SCY_CUDA_TRY(cudaStreamSynchronize(b->ctx.stream));
  for (auto& kv : b->ctx.graph_of_its) cudaGraphExecDestroy(kv.second);
  b->ctx.graph_of_its.clear();
  return SCY_OK;
}

scy_status scy_batch_set_graphs(scy_batch* b, int on) {
  if (!b) return SCY_ERR_ARG;
  b->ctx.graphs = on ? 1 : 0;
  return SCY_OK;
}

scy_status scy_batch_profile(scy_batch* b, int on) {
  if (!b) return SCY_ERR_ARG;
  b->ctx.prof = on ? 1 : 0;
  return SCY_OK;
}

scy_status scy_batch_profile_collect(scy_batch* b, int kernel, double* ms, long long* launches, double* bytes) {
  if (!b || !ms || !launches || !bytes || kernel < 0 || kernel > 4) return SCY_ERR_ARG;
  SCY_TRY(b->ctx.prof_collect(kernel, ms, launches, bytes));
  return SCY_OK;
}

scy_status scy_batch_tuning(scy_batch* b, int g, int* kpb, int* sweep_variant, int* ztransform, double* us) {
  if (!b || g < 0 || g >= (int)b->ctx.groups.size()) return SCY_ERR_ARG;
  const scy::BatchGroup& G = *b->ctx.groups[g];
  if (kpb) *kpb = G.kpb;
  if (sweep_variant) *sweep_variant = G.ys_variant;
  if (ztransform) *ztransform = (G.zt_pair == 1 ? 1 : 0) | (G.zt_bf16 << 1) | (G.zt_pair == 2 ? 4 : 0);
  if (us)
    for (int i = 0; i < 22; ++i) us[i] = G.tune_us[i];
  return SCY_OK;
}

scy_status scy_batch_operator_form(scy_batch* b, int g, int* rows_per_thread, int* min_blocks_per_sm) {
  if (!b || !rows_per_thread || g < 0 || g >= (int)b->ctx.groups.size()) return SCY_ERR_ARG;
  const int shape = b->ctx.groups[g]->full_shape;
  *rows_per_thread = shape >= 0 ? scy::kFullRpt[shape] : 0;
  if (min_blocks_per_sm) *min_blocks_per_sm = shape >= 0 ? scy::kFullMinb[shape] : 0;
  return SCY_OK;
}

scy_status scy_batch_profile_clear(scy_batch* b) {
  if (!b) return SCY_ERR_ARG;
  for (auto& r : b->ctx.precs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  b->ctx.precs.clear();
  return SCY_OK;
}

scy_status scy_batch_run(scy_batch* b, long nsteps, scy_batch_stats* st) {
  if (!b || nsteps < 0) {
    scy::set_error("scy_batch_run: invalid argument");
    return SCY_ERR_ARG;
  }
  return b->ctx.run(nsteps, st);
}

}  // extern "C"
