// Matrix-free SBP-SAT operator on the device.
//
// A = H*(Dyy^mu + Dzz^mu) + SAT_L + SAT_R + SAT_T + SAT_B, applied as two
// banded stages per direction:
//   stage 1 (at row k):  g1 = c_k (D x)_k,  g3 = w3_k m3_k (R3 x)_k,  g4 = w4_k c_k (R4 x)_k
//   stage 2 (at row i):  (A x)_i = w_i [ (Q g1)_i - (R3^T g3)_i - (R4^T g4)_i ] + SAT_i
// with Q = H_d*D, (R3, R4) = (D3, D4) for order 4 or (D2, 0) for order 2,
// c = mu (constant grid) or mu*qy / mu*rz (curvilinear grid), m3 the
// flattened-index average of c, w = Hz*zr (y part) or Hy*yq (z part).  This is
// the product the reference assembles as a sparse matrix in
// SbpOps_m_constGrid::constructA / SbpOps_m_varGrid::constructA.
#pragma once
#include "common.cuh"

namespace scy {

constexpr int BAND = 9;  // coefficients per row, column offsets -4..+4
constexpr int HALF = 4;
constexpr int TY = 8;    // tile rows (y, slow index)
constexpr int TZ = 32;   // tile columns (z, fast index: one warp per row)
constexpr int HX = 8;    // x halo: stage-2 reach + stage-1 reach
constexpr int HG = 4;    // stage-1 result halo: stage-2 reach

template <typename T>
struct DirDev {
  int n;
  const T *D, *R3, *R4, *Q, *R3T, *R4T;  // banded n*9
  const T *w3, *w4, *Hd, *Hinvd;         // n
  T bs0[BAND], bsN[BAND];
  T alphaD;
  int bc_lo, bc_hi;  // 0 Dirichlet, 1 Neumann (y: lo=L, hi=R; z: lo=T, hi=B)
  // Interior stencil of the order-4 operators (rows 4 .. n-6 of the stage-1
  // operators, 6 .. n-8 of the stage-2 operators), copied from an interior
  // row of the tables: D at offsets -2,-1,1,2; D3 at -1..2; D4 at -2..2; Q at
  // -2,-1,1,2; D3^T at -2..1; D4^T at -2..2; and the interior R weights.
  int fast;  // 1 when these are valid (order 4, n >= 17)
  T cD[4], cR3[4], cR4[5], cQ[4], cR3T[4], cR4T[5], cw3, cw4;
};

template <typename T>
struct LevelDev {
  int Ny, Nz, var;
  DirDev<T> y, z;
  const T *cy, *cz, *m3y, *m3z, *wy, *wz, *mu, *qy, *rz, *dinv;
  // Separable interior: when sep = 1 every node of the interior box
  // [4, Ny-6] x [4, Nz-6] has cy, m3y, wz depending on iy only and cz, m3z,
  // wy on iz only (checked bitwise on the host), so interior tiles read these
  // 1D arrays (L1-resident) instead of six per-node fields.
  int sep;
  const T *cy1, *m3y1, *wz1;  // Ny
  const T *cz1, *m3z1, *wy1;  // Nz
  // With sep = 1 the two stages compose, for an interior output row i, into
  // one 9-point stencil per direction: sy(i) = sum_o Cy[i*9 + o+4] x(i+o, iz)
  // and sz at column iz = sum_o CzT[(o+4)*Nz + iz] x(iy, iz+o) (host-built).
  const T *Cy, *CzT;
  // full = 1: the outer weights are separable over every node (wy = wy1[iz],
  // wz = wz1[iy]) and the line coefficients (cy, m3y down a column; cz, m3z
  // along a row) are those of the separable interior on all but a few
  // lines, so the whole operator (closures and SAT terms included) composes
  // into one 17-point stencil per row and per column (offsets -8..8), one
  // table per line class (class 0: the separable lines; one class per
  // exceptional line, e.g. the flattened-index m3 average at the grid's
  // corners):
  // (A x)(iy,iz) = wy1[iz] sum_o Cy17[(ycls[iz]*Ny + iy)*17 + o+8] x(iy+o, iz)
  //              + wz1[iy] sum_o CzT17[(zcls[iy]*17 + o+8)*Nz + iz] x(iy, iz+o)
  int full;
  const T *Cy17, *CzT17;
  const int *ycls, *zcls;  // Nz, Ny
  // Full form only: rows [ylo, yhi] and columns [zlo, zhi] of class 0 whose
  // class-0 stencils have no entry beyond offsets -4..4 (bitwise zeros
  // there), so a tile inside both ranges needs a halo of 4; crow / ccol = 1
  // when all those rows (columns) carry the same 9 entries, held in cyc /
  // czc (a constant grid's interior).  rpt: output rows per thread of the
  // full-form tile.
  int ylo, yhi, zlo, zhi, crow, ccol, rpt;
  T cyc[BAND], czc[BAND];
};

// -------------------------------------------------------------------------
// Loaders: the value of the operand at an in-domain node.
template <typename T>
struct LoadPlain {
  const T* x;
  __device__ __forceinline__ T operator()(long node, int, int) const { return x[node]; }
};

// p = z + beta*p_old (beta = rz_new/rz_old read from device scalars, or p = z
// on the first iteration).
template <typename Tz>
struct LoadPUpdate {
  const Tz* z;
  const double* pold;
  const double* rz_new;
  const double* rz_old;
  int first;
  __device__ __forceinline__ double operator()(long node, int, int) const {
    double zv = (double)z[node];
    if (first) return zv;
    const double ro = *rz_old;
    const double beta = ro != 0.0 ? *rz_new / ro : 0.0;  // a converged residual gives rz = 0
    return zv + beta * pold[node];
  }
};

// x + P*xc: coarse-grid correction folded into the load.
template <typename T>
struct LoadProlong {
  const T* x;
  const T* xc;
  int Ncz;
  const int *jy, *jz;
  const T *wy0, *wy1, *wz0, *wz1;
  __device__ __forceinline__ T operator()(long node, int iy, int iz) const {
    int a = jy[iy], b = jz[iz];
    const T* c0 = xc + (long)a * Ncz + b;
    const T* c1 = c0 + Ncz;
    T v = wy0[iy] * (wz0[iz] * c0[0] + wz1[iz] * c0[1]) + wy1[iy] * (wz0[iz] * c1[0] + wz1[iz] * c1[1]);
    return (x ? x[node] : T(0)) + v;
  }
};

// -------------------------------------------------------------------------
// Epilogues: consume (A x) and the operand value x at the node (index and
// coordinates); return a contribution to the optional block/grid sum.
template <typename T>
struct EpiStore {
  T* out;
  T scale;
  static constexpr bool kReduce = false;
  __device__ __forceinline__ double operator()(long node, int, int, T Ax, T) const {
    out[node] = scale * Ax;
    return 0.0;
  }
};

// r = f - K x with K = -A and f = sign_f * b  ->  r = sign_f*b + A x; returns r.r
template <typename T, typename Tb>
struct EpiResidual {
  const Tb* b;
  T* r;
  T sign_b;
  static constexpr bool kReduce = true;
  __device__ __forceinline__ double operator()(long node, int, int, T Ax, T) const {
    T v = sign_b * (T)b[node] + Ax;
    r[node] = v;
    return (double)v * (double)v;
  }
};

// CG: q = K p = -A p, store p; returns p.q
struct EpiCGMatvec {
  double* pnew;
  double* q;
  static constexpr bool kReduce = true;
  __device__ __forceinline__ double operator()(long node, int, int, double Ax, double p) const {
    double qv = -Ax;
    pnew[node] = p;
    q[node] = qv;
    return p * qv;
  }
};

// Chebyshev-Jacobi step: res = b - K x = b + A x; d = c1*d + c2*dinv*res; xout = x + d
template <typename T>
struct EpiCheb {
  const T* b;
  const T* dinv;
  T* d;
  T* xout;
  T c1, c2;
  static constexpr bool kReduce = false;
  __device__ __forceinline__ double operator()(long node, int, int, T Ax, T xv) const {
    T res = b[node] + Ax;
    T dv = c2 * dinv[node] * res;
    if (c1 != T(0)) dv += c1 * d[node];
    d[node] = dv;
    xout[node] = xv + dv;
    return 0.0;
  }
};

// -------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T band_dot(const T* __restrict__ row, const T* s, int stride) {
  T acc = T(0);
#pragma unroll
  for (int j = 0; j < BAND; ++j) acc += row[j] * s[j * stride];
  return acc;
}

// One 8x32 tile of outputs per block; 256 threads.
template <typename T, class Loader, class Epi>
__device__ __forceinline__ void stencil_tile(const LevelDev<T>& L, const Loader& ld, const Epi& ep, double* partials,
                                             unsigned int* counter, double* red_out) {
  __shared__ T xs_y[(TY + 2 * HX) * TZ];
  __shared__ T xs_z[TY * (TZ + 2 * HX)];
  __shared__ T gy[3][(TY + 2 * HG) * TZ];
  __shared__ T gz[3][TY * (TZ + 2 * HG)];
  __shared__ double red[32];
  const int Ny = L.Ny, Nz = L.Nz;
  const int y0 = blockIdx.y * TY, z0 = blockIdx.x * TZ;
  const int tid = threadIdx.x;

  for (int i = tid; i < (TY + 2 * HX) * TZ; i += blockDim.x) {
    int r = i / TZ, c = i % TZ;
    int iy = y0 - HX + r, iz = z0 + c;
    T v = T(0);
    if (iy >= 0 && iy < Ny && iz < Nz) v = ld((long)iy * Nz + iz, iy, iz);
    xs_y[i] = v;
  }
  for (int i = tid; i < TY * (TZ + 2 * HX); i += blockDim.x) {
    int r = i / (TZ + 2 * HX), c = i % (TZ + 2 * HX);
    int iy = y0 + r, iz = z0 - HX + c;
    T v = T(0);
    if (iy < Ny && iz >= 0 && iz < Nz) v = ld((long)iy * Nz + iz, iy, iz);
    xs_z[i] = v;
  }
  __syncthreads();
  // (full-form levels take full_tile instead)
  const bool fast = L.y.fast && L.z.fast && y0 - HG >= 4 && y0 + TY + HG - 1 <= Ny - 6 && z0 - HG >= 4 &&
                    z0 + TZ + HG - 1 <= Nz - 6;
  if (fast && L.sep) {
    // separable interior: the composed 9-point stencils, straight from the
    // two staged tiles of x (a warp is one output row, so Cy is a broadcast)
    const int ty = tid / TZ, tz = tid % TZ;
    const int iy = y0 + ty, iz = z0 + tz;
    const long node = (long)iy * Nz + iz;
    const T* cy = L.Cy + (long)iy * BAND;
    const T* xy = xs_y + (ty + HX) * TZ + tz;
    const T* xz = xs_z + ty * (TZ + 2 * HX) + tz + HX;
    T sy = T(0), sz = T(0);
#pragma unroll
    for (int o = 0; o < BAND; ++o) {
      sy += cy[o] * xy[(o - HALF) * TZ];
      sz += L.CzT[(long)o * Nz + iz] * xz[o - HALF];
    }
    T Ax = L.wy1[iz] * sy + L.wz1[iy] * sz;
    double contrib = ep(node, iy, iz, Ax, xy[0]);
    if constexpr (Epi::kReduce) {
      if (partials != nullptr) {
        double tot = block_sum(contrib, red);
        grid_reduce_finish(tot, partials, counter, red_out, red);
      }
    }
    return;
  }
  if (fast) {
    for (int i = tid; i < (TY + 2 * HG) * TZ; i += blockDim.x) {
      int r = i / TZ, c = i % TZ;
      int k = y0 - HG + r, iz = z0 + c;
      const T* x = xs_y + (r + HALF) * TZ + c;  // row k
      long node = (long)k * Nz + iz;
      const T cyv = L.sep ? L.cy1[k] : L.cy[node];
      const T m3v = L.sep ? L.m3y1[k] : L.m3y[node];
      T d1 = L.y.cD[0] * x[-2 * TZ] + L.y.cD[1] * x[-TZ] + L.y.cD[2] * x[TZ] + L.y.cD[3] * x[2 * TZ];
      T d3 = L.y.cR3[0] * x[-TZ] + L.y.cR3[1] * x[0] + L.y.cR3[2] * x[TZ] + L.y.cR3[3] * x[2 * TZ];
      T d4 = L.y.cR4[0] * x[-2 * TZ] + L.y.cR4[1] * x[-TZ] + L.y.cR4[2] * x[0] + L.y.cR4[3] * x[TZ] +
             L.y.cR4[4] * x[2 * TZ];
      gy[0][i] = cyv * d1;
      gy[1][i] = L.y.cw3 * m3v * d3;
      gy[2][i] = L.y.cw4 * cyv * d4;
    }
    for (int i = tid; i < TY * (TZ + 2 * HG); i += blockDim.x) {
      int r = i / (TZ + 2 * HG), c = i % (TZ + 2 * HG);
      int iy = y0 + r, k = z0 - HG + c;
      const T* x = xs_z + r * (TZ + 2 * HX) + c + HALF;  // column k
      long node = (long)iy * Nz + k;
      const T czv = L.sep ? L.cz1[k] : L.cz[node];
      const T m3v = L.sep ? L.m3z1[k] : L.m3z[node];
      T d1 = L.z.cD[0] * x[-2] + L.z.cD[1] * x[-1] + L.z.cD[2] * x[1] + L.z.cD[3] * x[2];
      T d3 = L.z.cR3[0] * x[-1] + L.z.cR3[1] * x[0] + L.z.cR3[2] * x[1] + L.z.cR3[3] * x[2];
      T d4 = L.z.cR4[0] * x[-2] + L.z.cR4[1] * x[-1] + L.z.cR4[2] * x[0] + L.z.cR4[3] * x[1] + L.z.cR4[4] * x[2];
      gz[0][i] = czv * d1;
      gz[1][i] = L.z.cw3 * m3v * d3;
      gz[2][i] = L.z.cw4 * czv * d4;
    }
    __syncthreads();
    const int ty = tid / TZ, tz = tid % TZ;
    const int iy = y0 + ty, iz = z0 + tz;
    const long node = (long)iy * Nz + iz;
    const int gc = (ty + HG) * TZ + tz;  // g row of iy
    const T* g0 = gy[0] + gc;
    const T* g1 = gy[1] + gc;
    const T* g2 = gy[2] + gc;
    T sy = L.y.cQ[0] * g0[-2 * TZ] + L.y.cQ[1] * g0[-TZ] + L.y.cQ[2] * g0[TZ] + L.y.cQ[3] * g0[2 * TZ];
    sy -= L.y.cR3T[0] * g1[-2 * TZ] + L.y.cR3T[1] * g1[-TZ] + L.y.cR3T[2] * g1[0] + L.y.cR3T[3] * g1[TZ];
    sy -= L.y.cR4T[0] * g2[-2 * TZ] + L.y.cR4T[1] * g2[-TZ] + L.y.cR4T[2] * g2[0] + L.y.cR4T[3] * g2[TZ] +
          L.y.cR4T[4] * g2[2 * TZ];
    const int zc = ty * (TZ + 2 * HG) + tz + HG;  // g column of iz
    const T* h0 = gz[0] + zc;
    const T* h1 = gz[1] + zc;
    const T* h2 = gz[2] + zc;
    T sz = L.z.cQ[0] * h0[-2] + L.z.cQ[1] * h0[-1] + L.z.cQ[2] * h0[1] + L.z.cQ[3] * h0[2];
    sz -= L.z.cR3T[0] * h1[-2] + L.z.cR3T[1] * h1[-1] + L.z.cR3T[2] * h1[0] + L.z.cR3T[3] * h1[1];
    sz -= L.z.cR4T[0] * h2[-2] + L.z.cR4T[1] * h2[-1] + L.z.cR4T[2] * h2[0] + L.z.cR4T[3] * h2[1] +
          L.z.cR4T[4] * h2[2];
    const T wyv = L.sep ? L.wy1[iz] : L.wy[node];
    const T wzv = L.sep ? L.wz1[iy] : L.wz[node];
    T Ax = wyv * sy + wzv * sz;
    T xv = xs_y[(ty + HX) * TZ + tz];
    double contrib = ep(node, iy, iz, Ax, xv);
    if constexpr (Epi::kReduce) {
      if (partials != nullptr) {
        double tot = block_sum(contrib, red);
        grid_reduce_finish(tot, partials, counter, red_out, red);
      }
    }
    return;
  }
  // stage 1, y direction: rows y0-HG .. y0+TY+HG
  for (int i = tid; i < (TY + 2 * HG) * TZ; i += blockDim.x) {
    int r = i / TZ, c = i % TZ;
    int k = y0 - HG + r, iz = z0 + c;
    T g1 = T(0), g3 = T(0), g4 = T(0);
    if (k >= 0 && k < Ny && iz < Nz) {
      const T* xcol = xs_y + r * TZ + c;  // row k-4 of xs_y sits at (r + HX - HG - HALF) = r
      long node = (long)k * Nz + iz;
      T cyv = L.cy[node];
      g1 = cyv * band_dot(L.y.D + (long)k * BAND, xcol, TZ);
      g3 = L.y.w3[k] * L.m3y[node] * band_dot(L.y.R3 + (long)k * BAND, xcol, TZ);
      if (L.y.R4) g4 = L.y.w4[k] * cyv * band_dot(L.y.R4 + (long)k * BAND, xcol, TZ);
    }
    gy[0][i] = g1;
    gy[1][i] = g3;
    gy[2][i] = g4;
  }
  // stage 1, z direction: columns z0-HG .. z0+TZ+HG
  for (int i = tid; i < TY * (TZ + 2 * HG); i += blockDim.x) {
    int r = i / (TZ + 2 * HG), c = i % (TZ + 2 * HG);
    int iy = y0 + r, k = z0 - HG + c;
    T g1 = T(0), g3 = T(0), g4 = T(0);
    if (iy < Ny && k >= 0 && k < Nz) {
      const T* xrow = xs_z + r * (TZ + 2 * HX) + c;  // column k-4 sits at c
      long node = (long)iy * Nz + k;
      T czv = L.cz[node];
      g1 = czv * band_dot(L.z.D + (long)k * BAND, xrow, 1);
      g3 = L.z.w3[k] * L.m3z[node] * band_dot(L.z.R3 + (long)k * BAND, xrow, 1);
      if (L.z.R4) g4 = L.z.w4[k] * czv * band_dot(L.z.R4 + (long)k * BAND, xrow, 1);
    }
    gz[0][i] = g1;
    gz[1][i] = g3;
    gz[2][i] = g4;
  }
  __syncthreads();
  const int ty = tid / TZ, tz = tid % TZ;
  const int iy = y0 + ty, iz = z0 + tz;
  double contrib = 0.0;
  if (iy < Ny && iz < Nz) {
    const long node = (long)iy * Nz + iz;
    // y part: g rows iy-4..iy+4 sit at gy rows ty..ty+8
    const T* qrow = L.y.Q + (long)iy * BAND;
    const T* r3 = L.y.R3T + (long)iy * BAND;
    const T* r4 = L.y.R4T + (long)iy * BAND;
    T sy = T(0);
#pragma unroll
    for (int j = 0; j < BAND; ++j) {
      int gi = (ty + j) * TZ + tz;
      sy += qrow[j] * gy[0][gi] - r3[j] * gy[1][gi];
      if (L.y.R4T) sy -= r4[j] * gy[2][gi];
    }
    const int gcen_y = (ty + HG) * TZ + tz;
    // SAT on the y = 0 (L) and y = Ly (R) boundaries
    if (L.y.bc_lo == 0) {
      if (iy < BAND) sy += (L.y.bs0[iy] + (iy == 0 ? L.y.alphaD : T(0))) * L.cy[iz] * xs_y[(0 - y0 + HX) * TZ + tz];
    } else if (iy == 0) {
      sy += gy[0][gcen_y];
    }
    if (L.y.bc_hi == 0) {
      if (iy >= Ny - BAND) {
        long bn = (long)(Ny - 1) * Nz + iz;
        int rr = Ny - 1 - y0 + HX;  // row of xs_y holding iy = Ny-1 (inside the tile halo)
        sy += (L.y.bsN[iy - (Ny - BAND)] + (iy == Ny - 1 ? L.y.alphaD : T(0))) * L.cy[bn] * xs_y[rr * TZ + tz];
      }
    } else if (iy == Ny - 1) {
      sy -= gy[0][gcen_y];
    }
    // z part: g columns iz-4..iz+4 sit at gz columns tz..tz+8
    const T* qz = L.z.Q + (long)iz * BAND;
    const T* z3 = L.z.R3T + (long)iz * BAND;
    const T* z4 = L.z.R4T + (long)iz * BAND;
    T sz = T(0);
#pragma unroll
    for (int j = 0; j < BAND; ++j) {
      int gi = ty * (TZ + 2 * HG) + tz + j;
      sz += qz[j] * gz[0][gi] - z3[j] * gz[1][gi];
      if (L.z.R4T) sz -= z4[j] * gz[2][gi];
    }
    const int gcen_z = ty * (TZ + 2 * HG) + tz + HG;
    if (L.z.bc_lo == 0) {
      if (iz < BAND) sz += (L.z.bs0[iz] + (iz == 0 ? L.z.alphaD : T(0))) * L.cz[(long)iy * Nz] * xs_z[ty * (TZ + 2 * HX) + (0 - z0 + HX)];
    } else if (iz == 0) {
      sz += gz[0][gcen_z];
    }
    if (L.z.bc_hi == 0) {
      if (iz >= Nz - BAND) {
        long bn = (long)iy * Nz + Nz - 1;
        int cc = Nz - 1 - z0 + HX;
        sz += (L.z.bsN[iz - (Nz - BAND)] + (iz == Nz - 1 ? L.z.alphaD : T(0))) * L.cz[bn] * xs_z[ty * (TZ + 2 * HX) + cc];
      }
    } else if (iz == Nz - 1) {
      sz -= gz[0][gcen_z];
    }
    T Ax = L.wy[node] * sy + L.wz[node] * sz;
    T xv = xs_y[(ty + HX) * TZ + tz];
    contrib = ep(node, iy, iz, Ax, xv);
  }
  if constexpr (Epi::kReduce) {
    if (partials != nullptr) {  // uniform across the grid
      double tot = block_sum(contrib, red);
      grid_reduce_finish(tot, partials, counter, red_out, red);
    }
  }
}

// -------------------------------------------------------------------------
// Full-form tile (L.full = 1: the whole operator is one 17-point stencil per
// row and per column, see LevelDev).  A block of 256 threads owns 8*RPT rows x
// 32 columns: warp w the rows w*RPT .. w*RPT+RPT-1, a lane one column.  The
// tile and its halo are staged once in shared memory.  In an interior tile
// (rows in [ylo, yhi], columns in [zlo, zhi]) a thread keeps its column's
// RPT+8 values along y and its column's 9 z entries in registers, so an
// output costs 9 + 9 multiply-adds and 8 shared-memory reads; the other tiles
// use all 17 offsets (halo 8, zeros outside the grid).  Sums run over the
// offsets in increasing order as in the 17-point form (the skipped entries
// are zeros).

// values of the shared array full_apply stages into
template <int RPT>
constexpr int full_smem_values() {
  return (8 * RPT + 16) * (TZ + 16);
}

// Stages rows y0-H .. y0+TYB+H-1 of columns z0 .. z0+31 at (r, H + c) and
// columns z0-H .. z0-1, z0+32 .. z0+31+H of rows y0 .. y0+TYB-1 at
// (r + H, c) of xs (pitch 32 + 2H) through ld(node, iy, iz), zeros outside
// the grid when CHECK (else every node is inside).  256 threads; a thread
// issues all its loads before its stores, so they are in flight together.
template <typename T, int TYB, int H, bool CHECK, class Loader>
__device__ __forceinline__ void full_stage(const Loader& ld, T* xs, int y0, int z0, int Ny, int Nz) {
  constexpr int W = TZ + 2 * H, NM = (TYB + 2 * H) * TZ, NT = NM + TYB * 2 * H, NV = (NT + 255) / 256;
  const int tid = threadIdx.x;
  T v[NV];
  int at[NV];
#pragma unroll
  for (int a = 0; a < NV; ++a) {
    const int i = tid + 256 * a;
    int iy, iz, sx;
    if (i < NM) {
      const int r = i >> 5, c = i & 31;
      iy = y0 - H + r;
      iz = z0 + c;
      sx = r * W + H + c;
    } else {
      const int j = i - NM, r = j / (2 * H), k = j % (2 * H), c = k < H ? k : TZ + k;
      iy = y0 + r;
      iz = z0 - H + c;
      sx = (r + H) * W + c;
    }
    at[a] = i < NT ? sx : -1;
    v[a] = T(0);
    if (i < NT && (!CHECK || (iy >= 0 && iy < Ny && iz >= 0 && iz < Nz))) v[a] = ld((long)iy * Nz + iz, iy, iz);
  }
#pragma unroll
  for (int a = 0; a < NV; ++a)
    if (at[a] >= 0) xs[at[a]] = v[a];
}

// The tile of block (blockIdx.x, blockIdx.y): stages the operand through
// ld(node, iy, iz) into xs; then pre(node, iy, iz) is called for each of
// the thread's output nodes (the epilogue's own loads, issued before the
// operator is applied so their latency is hidden; default value where the
// node is outside the grid), and out(node, iy, iz, A x, x, pre value) once
// per output node of the tile; after each of its RPT rows j every thread of
// the block calls row(j) (warp-uniform, so a row's values can be summed
// across the warp there).  The interior path also stages the class-0 rows
// of the tile's y stencils in shared memory (past the operand) when they
// differ from row to row.
template <typename T, int RPT, class Loader, class Pre, class Out, class Row>
__device__ __forceinline__ void full_apply(const LevelDev<T>& L, const Loader& ld, const Pre& pre, Out& out, Row& row,
                                           T* xs) {
  constexpr int TYB = 8 * RPT;
  using P = decltype(pre(0L, 0, 0));
  const int Ny = L.Ny, Nz = L.Nz;
  const int y0 = blockIdx.y * TYB, z0 = blockIdx.x * TZ;
  const int tid = threadIdx.x, lane = tid & 31, r0 = (tid >> 5) * RPT;
  const int iz = z0 + lane;
  const bool inner = y0 >= L.ylo && y0 + TYB - 1 <= L.yhi && z0 >= L.zlo && z0 + TZ - 1 <= L.zhi;
  P pv[RPT];
  if (inner) {
    constexpr int H = HALF, W = TZ + 2 * H;
    T* cys = xs + (TYB + 2 * H) * W;  // [TYB][BAND] (within the generic layout's size)
    const bool rows_differ = !L.crow;
    constexpr int NC = (TYB * BAND + 255) / 256;
    T cyv[NC];
#pragma unroll
    for (int a = 0; a < NC; ++a) {
      const int i = tid + 256 * a;
      cyv[a] = (rows_differ && i < TYB * BAND) ? L.Cy17[(long)(y0 + i / BAND) * 17 + (8 - HALF) + i % BAND] : T(0);
    }
    full_stage<T, TYB, H, false>(ld, xs, y0, z0, Ny, Nz);  // all inside the grid
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int iy = y0 + r0 + j;
      pv[j] = pre((long)iy * Nz + iz, iy, iz);
    }
#pragma unroll
    for (int a = 0; a < NC; ++a)
      if (rows_differ && tid + 256 * a < TYB * BAND) cys[tid + 256 * a] = cyv[a];
    T cz[BAND];
#pragma unroll
    for (int o = 0; o < BAND; ++o) cz[o] = L.ccol ? L.czc[o] : L.CzT17[(long)(o + 8 - HALF) * Nz + iz];
    const T wyv = L.wy1[iz];
    __syncthreads();
    T win[RPT + 2 * H];
#pragma unroll
    for (int k = 0; k < RPT + 2 * H; ++k) win[k] = xs[(r0 + k) * W + H + lane];
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int iy = y0 + r0 + j;
      const T* cy = cys + (r0 + j) * BAND;
      const T* xr = xs + (r0 + j + H) * W + lane;  // columns iz-4 .. iz+4
      T sy = T(0), sz = T(0);
#pragma unroll
      for (int o = 0; o < BAND; ++o) {
        sy += (rows_differ ? cy[o] : L.cyc[o]) * win[j + o];
        sz += cz[o] * (o == HALF ? win[j + HALF] : xr[o]);
      }
      const T Ax = wyv * sy + L.wz1[iy] * sz;
      out((long)iy * Nz + iz, iy, iz, Ax, win[j + HALF], pv[j]);
      row(j);
    }
  } else {
    constexpr int H = 8, W = TZ + 2 * H;
    full_stage<T, TYB, H, true>(ld, xs, y0, z0, Ny, Nz);
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int iy = y0 + r0 + j;
      pv[j] = (iz < Nz && iy < Ny) ? pre((long)iy * Nz + iz, iy, iz) : P{};
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int iy = y0 + r0 + j;
      if (iz < Nz && iy < Ny) {
        const int yc = L.ycls[iz], zc = L.zcls[iy];
        const T* cy = L.Cy17 + ((long)yc * Ny + iy) * 17;
        const T* cz = L.CzT17 + (long)zc * 17 * Nz + iz;
        const T* xy = xs + (r0 + j) * W + H + lane;  // rows iy-8 .. iy+8, stride W
        const T* xz = xs + (r0 + j + H) * W + lane;  // columns iz-8 .. iz+8
        T sy = T(0), sz = T(0);
        // the 9 middle offsets where the line's stencil has no others
        if (yc == 0 && iy >= L.ylo && iy <= L.yhi) {
#pragma unroll
          for (int o = 8 - HALF; o <= 8 + HALF; ++o) sy += cy[o] * xy[o * W];
        } else {
#pragma unroll
          for (int o = 0; o < 17; ++o) sy += cy[o] * xy[o * W];
        }
        if (zc == 0 && iz >= L.zlo && iz <= L.zhi) {
#pragma unroll
          for (int o = 8 - HALF; o <= 8 + HALF; ++o) sz += cz[(long)o * Nz] * xz[o];
        } else {
#pragma unroll
          for (int o = 0; o < 17; ++o) sz += cz[(long)o * Nz] * xz[o];
        }
        const T Ax = L.wy1[iz] * sy + L.wz1[iy] * sz;
        out((long)iy * Nz + iz, iy, iz, Ax, xy[H * W], pv[j]);
      }
      row(j);
    }
  }
}

// No epilogue loads to prefetch.
struct NoPre {
  __device__ __forceinline__ int operator()(long, int, int) const { return 0; }
};

template <typename T, int RPT, class Loader, class Epi>
__device__ __forceinline__ void full_tile(const LevelDev<T>& L, const Loader& ld, const Epi& ep, double* partials,
                                          unsigned int* counter, double* red_out) {
  __shared__ T xs[full_smem_values<RPT>()];
  __shared__ double red[32];
  double contrib = 0.0;
  auto out = [&](long node, int iy, int iz, T Ax, T xv, int) { contrib += ep(node, iy, iz, Ax, xv); };
  auto row = [](int) {};
  full_apply<T, RPT>(L, ld, NoPre{}, out, row, xs);
  if constexpr (Epi::kReduce) {
    if (partials != nullptr) {  // uniform across the grid
      double tot = block_sum(contrib, red);
      grid_reduce_finish(tot, partials, counter, red_out, red);
    }
  }
}

template <typename T, int RPT, class Loader, class Epi>
__global__ void __launch_bounds__(256) full_kernel(LevelDev<T> L, Loader ld, Epi ep, double* partials,
                                                   unsigned int* counter, double* red_out) {
  full_tile<T, RPT, Loader, Epi>(L, ld, ep, partials, counter, red_out);
}

// rhs at one node from the boundary data (SbpOps::setRhs,
// sbpOps_m_constGrid.cpp:877-914): the SAT columns of the Dirichlet
// boundaries and the Neumann boundary values, times the outer weights.
__device__ __forceinline__ double set_rhs_node(const LevelDev<double>& L, const double* __restrict__ bcL,
                                               const double* __restrict__ bcR, const double* __restrict__ bcT,
                                               const double* __restrict__ bcB, long node) {
  const int Ny = L.Ny, Nz = L.Nz;
  const int iy = (int)(node / Nz), iz = (int)(node % Nz);
  double sy = 0.0, sz = 0.0;
  if (L.y.bc_lo == 0) {
    if (iy < BAND) sy += (L.y.bs0[iy] + (iy == 0 ? L.y.alphaD : 0.0)) * L.cy[iz] * bcL[iz];
  } else if (iy == 0) {
    sy += bcL[iz];
  }
  if (L.y.bc_hi == 0) {
    if (iy >= Ny - BAND)
      sy += (L.y.bsN[iy - (Ny - BAND)] + (iy == Ny - 1 ? L.y.alphaD : 0.0)) * L.cy[(long)(Ny - 1) * Nz + iz] * bcR[iz];
  } else if (iy == Ny - 1) {
    sy -= bcR[iz];
  }
  if (L.z.bc_lo == 0) {
    if (iz < BAND) sz += (L.z.bs0[iz] + (iz == 0 ? L.z.alphaD : 0.0)) * L.cz[(long)iy * Nz] * bcT[iy];
  } else if (iz == 0) {
    sz += bcT[iy];
  }
  if (L.z.bc_hi == 0) {
    if (iz >= Nz - BAND)
      sz += (L.z.bsN[iz - (Nz - BAND)] + (iz == Nz - 1 ? L.z.alphaD : 0.0)) * L.cz[(long)iy * Nz + Nz - 1] * bcB[iy];
  } else if (iz == Nz - 1) {
    sz -= bcB[iy];
  }
  return L.wy[node] * sy + L.wz[node] * sz;
}

// Shear stress mu * Dy u on the fault row iy = 0 at column iz (muxDy of
// sbpOps_m_constGrid.cpp:1481-1500 scattered to the fault,
// strikeSlip_linearElastic_qd.cpp:785-788): Dy row 0 reaches columns 0..4.
__device__ __forceinline__ double fault_row_sxy(const LevelDev<double>& L, const double* __restrict__ u, int iz) {
  const int Nz = L.Nz;
  double d = 0.0;
#pragma unroll
  for (int j = HALF; j < BAND; ++j) {
    int k = j - HALF;
    if (k < L.Ny) d += L.y.D[j] * u[(long)k * Nz + iz];
  }
  if (L.var) d *= L.qy[iz];
  return L.mu[iz] * d;
}

template <typename T, class Loader, class Epi>
__global__ void __launch_bounds__(256) stencil_kernel(LevelDev<T> L, Loader ld, Epi ep, double* partials,
                                                      unsigned int* counter, double* red_out) {
  stencil_tile<T, Loader, Epi>(L, ld, ep, partials, counter, red_out);
}

// Launch grid of an operator application: full-form tiles of 8*rpt x 32 when
// L.full, else the 8 x 32 tiles of stencil_tile.
template <typename T>
inline dim3 apply_grid(const LevelDev<T>& L) {
  const int ty = L.full ? 8 * L.rpt : TY;
  return dim3((L.Nz + TZ - 1) / TZ, (L.Ny + ty - 1) / ty);
}

// One operator application with the loader / epilogue given (the kernel the
// level's form calls for); 256 threads per block.
template <typename T, class Loader, class Epi>
inline void launch_apply(const LevelDev<T>& L, const Loader& ld, const Epi& ep, double* partials,
                         unsigned int* counter, double* red_out, cudaStream_t s) {
  const dim3 g = apply_grid(L);
  if (!L.full)
    stencil_kernel<T, Loader, Epi><<<g, 256, 0, s>>>(L, ld, ep, partials, counter, red_out);
  else if (L.rpt == 4)
    full_kernel<T, 4, Loader, Epi><<<g, 256, 0, s>>>(L, ld, ep, partials, counter, red_out);
  else if (L.rpt == 2)
    full_kernel<T, 2, Loader, Epi><<<g, 256, 0, s>>>(L, ld, ep, partials, counter, red_out);
  else
    full_kernel<T, 1, Loader, Epi><<<g, 256, 0, s>>>(L, ld, ep, partials, counter, red_out);
}

}  // namespace scy
