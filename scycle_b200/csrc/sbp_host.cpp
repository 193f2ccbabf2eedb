// Host construction of the SBP-SAT operator data consumed by the device
// stencil.  The 1D operators follow the reference's sbp_Spmat / sbp_Spmat2 /
// sbp_Spmat4 (source/spmat.cpp:310-627); the 2D composition follows
// SbpOps_m_constGrid / SbpOps_m_varGrid with multiplyByH = 1
// (source/sbpOps_m_constGrid.cpp:606-701, 963-1315;
//  source/sbpOps_m_varGrid.cpp:333-436, 1133-1504).
#include <algorithm>
#include "sbp_host.hpp"

#include <cmath>
#include <stdexcept>

namespace scy {

Sparse1D Sparse1D::transpose() const {
  Sparse1D t(n);
  for (int r = 0; r < n; ++r)
    for (auto& kv : rows[r]) t.rows[kv.first][r] = kv.second;
  return t;
}

Ops1D build_ops1d(int order, int n, double scale, int compat) {
  Ops1D o;
  o.order = order;
  o.n = n;
  o.scale = scale;
  o.D1 = Sparse1D(n);
  o.BS = Sparse1D(n);
  o.D2 = Sparse1D(n);
  o.D3 = Sparse1D(n);
  o.D4 = Sparse1D(n);
  o.H.assign(n, 1.0);
  o.Hinv.assign(n, 0.0);
  if (order == 2) {
    if (n < 3) throw std::invalid_argument("order-2 SBP needs at least 3 points");
    // spmat.cpp:330-380
    o.H[0] = 0.5;
    o.H[n - 1] = 0.5;
    for (int i = 0; i < n; ++i) o.H[i] /= scale;
    for (int i = 0; i < n; ++i) o.Hinv[i] = 1.0 / o.H[i];
    Sparse1D Dint(n);
    Dint.set(0, 0, -1.0 * scale);
    Dint.set(0, 1, scale);
    for (int i = 1; i < n - 1; ++i) {
      Dint.set(i, i - 1, -0.5 * scale);
      Dint.set(i, i + 1, 0.5 * scale);
    }
    Dint.set(n - 1, n - 1, scale);
    Dint.set(n - 1, n - 2, -1.0 * scale);
    o.D1 = Dint;
    if (compat == 0) {
      o.BS.set(0, 0, -Dint.get(0, 0));
      o.BS.set(0, 1, -Dint.get(0, 1));
      o.BS.set(n - 1, n - 2, Dint.get(n - 1, n - 2));
      o.BS.set(n - 1, n - 1, Dint.get(n - 1, n - 1));
    } else {
      o.BS.set(0, 0, 1.5 * scale);
      o.BS.set(0, 1, -2.0 * scale);
      o.BS.set(0, 2, 0.5 * scale);
      o.BS.set(n - 1, n - 3, 0.5 * scale);
      o.BS.set(n - 1, n - 2, -2.0 * scale);
      o.BS.set(n - 1, n - 1, 1.5 * scale);
      o.D1.set(0, 0, -o.BS.get(0, 0));
      o.D1.set(0, 1, -o.BS.get(0, 1));
      o.D1.set(0, 2, -o.BS.get(0, 2));
      o.D1.set(n - 1, n - 3, o.BS.get(n - 1, n - 3));
      o.D1.set(n - 1, n - 2, o.BS.get(n - 1, n - 2));
      o.D1.set(n - 1, n - 1, o.BS.get(n - 1, n - 1));
    }
    // sbp_Spmat2 (spmat.cpp:494-544)
    const double s2 = scale * scale;
    o.D2.set(0, 0, s2);
    o.D2.set(0, 1, -2.0 * s2);
    o.D2.set(0, 2, s2);
    for (int i = 1; i < n - 1; ++i) {
      o.D2.set(i, i - 1, s2);
      o.D2.set(i, i, -2.0 * s2);
      o.D2.set(i, i + 1, s2);
    }
    o.D2.set(n - 1, n - 3, s2);
    o.D2.set(n - 1, n - 2, -2.0 * s2);
    o.D2.set(n - 1, n - 1, s2);
    o.C2.assign(n, 1.0);
    o.C2[0] = 0.0;
    o.C2[n - 1] = 0.0;
    return o;
  }
  if (order != 4) throw std::invalid_argument("order must be 2 or 4");
  if (n <= 8) throw std::invalid_argument("order-4 SBP needs more than 8 points");
  // spmat.cpp:382-491
  const double hb[4] = {17.0 / 48.0, 59.0 / 48.0, 43.0 / 48.0, 49.0 / 48.0};
  for (int i = 0; i < 4; ++i) {
    o.H[i] = hb[i];
    o.H[n - 1 - i] = hb[i];
  }
  for (int i = 0; i < n; ++i) o.H[i] /= scale;
  for (int i = 0; i < n; ++i) o.Hinv[i] = 1.0 / o.H[i];
  Sparse1D Dint(n);
  auto hi = [&](int i) { return o.Hinv[i]; };
  for (int i = 4; i < n - 4; ++i) {
    Dint.set(i, i - 2, 1.0 / 12.0 * hi(i));
    Dint.set(i, i - 1, -2.0 / 3.0 * hi(i));
    Dint.set(i, i + 1, 2.0 / 3.0 * hi(i));
    Dint.set(i, i + 2, -1.0 / 12.0 * hi(i));
  }
  // boundary closure of the first-derivative operator, Q = H*D rows 0..3
  const double q[4][6] = {{-1.0 / 2.0, 59.0 / 96.0, -1.0 / 12.0, -1.0 / 32.0, 0, 0},
                          {-59.0 / 96.0, 0, 59.0 / 96.0, 0, 0, 0},
                          {1.0 / 12.0, -59.0 / 96.0, 0, 59.0 / 96.0, -1.0 / 12.0, 0},
                          {1.0 / 32.0, 0, -59.0 / 96.0, 0, 2.0 / 3.0, -1.0 / 12.0}};
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 6; ++c)
      if (q[r][c] != 0.0) {
        Dint.set(r, c, q[r][c] * hi(r));
        // mirrored closure at the far end: Q[n-1-r][n-1-c] = -Q[r][c]
        Dint.set(n - 1 - r, n - 1 - c, -q[r][c] * hi(n - 1 - r));
      }
  o.D1 = Dint;
  if (compat == 0) {
    const double bs[4] = {24.0 / 17.0, -59.0 / 34.0, 4.0 / 17.0, 3.0 / 34.0};
    for (int c = 0; c < 4; ++c) {
      o.BS.set(0, c, bs[c] * scale);
      o.BS.set(n - 1, n - 1 - c, bs[c] * scale);
    }
  } else {
    const double bs[4] = {11.0 / 6.0, -3.0, 1.5, -1.0 / 3.0};
    for (int c = 0; c < 4; ++c) {
      o.BS.set(0, c, bs[c] * scale);
      // the reference leaves the last row unscaled (spmat.cpp:463)
      o.BS.set(n - 1, n - 1 - c, bs[c]);
    }
    for (int c = 0; c < 4; ++c) o.D1.set(0, c, -o.BS.get(0, c));
    // the reference writes (n-1, n-4) twice and leaves (n-1, n-3) at its
    // interior-closure value (spmat.cpp:466)
    o.D1.set(n - 1, n - 4, o.BS.get(n - 1, n - 4));
    o.D1.set(n - 1, n - 2, o.BS.get(n - 1, n - 2));
    o.D1.set(n - 1, n - 1, o.BS.get(n - 1, n - 1));
  }
  // sbp_Spmat4 (spmat.cpp:547-627)
  for (int r = 0; r < 2; ++r) {
    o.D3.set(r, 0, -1); o.D3.set(r, 1, 3); o.D3.set(r, 2, -3); o.D3.set(r, 3, 1);
  }
  const double d3r2[6] = {-185893.0 / 301051.0, 79000249461.0 / 54642863857.0,
                          -33235054191.0 / 54642863857.0, -36887526683.0 / 54642863857.0,
                          26183621850.0 / 54642863857.0, -4386.0 / 181507.0};
  for (int c = 0; c < 6; ++c) o.D3.set(2, c, d3r2[c]);
  for (int i = 3; i < n - 4; ++i) {
    o.D3.set(i, i - 1, -1.0); o.D3.set(i, i, 3); o.D3.set(i, i + 1, -3); o.D3.set(i, i + 2, 1.0);
  }
  for (int c = 0; c < 6; ++c) o.D3.set(n - 3, n - 1 - c, -d3r2[c]);
  for (int r = n - 2; r < n; ++r) {
    o.D3.set(r, n - 4, -1); o.D3.set(r, n - 3, 3); o.D3.set(r, n - 2, -3); o.D3.set(r, n - 1, 1);
  }
  const double d4[5] = {1, -4, 6, -4, 1};
  for (int c = 0; c < 5; ++c) {
    o.D4.set(0, c, d4[c]);
    o.D4.set(1, c, d4[c]);
    o.D4.set(n - 2, n - 5 + c, d4[c]);
    o.D4.set(n - 1, n - 5 + c, d4[c]);
  }
  for (int i = 2; i < n - 2; ++i)
    for (int c = 0; c < 5; ++c) o.D4.set(i, i - 2 + c, d4[c]);
  o.C3.assign(n, 1.0);
  o.C3[0] = 0; o.C3[1] = 0;
  o.C3[2] = 163928591571.0 / 53268010936.0;
  o.C3[3] = 189284.0 / 185893.0;
  o.C3[n - 5] = o.C3[3];
  o.C3[n - 4] = 0;
  o.C3[n - 3] = o.C3[2];
  o.C3[n - 2] = 0;
  o.C3[n - 1] = 0;
  o.C4.assign(n, 1.0);
  o.C4[0] = 0; o.C4[1] = 0;
  o.C4[2] = 1644330.0 / 301051.0;
  o.C4[3] = 156114.0 / 181507.0;
  o.C4[n - 4] = o.C4[3];
  o.C4[n - 3] = o.C4[2];
  o.C4[n - 2] = 0;
  o.C4[n - 1] = 0;
  return o;
}

std::vector<double> to_band(const Sparse1D& m) {
  std::vector<double> b((size_t)m.n * kBand, 0.0);
  for (int r = 0; r < m.n; ++r)
    for (auto& kv : m.rows[r]) {
      int off = kv.first - r;
      if (off < -kHalf || off > kHalf) throw std::invalid_argument("operator row reaches beyond +-4");
      b[(size_t)r * kBand + off + kHalf] = kv.second;
    }
  return b;
}

DirTables build_dir_tables(int order, int n, double h, int compat) {
  Ops1D o = build_ops1d(order, n, 1.0 / h, compat);
  DirTables t;
  t.n = n;
  t.D = to_band(o.D1);
  Sparse1D Q(n);
  for (int r = 0; r < n; ++r)
    for (auto& kv : o.D1.rows[r]) Q.rows[r][kv.first] = o.H[r] * kv.second;
  t.Q = to_band(Q);
  if (order == 4) {
    t.nterms = 3;
    t.R3 = to_band(o.D3);
    t.R4 = to_band(o.D4);
    t.R3T = to_band(o.D3.transpose());
    t.R4T = to_band(o.D4.transpose());
    t.w3.resize(n);
    t.w4.resize(n);
    for (int k = 0; k < n; ++k) {
      t.w3[k] = o.C3[k] * (1.0 / h / 18.0);
      t.w4[k] = o.C4[k] * (1.0 / h / 144.0);
    }
    t.alphaD = 2.0 * -48.0 / 17.0 / h;
  } else {
    t.nterms = 2;
    t.R3 = to_band(o.D2);
    t.R3T = to_band(o.D2.transpose());
    t.R4.assign((size_t)n * kBand, 0.0);
    t.R4T.assign((size_t)n * kBand, 0.0);
    t.w3.resize(n);
    t.w4.assign(n, 0.0);
    for (int k = 0; k < n; ++k) t.w3[k] = o.C2[k] * (0.25 * h * h * h);
    t.alphaD = -4.0 / h;
  }
  t.Hd = o.H;
  t.Hinvd = o.Hinv;
  for (int j = 0; j < kBand; ++j) {
    t.bs0[j] = j < n ? o.BS.get(0, j) : 0.0;
    int c = n - kBand + j;
    t.bsN[j] = c >= 0 ? o.BS.get(n - 1, c) : 0.0;
  }
  return t;
}

namespace {
// mu3 averages in the flattened index (sbpOps_m_constGrid.cpp:1238-1257 for y,
// :1087-1112 for z).
std::vector<double> mu3_y(const std::vector<double>& v) {
  size_t n = v.size();
  std::vector<double> m(v);
  m[n - 1] += v[n - 2];
  for (size_t i = 1; i < n; ++i) m[i - 1] += v[i];
  for (auto& x : m) x *= 0.5;
  return m;
}
std::vector<double> mu3_z(const std::vector<double>& v) {
  size_t n = v.size();
  std::vector<double> m(v);
  m[0] += v[1];
  m[n - 1] += v[n - 2];
  for (size_t i = 1; i + 1 < n; ++i) m[i - 1] += v[i];
  for (auto& x : m) x *= 0.5;
  return m;
}
inline double bandc(const std::vector<double>& b, int row, int col) {
  int off = col - row;
  if (off < -kHalf || off > kHalf) return 0.0;
  return b[(size_t)row * kBand + off + kHalf];
}
}  // namespace

LevelHost build_level(int order, int Ny, int Nz, double Ly, double Lz, int grid_type, int compat,
                      const std::vector<double>& y, const std::vector<double>& z,
                      const std::vector<double>& mu, const int bc[4]) {
  LevelHost L;
  L.order = order;
  L.Ny = Ny;
  L.Nz = Nz;
  L.Ly = Ly;
  L.Lz = Lz;
  L.grid_type = grid_type;
  L.compat = compat;
  for (int i = 0; i < 4; ++i) L.bc[i] = bc[i];
  const size_t N = (size_t)Ny * Nz;
  if (mu.size() != N) throw std::invalid_argument("mu must hold Ny*Nz values");
  if (grid_type == 0) {
    L.dy = Ly / (Ny - 1.0);
    L.dz = Lz / (Nz - 1.0);
  } else {
    L.dy = 1.0 / (Ny - 1.0);
    L.dz = 1.0 / (Nz - 1.0);
  }
  L.ty = build_dir_tables(order, Ny, L.dy, compat);
  L.tz = build_dir_tables(order, Nz, L.dz, compat);
  L.mu = mu;
  L.yq.assign(N, 1.0);
  L.zr.assign(N, 1.0);
  if (grid_type == 1) {
    // yq = Dq*y, zr = Dr*z (sbpOps_m_varGrid.cpp:350-366)
    std::vector<double> yy(y), zz(z);
    if (yy.empty()) {
      yy.resize(N);
      for (size_t i = 0; i < N; ++i) yy[i] = Ly * (double)(i / Nz) / (Ny - 1.0);
    }
    if (zz.empty()) {
      zz.resize(N);
      for (size_t i = 0; i < N; ++i) zz[i] = Lz * (double)(i % Nz) / (Nz - 1.0);
    }
    for (int iy = 0; iy < Ny; ++iy)
      for (int iz = 0; iz < Nz; ++iz) {
        double sy = 0, sz = 0;
        for (int j = 0; j < kBand; ++j) {
          int cyi = iy + j - kHalf, czi = iz + j - kHalf;
          if (cyi >= 0 && cyi < Ny) sy += L.ty.D[(size_t)iy * kBand + j] * yy[(size_t)cyi * Nz + iz];
          if (czi >= 0 && czi < Nz) sz += L.tz.D[(size_t)iz * kBand + j] * zz[(size_t)iy * Nz + czi];
        }
        L.yq[(size_t)iy * Nz + iz] = sy;
        L.zr[(size_t)iy * Nz + iz] = sz;
      }
  }
  L.qy.resize(N);
  L.rz.resize(N);
  L.cy.resize(N);
  L.cz.resize(N);
  for (size_t i = 0; i < N; ++i) {
    L.qy[i] = 1.0 / L.yq[i];
    L.rz[i] = 1.0 / L.zr[i];
    L.cy[i] = grid_type == 1 ? mu[i] * L.qy[i] : mu[i];
    L.cz[i] = grid_type == 1 ? mu[i] * L.rz[i] : mu[i];
  }
  if (order == 4) {
    L.m3y = mu3_y(L.cy);
    L.m3z = mu3_z(L.cz);
  } else {
    L.m3y = L.cy;
    L.m3z = L.cz;
  }
  L.wy.resize(N);
  L.wz.resize(N);
  for (int iy = 0; iy < Ny; ++iy)
    for (int iz = 0; iz < Nz; ++iz) {
      size_t i = (size_t)iy * Nz + iz;
      L.wy[i] = L.tz.Hd[iz] * (grid_type == 1 ? L.zr[i] : 1.0);
      L.wz[i] = L.ty.Hd[iy] * (grid_type == 1 ? L.yq[i] : 1.0);
    }
  L.compute_diag();
  return L;
}

// One line of the two-stage composition: out_i = sum_k S2[i,k] g_k with
// g_k = coef_k * sum_l S1[k,l] x_l, for the three R/derivative terms.
void LevelHost::apply_A(const double* x, double* out) const {
  const int Ny_ = Ny, Nz_ = Nz;
  auto X = [&](int iy, int iz) { return x[(size_t)iy * Nz_ + iz]; };
  std::vector<double> g1(std::max(Ny_, Nz_)), g3(g1.size()), g4(g1.size());
  const size_t N = (size_t)Ny_ * Nz_;
  for (size_t i = 0; i < N; ++i) out[i] = 0.0;
  // y lines
  for (int iz = 0; iz < Nz_; ++iz) {
    for (int k = 0; k < Ny_; ++k) {
      double d1 = 0, d3 = 0, d4 = 0;
      for (int j = 0; j < kBand; ++j) {
        int l = k + j - kHalf;
        if (l < 0 || l >= Ny_) continue;
        double xv = X(l, iz);
        d1 += ty.D[(size_t)k * kBand + j] * xv;
        d3 += ty.R3[(size_t)k * kBand + j] * xv;
        d4 += ty.R4[(size_t)k * kBand + j] * xv;
      }
      size_t node = (size_t)k * Nz_ + iz;
      g1[k] = cy[node] * d1;
      g3[k] = ty.w3[k] * m3y[node] * d3;
      g4[k] = ty.w4[k] * cy[node] * d4;
    }
    for (int i = 0; i < Ny_; ++i) {
      double acc = 0;
      for (int j = 0; j < kBand; ++j) {
        int k = i + j - kHalf;
        if (k < 0 || k >= Ny_) continue;
        acc += ty.Q[(size_t)i * kBand + j] * g1[k] - ty.R3T[(size_t)i * kBand + j] * g3[k] -
               ty.R4T[(size_t)i * kBand + j] * g4[k];
      }
      size_t node = (size_t)i * Nz_ + iz;
      double s = acc;
      // L side (bc[2]) and R side (bc[0])
      if (bc[2] == 0 && i < kBand) s += (ty.bs0[i] + (i == 0 ? ty.alphaD : 0.0)) * cy[iz] * X(0, iz);
      if (bc[2] == 1 && i == 0) s += g1[0];
      if (bc[0] == 0 && i >= Ny_ - kBand) {
        size_t bn = (size_t)(Ny_ - 1) * Nz_ + iz;
        s += (ty.bsN[i - (Ny_ - kBand)] + (i == Ny_ - 1 ? ty.alphaD : 0.0)) * cy[bn] * X(Ny_ - 1, iz);
      }
      if (bc[0] == 1 && i == Ny_ - 1) s -= g1[Ny_ - 1];
      out[node] += wy[node] * s;
    }
  }
  // z lines
  for (int iy = 0; iy < Ny_; ++iy) {
    for (int k = 0; k < Nz_; ++k) {
      double d1 = 0, d3 = 0, d4 = 0;
      for (int j = 0; j < kBand; ++j) {
        int l = k + j - kHalf;
        if (l < 0 || l >= Nz_) continue;
        double xv = X(iy, l);
        d1 += tz.D[(size_t)k * kBand + j] * xv;
        d3 += tz.R3[(size_t)k * kBand + j] * xv;
        d4 += tz.R4[(size_t)k * kBand + j] * xv;
      }
      size_t node = (size_t)iy * Nz_ + k;
      g1[k] = cz[node] * d1;
      g3[k] = tz.w3[k] * m3z[node] * d3;
      g4[k] = tz.w4[k] * cz[node] * d4;
    }
    for (int i = 0; i < Nz_; ++i) {
      double acc = 0;
      for (int j = 0; j < kBand; ++j) {
        int k = i + j - kHalf;
        if (k < 0 || k >= Nz_) continue;
        acc += tz.Q[(size_t)i * kBand + j] * g1[k] - tz.R3T[(size_t)i * kBand + j] * g3[k] -
               tz.R4T[(size_t)i * kBand + j] * g4[k];
      }
      size_t node = (size_t)iy * Nz_ + i;
      double s = acc;
      // T side (bc[1]) and B side (bc[3])
      if (bc[1] == 0 && i < kBand) s += (tz.bs0[i] + (i == 0 ? tz.alphaD : 0.0)) * cz[(size_t)iy * Nz_] * X(iy, 0);
      if (bc[1] == 1 && i == 0) s += g1[0];
      if (bc[3] == 0 && i >= Nz_ - kBand) {
        size_t bn = (size_t)iy * Nz_ + Nz_ - 1;
        s += (tz.bsN[i - (Nz_ - kBand)] + (i == Nz_ - 1 ? tz.alphaD : 0.0)) * cz[bn] * X(iy, Nz_ - 1);
      }
      if (bc[3] == 1 && i == Nz_ - 1) s -= g1[Nz_ - 1];
      out[node] += wz[node] * s;
    }
  }
}

void LevelHost::compute_diag() {
  const size_t N = (size_t)Ny * Nz;
  diagK.assign(N, 0.0);
  for (int iy = 0; iy < Ny; ++iy)
    for (int iz = 0; iz < Nz; ++iz) {
      size_t node = (size_t)iy * Nz + iz;
      double sy = 0, sz = 0;
      for (int j = 0; j < kBand; ++j) {
        int k = iy + j - kHalf;
        if (k < 0 || k >= Ny) continue;
        size_t kn = (size_t)k * Nz + iz;
        sy += ty.Q[(size_t)iy * kBand + j] * cy[kn] * bandc(ty.D, k, iy) -
              ty.R3T[(size_t)iy * kBand + j] * ty.w3[k] * m3y[kn] * bandc(ty.R3, k, iy) -
              ty.R4T[(size_t)iy * kBand + j] * ty.w4[k] * cy[kn] * bandc(ty.R4, k, iy);
      }
      if (bc[2] == 0 && iy == 0) sy += (ty.bs0[0] + ty.alphaD) * cy[node];
      if (bc[2] == 1 && iy == 0) sy += cy[node] * bandc(ty.D, 0, 0);
      if (bc[0] == 0 && iy == Ny - 1) sy += (ty.bsN[kBand - 1] + ty.alphaD) * cy[node];
      if (bc[0] == 1 && iy == Ny - 1) sy -= cy[node] * bandc(ty.D, Ny - 1, Ny - 1);
      for (int j = 0; j < kBand; ++j) {
        int k = iz + j - kHalf;
        if (k < 0 || k >= Nz) continue;
        size_t kn = (size_t)iy * Nz + k;
        sz += tz.Q[(size_t)iz * kBand + j] * cz[kn] * bandc(tz.D, k, iz) -
              tz.R3T[(size_t)iz * kBand + j] * tz.w3[k] * m3z[kn] * bandc(tz.R3, k, iz) -
              tz.R4T[(size_t)iz * kBand + j] * tz.w4[k] * cz[kn] * bandc(tz.R4, k, iz);
      }
      if (bc[1] == 0 && iz == 0) sz += (tz.bs0[0] + tz.alphaD) * cz[node];
      if (bc[1] == 1 && iz == 0) sz += cz[node] * bandc(tz.D, 0, 0);
      if (bc[3] == 0 && iz == Nz - 1) sz += (tz.bsN[kBand - 1] + tz.alphaD) * cz[node];
      if (bc[3] == 1 && iz == Nz - 1) sz -= cz[node] * bandc(tz.D, Nz - 1, Nz - 1);
      diagK[node] = -(wy[node] * sy + wz[node] * sz);
    }
}

Interp1D make_interp(int nf, int nc) {
  Interp1D I;
  I.nf = nf;
  I.nc = nc;
  I.j0.resize(nf);
  I.w0.resize(nf);
  I.w1.resize(nf);
  for (int i = 0; i < nf; ++i) {
    double s = (double)i * (nc - 1) / (double)(nf - 1);
    int j = (int)std::floor(s);
    if (j > nc - 2) j = nc - 2;
    if (j < 0) j = 0;
    double w1 = s - j;
    I.j0[i] = j;
    I.w1[i] = w1;
    I.w0[i] = 1.0 - w1;
  }
  return I;
}

// One direction of A composed into 17-point rows: stage 2 (Q, R3^T, R4^T)
// applied to stage 1 (c D, w3 m3 R3, w4 c R4) over the band tables, plus the
// SAT terms the stencil adds at the ends (Dirichlet: (BS row + alphaD) * c *
// x(end); Neumann: +/- c D x at the end row).  C[i*17 + o+8] multiplies
// x(i+o); bc_lo / bc_hi: 0 Dirichlet, 1 Neumann.
void compose_line(const DirTables& t, int bc_lo, int bc_hi, const std::vector<double>& c1,
                         const std::vector<double>& m31, std::vector<double>& C) {
  const int n = t.n;
  C.assign((size_t)n * 17, 0.0);
  const bool r4 = t.nterms == 3;
  for (int i = 0; i < n; ++i) {
    double* row = &C[(size_t)i * 17];
    for (int a = 0; a < kBand; ++a) {
      const int k = i + a - kHalf;
      if (k < 0 || k >= n) continue;
      const double q = t.Q[(size_t)i * kBand + a], q3 = t.R3T[(size_t)i * kBand + a];
      const double q4 = r4 ? t.R4T[(size_t)i * kBand + a] : 0.0;
      for (int b = 0; b < kBand; ++b) {
        const int j = k + b - kHalf;
        if (j < 0 || j >= n) continue;
        double v = q * (c1[k] * t.D[(size_t)k * kBand + b]);
        v -= q3 * (t.w3[k] * m31[k] * t.R3[(size_t)k * kBand + b]);
        if (r4) v -= q4 * (t.w4[k] * c1[k] * t.R4[(size_t)k * kBand + b]);
        row[j - i + 8] += v;
      }
    }
    if (bc_lo == 0) {
      if (i < kBand) row[0 - i + 8] += (t.bs0[i] + (i == 0 ? t.alphaD : 0.0)) * c1[0];
    } else if (i == 0) {
      for (int b = kHalf; b < kBand; ++b) row[b - kHalf + 8] += c1[0] * t.D[b];
    }
    if (bc_hi == 0) {
      if (i >= n - kBand) row[(n - 1) - i + 8] += (t.bsN[i - (n - kBand)] + (i == n - 1 ? t.alphaD : 0.0)) * c1[n - 1];
    } else if (i == n - 1) {
      for (int b = 0; b <= kHalf; ++b) row[b - kHalf + 8] -= c1[n - 1] * t.D[(size_t)(n - 1) * kBand + b];
    }
  }
}


void build_cross_planes(const LevelHost& h, std::vector<double>& C) {
  const int Ny = h.Ny, Nz = h.Nz;
  const size_t N = (size_t)Ny * Nz;
  C.assign(33 * N, 0.0);
  std::vector<double> c1, m31, L;
  c1.resize(Ny);
  m31.resize(Ny);
  for (int iz = 0; iz < Nz; ++iz) {
    for (int iy = 0; iy < Ny; ++iy) {
      c1[iy] = h.cy[(size_t)iy * Nz + iz];
      m31[iy] = h.m3y[(size_t)iy * Nz + iz];
    }
    compose_line(h.ty, h.bc[2], h.bc[0], c1, m31, L);
    for (int iy = 0; iy < Ny; ++iy) {
      const size_t node = (size_t)iy * Nz + iz;
      for (int o = 0; o < 17; ++o) C[(size_t)o * N + node] = h.wy[node] * L[(size_t)iy * 17 + o];
    }
  }
  c1.resize(Nz);
  m31.resize(Nz);
  for (int iy = 0; iy < Ny; ++iy) {
    for (int iz = 0; iz < Nz; ++iz) {
      c1[iz] = h.cz[(size_t)iy * Nz + iz];
      m31[iz] = h.m3z[(size_t)iy * Nz + iz];
    }
    compose_line(h.tz, h.bc[1], h.bc[3], c1, m31, L);
    for (int iz = 0; iz < Nz; ++iz) {
      const size_t node = (size_t)iy * Nz + iz;
      for (int o = 0; o < 17; ++o) {
        const double v = h.wz[node] * L[(size_t)iz * 17 + o];
        if (o == 8)
          C[(size_t)8 * N + node] += v;
        else
          C[(size_t)(o < 8 ? 17 + o : 16 + o) * N + node] = v;
      }
    }
  }
}

void apply_cross_planes(const std::vector<double>& C, int Ny, int Nz, const double* x, double* out) {
  const size_t N = (size_t)Ny * Nz;
  for (int iy = 0; iy < Ny; ++iy)
    for (int iz = 0; iz < Nz; ++iz) {
      const size_t node = (size_t)iy * Nz + iz;
      double s = 0.0;
      for (int o = -8; o <= 8; ++o) {
        const int jy = iy + o;
        if (jy >= 0 && jy < Ny) s += C[(size_t)(o + 8) * N + node] * x[(size_t)jy * Nz + iz];
      }
      for (int o = -8; o <= 8; ++o) {
        const int jz = iz + o;
        if (o == 0 || jz < 0 || jz >= Nz) continue;
        s += C[(size_t)(o < 0 ? 25 + o : 24 + o) * N + node] * x[(size_t)iy * Nz + jz];
      }
      out[node] = s;
    }
}

bool build_full_form(const LevelHost& h, FullForm& f) {
  const int Ny = h.Ny, Nz = h.Nz;
  if (h.order != 4 || Ny < 17 || Nz < 17) return false;
  const int iy_ref = Ny / 2, iz_ref = Nz / 2;
  std::vector<double> cy1(Ny), m3y1(Ny), cz1(Nz), m3z1(Nz);
  f.wy1.assign(Nz, 0.0);
  f.wz1.assign(Ny, 0.0);
  for (int iy = 0; iy < Ny; ++iy) {
    const size_t i = (size_t)iy * Nz + iz_ref;
    cy1[iy] = h.cy[i];
    m3y1[iy] = h.m3y[i];
    f.wz1[iy] = h.wz[i];
  }
  for (int iz = 0; iz < Nz; ++iz) {
    const size_t i = (size_t)iy_ref * Nz + iz;
    cz1[iz] = h.cz[i];
    m3z1[iz] = h.m3z[i];
    f.wy1[iz] = h.wy[i];
  }
  f.ycls.assign(Nz, 0);
  f.zcls.assign(Ny, 0);
  std::vector<int> yexc, zexc;
  for (int iy = 0; iy < Ny; ++iy)
    for (int iz = 0; iz < Nz; ++iz) {
      const size_t i = (size_t)iy * Nz + iz;
      if (h.wy[i] != f.wy1[iz] || h.wz[i] != f.wz1[iy]) return false;
      if ((h.cy[i] != cy1[iy] || h.m3y[i] != m3y1[iy]) && !f.ycls[iz]) {
        yexc.push_back(iz);
        f.ycls[iz] = (int)yexc.size();
      }
      if ((h.cz[i] != cz1[iz] || h.m3z[i] != m3z1[iz]) && !f.zcls[iy]) {
        zexc.push_back(iy);
        f.zcls[iy] = (int)zexc.size();
      }
      if (yexc.size() > (size_t)kMaxLineClasses || zexc.size() > (size_t)kMaxLineClasses) return false;
    }
  const int ncy = 1 + (int)yexc.size(), ncz = 1 + (int)zexc.size();
  f.Cy17.assign((size_t)ncy * Ny * 17, 0.0);
  f.CzT17.assign((size_t)ncz * 17 * Nz, 0.0);
  std::vector<double> L17, c1, m31;
  for (int c = 0; c < ncy; ++c) {
    c1 = cy1;
    m31 = m3y1;
    if (c > 0)
      for (int iy = 0; iy < Ny; ++iy) {
        c1[iy] = h.cy[(size_t)iy * Nz + yexc[c - 1]];
        m31[iy] = h.m3y[(size_t)iy * Nz + yexc[c - 1]];
      }
    compose_line(h.ty, h.bc[2], h.bc[0], c1, m31, L17);
    std::copy(L17.begin(), L17.end(), f.Cy17.begin() + (size_t)c * Ny * 17);
  }
  for (int c = 0; c < ncz; ++c) {
    c1 = cz1;
    m31 = m3z1;
    if (c > 0) {
      const size_t r = (size_t)zexc[c - 1] * Nz;
      c1.assign(h.cz.begin() + r, h.cz.begin() + r + Nz);
      m31.assign(h.m3z.begin() + r, h.m3z.begin() + r + Nz);
    }
    compose_line(h.tz, h.bc[1], h.bc[3], c1, m31, L17);
    for (int iz = 0; iz < Nz; ++iz)
      for (int o = 0; o < 17; ++o) f.CzT17[((size_t)c * 17 + o) * Nz + iz] = L17[(size_t)iz * 17 + o];
  }
  // the interior box: class-0 lines around the middle whose class-0
  // stencils vanish beyond offsets -4..4 (cross: the other direction's
  // classes, since an interior tile holds class-0 lines only)
  auto range = [](int n, const std::vector<int>& cross, auto entry, int& lo, int& hi) {
    auto nine = [&](int i) {
      if (i < kHalf || i > n - 1 - kHalf || cross[i] != 0) return false;
      for (int o = 0; o < 8 - kHalf; ++o)
        if (entry(i, o) != 0.0 || entry(i, 16 - o) != 0.0) return false;
      return true;
    };
    lo = 1;
    hi = 0;
    const int m = n / 2;
    if (!nine(m)) return;
    lo = hi = m;
    while (nine(lo - 1)) --lo;
    while (nine(hi + 1)) ++hi;
  };
  range(Ny, f.zcls, [&](int i, int o) { return f.Cy17[(size_t)i * 17 + o]; }, f.ylo, f.yhi);
  range(Nz, f.ycls, [&](int i, int o) { return f.CzT17[(size_t)o * Nz + i]; }, f.zlo, f.zhi);
  return true;
}

void apply_full_form(const FullForm& f, int Ny, int Nz, const double* x, double* out) {
  for (int iy = 0; iy < Ny; ++iy)
    for (int iz = 0; iz < Nz; ++iz) {
      const bool inner = iy >= f.ylo && iy <= f.yhi && iz >= f.zlo && iz <= f.zhi;
      const int lo = inner ? 8 - kHalf : 0, hi = inner ? 8 + kHalf : 16;
      const double* cy = &f.Cy17[((size_t)f.ycls[iz] * Ny + iy) * 17];
      const double* cz = &f.CzT17[(size_t)f.zcls[iy] * 17 * Nz + iz];
      double sy = 0.0, sz = 0.0;
      for (int o = lo; o <= hi; ++o) {
        const int jy = iy + o - 8, jz = iz + o - 8;
        const double xy = jy >= 0 && jy < Ny ? x[(size_t)jy * Nz + iz] : 0.0;
        const double xz = jz >= 0 && jz < Nz ? x[(size_t)iy * Nz + jz] : 0.0;
        sy += cy[o] * xy;
        sz += cz[(size_t)o * Nz] * xz;
      }
      out[(size_t)iy * Nz + iz] = f.wy1[iz] * sy + f.wz1[iy] * sz;
    }
}

}  // namespace scy
