// Host-side construction of the 1D SBP operators and the per-level
// coefficient fields used by the matrix-free device stencil.
#pragma once
#include <map>
#include <string>
#include <vector>

namespace scy {

// Sparse 1D matrix (row -> col -> value), the same shape of container the
// reference builds its 1D operators in (source/spmat.hpp:18-75).
struct Sparse1D {
  int n = 0;
  std::vector<std::map<int, double>> rows;
  explicit Sparse1D(int n_ = 0) : n(n_), rows(n_) {}
  void set(int r, int c, double v) { rows[r][c] = v; }
  double get(int r, int c) const {
    auto it = rows[r].find(c);
    return it == rows[r].end() ? 0.0 : it->second;
  }
  Sparse1D transpose() const;
};

// All 1D operators of one direction (spmat.cpp:310-627).
struct Ops1D {
  int order = 4, n = 0;
  double scale = 1.0;            // 1/h
  std::vector<double> H, Hinv;   // diagonals
  Sparse1D D1, BS;               // first derivative and boundary derivative
  Sparse1D D3, D4, D2;           // R-term difference operators (unscaled D3/D4; D2 scaled)
  std::vector<double> C3, C4, C2;
};

// Builds the operators; throws std::invalid_argument on an unsupported size/order.
Ops1D build_ops1d(int order, int n, double scale, int compat /*0 fully,1 compatible*/);

// Centred band: 9 coefficients per row at column offsets -4..+4.
constexpr int kBand = 9;
constexpr int kHalf = 4;
std::vector<double> to_band(const Sparse1D& m);  // throws if a row reaches beyond +-4

// Per-direction tables in the order the device kernel consumes them.
struct DirTables {
  int n = 0;
  int nterms = 3;                // 3 (order 4: D, D3, D4) or 2 (order 2: D, D2)
  std::vector<double> D, R3, R4; // stage 1 (applied to x), banded n*9
  std::vector<double> Q, R3T, R4T; // stage 2 (applied to the stage-1 results), banded
  std::vector<double> w3, w4;    // per-row weights of the R terms
  std::vector<double> Hd, Hinvd; // H diagonal and its inverse
  double bs0[kBand];             // BS row 0, columns 0..8
  double bsN[kBand];             // BS row n-1, columns n-9..n-1
  double alphaD = 0.0;           // Dirichlet penalty
};
DirTables build_dir_tables(int order, int n, double h, int compat);

// One grid of the hierarchy: sizes, tables and per-node coefficient fields.
struct LevelHost {
  int order = 4, Ny = 0, Nz = 0, grid_type = 0, compat = 0;
  double Ly = 1, Lz = 1, dy = 1, dz = 1;
  int bc[4] = {0, 1, 0, 1};      // R, T, L, B
  DirTables ty, tz;
  // fields, length Ny*Nz
  std::vector<double> mu, cy, cz, m3y, m3z, wy, wz, yq, zr, qy, rz;
  std::vector<double> diagK;     // diagonal of K = -A
  double lambda_max = 0.0;       // spectral bound of diag(K)^-1 K (power iteration)
  void apply_A(const double* x, double* out) const;  // host reference of the device stencil
  void compute_diag();
};

// Builds a level from grid data; y/z may be empty (-> q*Ly, r*Lz).
LevelHost build_level(int order, int Ny, int Nz, double Ly, double Lz, int grid_type, int compat,
                      const std::vector<double>& y, const std::vector<double>& z,
                      const std::vector<double>& mu, const int bc[4]);

// 1D linear interpolation from a coarse logical grid of nc points onto a fine
// one of nf points: fine i = w0*coarse[j0] + w1*coarse[j0+1].
struct Interp1D {
  int nf = 0, nc = 0;
  std::vector<int> j0;
  std::vector<double> w0, w1;
};
Interp1D make_interp(int nf, int nc);

// One direction of A composed into 17-point rows (offsets -8..8): stage 2
// (Q, R3^T, R4^T) applied to stage 1 (c D, w3 m3 R3, w4 c R4) over the band
// tables, plus the SAT terms of the boundary rows (Dirichlet: (BS row +
// alphaD) * c * x(end); Neumann: +/- c D x at the end row).  C[i*17 + o+8]
// multiplies x(i+o); bc_lo / bc_hi: 0 Dirichlet, 1 Neumann.
void compose_line(const DirTables& t, int bc_lo, int bc_hi, const std::vector<double>& c1,
                  const std::vector<double>& m31, std::vector<double>& C);
// A as a 33-point cross stencil per node, exact for any coefficient fields:
// (A x)(iy, iz) = sum_{o=-8..8} C[(o+8) N + node] x(iy+o, iz)
//               + sum_{o=-8..-1} C[(25+o) N + node] x(iy, iz+o) + sum_{o=1..8} C[(24+o) N + node] x(iy, iz+o)
// (each column's y operator and each row's z operator composed with that
// line's coefficients, times the outer weights wy and wz).
void build_cross_planes(const LevelHost& h, std::vector<double>& C);

// The full form of a level: the outer weights separable over every node
// (wy = wy1[iz], wz = wz1[iy]) and the line coefficients (cy, m3y down a
// column; cz, m3z along a row) equal to those of the middle column / row on
// all but at most kMaxLineClasses exceptional lines per direction, so
// (A x)(iy,iz) = wy1[iz] sum_o Cy17[(ycls[iz]*Ny + iy)*17 + o+8] x(iy+o, iz)
//              + wz1[iy] sum_o CzT17[(zcls[iy]*17 + o+8)*Nz + iz] x(iy, iz+o)
// (class 0: the middle line's composition; class c > 0: exceptional line c).
// [ylo, yhi] x [zlo, zhi]: the class-0 rows / columns around the middle
// whose class-0 stencils vanish beyond offsets -4..4 (empty when lo > hi).
constexpr int kMaxLineClasses = 8;
struct FullForm {
  std::vector<double> Cy17, CzT17, wy1, wz1;
  std::vector<int> ycls, zcls;
  int ylo = 1, yhi = 0, zlo = 1, zhi = 0;
};
// false when the level has no full form (order 2, a direction shorter than
// 17 points, non-separable weights or too many exceptional lines)
bool build_full_form(const LevelHost& h, FullForm& f);
// A x from the full form, 9-point on the interior box and 17-point elsewhere
// (the device's arithmetic order)
void apply_full_form(const FullForm& f, int Ny, int Nz, const double* x, double* out);
// Host reference of the cross-plane form (for checking it against apply_A).
void apply_cross_planes(const std::vector<double>& C, int Ny, int Nz, const double* x, double* out);

}  // namespace scy
