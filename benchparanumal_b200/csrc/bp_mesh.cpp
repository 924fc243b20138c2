// Host-side setup of the Hex3D box: 1D basis, vertices, and the masked
// gathered numbering (GlobalToLocal + CSR) computed in closed form from the
// box structure.
//
// The numbering reproduces, integer for integer, what the reference computes
// with generic connectivity (libs/mesh/meshConnectNodes.cpp:32-82,
// libs/mesh/meshMaskedGatherScatterSetup.cpp:31-77, libs/ogs/ogsSetup.cpp:
// 492-579 and 833-849):
//   * a node's class is the set of local nodes at the same lattice point; its
//     representative is the local node of the lowest-numbered element of the
//     class (the reference's globalId = 1 + smallest local index);
//   * nodes on the box boundary are masked (GlobalToLocal = -1);
//   * gathered rows are the unmasked classes in order of first appearance
//     over the local index e*Np*Nf + f*Np + n;
//   * each CSR row lists its local nodes in ascending local index.
// Here those orders follow from the lattice coordinates, so every element is
// handled independently (OpenMP over elements) with no sort.
#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <map>
#include <numeric>
#include <unordered_map>

#include "bp_internal.hpp"

namespace bp {

// GLL nodes: Newton iteration on (1-x^2) P_N'(x) with the Legendre
// recurrence, started from the Chebyshev-Gauss-Lobatto points; weights
// 2 / (N (N+1) P_N(x)^2).
void gll_nodes_weights(int N, std::vector<double>& z, std::vector<double>& w) {
  const int n1 = N + 1;
  z.assign(n1, 0.0);
  w.assign(n1, 0.0);
  const double pi = 3.14159265358979323846;
  std::vector<double> x(n1), xold(n1, 2.0), PN(n1), PN1(n1);
  for (int i = 0; i < n1; ++i) x[i] = -std::cos(pi * i / N);
  for (int it = 0; it < 100; ++it) {
    double delta = 0.0;
    for (int i = 0; i < n1; ++i) delta = std::max(delta, std::fabs(x[i] - xold[i]));
    if (delta <= 1e-16) break;
    for (int i = 0; i < n1; ++i) {
      xold[i] = x[i];
      double p0 = 1.0, p1 = x[i];
      for (int k = 2; k <= N; ++k) {
        const double p2 = ((2 * k - 1) * x[i] * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      PN[i] = p1;     // P_N
      PN1[i] = p0;    // P_{N-1}
      if (N == 1) { PN[i] = x[i]; PN1[i] = 1.0; }
      x[i] = xold[i] - (x[i] * PN[i] - PN1[i]) / (n1 * PN[i]);
    }
  }
  x[0] = -1.0;
  x[N] = 1.0;
  for (int i = 0; i < n1; ++i) {
    double p0 = 1.0, p1 = x[i];
    for (int k = 2; k <= N; ++k) {
      const double p2 = ((2 * k - 1) * x[i] * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    z[i] = x[i];
    w[i] = 2.0 / (N * (N + 1.0) * p1 * p1);
  }
  // symmetrise
  for (int i = 0; i < n1 / 2; ++i) {
    const double a = 0.5 * (z[N - i] - z[i]);
    z[i] = -a;
    z[N - i] = a;
    const double b = 0.5 * (w[i] + w[N - i]);
    w[i] = w[N - i] = b;
  }
  if (n1 % 2) z[N / 2] = 0.0;
}

// Lagrange differentiation matrix by barycentric weights:
// D[i*Nq+m] = l_m'(z_i) = (b_m / b_i) / (z_i - z_m), diagonal = -(row sum).
void diff_matrix(const std::vector<double>& z, std::vector<double>& D) {
  const int n = (int)z.size();
  std::vector<double> b(n, 1.0);
  for (int j = 0; j < n; ++j)
    for (int k = 0; k < n; ++k)
      if (k != j) b[j] *= (z[j] - z[k]);
  for (int j = 0; j < n; ++j) b[j] = 1.0 / b[j];
  D.assign(n * n, 0.0);
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int m = 0; m < n; ++m) {
      if (m == i) continue;
      const double v = (b[m] / b[i]) / (z[i] - z[m]);
      D[i * n + m] = v;
      s += v;
    }
    D[i * n + i] = -s;
  }
}

// Legendre P_n(x) and P_n'(x) by the three-term recurrence and
// P'_{k+1} = P'_{k-1} + (2k+1) P_k.
static void legendre(int n, double x, double& p, double& dp) {
  double p0 = 1.0, p1 = x, d0 = 0.0, d1 = 1.0;
  if (n == 0) { p = 1.0; dp = 0.0; return; }
  for (int k = 1; k < n; ++k) {
    const double p2 = ((2 * k + 1) * x * p1 - k * p0) / (k + 1);
    const double d2 = d0 + (2 * k + 1) * p1;
    p0 = p1; p1 = p2; d0 = d1; d1 = d2;
  }
  p = p1;
  dp = d1;
}

// Gauss-Legendre points and weights, n points: Newton on P_n from the
// Chebyshev guesses cos(pi (i+3/4)/(n+1/2)); w = 2 / ((1-x^2) P_n'(x)^2).
void gauss_nodes_weights(int n, std::vector<double>& r, std::vector<double>& w) {
  const double pi = 3.14159265358979323846;
  r.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    double x = -std::cos(pi * (i + 0.75) / (n + 0.5)), p, dp;
    for (int it = 0; it < 100; ++it) {
      legendre(n, x, p, dp);
      const double dx = p / dp;
      x -= dx;
      if (std::fabs(dx) <= 1e-16) break;
    }
    legendre(n, x, p, dp);
    r[i] = x;
    w[i] = 2.0 / ((1.0 - x * x) * dp * dp);
  }
  for (int i = 0; i < n / 2; ++i) {   // symmetrise
    const double a = 0.5 * (r[n - 1 - i] - r[i]), b = 0.5 * (w[i] + w[n - 1 - i]);
    r[i] = -a; r[n - 1 - i] = a;
    w[i] = w[n - 1 - i] = b;
  }
  if (n % 2) r[n / 2] = 0.0;
}

// Lagrange interpolation from nodes z to points x: I[i*nz + m] = l_m(x_i).
static void interp_matrix(const std::vector<double>& z, const std::vector<double>& x, std::vector<double>& I) {
  const int nz = (int)z.size(), nx = (int)x.size();
  I.assign((size_t)nx * nz, 0.0);
  for (int i = 0; i < nx; ++i)
    for (int m = 0; m < nz; ++m) {
      double l = 1.0;
      for (int k = 0; k < nz; ++k)
        if (k != m) l *= (x[i] - z[k]) / (z[m] - z[k]);
      I[(size_t)i * nz + m] = l;
    }
}

// In-place inverse of a small dense matrix (Gauss-Jordan, partial pivoting).
static bool invert(int n, std::vector<double>& A) {
  std::vector<double> X((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) X[(size_t)i * n + i] = 1.0;
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(A[(size_t)r * n + c]) > std::fabs(A[(size_t)piv * n + c])) piv = r;
    if (A[(size_t)piv * n + c] == 0.0) return false;
    for (int k = 0; k < n; ++k) {
      std::swap(A[(size_t)c * n + k], A[(size_t)piv * n + k]);
      std::swap(X[(size_t)c * n + k], X[(size_t)piv * n + k]);
    }
    const double d = A[(size_t)c * n + c];
    for (int k = 0; k < n; ++k) { A[(size_t)c * n + k] /= d; X[(size_t)c * n + k] /= d; }
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = A[(size_t)r * n + c];
      if (f == 0.0) continue;
      for (int k = 0; k < n; ++k) {
        A[(size_t)r * n + k] -= f * A[(size_t)c * n + k];
        X[(size_t)r * n + k] -= f * X[(size_t)c * n + k];
      }
    }
  }
  A = X;
  return true;
}

// 1D data of the over-integrated operators (libs/mesh/meshCubatureSetupHex3D.cpp:
// 31-80): N+2 Gauss points, GLL->Gauss interpolation, differentiation on the
// Gauss points; the inverse orthonormal-Legendre Vandermonde on the GLL nodes,
// the modal differentiation matrix invV*Vr and the exact GLL mass matrix
// MM = invV^T invV (= (V V^T)^-1).
void cubature_basis(int N, const std::vector<double>& gllz, CubBasis& cb) {
  const int Nq = N + 1, cNq = N + 2;
  cb.cNq = cNq;
  gauss_nodes_weights(cNq, cb.r, cb.w);
  interp_matrix(gllz, cb.r, cb.I);
  diff_matrix(cb.r, cb.D);
  std::vector<double> V((size_t)Nq * Nq), Vr((size_t)Nq * Nq);
  for (int i = 0; i < Nq; ++i)
    for (int n = 0; n < Nq; ++n) {
      double p, dp;
      legendre(n, gllz[i], p, dp);
      const double s = std::sqrt((2.0 * n + 1.0) / 2.0);
      V[(size_t)i * Nq + n] = s * p;
      Vr[(size_t)i * Nq + n] = s * dp;
    }
  cb.invV = V;
  invert(Nq, cb.invV);
  cb.Dmodal.assign((size_t)Nq * Nq, 0.0);
  cb.MM.assign((size_t)Nq * Nq, 0.0);
  for (int a = 0; a < Nq; ++a)
    for (int b = 0; b < Nq; ++b) {
      double d = 0.0, mm = 0.0;
      for (int k = 0; k < Nq; ++k) {
        d += cb.invV[(size_t)a * Nq + k] * Vr[(size_t)k * Nq + b];
        mm += cb.invV[(size_t)k * Nq + a] * cb.invV[(size_t)k * Nq + b];
      }
      cb.Dmodal[(size_t)a * Nq + b] = d;
      cb.MM[(size_t)a * Nq + b] = mm;
    }
}

// Box vertices as in libs/mesh/meshSetupBoxHex3D.cpp:31-131 (one rank), with
// interior vertices moved by pert*h*(2u-1) per coordinate; u is the reference
// LCG stream (libs/primitives/random.cpp) seeded with `seed`, three values per
// global vertex id, x/y/z interleaved.
void box_vertices(HostMesh& m, double pert, uint64_t seed) {
  const int nx = m.nx, ny = m.ny, nz = m.nz;
  const int64_t NnX = nx + 1, NnY = ny + 1, NnZ = nz + 1;
  const double dx = 2.0 / nx, dy = 2.0 / ny, dz = 2.0 / nz;
  m.EX.resize((size_t)m.E * 8);
  m.EY.resize((size_t)m.E * 8);
  m.EZ.resize((size_t)m.E * 8);
  std::vector<double> u;
  if (pert != 0.0) {
    u.resize((size_t)3 * NnX * NnY * NnZ);
    uint64_t x = 6364136223846793005ULL * (~seed) + 1ULL;
    const double scale = 1.0 / (double)std::numeric_limits<uint64_t>::max();
    for (size_t r = 0; r < u.size(); ++r) {
      u[r] = (double)x * scale;
      x = 6364136223846793005ULL * x + 1ULL;
    }
  }
  static const int ci[8] = {0, 1, 1, 0, 0, 1, 1, 0};
  static const int cj[8] = {0, 0, 1, 1, 0, 0, 1, 1};
  static const int ck[8] = {0, 0, 0, 0, 1, 1, 1, 1};
#pragma omp parallel for
  for (int e = 0; e < m.E; ++e) {
    const int i = e % nx, j = (e / nx) % ny, k = e / (nx * ny);
    const double x0 = -1.0 + dx * i, y0 = -1.0 + dy * j, z0 = -1.0 + dz * k;
    for (int c = 0; c < 8; ++c) {
      double X = ci[c] ? x0 + dx : x0;
      double Y = cj[c] ? y0 + dy : y0;
      double Z = ck[c] ? z0 + dz : z0;
      const int64_t I = i + ci[c], J = j + cj[c], K = k + ck[c];
      if (pert != 0.0 && I > 0 && I < nx && J > 0 && J < ny && K > 0 && K < nz) {
        const int64_t g = I + J * NnX + K * NnX * NnY;
        X += pert * dx * (2 * u[3 * g + 0] - 1);
        Y += pert * dy * (2 * u[3 * g + 1] - 1);
        Z += pert * dz * (2 * u[3 * g + 2] - 1);
      }
      m.EX[(size_t)e * 8 + c] = X;
      m.EY[(size_t)e * 8 + c] = Y;
      m.EZ[(size_t)e * 8 + c] = Z;
    }
  }
}

namespace {
// Per-direction lattice helpers for lattice index L in [0, n*N]:
//  first(L) : element index of the first (lowest) element containing L
//  count(L) : number of elements containing L (1 or 2)
struct Axis {
  int n, N;
  int first(int L) const { return (L > 0 && L % N == 0) ? L / N - 1 : std::min(L / N, n - 1); }
  int count(int L) const { return (L > 0 && L < n * N && L % N == 0) ? 2 : 1; }
  bool boundary(int L) const { return L == 0 || L == n * N; }
  // representatives of element index a: local indices 1..N-1, plus N if a < n-1
  int reps(int a) const { return N - 1 + (a < n - 1 ? 1 : 0); }
};
}  // namespace

void box_numbering(HostMesh& m) {
  const int N = m.N, Nq = m.Nq, Np = m.Np, Nf = m.Nfields;
  const Axis ax{m.nx, N}, ay{m.ny, N}, az{m.nz, N};
  const int E = m.E;
  // rows contributed by each element, in element order
  std::vector<int64_t> rowBase((size_t)E + 1, 0);
  for (int e = 0; e < E; ++e) {
    const int ex = e % m.nx, ey = (e / m.nx) % m.ny, ez = e / (m.nx * m.ny);
    rowBase[e + 1] = rowBase[e] + (int64_t)Nf * ax.reps(ex) * ay.reps(ey) * az.reps(ez);
  }
  m.Ngather = (int32_t)rowBase[E];
  auto row_of = [&](int ex, int ey, int ez, int i, int j, int k, int f) -> int32_t {
    // (ex,ey,ez) is the representative element, (i,j,k) >= 1 its local indices
    const int e = ex + m.nx * (ey + m.ny * ez);
    const int ci = ax.reps(ex), cj = ay.reps(ey), ck = az.reps(ez);
    return (int32_t)(rowBase[e] + (int64_t)f * ci * cj * ck + ((int64_t)(k - 1) * cj + (j - 1)) * ci + (i - 1));
  };
  // multiplicities -> rowStarts
  m.rowStarts.assign((size_t)m.Ngather + 1, 0);
#pragma omp parallel for
  for (int e = 0; e < E; ++e) {
    const int ex = e % m.nx, ey = (e / m.nx) % m.ny, ez = e / (m.nx * m.ny);
    for (int k = 1; k <= az.reps(ez); ++k)
      for (int j = 1; j <= ay.reps(ey); ++j)
        for (int i = 1; i <= ax.reps(ex); ++i) {
          const int mult = ax.count(ex * N + i) * ay.count(ey * N + j) * az.count(ez * N + k);
          for (int f = 0; f < Nf; ++f) m.rowStarts[(size_t)row_of(ex, ey, ez, i, j, k, f) + 1] = mult;
        }
  }
  for (int32_t r = 0; r < m.Ngather; ++r) m.rowStarts[r + 1] += m.rowStarts[r];
  m.nnz = m.rowStarts[m.Ngather];
  m.colIds.assign((size_t)m.nnz, 0);
  m.G2L.assign((size_t)E * Np * Nf, -1);
#pragma omp parallel for
  for (int e = 0; e < E; ++e) {
    const int ex = e % m.nx, ey = (e / m.nx) % m.ny, ez = e / (m.nx * m.ny);
    for (int k = 0; k < Nq; ++k) {
      const int LK = ez * N + k;
      if (az.boundary(LK)) continue;
      const int rz = az.first(LK);
      for (int j = 0; j < Nq; ++j) {
        const int LJ = ey * N + j;
        if (ay.boundary(LJ)) continue;
        const int ry = ay.first(LJ);
        for (int i = 0; i < Nq; ++i) {
          const int LI = ex * N + i;
          if (ax.boundary(LI)) continue;
          const int rx = ax.first(LI);
          const int n = i + Nq * (j + Nq * k);
          // position among the class members (ascending element index)
          const int cx = ax.count(LI), cy = ay.count(LJ);
          const int pos = ((ez - rz) * cy + (ey - ry)) * cx + (ex - rx);
          for (int f = 0; f < Nf; ++f) {
            const int32_t row = row_of(rx, ry, rz, LI - rx * N, LJ - ry * N, LK - rz * N, f);
            const int64_t l = ((int64_t)e * Nf + f) * Np + n;
            m.G2L[(size_t)l] = row;
            m.colIds[(size_t)m.rowStarts[row] + pos] = (int32_t)l;
          }
        }
      }
    }
  }
}

// Quad2D box (meshSetupBoxQuad2D.cpp:30-100): element e = i + j nx, vertices
// (i,j), (i+1,j), (i+1,j+1), (i,j+1); the seeded perturbation of the Hex3D box
// in two coordinates (two draws per vertex id, x and y interleaved).
void box_vertices_2d(HostMesh& m, double pert, uint64_t seed) {
  const int nx = m.nx, ny = m.ny;
  const int64_t NnX = nx + 1, NnY = ny + 1;
  const double dx = 2.0 / nx, dy = 2.0 / ny;
  m.EX.resize((size_t)m.E * 4);
  m.EY.resize((size_t)m.E * 4);
  m.EZ.clear();
  std::vector<double> u;
  if (pert != 0.0) {
    u.resize((size_t)2 * NnX * NnY);
    uint64_t x = 6364136223846793005ULL * (~seed) + 1ULL;
    const double scale = 1.0 / (double)std::numeric_limits<uint64_t>::max();
    for (size_t r = 0; r < u.size(); ++r) {
      u[r] = (double)x * scale;
      x = 6364136223846793005ULL * x + 1ULL;
    }
  }
  static const int ci[4] = {0, 1, 1, 0};
  static const int cj[4] = {0, 0, 1, 1};
  for (int e = 0; e < m.E; ++e) {
    const int i = e % nx, j = e / nx;
    const double x0 = -1.0 + dx * i, y0 = -1.0 + dy * j;
    for (int c = 0; c < 4; ++c) {
      double X = ci[c] ? x0 + dx : x0;
      double Y = cj[c] ? y0 + dy : y0;
      const int64_t I = i + ci[c], J = j + cj[c];
      if (pert != 0.0 && I > 0 && I < nx && J > 0 && J < ny) {
        const int64_t g = I + J * NnX;
        X += pert * dx * (2 * u[2 * g + 0] - 1);
        Y += pert * dy * (2 * u[2 * g + 1] - 1);
      }
      m.EX[(size_t)e * 4 + c] = X;
      m.EY[(size_t)e * 4 + c] = Y;
    }
  }
}

// The masked numbering of the Quad2D box in the closed form of box_numbering:
// row r is the r-th unmasked connectivity class in order of first appearance
// over the local index e*Np*Nf + f*Np + n (the reference's order at one rank).
void box_numbering_2d(HostMesh& m) {
  const int N = m.N, Nq = m.Nq, Np = m.Np, Nf = m.Nfields;
  const Axis ax{m.nx, N}, ay{m.ny, N};
  const int E = m.E;
  std::vector<int64_t> rowBase((size_t)E + 1, 0);
  for (int e = 0; e < E; ++e) {
    const int ex = e % m.nx, ey = e / m.nx;
    rowBase[e + 1] = rowBase[e] + (int64_t)Nf * ax.reps(ex) * ay.reps(ey);
  }
  m.Ngather = (int32_t)rowBase[E];
  auto row_of = [&](int ex, int ey, int i, int j, int f) -> int32_t {
    const int e = ex + m.nx * ey;
    const int ci = ax.reps(ex), cj = ay.reps(ey);
    return (int32_t)(rowBase[e] + (int64_t)f * ci * cj + (int64_t)(j - 1) * ci + (i - 1));
  };
  m.rowStarts.assign((size_t)m.Ngather + 1, 0);
  for (int e = 0; e < E; ++e) {
    const int ex = e % m.nx, ey = e / m.nx;
    for (int j = 1; j <= ay.reps(ey); ++j)
      for (int i = 1; i <= ax.reps(ex); ++i) {
        const int mult = ax.count(ex * N + i) * ay.count(ey * N + j);
        for (int f = 0; f < Nf; ++f) m.rowStarts[(size_t)row_of(ex, ey, i, j, f) + 1] = mult;
      }
  }
  for (int32_t r = 0; r < m.Ngather; ++r) m.rowStarts[r + 1] += m.rowStarts[r];
  m.nnz = m.rowStarts[m.Ngather];
  m.colIds.assign((size_t)m.nnz, 0);
  m.G2L.assign((size_t)E * Np * Nf, -1);
  for (int e = 0; e < E; ++e) {
    const int ex = e % m.nx, ey = e / m.nx;
    for (int j = 0; j < Nq; ++j) {
      const int LJ = ey * N + j;
      if (ay.boundary(LJ)) continue;
      const int ry = ay.first(LJ);
      for (int i = 0; i < Nq; ++i) {
        const int LI = ex * N + i;
        if (ax.boundary(LI)) continue;
        const int rx = ax.first(LI);
        const int n = i + Nq * j;
        const int pos = (ey - ry) * ax.count(LI) + (ex - rx);
        for (int f = 0; f < Nf; ++f) {
          const int32_t row = row_of(rx, ry, LI - rx * N, LJ - ry * N, f);
          const int64_t l = ((int64_t)e * Nf + f) * Np + n;
          m.G2L[(size_t)l] = row;
          m.colIds[(size_t)m.rowStarts[row] + pos] = (int32_t)l;
        }
      }
    }
  }
}

// ---- Tri2D ----------------------------------------------------------------

// Orthonormal Jacobi polynomial P_n^(a,b)(x) by its three-term recurrence, and
// its derivative sqrt(n (n+a+b+1)) P_{n-1}^(a+1,b+1)(x).
static double jacobi_on(double x, double a, double b, int n) {
  const double g0 = std::pow(2.0, a + b + 1) / (a + b + 1) * std::tgamma(a + 1) * std::tgamma(b + 1) /
                    std::tgamma(a + b + 1);
  double pm = 1.0 / std::sqrt(g0);
  if (n == 0) return pm;
  const double g1 = (a + 1) * (b + 1) / (a + b + 3) * g0;
  double p = ((a + b + 2) * x / 2 + (a - b) / 2) / std::sqrt(g1);
  double aold = 2 / (2 + a + b) * std::sqrt((a + 1) * (b + 1) / (a + b + 3));
  for (int i = 1; i < n; ++i) {
    const double h1 = 2 * i + a + b;
    const double anew =
        2 / (h1 + 2) * std::sqrt((i + 1) * (i + 1 + a + b) * (i + 1 + a) * (i + 1 + b) / (h1 + 1) / (h1 + 3));
    const double bnew = -(a * a - b * b) / h1 / (h1 + 2);
    const double pn = (-aold * pm + (x - bnew) * p) / anew;
    pm = p;
    p = pn;
    aold = anew;
  }
  return p;
}
static double jacobi_on_deriv(double x, double a, double b, int n) {
  return n == 0 ? 0.0 : std::sqrt(n * (n + a + b + 1)) * jacobi_on(x, a + 1, b + 1, n - 1);
}

// Warp & blend nodes of the triangle (Warburton 2006): equispaced (r, s) rows
// in the reference's order (meshBasisTri2D.cpp:200-217), each edge warped
// toward the GLL distribution by the equispaced-to-GLL displacement,
// interpolated and divided by 1 - r^2, blended into the interior with the
// optimised alpha of each degree (:509-585).
static void tri_nodes(int N, std::vector<double>& r, std::vector<double>& s) {
  static const double alpha_opt[15] = {0.0000, 0.0000, 1.4152, 0.1001, 0.2751, 0.9800, 1.0999, 1.2832,
                                       1.3648, 1.4773, 1.4959, 1.5743, 1.5770, 1.6223, 1.6258};
  const double alpha = N < 16 ? alpha_opt[N - 1] : 5.0 / 3.0;
  r.clear();
  s.clear();
  for (int n = 0; n <= N; ++n)
    for (int m = 0; m + n <= N; ++m) {
      r.push_back(-1.0 + 2.0 * m / N);
      s.push_back(-1.0 + 2.0 * n / N);
    }
  std::vector<double> gll, w, req(N + 1);
  gll_nodes_weights(N, gll, w);
  for (int i = 0; i <= N; ++i) req[i] = -1.0 + 2.0 * i / N;
  auto warp = [&](double x) {
    std::vector<double> I;
    interp_matrix(req, std::vector<double>{x}, I);
    double v = 0.0;
    for (int i = 0; i <= N; ++i) v += I[i] * (gll[i] - req[i]);
    const double inside = std::fabs(x) < 1.0 - 1.0e-10 ? 1.0 : 0.0;
    const double sf = 1.0 - (inside * x) * (inside * x);
    return v / sf + v * (inside - 1.0);
  };
  const double pi = 3.14159265358979323846, r3 = std::sqrt(3.0);
  for (size_t k = 0; k < r.size(); ++k) {
    const double L1 = 0.5 * (1 + s[k]), L2 = -0.5 * (r[k] + s[k]), L3 = 0.5 * (1 + r[k]);
    double x = -L2 + L3, y = (-L2 - L3 + 2 * L1) / r3;
    const double w1 = 4 * L2 * L3 * warp(L3 - L2) * (1 + alpha * alpha * L1 * L1);
    const double w2 = 4 * L3 * L1 * warp(L1 - L3) * (1 + alpha * alpha * L2 * L2);
    const double w3 = 4 * L1 * L2 * warp(L2 - L1) * (1 + alpha * alpha * L3 * L3);
    x += w1 + std::cos(2 * pi / 3) * w2 + std::cos(4 * pi / 3) * w3;
    y += std::sin(2 * pi / 3) * w2 + std::sin(4 * pi / 3) * w3;
    const double l1 = (r3 * y + 1) / 3, l2 = (-3 * x - r3 * y + 2) / 6, l3 = (3 * x - r3 * y + 2) / 6;
    r[k] = -l2 + l3 - l1;
    s[k] = -l2 - l3 + l1;
  }
}

// Reference-element matrices of the triangle: the Vandermonde V (and Vr, Vs)
// of the orthonormal basis sqrt(2) P_i(a) P_j^(2i+1,0)(b) (1-b)^i of P_N at
// the nodes, Dr = Vr V^-1, Ds = Vs V^-1, MM = (V V^T)^-1
// (meshReferenceNodesTri2D.cpp:41-52) and the stiffness matrices
// Srr = Dr^T MM Dr, Srs = Dr^T MM Ds + Ds^T MM Dr, Sss = Ds^T MM Ds
// (meshBasisTri2D.cpp:406-430).  The matrices do not depend on the basis of
// P_N that builds V.  All row-major: X[n*Np + m] maps node m to node n.
bool tri_basis(int N, TriBasis& b) {
  const int Np = (N + 1) * (N + 2) / 2;
  b.N = N;
  b.Np = Np;
  tri_nodes(N, b.r, b.s);
  std::vector<double> V((size_t)Np * Np), Vr(V.size()), Vs(V.size());
  for (int k = 0; k < Np; ++k) {
    const double r = b.r[k], s = b.s[k];
    const double a = s != 1.0 ? 2 * (1 + r) / (1 - s) - 1 : -1.0, bb = s;
    int col = 0;
    for (int i = 0; i <= N; ++i)
      for (int j = 0; i + j <= N; ++j, ++col) {
        const double fa = jacobi_on(a, 0, 0, i), dfa = jacobi_on_deriv(a, 0, 0, i);
        const double gb = jacobi_on(bb, 2 * i + 1, 0, j), dgb = jacobi_on_deriv(bb, 2 * i + 1, 0, j);
        const double h = 0.5 * (1 - bb);
        const double hm1 = i > 0 ? std::pow(h, i - 1) : 1.0;
        V[(size_t)k * Np + col] = std::sqrt(2.0) * fa * gb * std::pow(1 - bb, i);
        const double dr = dfa * gb * hm1;
        double ds = dfa * gb * 0.5 * (1 + a) * hm1;
        double t = dgb * std::pow(h, i);
        if (i > 0) t -= 0.5 * i * gb * hm1;
        ds += fa * t;
        Vr[(size_t)k * Np + col] = std::pow(2.0, i + 0.5) * dr;
        Vs[(size_t)k * Np + col] = std::pow(2.0, i + 0.5) * ds;
      }
  }
  std::vector<double> Vi = V;
  if (!invert(Np, Vi)) return false;
  auto mul = [Np](const std::vector<double>& A, const std::vector<double>& B, bool ta) {
    std::vector<double> C((size_t)Np * Np, 0.0);
    for (int i = 0; i < Np; ++i)
      for (int k = 0; k < Np; ++k) {
        const double aik = ta ? A[(size_t)k * Np + i] : A[(size_t)i * Np + k];
        if (aik == 0.0) continue;
        for (int j = 0; j < Np; ++j) C[(size_t)i * Np + j] += aik * B[(size_t)k * Np + j];
      }
    return C;
  };
  b.Dr = mul(Vr, Vi, false);
  b.Ds = mul(Vs, Vi, false);
  std::vector<double> VVt((size_t)Np * Np, 0.0);
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) {
      double acc = 0.0;
      for (int k = 0; k < Np; ++k) acc += V[(size_t)i * Np + k] * V[(size_t)j * Np + k];
      VVt[(size_t)i * Np + j] = acc;
    }
  if (!invert(Np, VVt)) return false;
  b.MM = VVt;
  const std::vector<double> MDr = mul(b.MM, b.Dr, false), MDs = mul(b.MM, b.Ds, false);
  const std::vector<double> Srr = mul(b.Dr, MDr, true), Sss = mul(b.Ds, MDs, true);
  const std::vector<double> Srs1 = mul(b.Dr, MDs, true), Srs2 = mul(b.Ds, MDr, true);
  b.S.assign((size_t)3 * Np * Np, 0.0);
  for (size_t k = 0; k < (size_t)Np * Np; ++k) {
    b.S[k] = Srr[k];
    b.S[(size_t)Np * Np + k] = Srs1[k] + Srs2[k];
    b.S[(size_t)2 * Np * Np + k] = Sss[k];
  }
  return true;
}

// Tri2D box (meshSetupBoxTri2D.cpp:78-107): cell (i, j) holds triangles
// 2(i + j nx) with vertices (i,j), (i+1,j), (i+1,j+1) and 2(i + j nx) + 1 with
// (i,j), (i+1,j+1), (i,j+1); affine geometric factors per element
// (wJ = J; ggeo = J (rx^2+ry^2), J (rx sx + ry sy), J (sx^2+sy^2)); the masked
// numbering: a node's copies are found by topology (vertex, edge position,
// interior), its global id is its lowest copy (meshConnectNodes.cpp:32-82),
// the copies on boundary faces (faces 0, 1, 2: s = -1, r + s = 0, r = -1) are
// masked copy by copy, so a boundary vertex stays live through the elements
// that touch the boundary only there (meshMaskedGatherScatterSetup.cpp:31-56),
// rows follow each node's first unmasked copy and each row's columns ascend.
// Returns false on a non-positive Jacobian.
bool box_tri(HostMesh& m, const TriBasis& b, std::vector<double>& wJ, std::vector<double>& ggeo) {
  const int nx = m.nx, ny = m.ny, N = b.N, Np = b.Np, E = m.E;
  const int64_t NnX = nx + 1;
  const double dx = 2.0 / nx, dy = 2.0 / ny;
  std::vector<int64_t> EToV((size_t)E * 3);
  m.EX.resize((size_t)E * 3);
  m.EY.resize((size_t)E * 3);
  m.EZ.clear();
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const int e = 2 * (i + j * nx);
      const double x0 = -1.0 + dx * i, y0 = -1.0 + dy * j;
      const int64_t v00 = i + j * NnX, v10 = v00 + 1, v11 = v10 + NnX, v01 = v00 + NnX;
      const int64_t va[6] = {v00, v10, v11, v00, v11, v01};
      const double xa[6] = {x0, x0 + dx, x0 + dx, x0, x0 + dx, x0};
      const double ya[6] = {y0, y0, y0 + dy, y0, y0 + dy, y0 + dy};
      for (int c = 0; c < 6; ++c) {
        EToV[(size_t)e * 3 + c] = va[c];
        m.EX[(size_t)e * 3 + c] = xa[c];
        m.EY[(size_t)e * 3 + c] = ya[c];
      }
    }
  wJ.resize(E);
  ggeo.resize((size_t)3 * E);
  for (int e = 0; e < E; ++e) {
    const double* X = &m.EX[(size_t)e * 3];
    const double* Y = &m.EY[(size_t)e * 3];
    const double xr = 0.5 * (X[1] - X[0]), xs = 0.5 * (X[2] - X[0]);
    const double yr = 0.5 * (Y[1] - Y[0]), ys = 0.5 * (Y[2] - Y[0]);
    const double J = xr * ys - xs * yr;
    if (!(J > 0.0)) return false;
    const double rx = ys / J, ry = -xs / J, sx = -yr / J, sy = xr / J;
    wJ[e] = J;
    ggeo[(size_t)3 * e + 0] = J * (rx * rx + ry * ry);
    ggeo[(size_t)3 * e + 1] = J * (rx * sx + ry * sy);
    ggeo[(size_t)3 * e + 2] = J * (sx * sx + sy * sy);
  }
  // node roles in the reference element: vertex v (0..2), or edge f (0..2)
  // at position k from the edge's first vertex, or interior
  const double tol = 1.0e-5;
  std::vector<int> vert(Np, -1), edge(Np, -1), epos(Np, 0);
  static const int fv[3][2] = {{0, 1}, {1, 2}, {0, 2}};   // faces s=-1, r+s=0, r=-1, oriented by local index
  std::vector<std::vector<int>> fn(3);
  for (int n = 0; n < Np; ++n) {
    const bool on[3] = {std::fabs(b.s[n] + 1) < tol, std::fabs(b.r[n] + b.s[n]) < tol, std::fabs(b.r[n] + 1) < tol};
    for (int f = 0; f < 3; ++f)
      if (on[f]) fn[f].push_back(n);
    if (on[0] && on[2]) vert[n] = 0;
    else if (on[0] && on[1]) vert[n] = 1;
    else if (on[1] && on[2]) vert[n] = 2;
  }
  for (int f = 0; f < 3; ++f)
    for (size_t k = 0; k < fn[f].size(); ++k)
      if (vert[fn[f][k]] < 0) {
        edge[fn[f][k]] = f;
        epos[fn[f][k]] = (int)k;   // 1..N-1 from the face's first vertex (local index order)
      }
  // key of each copy: vertex id, or (edge's vertex pair, position from its lower vertex), or the copy itself
  const int64_t NV = (int64_t)(nx + 1) * (ny + 1);
  const int64_t NL = (int64_t)E * Np;
  std::vector<int64_t> key((size_t)NL);
  std::unordered_map<int64_t, int64_t> edge_key;   // undirected vertex pair -> base key
  int64_t next = NV;
  for (int e = 0; e < E; ++e)
    for (int n = 0; n < Np; ++n) {
      const int64_t l = (int64_t)e * Np + n;
      if (vert[n] >= 0) {
        key[(size_t)l] = EToV[(size_t)e * 3 + vert[n]];
      } else if (edge[n] >= 0) {
        int64_t a = EToV[(size_t)e * 3 + fv[edge[n]][0]], c = EToV[(size_t)e * 3 + fv[edge[n]][1]];
        int k = epos[n];
        if (a > c) {
          std::swap(a, c);
          k = N - k;
        }
        const int64_t pair = a * NV + c;
        auto it = edge_key.find(pair);
        if (it == edge_key.end()) it = edge_key.emplace(pair, (next += N) - N).first;
        key[(size_t)l] = it->second + k;
      } else {
        key[(size_t)l] = -1 - l;   // interior: its own class
      }
    }
  // copies on boundary faces are masked
  std::vector<char> masked((size_t)NL, 0);
  for (int e = 0; e < E; ++e) {
    const double* X = &m.EX[(size_t)e * 3];
    const double* Y = &m.EY[(size_t)e * 3];
    for (int f = 0; f < 3; ++f) {
      const int a = fv[f][0], c = fv[f][1];
      auto at = [](double v, double w) { return std::fabs(v - w) < 1.0e-12; };
      const bool bnd = (at(X[a], -1.0) && at(X[c], -1.0)) || (at(X[a], 1.0) && at(X[c], 1.0)) ||
                       (at(Y[a], -1.0) && at(Y[c], -1.0)) || (at(Y[a], 1.0) && at(Y[c], 1.0));
      if (bnd)
        for (int n : fn[f]) masked[(size_t)e * Np + n] = 1;
    }
  }
  std::unordered_map<int64_t, int32_t> row;
  m.G2L.assign((size_t)NL, -1);
  std::vector<int32_t> count;
  for (int64_t l = 0; l < NL; ++l) {
    if (masked[(size_t)l]) continue;
    auto it = row.find(key[(size_t)l]);
    if (it == row.end()) {
      it = row.emplace(key[(size_t)l], (int32_t)count.size()).first;
      count.push_back(0);
    }
    m.G2L[(size_t)l] = it->second;
    ++count[it->second];
  }
  m.Ngather = (int32_t)count.size();
  m.rowStarts.assign((size_t)m.Ngather + 1, 0);
  for (int32_t r = 0; r < m.Ngather; ++r) m.rowStarts[r + 1] = m.rowStarts[r] + count[r];
  m.nnz = m.rowStarts[m.Ngather];
  m.colIds.assign((size_t)m.nnz, 0);
  std::vector<int32_t> fill(m.rowStarts.begin(), m.rowStarts.end() - 1);
  for (int64_t l = 0; l < NL; ++l)
    if (m.G2L[(size_t)l] >= 0) m.colIds[(size_t)fill[m.G2L[(size_t)l]]++] = (int32_t)l;
  return true;
}

// the affine map of each triangle's vertices at the reference nodes
// (meshPhysicalNodesTri2D.cpp): x = -(r+s)/2 x1 + (1+r)/2 x2 + (1+s)/2 x3
void tri_nodes_xy(const HostMesh& m, const TriBasis& b, std::vector<double>& x, std::vector<double>& y) {
  const int Np = b.Np;
  x.resize((size_t)m.E * Np);
  y.resize((size_t)m.E * Np);
  for (int e = 0; e < m.E; ++e) {
    const double* X = &m.EX[(size_t)e * 3];
    const double* Y = &m.EY[(size_t)e * 3];
    for (int n = 0; n < Np; ++n) {
      const double r = b.r[n], s = b.s[n];
      x[(size_t)e * Np + n] = -0.5 * (r + s) * X[0] + 0.5 * (1 + r) * X[1] + 0.5 * (1 + s) * X[2];
      y[(size_t)e * Np + n] = -0.5 * (r + s) * Y[0] + 0.5 * (1 + r) * Y[1] + 0.5 * (1 + s) * Y[2];
    }
  }
}

// ---- Tet3D ----------------------------------------------------------------

// the 2D warp of one face of the tetrahedron, in its two tangential directions
// (WarpShiftFace3D, meshBasisTet3D.cpp:604-645)
static void face_warp(int N, double alpha, double L1, double L2, double L3, const std::vector<double>& gll,
                      const std::vector<double>& req, double& w1, double& w2) {
  auto warp = [&](double x) {
    std::vector<double> I;
    interp_matrix(req, std::vector<double>{x}, I);
    double v = 0.0;
    for (int i = 0; i <= N; ++i) v += I[i] * (gll[i] - req[i]);
    const double inside = std::fabs(x) < 1.0 - 1.0e-10 ? 1.0 : 0.0;
    const double sf = 1.0 - (inside * x) * (inside * x);
    return v / sf + v * (inside - 1.0);
  };
  const double pi = 3.14159265358979323846;
  const double a = 4 * L2 * L3 * warp(L3 - L2) * (1 + alpha * alpha * L1 * L1);
  const double b = 4 * L3 * L1 * warp(L1 - L3) * (1 + alpha * alpha * L2 * L2);
  const double c = 4 * L1 * L2 * warp(L2 - L1) * (1 + alpha * alpha * L3 * L3);
  w1 = a + std::cos(2 * pi / 3) * b + std::cos(4 * pi / 3) * c;
  w2 = std::sin(2 * pi / 3) * b + std::sin(4 * pi / 3) * c;
}

// Warp & blend nodes of the tetrahedron (Warburton 2006; meshBasisTet3D.cpp:
// 227-248, 647-763): equispaced (r, s, t) layers in the reference's order, the
// face warps along each face's unit tangents blended by Lb Lc Ld (with the
// alpha of each degree), a face's own warp on its edges, mapped back from the
// equilateral tetrahedron.  Also the nodes' lattice weights on the vertices.
static void tet_nodes(int N, TetBasis& b) {
  static const double alpha_opt[15] = {0.0000, 0.0000, 0.00000, 0.1002, 1.1332, 1.5608, 1.3413, 1.2577,
                                       1.1603, 1.10153, 0.6080, 0.4523, 0.8856, 0.8717, 0.9655};
  const double alpha = N < 16 ? alpha_opt[N - 1] : 1.0;
  const double r3 = std::sqrt(3.0), r6 = std::sqrt(6.0);
  const double v[4][3] = {{-1.0, -1 / r3, -1 / r6}, {1.0, -1 / r3, -1 / r6}, {0.0, 2 / r3, -1 / r6}, {0.0, 0.0, 3 / r6}};
  double t1[4][3], t2[4][3];
  for (int i = 0; i < 3; ++i) {
    t1[0][i] = v[1][i] - v[0][i];
    t1[1][i] = v[1][i] - v[0][i];
    t1[2][i] = v[2][i] - v[1][i];
    t1[3][i] = v[2][i] - v[0][i];
    t2[0][i] = v[2][i] - 0.5 * (v[0][i] + v[1][i]);
    t2[1][i] = v[3][i] - 0.5 * (v[0][i] + v[1][i]);
    t2[2][i] = v[3][i] - 0.5 * (v[1][i] + v[2][i]);
    t2[3][i] = v[3][i] - 0.5 * (v[0][i] + v[2][i]);
  }
  for (int f = 0; f < 4; ++f) {
    const double n1 = std::sqrt(t1[f][0] * t1[f][0] + t1[f][1] * t1[f][1] + t1[f][2] * t1[f][2]);
    const double n2 = std::sqrt(t2[f][0] * t2[f][0] + t2[f][1] * t2[f][1] + t2[f][2] * t2[f][2]);
    for (int i = 0; i < 3; ++i) {
      t1[f][i] /= n1;
      t2[f][i] /= n2;
    }
  }
  std::vector<double> gll, w, req(N + 1);
  gll_nodes_weights(N, gll, w);
  for (int i = 0; i <= N; ++i) req[i] = -1.0 + 2.0 * i / N;
  b.r.clear(); b.s.clear(); b.t.clear(); b.bary.clear();
  for (int k = 0; k <= N; ++k)
    for (int n = 0; n + k <= N; ++n)
      for (int m = 0; m + n + k <= N; ++m) {
        const double r = -1.0 + 2.0 * m / N, s = -1.0 + 2.0 * n / N, t = -1.0 + 2.0 * k / N;
        const double L[4] = {0.5 * (1 + t), 0.5 * (1 + s), -0.5 * (1 + r + s + t), 0.5 * (1 + r)};   // L1..L4
        double X[3];
        for (int i = 0; i < 3; ++i) X[i] = L[2] * v[0][i] + L[3] * v[1][i] + L[1] * v[2][i] + L[0] * v[3][i];
        double sh[3] = {0, 0, 0};
        static const int perm[4][4] = {{0, 1, 2, 3}, {1, 0, 2, 3}, {2, 0, 3, 1}, {3, 0, 2, 1}};   // La, Lb, Lc, Ld
        for (int f = 0; f < 4; ++f) {
          const double La = L[perm[f][0]], Lb = L[perm[f][1]], Lc = L[perm[f][2]], Ld = L[perm[f][3]];
          double w1, w2;
          face_warp(N, alpha, Lb, Lc, Ld, gll, req, w1, w2);
          double blend = Lb * Lc * Ld;
          const double denom = (Lb + 0.5 * La) * (Lc + 0.5 * La) * (Ld + 0.5 * La);
          if (denom > 1.0e-10) blend = (1 + (alpha * La) * (alpha * La)) * blend / denom;
          for (int i = 0; i < 3; ++i) sh[i] += (blend * w1) * t1[f][i] + (blend * w2) * t2[f][i];
          if (La < 1.0e-10 && (Lb < 1.0e-10 || Lc < 1.0e-10 || Ld < 1.0e-10))
            for (int i = 0; i < 3; ++i) sh[i] = w1 * t1[f][i] + w2 * t2[f][i];
        }
        for (int i = 0; i < 3; ++i) X[i] += sh[i];
        // back to (r, s, t): X - c = r a1 + s a2 + t a3, a_j = (v_{j+1} - v_0)/2
        double A[9], B[3];
        for (int i = 0; i < 3; ++i) {
          A[i * 3 + 0] = 0.5 * (v[1][i] - v[0][i]);
          A[i * 3 + 1] = 0.5 * (v[2][i] - v[0][i]);
          A[i * 3 + 2] = 0.5 * (v[3][i] - v[0][i]);
          B[i] = X[i] - 0.5 * (v[1][i] + v[2][i] + v[3][i] - v[0][i]);
        }
        std::vector<double> Ai(A, A + 9);
        invert(3, Ai);
        b.r.push_back(Ai[0] * B[0] + Ai[1] * B[1] + Ai[2] * B[2]);
        b.s.push_back(Ai[3] * B[0] + Ai[4] * B[1] + Ai[5] * B[2]);
        b.t.push_back(Ai[6] * B[0] + Ai[7] * B[1] + Ai[8] * B[2]);
        const int bw[4] = {N - m - n - k, m, n, k};   // on vertices (-1,-1,-1), r = 1, s = 1, t = 1
        b.bary.insert(b.bary.end(), bw, bw + 4);
      }
}

// Reference-element matrices of the tetrahedron: the Vandermonde (and its r,
// s, t derivatives) of the orthonormal basis of P_N in collapsed coordinates,
// Dr, Ds, Dt = Vr,s,t V^-1, MM = (V V^T)^-1, and the six stiffness matrices
// S_ab = Da^T MM Db (+ Db^T MM Da for a != b) (meshBasisTet3D.cpp:494-527).
bool tet_basis(int N, TetBasis& b) {
  const int Np = (N + 1) * (N + 2) * (N + 3) / 6;
  b.N = N;
  b.Np = Np;
  tet_nodes(N, b);
  std::vector<double> V((size_t)Np * Np), Vr(V.size()), Vs(V.size()), Vt(V.size());
  for (int p = 0; p < Np; ++p) {
    const double r = b.r[p], s = b.s[p], t = b.t[p];
    const double a = std::fabs(s + t) > 1e-14 ? 2 * (1 + r) / (-s - t) - 1 : -1.0;
    const double bb = std::fabs(t - 1) > 1e-14 ? 2 * (1 + s) / (1 - t) - 1 : -1.0;
    const double c = t;
    int col = 0;
    for (int i = 0; i <= N; ++i)
      for (int j = 0; i + j <= N; ++j)
        for (int k = 0; i + j + k <= N; ++k, ++col) {
          const double fa = jacobi_on(a, 0, 0, i), dfa = jacobi_on_deriv(a, 0, 0, i);
          const double gb = jacobi_on(bb, 2 * i + 1, 0, j), dgb = jacobi_on_deriv(bb, 2 * i + 1, 0, j);
          const double hc = jacobi_on(c, 2 * (i + j) + 2, 0, k), dhc = jacobi_on_deriv(c, 2 * (i + j) + 2, 0, k);
          const double hb = 0.5 * (1 - bb), hcc = 0.5 * (1 - c);
          V[(size_t)p * Np + col] = 2 * std::sqrt(2.0) * fa * gb * std::pow(1 - bb, i) * hc * std::pow(1 - c, i + j);
          double dr = dfa * gb * hc;
          if (i > 0) dr *= std::pow(hb, i - 1);
          if (i + j > 0) dr *= std::pow(hcc, i + j - 1);
          double ds = 0.5 * (1 + a) * dr;
          double tmp = dgb * std::pow(hb, i);
          if (i > 0) tmp -= 0.5 * i * gb * std::pow(hb, i - 1);
          if (i + j > 0) tmp *= std::pow(hcc, i + j - 1);
          tmp = fa * tmp * hc;
          ds += tmp;
          double dt = 0.5 * (1 + a) * dr + 0.5 * (1 + bb) * tmp;
          tmp = dhc * std::pow(hcc, i + j);
          if (i + j > 0) tmp -= 0.5 * (i + j) * hc * std::pow(hcc, i + j - 1);
          tmp = fa * gb * tmp * std::pow(hb, i);
          dt += tmp;
          const double sc = std::pow(2.0, 2 * i + j + 1.5);
          Vr[(size_t)p * Np + col] = dr * sc;
          Vs[(size_t)p * Np + col] = ds * sc;
          Vt[(size_t)p * Np + col] = dt * sc;
        }
  }
  std::vector<double> Vi = V;
  if (!invert(Np, Vi)) return false;
  auto mul = [Np](const std::vector<double>& A, const std::vector<double>& B, bool ta) {
    std::vector<double> C((size_t)Np * Np, 0.0);
    for (int i = 0; i < Np; ++i)
      for (int k = 0; k < Np; ++k) {
        const double aik = ta ? A[(size_t)k * Np + i] : A[(size_t)i * Np + k];
        if (aik == 0.0) continue;
        for (int j = 0; j < Np; ++j) C[(size_t)i * Np + j] += aik * B[(size_t)k * Np + j];
      }
    return C;
  };
  b.Dr = mul(Vr, Vi, false);
  b.Ds = mul(Vs, Vi, false);
  b.Dt = mul(Vt, Vi, false);
  std::vector<double> VVt((size_t)Np * Np, 0.0);
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) {
      double acc = 0.0;
      for (int k = 0; k < Np; ++k) acc += V[(size_t)i * Np + k] * V[(size_t)j * Np + k];
      VVt[(size_t)i * Np + j] = acc;
    }
  if (!invert(Np, VVt)) return false;
  b.MM = VVt;
  const std::vector<double>* D[3] = {&b.Dr, &b.Ds, &b.Dt};
  std::vector<double> MD[3];
  for (int a = 0; a < 3; ++a) MD[a] = mul(b.MM, *D[a], false);
  static const int pairs[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  const size_t NP2 = (size_t)Np * Np;
  b.S.assign(6 * NP2, 0.0);
  for (int q = 0; q < 6; ++q) {
    const int a = pairs[q][0], c = pairs[q][1];
    std::vector<double> X = mul(*D[a], MD[c], true);
    if (a != c) {
      const std::vector<double> Y = mul(*D[c], MD[a], true);
      for (size_t k = 0; k < NP2; ++k) X[k] += Y[k];
    }
    std::copy(X.begin(), X.end(), b.S.begin() + q * NP2);
  }
  return true;
}

// Tet3D box (meshSetupBoxTet3D.cpp): cell (i, j, k) holds tetrahedra
// 6(i + j nx + k nx ny) + 0..5 on the cell corners (0,3,2,7), (0,1,3,7),
// (0,2,6,7), (0,6,4,7), (0,5,1,7), (0,4,5,7) (corner bits: x, y, z); affine
// factors per element (wJ = J; ggeo = J grad a . grad b for ab = rr, rs, rt,
// ss, st, tt; meshGeometricFactorsTet3D.cpp:31-110); the masked numbering as
// for Tri2D, a node identified by its lattice weights on the global vertices;
// boundary faces 0..3 (t = -1, s = -1, r + s + t = -1, r = -1).  Returns false
// on a non-positive Jacobian.
bool box_tet(HostMesh& m, const TetBasis& b, std::vector<double>& wJ, std::vector<double>& ggeo,
             std::vector<double>& x, std::vector<double>& y, std::vector<double>& z) {
  static const int tets[6][4] = {{0, 3, 2, 7}, {0, 1, 3, 7}, {0, 2, 6, 7}, {0, 6, 4, 7}, {0, 5, 1, 7}, {0, 4, 5, 7}};
  const int nx = m.nx, ny = m.ny, nz = m.nz, N = b.N, Np = b.Np, E = m.E;
  const int64_t NnX = nx + 1, NnY = ny + 1;
  const double dx = 2.0 / nx, dy = 2.0 / ny, dz = 2.0 / nz;
  std::vector<int64_t> EToV((size_t)E * 4);
  m.EX.resize((size_t)E * 4);
  m.EY.resize((size_t)E * 4);
  m.EZ.resize((size_t)E * 4);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const double x0 = -1.0 + dx * i, y0 = -1.0 + dy * j, z0 = -1.0 + dz * k;
        for (int q = 0; q < 6; ++q) {
          const int e = 6 * (i + j * nx + k * nx * ny) + q;
          for (int c = 0; c < 4; ++c) {
            const int cn = tets[q][c], ci = cn & 1, cj = (cn >> 1) & 1, ck = (cn >> 2) & 1;
            EToV[(size_t)e * 4 + c] = (i + ci) + (j + cj) * NnX + (k + ck) * NnX * NnY;
            m.EX[(size_t)e * 4 + c] = ci ? x0 + dx : x0;
            m.EY[(size_t)e * 4 + c] = cj ? y0 + dy : y0;
            m.EZ[(size_t)e * 4 + c] = ck ? z0 + dz : z0;
          }
        }
      }
  wJ.resize(E);
  ggeo.resize((size_t)6 * E);
  x.resize((size_t)E * Np);
  y.resize((size_t)E * Np);
  z.resize((size_t)E * Np);
  for (int e = 0; e < E; ++e) {
    const double* X = &m.EX[(size_t)e * 4];
    const double* Y = &m.EY[(size_t)e * 4];
    const double* Z = &m.EZ[(size_t)e * 4];
    const double xr = 0.5 * (X[1] - X[0]), xs = 0.5 * (X[2] - X[0]), xt = 0.5 * (X[3] - X[0]);
    const double yr = 0.5 * (Y[1] - Y[0]), ys = 0.5 * (Y[2] - Y[0]), yt = 0.5 * (Y[3] - Y[0]);
    const double zr = 0.5 * (Z[1] - Z[0]), zs = 0.5 * (Z[2] - Z[0]), zt = 0.5 * (Z[3] - Z[0]);
    const double J = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt);
    if (!(J > 0.0)) return false;
    const double rx = (ys * zt - zs * yt) / J, ry = -(xs * zt - zs * xt) / J, rz = (xs * yt - ys * xt) / J;
    const double sx = -(yr * zt - zr * yt) / J, sy = (xr * zt - zr * xt) / J, sz = -(xr * yt - yr * xt) / J;
    const double tx = (yr * zs - zr * ys) / J, ty = -(xr * zs - zr * xs) / J, tz = (xr * ys - yr * xs) / J;
    wJ[e] = J;
    double* g = &ggeo[(size_t)6 * e];
    g[0] = J * (rx * rx + ry * ry + rz * rz);
    g[1] = J * (rx * sx + ry * sy + rz * sz);
    g[2] = J * (rx * tx + ry * ty + rz * tz);
    g[3] = J * (sx * sx + sy * sy + sz * sz);
    g[4] = J * (sx * tx + sy * ty + sz * tz);
    g[5] = J * (tx * tx + ty * ty + tz * tz);
    for (int n = 0; n < Np; ++n) {
      const double r = b.r[n], s = b.s[n], t = b.t[n];
      const double w[4] = {-0.5 * (1 + r + s + t), 0.5 * (1 + r), 0.5 * (1 + s), 0.5 * (1 + t)};
      double px = 0, py = 0, pz = 0;
      for (int c = 0; c < 4; ++c) {
        px += w[c] * X[c];
        py += w[c] * Y[c];
        pz += w[c] * Z[c];
      }
      x[(size_t)e * Np + n] = px;
      y[(size_t)e * Np + n] = py;
      z[(size_t)e * Np + n] = pz;
    }
  }
  // a node's identity: its nonzero lattice weights on global vertex ids
  const int64_t NL = (int64_t)E * Np;
  std::map<std::array<int64_t, 4>, int64_t> cls;
  std::vector<int64_t> key((size_t)NL);
  for (int e = 0; e < E; ++e)
    for (int n = 0; n < Np; ++n) {
      std::array<int64_t, 4> k4;
      int cnt = 0;
      for (int c = 0; c < 4; ++c)
        if (b.bary[(size_t)n * 4 + c] > 0) k4[cnt++] = EToV[(size_t)e * 4 + c] * (N + 1) + b.bary[(size_t)n * 4 + c];
      std::sort(k4.begin(), k4.begin() + cnt);
      for (int c = cnt; c < 4; ++c) k4[c] = -1;
      auto it = cls.emplace(k4, (int64_t)cls.size()).first;
      key[(size_t)e * Np + n] = it->second;
    }
  // copies on boundary faces are masked
  const double tol = 1.0e-5;
  std::vector<std::vector<int>> fn(4);
  for (int n = 0; n < Np; ++n) {
    const double r = b.r[n], s = b.s[n], t = b.t[n];
    if (std::fabs(t + 1) < tol) fn[0].push_back(n);
    if (std::fabs(s + 1) < tol) fn[1].push_back(n);
    if (std::fabs(r + s + t + 1) < tol) fn[2].push_back(n);
    if (std::fabs(r + 1) < tol) fn[3].push_back(n);
  }
  static const int fv[4][3] = {{0, 1, 2}, {0, 1, 3}, {1, 2, 3}, {0, 2, 3}};
  std::vector<char> masked((size_t)NL, 0);
  auto at = [](double v, double w) { return std::fabs(v - w) < 1.0e-12; };
  for (int e = 0; e < E; ++e) {
    const double* C[3] = {&m.EX[(size_t)e * 4], &m.EY[(size_t)e * 4], &m.EZ[(size_t)e * 4]};
    for (int f = 0; f < 4; ++f) {
      bool bnd = false;
      for (int d = 0; d < 3 && !bnd; ++d)
        for (double side : {-1.0, 1.0})
          if (at(C[d][fv[f][0]], side) && at(C[d][fv[f][1]], side) && at(C[d][fv[f][2]], side)) bnd = true;
      if (bnd)
        for (int n : fn[f]) masked[(size_t)e * Np + n] = 1;
    }
  }
  std::vector<int32_t> row(cls.size(), -1), count;
  m.G2L.assign((size_t)NL, -1);
  for (int64_t l = 0; l < NL; ++l) {
    if (masked[(size_t)l]) continue;
    int32_t& rw = row[(size_t)key[(size_t)l]];
    if (rw < 0) {
      rw = (int32_t)count.size();
      count.push_back(0);
    }
    m.G2L[(size_t)l] = rw;
    ++count[rw];
  }
  m.Ngather = (int32_t)count.size();
  m.rowStarts.assign((size_t)m.Ngather + 1, 0);
  for (int32_t r = 0; r < m.Ngather; ++r) m.rowStarts[r + 1] = m.rowStarts[r] + count[r];
  m.nnz = m.rowStarts[m.Ngather];
  m.colIds.assign((size_t)m.nnz, 0);
  std::vector<int32_t> fill(m.rowStarts.begin(), m.rowStarts.end() - 1);
  for (int64_t l = 0; l < NL; ++l)
    if (m.G2L[(size_t)l] >= 0) m.colIds[(size_t)fill[m.G2L[(size_t)l]]++] = (int32_t)l;
  return true;
}

// GeometricFactorsQuad2D (meshGeometricFactorsQuad2D.cpp:31-120) from the
// bilinear map of the vertices at the GLL nodes (meshPhysicalNodesQuad2D.cpp)
bool quad_geometry(const HostMesh& m, std::vector<double>& wJ, std::vector<double>& ggeo) {
  const int Nq = m.Nq, Np = m.Np;
  bool ok = true;
  if (m.affine) {
    wJ.resize(m.E);
    ggeo.resize((size_t)3 * m.E);
    for (int e = 0; e < m.E; ++e) {
      const double* ex = &m.EX[(size_t)e * 4];
      const double* ey = &m.EY[(size_t)e * 4];
      const double xr = 0.5 * (ex[1] - ex[0]), xs = 0.5 * (ex[3] - ex[0]);
      const double yr = 0.5 * (ey[1] - ey[0]), ys = 0.5 * (ey[3] - ey[0]);
      const double J = xr * ys - xs * yr;
      if (!(J >= 1e-8)) ok = false;
      const double rx = ys / J, ry = -xs / J, sx = -yr / J, sy = xr / J;
      wJ[e] = J;
      ggeo[3 * (size_t)e + 0] = J * (rx * rx + ry * ry);
      ggeo[3 * (size_t)e + 1] = J * (rx * sx + ry * sy);
      ggeo[3 * (size_t)e + 2] = J * (sx * sx + sy * sy);
    }
    return ok;
  }
  wJ.resize((size_t)m.E * Np);
  ggeo.resize((size_t)3 * m.E * Np);
  std::vector<double> x(Np), y(Np);
#pragma omp parallel for firstprivate(x, y) reduction(&& : ok)
  for (int e = 0; e < m.E; ++e) {
    const double* ex = &m.EX[(size_t)e * 4];
    const double* ey = &m.EY[(size_t)e * 4];
    for (int j = 0; j < Nq; ++j)
      for (int i = 0; i < Nq; ++i) {
        const double r = m.gllz[i], s = m.gllz[j];
        const double a0 = 0.25 * (1 - r) * (1 - s), a1 = 0.25 * (1 + r) * (1 - s), a2 = 0.25 * (1 + r) * (1 + s),
                     a3 = 0.25 * (1 - r) * (1 + s);
        x[i + j * Nq] = a0 * ex[0] + a1 * ex[1] + a2 * ex[2] + a3 * ex[3];
        y[i + j * Nq] = a0 * ey[0] + a1 * ey[1] + a2 * ey[2] + a3 * ey[3];
      }
    for (int j = 0; j < Nq; ++j)
      for (int i = 0; i < Nq; ++i) {
        double xr = 0, xs = 0, yr = 0, ys = 0;
        for (int mm = 0; mm < Nq; ++mm) {
          xr += m.D[i * Nq + mm] * x[j * Nq + mm];
          xs += m.D[j * Nq + mm] * x[mm * Nq + i];
          yr += m.D[i * Nq + mm] * y[j * Nq + mm];
          ys += m.D[j * Nq + mm] * y[mm * Nq + i];
        }
        const double J = xr * ys - xs * yr;
        if (!(J >= 1e-8)) ok = false;
        const double rx = ys / J, ry = -xs / J, sx = -yr / J, sy = xr / J;
        const double JW = J * m.gllw[i] * m.gllw[j];
        const size_t id = (size_t)e * Np + i + j * Nq;
        wJ[id] = JW;
        ggeo[3 * id + 0] = JW * (rx * rx + ry * ry);
        ggeo[3 * id + 1] = JW * (rx * sx + ry * sy);
        ggeo[3 * id + 2] = JW * (sx * sx + sy * sy);
      }
  }
  return ok;
}

}  // namespace bp

// ---------------------------------------------------------------------------
// host-only C entry points
// ---------------------------------------------------------------------------
namespace {
int host_mesh_from_desc(const bp_box_desc_t* d, bp::HostMesh& m) {
  if (!d) return bp::fail(BP_ERROR_ARG, "null descriptor");
  if (d->dim != 0 && d->dim != 2 && d->dim != 3) return bp::fail(BP_ERROR_ARG, "box dim must be 2 or 3");
  m.dim = d->dim == 2 ? 2 : 3;
  if (d->simplex) {
    const int nzs = m.dim == 2 ? 1 : d->nz;
    if (d->nx < 1 || d->ny < 1 || nzs < 1 || d->N < 1 || d->N > 15 || d->Nfields != 1)
      return bp::fail(BP_ERROR_ARG, "bad simplex box descriptor");
    m.N = d->N; m.Nq = d->N + 1;
    m.Np = m.dim == 2 ? (d->N + 1) * (d->N + 2) / 2 : (d->N + 1) * (d->N + 2) * (d->N + 3) / 6;
    m.nx = d->nx; m.ny = d->ny; m.nz = nzs;
    const int64_t E = (m.dim == 2 ? 2 : 6) * (int64_t)d->nx * d->ny * nzs;
    if (E * m.Np >= (int64_t)INT32_MAX) return bp::fail(BP_ERROR_ARG, "local node count exceeds int32");
    m.E = (int)E; m.affine = 1; m.Nfields = 1;
    return BP_SUCCESS;
  }
  const int nz = m.dim == 2 ? 1 : d->nz;
  if (d->nx < 1 || d->ny < 1 || nz < 1 || d->N < 1 || d->N > 15 ||
      (m.dim == 3 && d->Nfields != 1 && d->Nfields != 3) || (m.dim == 2 && d->Nfields != 1 && d->Nfields != 2))
    return bp::fail(BP_ERROR_ARG, "bad box descriptor");
  m.N = d->N; m.Nq = d->N + 1; m.Np = m.dim == 2 ? m.Nq * m.Nq : m.Nq * m.Nq * m.Nq;
  m.nx = d->nx; m.ny = d->ny; m.nz = nz;
  const int64_t E = (int64_t)d->nx * d->ny * nz;
  if (E * m.Np * d->Nfields >= (int64_t)INT32_MAX) return bp::fail(BP_ERROR_ARG, "local node count exceeds int32");
  m.E = (int)E; m.affine = d->affine ? 1 : 0; m.Nfields = d->Nfields;
  return BP_SUCCESS;
}
}  // namespace

extern "C" int bp_box_numbering(const bp_box_desc_t* d, int32_t* Ngather, int32_t* nnz, int32_t* G2L,
                                int32_t* rowStarts, int32_t* colIds) {
  bp::HostMesh m;
  int rc = host_mesh_from_desc(d, m);
  if (rc) return rc;
  if (d->simplex && m.dim == 3) {
    bp::TetBasis tb;
    std::vector<double> wJ, ggeo, x, y, z;
    if (!bp::tet_basis(m.N, tb) || !bp::box_tet(m, tb, wJ, ggeo, x, y, z))
      return bp::fail(BP_ERROR_NUMERIC, "bp_box_numbering: Tet3D set-up failed");
  } else if (d->simplex) {
    bp::TriBasis tb;
    std::vector<double> wJ, ggeo;
    if (!bp::tri_basis(m.N, tb) || !bp::box_tri(m, tb, wJ, ggeo))
      return bp::fail(BP_ERROR_NUMERIC, "bp_box_numbering: Tri2D set-up failed");
  } else if (m.dim == 2) {
    bp::box_numbering_2d(m);
  } else {
    bp::box_numbering(m);
  }
  if (Ngather) *Ngather = m.Ngather;
  if (nnz) *nnz = m.nnz;
  if (G2L) std::copy(m.G2L.begin(), m.G2L.end(), G2L);
  if (rowStarts) std::copy(m.rowStarts.begin(), m.rowStarts.end(), rowStarts);
  if (colIds) std::copy(m.colIds.begin(), m.colIds.end(), colIds);
  return BP_SUCCESS;
}

extern "C" int bp_basis_gll(int32_t N, double* z, double* w, double* D) {
  if (N < 1 || N > 15) return bp::fail(BP_ERROR_ARG, "degree must be in 1..15");
  std::vector<double> zz, ww, DD;
  bp::gll_nodes_weights(N, zz, ww);
  bp::diff_matrix(zz, DD);
  if (z) std::copy(zz.begin(), zz.end(), z);
  if (w) std::copy(ww.begin(), ww.end(), w);
  if (D) std::copy(DD.begin(), DD.end(), D);
  return BP_SUCCESS;
}

extern "C" int bp_basis_tri2d(int32_t N, double* r, double* s, double* D, double* MM, double* S) {
  if (N < 1 || N > 15) return bp::fail(BP_ERROR_ARG, "bp_basis_tri2d: degree must be in 1..15");
  bp::TriBasis tb;
  if (!bp::tri_basis(N, tb)) return bp::fail(BP_ERROR_NUMERIC, "bp_basis_tri2d: singular Vandermonde matrix");
  const int Np = tb.Np;
  const size_t NP2 = (size_t)Np * Np;
  auto put = [&](const std::vector<double>& rm, double* out, size_t off) {   // node-fastest
    for (int n = 0; n < Np; ++n)
      for (int k = 0; k < Np; ++k) out[off + (size_t)k * Np + n] = rm[(size_t)n * Np + k];
  };
  if (r) std::copy(tb.r.begin(), tb.r.end(), r);
  if (s) std::copy(tb.s.begin(), tb.s.end(), s);
  if (D) {
    put(tb.Dr, D, 0);
    put(tb.Ds, D, NP2);
  }
  if (MM) std::copy(tb.MM.begin(), tb.MM.end(), MM);
  if (S)
    for (int b = 0; b < 3; ++b) {
      const std::vector<double> blk(tb.S.begin() + b * NP2, tb.S.begin() + (b + 1) * NP2);
      put(blk, S, b * NP2);
    }
  return BP_SUCCESS;
}

extern "C" int bp_basis_tet3d(int32_t N, double* r, double* s, double* t, double* D, double* MM, double* S) {
  if (N < 1 || N > 15) return bp::fail(BP_ERROR_ARG, "bp_basis_tet3d: degree must be in 1..15");
  bp::TetBasis tb;
  if (!bp::tet_basis(N, tb)) return bp::fail(BP_ERROR_NUMERIC, "bp_basis_tet3d: singular Vandermonde matrix");
  const int Np = tb.Np;
  const size_t NP2 = (size_t)Np * Np;
  auto put = [&](const double* rm, double* out) {   // node-fastest
    for (int n = 0; n < Np; ++n)
      for (int k = 0; k < Np; ++k) out[(size_t)k * Np + n] = rm[(size_t)n * Np + k];
  };
  if (r) std::copy(tb.r.begin(), tb.r.end(), r);
  if (s) std::copy(tb.s.begin(), tb.s.end(), s);
  if (t) std::copy(tb.t.begin(), tb.t.end(), t);
  if (D) {
    put(tb.Dr.data(), D);
    put(tb.Ds.data(), D + NP2);
    put(tb.Dt.data(), D + 2 * NP2);
  }
  if (MM) std::copy(tb.MM.begin(), tb.MM.end(), MM);
  if (S)
    for (int q = 0; q < 6; ++q) put(tb.S.data() + q * NP2, S + q * NP2);
  return BP_SUCCESS;
}

extern "C" int bp_basis_cubature(int32_t N, double* r, double* w, double* I, double* D, double* invV,
                                 double* Dmodal, double* MM) {
  if (N < 1 || N > 15) return bp::fail(BP_ERROR_ARG, "bp_basis_cubature: degree must be in 1..15");
  if (!r || !w || !I || !D || !invV || !Dmodal || !MM) return bp::fail(BP_ERROR_ARG, "bp_basis_cubature: null array");
  std::vector<double> z, zw;
  bp::gll_nodes_weights(N, z, zw);
  bp::CubBasis cb;
  bp::cubature_basis(N, z, cb);
  std::copy(cb.r.begin(), cb.r.end(), r);
  std::copy(cb.w.begin(), cb.w.end(), w);
  std::copy(cb.I.begin(), cb.I.end(), I);
  std::copy(cb.D.begin(), cb.D.end(), D);
  std::copy(cb.invV.begin(), cb.invV.end(), invV);
  std::copy(cb.Dmodal.begin(), cb.Dmodal.end(), Dmodal);
  std::copy(cb.MM.begin(), cb.MM.end(), MM);
  return BP_SUCCESS;
}

extern "C" int bp_box_vertices(const bp_box_desc_t* d, double* EX, double* EY, double* EZ) {
  bp::HostMesh m;
  int rc = host_mesh_from_desc(d, m);
  if (rc) return rc;
  if (m.dim == 2) bp::box_vertices_2d(m, d->pert, d->pert_seed);
  else bp::box_vertices(m, d->pert, d->pert_seed);
  if (EX) std::copy(m.EX.begin(), m.EX.end(), EX);
  if (EY) std::copy(m.EY.begin(), m.EY.end(), EY);
  if (EZ) std::copy(m.EZ.begin(), m.EZ.end(), EZ);
  return BP_SUCCESS;
}

// Host validation of an externally built masked numbering (rules in bp_b200.h).
extern "C" int bp_ogs_check(int64_t Nlocal, const int32_t* G2L, int32_t Ngather, const int32_t* rowStarts,
                            const int32_t* colIds) {
  using bp::fail;
  if (Nlocal < 0 || Ngather < 0) return fail(BP_ERROR_ARG, "bp_ogs_check: negative size");
  if (!rowStarts || (Nlocal > 0 && !G2L)) return fail(BP_ERROR_ARG, "bp_ogs_check: null array");
  int64_t unmasked = 0;
  for (int64_t l = 0; l < Nlocal; ++l) {
    const int32_t r = G2L[l];
    if (r < -1 || r >= Ngather)
      return fail(BP_ERROR_ARG, "bp_ogs_check: GlobalToLocal[" + std::to_string(l) + "] = " + std::to_string(r) +
                                    " is outside [-1, Ngather = " + std::to_string(Ngather) + ")");
    unmasked += r >= 0;
  }
  if (rowStarts[0] != 0) return fail(BP_ERROR_ARG, "bp_ogs_check: rowStarts[0] is not 0");
  for (int32_t r = 0; r < Ngather; ++r)
    if (rowStarts[r + 1] <= rowStarts[r])
      return fail(BP_ERROR_ARG, "bp_ogs_check: row " + std::to_string(r) + " is empty or rowStarts decrease there");
  if (rowStarts[Ngather] != unmasked)
    return fail(BP_ERROR_ARG, "bp_ogs_check: rowStarts[Ngather] = " + std::to_string(rowStarts[Ngather]) +
                                  " but GlobalToLocal has " + std::to_string(unmasked) + " unmasked entries");
  if (unmasked > 0 && !colIds) return fail(BP_ERROR_ARG, "bp_ogs_check: null colIds");
  for (int32_t r = 0; r < Ngather; ++r)
    for (int32_t c = rowStarts[r]; c < rowStarts[r + 1]; ++c) {
      const int32_t l = colIds[c];
      if (l < 0 || l >= Nlocal || G2L[l] != r)
        return fail(BP_ERROR_ARG, "bp_ogs_check: colIds[" + std::to_string(c) + "] = " + std::to_string(l) +
                                      " is not a local node of row " + std::to_string(r));
      if (c > rowStarts[r] && l <= colIds[c - 1])
        return fail(BP_ERROR_ARG, "bp_ogs_check: the columns of row " + std::to_string(r) + " do not ascend at colIds[" +
                                      std::to_string(c) + "]");
    }
  return BP_SUCCESS;
}
