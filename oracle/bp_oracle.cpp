/*
 * bp_oracle.cpp -- CPU restatement of the benchParanumal BK/BP Hex3D hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the pytest suite, the
 * smoke check in __graft_entry__.py and the CPU-baseline leg of bench.py load
 * it to produce reference answers and CPU timings.  The product library under
 * benchparanumal_b200/ never links, loads or calls it.
 *
 * Every routine restates one piece of the reference (paths are relative to the
 * reference project root):
 *   - seeded LCG               libs/primitives/random.cpp:29-170
 *   - 1D basis                 libs/mesh/meshBasis1D.cpp:61-338
 *   - hex reference nodes      libs/mesh/meshBasisHex3D.cpp:31-130,
 *                              libs/mesh/meshReferenceNodesHex3D.cpp:31-70
 *   - box mesh                 libs/mesh/meshSetupBoxHex3D.cpp:31-131
 *   - connectivity             libs/mesh/meshConnect.cpp:48-140,
 *                              libs/mesh/meshConnectFaceNodes.cpp:31-98,
 *                              libs/mesh/meshBasisHex3D.cpp:132-260
 *   - global node numbering    libs/mesh/meshConnectNodes.cpp:32-82
 *   - physical nodes           libs/mesh/meshPhysicalNodesHex3D.cpp:31-116
 *   - geometric factors        libs/mesh/meshGeometricFactorsHex3D.cpp:31-153
 *   - masked ogs numbering     libs/mesh/meshMaskedGatherScatterSetup.cpp:31-77,
 *                              libs/ogs/ogsSetup.cpp:87-290,492-579,833-849,
 *                              libs/ogs/ogsOperator.cpp:474-617
 *   - BP5 Ax (3D-shmem order)  okl/bp5AxHex3D.okl:415-569
 *   - BP5 Ax affine            okl/bp5AxAffineHex3D.okl:419-579
 *   - BP5 Ax pencil order      okl/bp5AxHex3D.okl:50-185 (p>8)
 *   - ogs gather / scatter     libs/ogs/ogsOperator.cpp:61-98,207-239
 *   - forcing                  okl/rhsHex3D.okl:29-128
 *   - CG                       libs/core/linearSolverCG.cpp:62-156,
 *                              libs/core/okl/linearSolverUpdateCG.okl:29-103,
 *                              libs/core/okl/linAlg{InnerProd,Norm2,AXPY}.okl,
 *                              libs/core/linAlg.cpp:38-89
 * Extensions that the reference does not have (seeded nodal forcing, vertex
 * perturbation, Jacobi diagonal, preconditioned CG) are restated here from
 * their mathematical definition so the product can be checked against them.
 * The BP1-BP4 over-integrated forms follow libs/mesh/meshCubatureSetupHex3D.cpp
 * and okl/bp{1,3}Ax{,Affine}Hex3D.okl.
 *
 * Quad2D (the reference's other tensor-product element, BP5/BP6 with Nfields
 * = dim): libs/mesh/meshSetupBoxQuad2D.cpp:30-100, meshBasisQuad2D.cpp:55-170,
 * meshPhysicalNodesQuad2D.cpp, meshGeometricFactorsQuad2D.cpp:31-120,
 * okl/bp5AxQuad2D.okl, okl/bp5AxAffineQuad2D.okl, okl/rhsQuad2D.okl.
 *
 * Parity pin: the reference ships no tests or golden vectors for this path and
 * its full build needs OCCA, MPI and LAPACK, none present; its host set-up
 * code, though, is compiled here against host-only shims (oracle/Makefile,
 * target ref) and its numbering, CSR, basis, geometric factors and host
 * gather/scatter are stored as fixtures (tests/golden/); tests/test_ref_golden.py
 * holds this restatement to them (integers bit-exact).  The element kernels
 * (OKL) need OCCA; their restatement here is pinned by known answers of the
 * mathematics (tests/test_oracle.py, tests/test_cub_host.py): quadrature and
 * differentiation exactness, affine/curved agreement, symmetry and positivity,
 * and spectral convergence of a manufactured solution.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef int32_t dlong;   // include/types.h: dlong = int
typedef int64_t hlong;   // include/types.h: hlong = long long int

/* ------------------------------------------------------------------------ */
/* seeded LCG, libs/primitives/random.cpp:29-170                              */
/* ------------------------------------------------------------------------ */
static const uint64_t kLcgA = 6364136223846793005ULL;
static const uint64_t kLcgC = 1ULL;

/* prim::seedRNG(seed); prim::random<double>(n, v).  The state starts at
   a*(~seed)+c and each value is state/UINT64_MAX taken before the step. */
extern "C" void bpo_random(uint64_t seed, int64_t n, double* v) {
  uint64_t x = kLcgA * (std::numeric_limits<uint64_t>::max() ^ seed) + kLcgC;
  const double scale = 1.0 / (double)std::numeric_limits<uint64_t>::max();
  for (int64_t i = 0; i < n; ++i) {
    v[i] = (double)x * scale;
    x = kLcgA * x + kLcgC;
  }
}

/* ------------------------------------------------------------------------ */
/* small dense linear algebra (stands in for LAPACK dgesv/dgetri/dgeev)       */
/* ------------------------------------------------------------------------ */
/* LU with partial pivoting; solves A X = B for X (A n x n, B n x m, row major) */
static int dense_solve(int n, std::vector<double> A, std::vector<double>& B, int m) {
  std::vector<int> piv(n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    double amax = std::fabs(A[k * n + k]);
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(A[i * n + k]) > amax) { amax = std::fabs(A[i * n + k]); p = i; }
    if (amax == 0.0) return -1;
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(A[k * n + j], A[p * n + j]);
      for (int j = 0; j < m; ++j) std::swap(B[k * m + j], B[p * m + j]);
    }
    for (int i = k + 1; i < n; ++i) {
      double l = A[i * n + k] / A[k * n + k];
      A[i * n + k] = l;
      for (int j = k + 1; j < n; ++j) A[i * n + j] -= l * A[k * n + j];
      for (int j = 0; j < m; ++j) B[i * m + j] -= l * B[k * m + j];
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    for (int j = 0; j < m; ++j) {
      double s = B[k * m + j];
      for (int i = k + 1; i < n; ++i) s -= A[k * n + i] * B[i * m + j];
      B[k * m + j] = s / A[k * n + k];
    }
  }
  return 0;
}

static int dense_inverse(int n, std::vector<double>& A) {
  std::vector<double> I(n * n, 0.0);
  for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
  int rc = dense_solve(n, A, I, n);
  A = I;
  return rc;
}

/* X = B / A, i.e. X A = B with B (nb x n), A (n x n): transpose to A^T X^T = B^T
   (linAlg_t::matrixRightSolve, libs/core/linAlgMatrixRightSolve.cpp). */
static int dense_right_solve(int nb, int n, const std::vector<double>& B,
                             const std::vector<double>& A, std::vector<double>& X) {
  std::vector<double> At(n * n), Bt(n * nb);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) At[i * n + j] = A[j * n + i];
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < n; ++j) Bt[j * nb + i] = B[i * n + j];
  int rc = dense_solve(n, At, Bt, nb);
  X.assign(nb * n, 0.0);
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < n; ++j) X[i * n + j] = Bt[j * nb + i];
  return rc;
}

/* Symmetric tridiagonal eigen-decomposition by the implicit QL method with
   Wilkinson shifts.  d: diagonal (n), e: sub-diagonal (n, e[n-1] unused).
   Z returns the eigenvectors as columns (row major n x n).  Replaces the
   dgeev call of JacobiGQ (libs/mesh/meshBasis1D.cpp:318). */
static int tridiag_ql(int n, std::vector<double>& d, std::vector<double>& e,
                      std::vector<double>& Z) {
  Z.assign(n * n, 0.0);
  for (int i = 0; i < n; ++i) Z[i * n + i] = 1.0;
  e[n - 1] = 0.0;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    int m;
    do {
      for (m = l; m < n - 1; ++m) {
        double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= std::numeric_limits<double>::epsilon() * dd) break;
      }
      if (m != l) {
        if (iter++ == 60) return -1;
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = std::hypot(g, 1.0);
        g = d[m] - d[l] + e[l] / (g + (g >= 0 ? std::fabs(r) : -std::fabs(r)));
        double s = 1.0, c = 1.0, p = 0.0;
        int i;
        for (i = m - 1; i >= l; --i) {
          double f = s * e[i], b = c * e[i];
          r = std::hypot(f, g);
          e[i + 1] = r;
          if (r == 0.0) { d[i + 1] -= p; e[m] = 0.0; break; }
          s = f / r; c = g / r;
          g = d[i + 1] - p;
          r = (d[i] - g) * s + 2.0 * c * b;
          p = s * r;
          d[i + 1] = g + p;
          g = c * r - b;
          for (int k = 0; k < n; ++k) {
            f = Z[k * n + i + 1];
            Z[k * n + i + 1] = s * Z[k * n + i] + c * f;
            Z[k * n + i] = c * Z[k * n + i] - s * f;
          }
        }
        if (r == 0.0 && i >= l) continue;
        d[l] -= p; e[l] = g; e[m] = 0.0;
      }
    } while (m != l);
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* 1D basis, libs/mesh/meshBasis1D.cpp                                        */
/* ------------------------------------------------------------------------ */
static double mygamma(double x) { return std::tgamma(x); }

/* JacobiP, meshBasis1D.cpp:180-214 (orthonormal Jacobi polynomial) */
static double jacobiP(double a, double alpha, double beta, int N) {
  const double gamma0 = std::pow(2.0, alpha + beta + 1) / (alpha + beta + 1) *
                        mygamma(1 + alpha) * mygamma(1 + beta) / mygamma(1 + alpha + beta);
  const double p0 = 1.0 / std::sqrt(gamma0);
  if (N == 0) return p0;
  const double gamma1 = (alpha + 1) * (beta + 1) / (alpha + beta + 3) * gamma0;
  const double p1 = ((alpha + beta + 2) * a / 2 + (alpha - beta) / 2) / std::sqrt(gamma1);
  if (N == 1) return p1;
  std::vector<double> P(N + 1);
  P[0] = p0; P[1] = p1;
  double aold = 2 / (2 + alpha + beta) * std::sqrt((alpha + 1.) * (beta + 1.) / (alpha + beta + 3.));
  for (int i = 1; i <= N - 1; ++i) {
    double h1 = 2. * i + alpha + beta;
    double anew = 2. / (h1 + 2.) * std::sqrt((i + 1.) * (i + 1. + alpha + beta) * (i + 1 + alpha) *
                                             (i + 1 + beta) / (h1 + 1) / (h1 + 3));
    double bnew = -(alpha * alpha - beta * beta) / h1 / (h1 + 2);
    P[i + 1] = 1. / anew * (-aold * P[i - 1] + (a - bnew) * P[i]);
    aold = anew;
  }
  return P[N];
}

/* GradJacobiP, meshBasis1D.cpp:216-224 */
static double gradJacobiP(double a, double alpha, double beta, int N) {
  if (N == 0) return 0.0;
  return std::sqrt(N * (N + alpha + beta + 1.)) * jacobiP(a, alpha + 1.0, beta + 1.0, N - 1);
}

/* JacobiGQ, meshBasis1D.cpp:266-338 (Golub-Welsch) */
extern "C" int bpo_jacobi_gq(double alpha, double beta, int N, double* x, double* w) {
  if (N == 0) {
    x[0] = (alpha - beta) / (alpha + beta + 2);
    w[0] = 2;
    return 0;
  }
  const int n = N + 1;
  std::vector<double> h1(n), d(n), e(n, 0.0);
  for (int i = 0; i < n; ++i) h1[i] = 2 * i + alpha + beta;
  for (int i = 0; i < n; ++i) {
    d[i] = -0.5 * (alpha * alpha - beta * beta) / ((h1[i] + 2) * h1[i]) * 2;
    if (i < N)
      e[i] = (2. / (h1[i] + 2.)) *
             std::sqrt((i + 1) * (i + 1 + alpha + beta) * (i + 1 + alpha) * (i + 1 + beta) /
                       ((h1[i] + 1) * (h1[i] + 3)));
  }
  if (alpha + beta < 10 * std::numeric_limits<double>::epsilon()) d[0] = 0;
  std::vector<double> Z;
  if (tridiag_ql(n, d, e, Z)) return -1;
  const double c = std::pow(2, alpha + beta + 1) / (alpha + beta + 1) * mygamma(alpha + 1) *
                   mygamma(beta + 1) / mygamma(alpha + beta + 1);
  for (int i = 0; i < n; ++i) { x[i] = d[i]; w[i] = Z[0 * n + i] * Z[0 * n + i] * c; }
  /* sort ascending (the reference's "sloppy sort") */
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j)
      if (x[i] > x[j]) { std::swap(x[i], x[j]); std::swap(w[i], w[j]); }
  return 0;
}

static void vandermonde1d(int N, const std::vector<double>& r, std::vector<double>& V) {
  const int n = N + 1, np = (int)r.size();
  V.assign(np * n, 0.0);
  for (int p = 0; p < np; ++p)
    for (int i = 0; i < n; ++i) V[p * n + i] = jacobiP(r[p], 0, 0, i);
}

static void grad_vandermonde1d(int N, const std::vector<double>& r, std::vector<double>& Vr) {
  const int n = N + 1, np = (int)r.size();
  Vr.assign(np * n, 0.0);
  for (int p = 0; p < np; ++p)
    for (int i = 0; i < n; ++i) Vr[p * n + i] = gradJacobiP(r[p], 0, 0, i);
}

/* MassMatrix1D, meshBasis1D.cpp:96-112: MM = inv(V V^T) */
static int mass_matrix1d(int n, const std::vector<double>& V, std::vector<double>& MM) {
  MM.assign(n * n, 0.0);
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      double s = 0;
      for (int i = 0; i < n; ++i) s += V[a * n + i] * V[b * n + i];
      MM[a * n + b] = s;
    }
  return dense_inverse(n, MM);
}

/* JacobiGLL with lumped weights, meshBasis1D.cpp:233-264 */
extern "C" int bpo_jacobi_gll(int N, double* x, double* w) {
  x[0] = -1.0;
  x[N] = 1.0;
  if (N > 1) {
    std::vector<double> xi(N - 1), wi(N - 1);
    if (bpo_jacobi_gq(1, 1, N - 2, xi.data(), wi.data())) return -1;
    for (int i = 0; i < N - 1; ++i) x[i + 1] = xi[i];
  }
  std::vector<double> r(x, x + N + 1), V, MM;
  vandermonde1d(N, r, V);
  if (mass_matrix1d(N + 1, V, MM)) return -1;
  for (int a = 0; a <= N; ++a) {
    double s = 0;
    for (int b = 0; b <= N; ++b) s += MM[a * (N + 1) + b];
    w[a] = s;
  }
  return 0;
}

/* Dmatrix1D, meshBasis1D.cpp:114-136: D = Vr / V, D[i*Nin + m] = l_m'(rout_i) */
extern "C" int bpo_dmatrix1d(int N, const double* rin, int nout, const double* rout, double* D) {
  std::vector<double> ri(rin, rin + N + 1), ro(rout, rout + nout), V, Vr, X;
  vandermonde1d(N, ri, V);
  grad_vandermonde1d(N, ro, Vr);
  if (dense_right_solve(nout, N + 1, Vr, V, X)) return -1;
  std::copy(X.begin(), X.end(), D);
  return 0;
}

/* InterpolationMatrix1D, meshBasis1D.cpp:138-160: I = Vout / Vin */
extern "C" int bpo_interp_matrix1d(int N, const double* rin, int nout, const double* rout,
                                   double* I) {
  std::vector<double> ri(rin, rin + N + 1), ro(rout, rout + nout), Vin, Vout, X;
  vandermonde1d(N, ri, Vin);
  vandermonde1d(N, ro, Vout);
  if (dense_right_solve(nout, N + 1, Vout, Vin, X)) return -1;
  std::copy(X.begin(), X.end(), I);
  return 0;
}

extern "C" int bpo_mass_matrix1d(int N, const double* r, double* MMout) {
  std::vector<double> rr(r, r + N + 1), V, MM;
  vandermonde1d(N, rr, V);
  if (mass_matrix1d(N + 1, V, MM)) return -1;
  std::copy(MM.begin(), MM.end(), MMout);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* mesh                                                                       */
/* ------------------------------------------------------------------------ */
struct bpo_mesh {
  int N, Nq, Np, Nfp, nx, ny, nz, E, affine, Nfields;
  int dim = 3, Nfaces = 6, Nverts = 8, Nggeo = 6;   // Quad2D: 2, 4, 4, 3
  std::vector<double> gllz, gllw, D, MM;
  std::vector<double> r, s, t;          // reference node coordinates (Np)
  std::vector<int> faceNodes;            // 6*Nfp
  std::vector<hlong> EToV;               // E*8
  std::vector<double> EX, EY, EZ;        // E*8
  std::vector<dlong> EToE;               // E*6
  std::vector<int> EToF;                 // E*6
  std::vector<dlong> vmapM, vmapP;       // E*6*Nfp
  std::vector<hlong> globalIds;          // E*Np
  std::vector<double> x, y, z;           // E*Np
  std::vector<double> wJ, ggeo;          // affine: E, 6E; else E*Np, 6*E*Np
  std::vector<hlong> maskedIds;          // E*Np*Nfields
  dlong Ngather, nnz;
  std::vector<dlong> rowStarts, colIds, G2L, blockRowStarts;
  std::vector<dlong> elementList;
  // cubature for BP1-BP4 (cubNq = N+2 Gauss points), set up on first use
  int cubNq = 0, cubNp = 0;
  std::vector<double> cubr, cubw, cubInterp;   // cubInterp [cubNq*Nq]
  std::vector<double> cubD;                    // curved: [cubNq^2]; affine: modal [Nq^2]
  std::vector<double> invV;                    // affine: inverse Legendre Vandermonde [Nq^2]
  std::vector<double> cubwJ, cubggeo;          // curved: [E*cubNp], [6*E*cubNp]; affine: wJ, ggeo
};

static const int kFaceVertices[6][4] = {{0, 1, 2, 3}, {0, 4, 5, 1}, {1, 5, 6, 2},
                                        {2, 6, 7, 3}, {0, 3, 7, 4}, {4, 7, 6, 5}};

/* NodesHex3D / FaceNodesHex3D, meshBasisHex3D.cpp:31-93 */
static void reference_nodes(bpo_mesh& m) {
  const int Nq = m.Nq;
  m.r.resize(m.Np); m.s.resize(m.Np); m.t.resize(m.Np);
  for (int k = 0; k < Nq; ++k)
    for (int j = 0; j < Nq; ++j)
      for (int i = 0; i < Nq; ++i) {
        int n = i + j * Nq + k * Nq * Nq;
        m.r[n] = m.gllz[i]; m.s[n] = m.gllz[j]; m.t[n] = m.gllz[k];
      }
  const double tol = 1000. * std::numeric_limits<double>::epsilon() * 0.5;
  m.faceNodes.assign(6 * m.Nfp, 0);
  int cnt[6] = {0, 0, 0, 0, 0, 0};
  for (int n = 0; n < m.Np; ++n) {
    if (std::fabs(m.t[n] + 1) < tol) m.faceNodes[0 * m.Nfp + cnt[0]++] = n;
    if (std::fabs(m.s[n] + 1) < tol) m.faceNodes[1 * m.Nfp + cnt[1]++] = n;
    if (std::fabs(m.r[n] - 1) < tol) m.faceNodes[2 * m.Nfp + cnt[2]++] = n;
    if (std::fabs(m.s[n] - 1) < tol) m.faceNodes[3 * m.Nfp + cnt[3]++] = n;
    if (std::fabs(m.r[n] + 1) < tol) m.faceNodes[4 * m.Nfp + cnt[4]++] = n;
    if (std::fabs(m.t[n] - 1) < tol) m.faceNodes[5 * m.Nfp + cnt[5]++] = n;
  }
}

static inline double trilinear(const double* v, double rn, double sn, double tn) {
  return +0.125 * (1 - rn) * (1 - sn) * (1 - tn) * v[0] + 0.125 * (1 + rn) * (1 - sn) * (1 - tn) * v[1] +
         0.125 * (1 + rn) * (1 + sn) * (1 - tn) * v[2] + 0.125 * (1 - rn) * (1 + sn) * (1 - tn) * v[3] +
         0.125 * (1 - rn) * (1 - sn) * (1 + tn) * v[4] + 0.125 * (1 + rn) * (1 - sn) * (1 + tn) * v[5] +
         0.125 * (1 + rn) * (1 + sn) * (1 + tn) * v[6] + 0.125 * (1 - rn) * (1 + sn) * (1 + tn) * v[7];
}

/* SetupBoxHex3D at one rank, meshSetupBoxHex3D.cpp:31-131, plus the seeded
   interior-vertex perturbation: every global vertex draws three uniforms in
   vertex-id order (x,y,z interleaved) and interior vertices move by
   pert*h*(2u-1) per coordinate, h the element width in that direction. */
static void setup_box(bpo_mesh& m, double pert, uint64_t seed) {
  const int nx = m.nx, ny = m.ny, nz = m.nz;
  const hlong NnX = nx + 1, NnY = ny + 1, NnZ = nz + 1;
  const double dx = 2.0 / nx, dy = 2.0 / ny, dz = 2.0 / nz;
  m.EToV.resize(m.E * 8); m.EX.resize(m.E * 8); m.EY.resize(m.E * 8); m.EZ.resize(m.E * 8);
  std::vector<double> u;
  if (pert != 0.0) {
    u.resize(3 * NnX * NnY * NnZ);
    bpo_random(seed, (int64_t)u.size(), u.data());
  }
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const dlong e = i + j * nx + k * nx * ny;
        const hlong i0 = i, i1 = (i + 1) % NnX, j0 = j, j1 = (j + 1) % NnY, k0 = k, k1 = (k + 1) % NnZ;
        hlong* v = &m.EToV[e * 8];
        v[0] = i0 + j0 * NnX + k0 * NnX * NnY; v[1] = i1 + j0 * NnX + k0 * NnX * NnY;
        v[2] = i1 + j1 * NnX + k0 * NnX * NnY; v[3] = i0 + j1 * NnX + k0 * NnX * NnY;
        v[4] = i0 + j0 * NnX + k1 * NnX * NnY; v[5] = i1 + j0 * NnX + k1 * NnX * NnY;
        v[6] = i1 + j1 * NnX + k1 * NnX * NnY; v[7] = i0 + j1 * NnX + k1 * NnX * NnY;
        const double x0 = -1.0 + dx * i, y0 = -1.0 + dy * j, z0 = -1.0 + dz * k;
        double* ex = &m.EX[e * 8]; double* ey = &m.EY[e * 8]; double* ez = &m.EZ[e * 8];
        ex[0] = x0;      ey[0] = y0;      ez[0] = z0;
        ex[1] = x0 + dx; ey[1] = y0;      ez[1] = z0;
        ex[2] = x0 + dx; ey[2] = y0 + dy; ez[2] = z0;
        ex[3] = x0;      ey[3] = y0 + dy; ez[3] = z0;
        ex[4] = x0;      ey[4] = y0;      ez[4] = z0 + dz;
        ex[5] = x0 + dx; ey[5] = y0;      ez[5] = z0 + dz;
        ex[6] = x0 + dx; ey[6] = y0 + dy; ez[6] = z0 + dz;
        ex[7] = x0;      ey[7] = y0 + dy; ez[7] = z0 + dz;
        if (pert != 0.0) {
          for (int c = 0; c < 8; ++c) {
            const hlong g = v[c];
            const hlong I = g % NnX, J = (g / NnX) % NnY, K = g / (NnX * NnY);
            if (I == 0 || I == nx || J == 0 || J == ny || K == 0 || K == nz) continue;
            ex[c] += pert * dx * (2 * u[3 * g + 0] - 1);
            ey[c] += pert * dy * (2 * u[3 * g + 1] - 1);
            ez[c] += pert * dz * (2 * u[3 * g + 2] - 1);
          }
        }
      }
}

/* Connect, meshConnect.cpp:48-140: match faces by their sorted vertex ids */
static void connect(bpo_mesh& m) {
  struct F { hlong v[4]; dlong e; int f; dlong eN; int fN; };
  std::vector<F> faces(m.E * 6);
  for (dlong e = 0; e < m.E; ++e)
    for (int f = 0; f < 6; ++f) {
      F& fc = faces[e * 6 + f];
      for (int n = 0; n < 4; ++n) fc.v[n] = m.EToV[e * 8 + kFaceVertices[f][n]];
      std::sort(fc.v, fc.v + 4);
      fc.e = e; fc.f = f; fc.eN = -1; fc.fN = -1;
    }
  std::sort(faces.begin(), faces.end(), [](const F& a, const F& b) {
    return std::lexicographical_compare(a.v, a.v + 4, b.v, b.v + 4);
  });
  for (size_t c = 0; c + 1 < faces.size(); ++c)
    if (std::equal(faces[c].v, faces[c].v + 4, faces[c + 1].v)) {
      faces[c].eN = faces[c + 1].e; faces[c].fN = faces[c + 1].f;
      faces[c + 1].eN = faces[c].e; faces[c + 1].fN = faces[c].f;
    }
  m.EToE.assign(m.E * 6, -1);
  m.EToF.assign(m.E * 6, -1);
  for (auto& fc : faces) { m.EToE[fc.e * 6 + fc.f] = fc.eN; m.EToF[fc.e * 6 + fc.f] = fc.fN; }
}

/* FaceNodeMatchingHex3D, meshBasisHex3D.cpp:132-260: for every (fM, fP, rot)
   find, for each node of face fM, the node of face fP at the same place when
   face fP is laid on top of fM with its vertex (rot) on fM's first vertex. */
static void face_node_matching(const bpo_mesh& m, std::vector<int>& R) {
  const int Nfp = m.Nfp;
  static const double V0[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
  static const double V1[4][2] = {{-1, -1}, {-1, 1}, {1, 1}, {1, -1}};
  R.assign(6 * 6 * 4 * Nfp, -1);
  std::vector<double> x0(Nfp), y0(Nfp), x1(Nfp), y1(Nfp);
  for (int fM = 0; fM < 6; ++fM) {
    double EX0[8] = {0}, EY0[8] = {0};
    for (int v = 0; v < 4; ++v) { EX0[kFaceVertices[fM][v]] = V0[v][0]; EY0[kFaceVertices[fM][v]] = V0[v][1]; }
    for (int n = 0; n < Nfp; ++n) {
      int fn = m.faceNodes[fM * Nfp + n];
      x0[n] = trilinear(EX0, m.r[fn], m.s[fn], m.t[fn]);
      y0[n] = trilinear(EY0, m.r[fn], m.s[fn], m.t[fn]);
    }
    for (int fP = 0; fP < 6; ++fP)
      for (int rot = 0; rot < 4; ++rot) {
        double EX1[8] = {0}, EY1[8] = {0};
        for (int v = 0; v < 4; ++v) {
          int fv = kFaceVertices[fP][(v + rot) % 4];
          EX1[fv] = V1[v][0]; EY1[fv] = V1[v][1];
        }
        for (int n = 0; n < Nfp; ++n) {
          int fn = m.faceNodes[fP * Nfp + n];
          x1[n] = trilinear(EX1, m.r[fn], m.s[fn], m.t[fn]);
          y1[n] = trilinear(EY1, m.r[fn], m.s[fn], m.t[fn]);
        }
        for (int n = 0; n < Nfp; ++n)
          for (int k = 0; k < Nfp; ++k) {
            double d = (x0[n] - x1[k]) * (x0[n] - x1[k]) + (y0[n] - y1[k]) * (y0[n] - y1[k]);
            if (d < 1.0e-5) { R[fM * 6 * Nfp * 4 + fP * Nfp * 4 + rot * Nfp + n] = k; break; }
          }
      }
  }
}

/* ConnectFaceNodes, meshConnectFaceNodes.cpp:31-98 */
static void connect_face_nodes(bpo_mesh& m) {
  std::vector<int> R;
  face_node_matching(m, R);
  const int Nfp = m.Nfp, Np = m.Np;
  m.vmapM.resize((size_t)m.E * 6 * Nfp);
  m.vmapP.resize((size_t)m.E * 6 * Nfp);
#pragma omp parallel for
  for (dlong eM = 0; eM < m.E; ++eM)
    for (int fM = 0; fM < 6; ++fM) {
      dlong eP = m.EToE[eM * 6 + fM];
      int fP = m.EToF[eM * 6 + fM];
      for (int nM = 0; nM < Nfp; ++nM) {
        const int idM = m.faceNodes[fM * Nfp + nM];
        const size_t id = (size_t)eM * 6 * Nfp + fM * Nfp + nM;
        m.vmapM[id] = idM + eM * Np;
        if (eP < 0 || fP < 0) { m.vmapP[id] = idM + eM * Np; continue; }
        hlong vf0P = m.EToV[eP * 8 + kFaceVertices[fP][0]];
        int rot = 0;
        for (; rot < 4; ++rot)
          if (m.EToV[eM * 8 + kFaceVertices[fM][rot]] == vf0P) break;
        const int nP = R[fM * 6 * Nfp * 4 + fP * Nfp * 4 + rot * Nfp + nM];
        m.vmapP[id] = m.faceNodes[fP * Nfp + nP] + eP * Np;
      }
    }
}

/* ConnectNodes, meshConnectNodes.cpp:32-82: globalId = 1 + smallest local
   index among the nodes connected through shared faces (min propagation to a
   fixed point). */
static void connect_nodes(bpo_mesh& m) {
  const size_t Ntot = (size_t)m.E * m.Np;
  m.globalIds.resize(Ntot);
  for (size_t i = 0; i < Ntot; ++i) m.globalIds[i] = 1 + (hlong)i;
  const size_t Ntr = m.vmapM.size();
  hlong change = 1;
  while (change > 0) {
    change = 0;
    for (size_t id = 0; id < Ntr; ++id) {
      hlong gM = m.globalIds[m.vmapM[id]], gP = m.globalIds[m.vmapP[id]];
      if (gP < gM) { ++change; m.globalIds[m.vmapM[id]] = gP; }
    }
  }
}

/* PhysicalNodesHex3D, meshPhysicalNodesHex3D.cpp:31-116 */
static void physical_nodes(bpo_mesh& m) {
  const size_t Ntot = (size_t)m.E * m.Np;
  m.x.resize(Ntot); m.y.resize(Ntot); m.z.resize(Ntot);
#pragma omp parallel for
  for (dlong e = 0; e < m.E; ++e)
    for (int n = 0; n < m.Np; ++n) {
      const size_t id = (size_t)e * m.Np + n;
      m.x[id] = trilinear(&m.EX[e * 8], m.r[n], m.s[n], m.t[n]);
      m.y[id] = trilinear(&m.EY[e * 8], m.r[n], m.s[n], m.t[n]);
      m.z[id] = trilinear(&m.EZ[e * 8], m.r[n], m.s[n], m.t[n]);
    }
}

/* GeometricFactorsHex3D, meshGeometricFactorsHex3D.cpp:31-153.
   ggeo order G00,G01,G02,G11,G12,G22.  Returns -1 on a non-positive Jacobian. */
static int geometric_factors(bpo_mesh& m) {
  int bad = 0;
  if (m.affine) {
    m.wJ.resize(m.E); m.ggeo.resize((size_t)6 * m.E);
    for (dlong e = 0; e < m.E; ++e) {
      const double* ex = &m.EX[e * 8]; const double* ey = &m.EY[e * 8]; const double* ez = &m.EZ[e * 8];
      double xr = 0.5 * (ex[1] - ex[0]), xs = 0.5 * (ex[3] - ex[0]), xt = 0.5 * (ex[4] - ex[0]);
      double yr = 0.5 * (ey[1] - ey[0]), ys = 0.5 * (ey[3] - ey[0]), yt = 0.5 * (ey[4] - ey[0]);
      double zr = 0.5 * (ez[1] - ez[0]), zs = 0.5 * (ez[3] - ez[0]), zt = 0.5 * (ez[4] - ez[0]);
      double J = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt);
      double rx = (ys * zt - zs * yt) / J, ry = -(xs * zt - zs * xt) / J, rz = (xs * yt - ys * xt) / J;
      double sx = -(yr * zt - zr * yt) / J, sy = (xr * zt - zr * xt) / J, sz = -(xr * yt - yr * xt) / J;
      double tx = (yr * zs - zr * ys) / J, ty = -(xr * zs - zr * xs) / J, tz = (xr * ys - yr * xs) / J;
      if (J < 0) bad = 1;
      m.wJ[e] = J;
      double* g = &m.ggeo[6 * (size_t)e];
      g[0] = J * (rx * rx + ry * ry + rz * rz); g[1] = J * (rx * sx + ry * sy + rz * sz);
      g[2] = J * (rx * tx + ry * ty + rz * tz); g[3] = J * (sx * sx + sy * sy + sz * sz);
      g[4] = J * (sx * tx + sy * ty + sz * tz); g[5] = J * (tx * tx + ty * ty + tz * tz);
    }
    return bad ? -1 : 0;
  }
  const int Nq = m.Nq, Np = m.Np;
  m.wJ.resize((size_t)m.E * Np); m.ggeo.resize((size_t)6 * m.E * Np);
#pragma omp parallel for reduction(| : bad)
  for (dlong e = 0; e < m.E; ++e)
    for (int k = 0; k < Nq; ++k)
      for (int j = 0; j < Nq; ++j)
        for (int i = 0; i < Nq; ++i) {
          const int n = i + j * Nq + k * Nq * Nq;
          double xr = 0, xs = 0, xt = 0, yr = 0, ys = 0, yt = 0, zr = 0, zs = 0, zt = 0;
          for (int mm = 0; mm < Nq; ++mm) {
            size_t idr = (size_t)e * Np + k * Nq * Nq + j * Nq + mm;
            size_t ids = (size_t)e * Np + k * Nq * Nq + mm * Nq + i;
            size_t idt = (size_t)e * Np + mm * Nq * Nq + j * Nq + i;
            xr += m.D[i * Nq + mm] * m.x[idr]; xs += m.D[j * Nq + mm] * m.x[ids]; xt += m.D[k * Nq + mm] * m.x[idt];
            yr += m.D[i * Nq + mm] * m.y[idr]; ys += m.D[j * Nq + mm] * m.y[ids]; yt += m.D[k * Nq + mm] * m.y[idt];
            zr += m.D[i * Nq + mm] * m.z[idr]; zs += m.D[j * Nq + mm] * m.z[ids]; zt += m.D[k * Nq + mm] * m.z[idt];
          }
          double J = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt);
          if (J < 1e-12) bad = 1;
          double rx = (ys * zt - zs * yt) / J, ry = -(xs * zt - zs * xt) / J, rz = (xs * yt - ys * xt) / J;
          double sx = -(yr * zt - zr * yt) / J, sy = (xr * zt - zr * xt) / J, sz = -(xr * yt - yr * xt) / J;
          double tx = (yr * zs - zr * ys) / J, ty = -(xr * zs - zr * xs) / J, tz = (xr * ys - yr * xs) / J;
          double JW = J * m.gllw[i] * m.gllw[j] * m.gllw[k];
          const size_t id = (size_t)e * Np + n;
          m.wJ[id] = JW;
          double* g = &m.ggeo[6 * id];
          g[0] = JW * (rx * rx + ry * ry + rz * rz); g[1] = JW * (rx * sx + ry * sy + rz * sz);
          g[2] = JW * (rx * tx + ry * ty + rz * tz); g[3] = JW * (sx * sx + sy * sy + sz * sz);
          g[4] = JW * (sx * tx + sy * ty + sz * tz); g[5] = JW * (tx * tx + ty * ty + tz * tz);
        }
  return bad ? -1 : 0;
}

/* blockRows, ogsOperator.cpp:474-546: bisect the rows into blocks holding at
   most 512 non-zeros */
static void block_rows(dlong Nrows, const std::vector<dlong>& rowStarts, std::vector<dlong>& blockStarts) {
  const dlong per = 512;
  blockStarts.clear();
  if (!Nrows) return;
  dlong maxNblocks = 1;
  while (maxNblocks < Nrows) maxNblocks *= 2;
  std::vector<dlong> oldS(maxNblocks + 1), newS(maxNblocks + 1), sizes(maxNblocks);
  dlong Nblocks = 1;
  oldS[0] = 0; oldS[1] = Nrows; newS[0] = 0;
  sizes[0] = rowStarts[Nrows];
  dlong maxSize = sizes[0];
  while (maxSize > per) {
    newS[2 * Nblocks] = Nrows;
    for (dlong n = 0; n < Nblocks; ++n) {
      const dlong start = oldS[n], end = oldS[n + 1];
      const dlong sz = rowStarts[end] - rowStarts[start];
      if (sz > per) {
        const dlong midSize = rowStarts[start] + (sz + 1) / 2;
        /* upperBound over rowStarts[start..end) */
        dlong first = start, count = end - start;
        while (count > 0) {
          dlong step = count / 2, mid = first + step;
          if (!(midSize < rowStarts[mid])) { first = mid + 1; count -= step + 1; } else count = step;
        }
        dlong mid = first;
        if (mid == end) --mid;
        newS[2 * n] = start; newS[2 * n + 1] = mid;
        sizes[2 * n] = rowStarts[mid] - rowStarts[start];
        sizes[2 * n + 1] = rowStarts[end] - rowStarts[mid];
      } else {
        newS[2 * n] = start; newS[2 * n + 1] = end;
        sizes[2 * n] = sz; sizes[2 * n + 1] = 0;
      }
    }
    std::swap(oldS, newS);
    Nblocks *= 2;
    maxSize = *std::max_element(sizes.begin(), sizes.begin() + Nblocks);
  }
  for (dlong n = 0; n <= Nblocks; ++n)
    if (blockStarts.empty() || blockStarts.back() != oldS[n]) blockStarts.push_back(oldS[n]);
}

/* MaskedGatherScatterSetup + ogs Setup (Signed, unique) + GlobalToLocal.
   meshMaskedGatherScatterSetup.cpp:31-77, ogsSetup.cpp:87-290, 492-579, 833-849,
   ogsOperator.cpp:549-617.  At one rank every group is local; the unique
   owner choice only affects the NoTrans gather, which the BPs do not use. */
static void masked_ogs(bpo_mesh& m) {
  const int Np = m.Np, Nf = m.Nfields, Nfp = m.Nfp;
  const size_t NL = (size_t)m.E * Np * Nf;
  m.maskedIds.resize(NL);
  for (dlong e = 0; e < m.E; ++e)
    for (int n = 0; n < Np; ++n)
      for (int f = 0; f < Nf; ++f)
        m.maskedIds[(size_t)e * Np * Nf + f * Np + n] = m.globalIds[(size_t)e * Np + n] * Nf + f;
  for (dlong e = 0; e < m.E; ++e)
    for (int f = 0; f < m.Nfaces; ++f)
      if (m.EToE[f + e * m.Nfaces] < 0)
        for (int n = 0; n < Nfp; ++n)
          for (int nf = 0; nf < Nf; ++nf)
            m.maskedIds[(size_t)e * Np * Nf + nf * Np + m.faceNodes[n + f * Nfp]] = 0;
  /* flag and compress out zero ids */
  std::vector<dlong> colIds;
  std::vector<hlong> baseIds;
  colIds.reserve(NL);
  for (size_t n = 0; n < NL; ++n)
    if (m.maskedIds[n] != 0) { colIds.push_back((dlong)n); baseIds.push_back(m.maskedIds[n]); }
  const dlong Nids = (dlong)colIds.size();
  /* EnumerateGatherGroups: stable sort by |baseId|, number groups in order of first appearance */
  std::vector<dlong> sortIds(Nids);
  std::iota(sortIds.begin(), sortIds.end(), 0);
  std::stable_sort(sortIds.begin(), sortIds.end(), [&](dlong a, dlong b) {
    return std::llabs(baseIds[a]) < std::llabs(baseIds[b]);
  });
  std::vector<dlong> gids(Nids, 0), groupStart;
  for (dlong i = 0; i < Nids; ++i)
    if (i == 0 || std::llabs(baseIds[sortIds[i]]) != std::llabs(baseIds[sortIds[i - 1]])) groupStart.push_back(i);
  const dlong Ngroups = (dlong)groupStart.size();
  groupStart.push_back(Nids);
  for (dlong g = 0; g < Ngroups; ++g) gids[sortIds[groupStart[g]]] = 1;  // every group owns a positive id
  std::vector<dlong> firsts;
  for (dlong n = 0; n < Nids; ++n) if (gids[n] == 1) firsts.push_back(n);
  for (dlong g = 0; g < Ngroups; ++g) gids[firsts[g]] = g;
  for (dlong g = 0; g < Ngroups; ++g) {
    const dlong gid = gids[sortIds[groupStart[g]]];
    for (dlong i = groupStart[g] + 1; i < groupStart[g + 1]; ++i) gids[sortIds[i]] = gid;
  }
  /* SortByRow: stable sort the (row, col) pairs by row */
  std::vector<dlong> order(Nids);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](dlong a, dlong b) { return gids[a] < gids[b]; });
  m.Ngather = Ngroups;
  m.nnz = Nids;
  m.rowStarts.assign(Ngroups + 1, 0);
  m.colIds.resize(Nids);
  for (dlong i = 0; i < Nids; ++i) {
    m.colIds[i] = colIds[order[i]];
    m.rowStarts[gids[order[i]] + 1]++;
  }
  for (dlong r = 0; r < Ngroups; ++r) m.rowStarts[r + 1] += m.rowStarts[r];
  block_rows(Ngroups, m.rowStarts, m.blockRowStarts);
  /* SetupGlobalToLocalMapping: NoTrans scatter of the row index */
  m.G2L.assign(NL, -1);
  for (dlong r = 0; r < Ngroups; ++r)
    for (dlong j = m.rowStarts[r]; j < m.rowStarts[r + 1]; ++j) m.G2L[m.colIds[j]] = r;
}

extern "C" bpo_mesh* bpo_mesh_create(int nx, int ny, int nz, int N, int affine, int Nfields,
                                     double pert, uint64_t pert_seed) {
  if (nx < 1 || ny < 1 || nz < 1 || N < 1 || N > 15 || (Nfields != 1 && Nfields != 3)) return nullptr;
  bpo_mesh* m = new bpo_mesh();
  m->N = N; m->Nq = N + 1; m->Np = m->Nq * m->Nq * m->Nq; m->Nfp = m->Nq * m->Nq;
  m->nx = nx; m->ny = ny; m->nz = nz; m->E = nx * ny * nz; m->affine = affine; m->Nfields = Nfields;
  m->gllz.resize(m->Nq); m->gllw.resize(m->Nq);
  if (bpo_jacobi_gll(N, m->gllz.data(), m->gllw.data())) { delete m; return nullptr; }
  m->D.resize(m->Nq * m->Nq);
  bpo_dmatrix1d(N, m->gllz.data(), m->Nq, m->gllz.data(), m->D.data());
  m->MM.resize(m->Nq * m->Nq);
  bpo_mass_matrix1d(N, m->gllz.data(), m->MM.data());
  reference_nodes(*m);
  setup_box(*m, pert, pert_seed);
  connect(*m);
  connect_face_nodes(*m);
  connect_nodes(*m);
  physical_nodes(*m);
  if (geometric_factors(*m)) { delete m; return nullptr; }
  masked_ogs(*m);
  m->elementList.resize(m->E);
  std::iota(m->elementList.begin(), m->elementList.end(), 0);
  return m;
}

/* ------------------------------------------------------------------------ */
/* Quad2D (2D tensor-product elements)                                        */
/* ------------------------------------------------------------------------ */
static const int kEdgeVertices[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};   // meshSetElementType.cpp:56

static inline double bilinear(const double* v, double rn, double sn) {
  return 0.25 * (1 - rn) * (1 - sn) * v[0] + 0.25 * (1 + rn) * (1 - sn) * v[1] + 0.25 * (1 + rn) * (1 + sn) * v[2] +
         0.25 * (1 - rn) * (1 + sn) * v[3];
}

/* NodesQuad2D / FaceNodesQuad2D, meshBasisQuad2D.cpp:31-86 */
static void reference_nodes_2d(bpo_mesh& m) {
  const int Nq = m.Nq;
  m.r.resize(m.Np); m.s.resize(m.Np); m.t.assign(m.Np, 0.0);
  for (int j = 0; j < Nq; ++j)
    for (int i = 0; i < Nq; ++i) {
      m.r[i + j * Nq] = m.gllz[i];
      m.s[i + j * Nq] = m.gllz[j];
    }
  const double tol = 1000. * std::numeric_limits<double>::epsilon() * 0.5;
  m.faceNodes.assign(4 * m.Nfp, 0);
  int cnt[4] = {0, 0, 0, 0};
  for (int n = 0; n < m.Np; ++n) {
    if (std::fabs(m.s[n] + 1) < tol) m.faceNodes[0 * m.Nfp + cnt[0]++] = n;
    if (std::fabs(m.r[n] - 1) < tol) m.faceNodes[1 * m.Nfp + cnt[1]++] = n;
    if (std::fabs(m.s[n] - 1) < tol) m.faceNodes[2 * m.Nfp + cnt[2]++] = n;
    if (std::fabs(m.r[n] + 1) < tol) m.faceNodes[3 * m.Nfp + cnt[3]++] = n;
  }
}

/* SetupBoxQuad2D at one rank, meshSetupBoxQuad2D.cpp:30-100, plus the seeded
   interior-vertex perturbation of the 3D box: every global vertex draws two
   uniforms in vertex-id order (x, y interleaved), interior vertices move by
   pert*h*(2u-1) per coordinate. */
static void setup_box_2d(bpo_mesh& m, double pert, uint64_t seed) {
  const int nx = m.nx, ny = m.ny;
  const hlong NnX = nx + 1, NnY = ny + 1;
  const double dx = 2.0 / nx, dy = 2.0 / ny;
  m.EToV.resize(m.E * 4); m.EX.resize(m.E * 4); m.EY.resize(m.E * 4); m.EZ.clear();
  std::vector<double> u;
  if (pert != 0.0) {
    u.resize(2 * NnX * NnY);
    bpo_random(seed, (int64_t)u.size(), u.data());
  }
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const dlong e = i + j * nx;
      const hlong i0 = i, i1 = (i + 1) % NnX, j0 = j, j1 = (j + 1) % NnY;
      hlong* v = &m.EToV[e * 4];
      v[0] = i0 + j0 * NnX; v[1] = i1 + j0 * NnX; v[2] = i1 + j1 * NnX; v[3] = i0 + j1 * NnX;
      const double x0 = -1.0 + dx * i, y0 = -1.0 + dy * j;
      double* ex = &m.EX[e * 4]; double* ey = &m.EY[e * 4];
      ex[0] = x0;      ey[0] = y0;
      ex[1] = x0 + dx; ey[1] = y0;
      ex[2] = x0 + dx; ey[2] = y0 + dy;
      ex[3] = x0;      ey[3] = y0 + dy;
      if (pert != 0.0)
        for (int c = 0; c < 4; ++c) {
          const hlong g = v[c];
          const hlong I = g % NnX, J = g / NnX;
          if (I == 0 || I == nx || J == 0 || J == ny) continue;
          ex[c] += pert * dx * (2 * u[2 * g + 0] - 1);
          ey[c] += pert * dy * (2 * u[2 * g + 1] - 1);
        }
    }
}

/* Connect, meshConnect.cpp:48-140, with the two-vertex faces of Quad2D */
static void connect_2d(bpo_mesh& m) {
  struct F { hlong v[2]; dlong e; int f; dlong eN; int fN; };
  std::vector<F> faces(m.E * 4);
  for (dlong e = 0; e < m.E; ++e)
    for (int f = 0; f < 4; ++f) {
      F& fc = faces[e * 4 + f];
      for (int n = 0; n < 2; ++n) fc.v[n] = m.EToV[e * 4 + kEdgeVertices[f][n]];
      std::sort(fc.v, fc.v + 2);
      fc.e = e; fc.f = f; fc.eN = -1; fc.fN = -1;
    }
  std::sort(faces.begin(), faces.end(), [](const F& a, const F& b) {
    return std::lexicographical_compare(a.v, a.v + 2, b.v, b.v + 2);
  });
  for (size_t c = 0; c + 1 < faces.size(); ++c)
    if (std::equal(faces[c].v, faces[c].v + 2, faces[c + 1].v)) {
      faces[c].eN = faces[c + 1].e; faces[c].fN = faces[c + 1].f;
      faces[c + 1].eN = faces[c].e; faces[c + 1].fN = faces[c].f;
    }
  m.EToE.assign(m.E * 4, -1);
  m.EToF.assign(m.E * 4, -1);
  for (auto& fc : faces) { m.EToE[fc.e * 4 + fc.f] = fc.eN; m.EToF[fc.e * 4 + fc.f] = fc.fN; }
}

/* FaceNodeMatchingQuad2D, meshBasisQuad2D.cpp:113-170: for (fM, fP, rot) the
   node of face fP at the place of each node of fM when fP is laid on fM */
static void face_node_matching_2d(const bpo_mesh& m, std::vector<int>& R) {
  const int Nfp = m.Nfp;
  static const double V[2] = {-1.0, 1.0};
  R.assign(4 * 4 * 2 * Nfp, -1);
  std::vector<double> x0(Nfp), x1(Nfp);
  for (int fM = 0; fM < 4; ++fM) {
    double EX0[4] = {0, 0, 0, 0};
    for (int v = 0; v < 2; ++v) EX0[kEdgeVertices[fM][v]] = V[v];
    for (int n = 0; n < Nfp; ++n) {
      const int fn = m.faceNodes[fM * Nfp + n];
      x0[n] = bilinear(EX0, m.r[fn], m.s[fn]);
    }
    for (int fP = 0; fP < 4; ++fP)
      for (int rot = 0; rot < 2; ++rot) {
        double EX1[4] = {0, 0, 0, 0};
        for (int v = 0; v < 2; ++v) EX1[kEdgeVertices[fP][(v + rot) % 2]] = V[v];
        for (int n = 0; n < Nfp; ++n) {
          const int fn = m.faceNodes[fP * Nfp + n];
          x1[n] = bilinear(EX1, m.r[fn], m.s[fn]);
        }
        for (int n = 0; n < Nfp; ++n)
          for (int k = 0; k < Nfp; ++k)
            if ((x0[n] - x1[k]) * (x0[n] - x1[k]) < 1.0e-5) {
              R[fM * 4 * Nfp * 2 + fP * Nfp * 2 + rot * Nfp + n] = k;
              break;
            }
      }
  }
}

/* ConnectFaceNodes, meshConnectFaceNodes.cpp:31-98, Quad2D faces */
static void connect_face_nodes_2d(bpo_mesh& m) {
  std::vector<int> R;
  face_node_matching_2d(m, R);
  const int Nfp = m.Nfp, Np = m.Np;
  m.vmapM.resize((size_t)m.E * 4 * Nfp);
  m.vmapP.resize((size_t)m.E * 4 * Nfp);
  for (dlong eM = 0; eM < m.E; ++eM)
    for (int fM = 0; fM < 4; ++fM) {
      const dlong eP = m.EToE[eM * 4 + fM];
      const int fP = m.EToF[eM * 4 + fM];
      for (int nM = 0; nM < Nfp; ++nM) {
        const int idM = m.faceNodes[fM * Nfp + nM];
        const size_t id = (size_t)eM * 4 * Nfp + fM * Nfp + nM;
        m.vmapM[id] = idM + eM * Np;
        if (eP < 0 || fP < 0) { m.vmapP[id] = idM + eM * Np; continue; }
        const hlong vf0P = m.EToV[eP * 4 + kEdgeVertices[fP][0]];
        int rot = 0;
        for (; rot < 2; ++rot)
          if (m.EToV[eM * 4 + kEdgeVertices[fM][rot]] == vf0P) break;
        const int nP = R[fM * 4 * Nfp * 2 + fP * Nfp * 2 + rot * Nfp + nM];
        m.vmapP[id] = m.faceNodes[fP * Nfp + nP] + eP * Np;
      }
    }
}

/* PhysicalNodesQuad2D, meshPhysicalNodesQuad2D.cpp */
static void physical_nodes_2d(bpo_mesh& m) {
  const size_t Ntot = (size_t)m.E * m.Np;
  m.x.resize(Ntot); m.y.resize(Ntot); m.z.clear();
  for (dlong e = 0; e < m.E; ++e)
    for (int n = 0; n < m.Np; ++n) {
      m.x[(size_t)e * m.Np + n] = bilinear(&m.EX[e * 4], m.r[n], m.s[n]);
      m.y[(size_t)e * m.Np + n] = bilinear(&m.EY[e * 4], m.r[n], m.s[n]);
    }
}

/* GeometricFactorsQuad2D, meshGeometricFactorsQuad2D.cpp:31-120: ggeo
   G00, G01, G11 (3 per node, GLL weights folded in; affine: per element) */
static int geometric_factors_2d(bpo_mesh& m) {
  int bad = 0;
  if (m.affine) {
    m.wJ.resize(m.E); m.ggeo.resize((size_t)3 * m.E);
    for (dlong e = 0; e < m.E; ++e) {
      const double* ex = &m.EX[e * 4]; const double* ey = &m.EY[e * 4];
      const double xr = 0.5 * (ex[1] - ex[0]), xs = 0.5 * (ex[3] - ex[0]);
      const double yr = 0.5 * (ey[1] - ey[0]), ys = 0.5 * (ey[3] - ey[0]);
      const double J = xr * ys - xs * yr;
      if (J < 1e-8) bad = 1;
      const double rx = ys / J, ry = -xs / J, sx = -yr / J, sy = xr / J;
      m.wJ[e] = J;
      m.ggeo[3 * e + 0] = J * (rx * rx + ry * ry);
      m.ggeo[3 * e + 1] = J * (rx * sx + ry * sy);
      m.ggeo[3 * e + 2] = J * (sx * sx + sy * sy);
    }
    return bad ? -1 : 0;
  }
  const int Nq = m.Nq, Np = m.Np;
  m.wJ.resize((size_t)m.E * Np); m.ggeo.resize((size_t)3 * m.E * Np);
  for (dlong e = 0; e < m.E; ++e)
    for (int j = 0; j < Nq; ++j)
      for (int i = 0; i < Nq; ++i) {
        double xr = 0, xs = 0, yr = 0, ys = 0;
        for (int mm = 0; mm < Nq; ++mm) {
          const size_t idr = (size_t)e * Np + j * Nq + mm, ids = (size_t)e * Np + mm * Nq + i;
          xr += m.D[i * Nq + mm] * m.x[idr];
          xs += m.D[j * Nq + mm] * m.x[ids];
          yr += m.D[i * Nq + mm] * m.y[idr];
          ys += m.D[j * Nq + mm] * m.y[ids];
        }
        const double J = xr * ys - xs * yr;
        if (J < 1e-8) bad = 1;
        const double rx = ys / J, ry = -xs / J, sx = -yr / J, sy = xr / J;
        const double JW = J * m.gllw[i] * m.gllw[j];
        const size_t id = (size_t)e * Np + i + j * Nq;
        m.wJ[id] = JW;
        m.ggeo[3 * id + 0] = JW * (rx * rx + ry * ry);
        m.ggeo[3 * id + 1] = JW * (rx * sx + ry * sy);
        m.ggeo[3 * id + 2] = JW * (sx * sx + sy * sy);
      }
  return bad ? -1 : 0;
}

/* A Quad2D box of nx x ny elements (Nfields 1 or 2: BP5, BP6 with Nfields =
   dim) with the reference's set-up sequence */
extern "C" bpo_mesh* bpo_mesh_create2d(int nx, int ny, int N, int affine, int Nfields, double pert,
                                       uint64_t pert_seed) {
  if (nx < 1 || ny < 1 || N < 1 || N > 15 || (Nfields != 1 && Nfields != 2)) return nullptr;
  bpo_mesh* m = new bpo_mesh();
  m->dim = 2; m->Nfaces = 4; m->Nverts = 4; m->Nggeo = 3;
  m->N = N; m->Nq = N + 1; m->Np = m->Nq * m->Nq; m->Nfp = m->Nq;
  m->nx = nx; m->ny = ny; m->nz = 1; m->E = nx * ny; m->affine = affine; m->Nfields = Nfields;
  m->gllz.resize(m->Nq); m->gllw.resize(m->Nq);
  if (bpo_jacobi_gll(N, m->gllz.data(), m->gllw.data())) { delete m; return nullptr; }
  m->D.resize(m->Nq * m->Nq);
  bpo_dmatrix1d(N, m->gllz.data(), m->Nq, m->gllz.data(), m->D.data());
  m->MM.resize(m->Nq * m->Nq);
  bpo_mass_matrix1d(N, m->gllz.data(), m->MM.data());
  reference_nodes_2d(*m);
  setup_box_2d(*m, pert, pert_seed);
  connect_2d(*m);
  connect_face_nodes_2d(*m);
  connect_nodes(*m);
  physical_nodes_2d(*m);
  if (geometric_factors_2d(*m)) { delete m; return nullptr; }
  masked_ogs(*m);
  m->elementList.resize(m->E);
  std::iota(m->elementList.begin(), m->elementList.end(), 0);
  return m;
}

/* bp5AxQuad2D / bp5AxAffineQuad2D (okl/bp5AxQuad2D.okl, okl/bp5AxAffineQuad2D.okl)
   and the field loop of okl/bp6AxQuad2D.okl, in their arithmetic order */
static void ax_bp5_e_2d(const bpo_mesh& m, dlong e, const dlong* G2L, double lambda, const double* q, double* AqL,
                        int f) {
  const int Nq = m.Nq, Np = m.Np, Nf = m.Nfields;
  const double* D = m.D.data();
  thread_local std::vector<double> sq, Gqr, Gqs;
  sq.resize(Np); Gqr.resize(Np); Gqs.resize(Np);
  const size_t lbase = (size_t)e * Np * Nf + (size_t)f * Np;
  for (int n = 0; n < Np; ++n) {
    const dlong id = G2L[lbase + n];
    sq[n] = (id != -1) ? q[id] : 0.0;
  }
  for (int j = 0; j < Nq; ++j)
    for (int i = 0; i < Nq; ++i) {
      double G00, G01, G11;
      if (m.affine) {
        G00 = m.ggeo[3 * (size_t)e + 0]; G01 = m.ggeo[3 * (size_t)e + 1]; G11 = m.ggeo[3 * (size_t)e + 2];
      } else {
        const size_t gb = (size_t)e * Np + i + j * Nq;
        G00 = m.ggeo[3 * gb + 0]; G01 = m.ggeo[3 * gb + 1]; G11 = m.ggeo[3 * gb + 2];
      }
      double tmp = 0;
      for (int mm = 0; mm < Nq; ++mm) tmp += D[i * Nq + mm] * sq[j * Nq + mm];
      double gr = G00 * tmp, gs = G01 * tmp;
      tmp = 0;
      for (int mm = 0; mm < Nq; ++mm) tmp += D[j * Nq + mm] * sq[mm * Nq + i];
      gr += G01 * tmp;
      gs += G11 * tmp;
      if (m.affine) {
        const double w = m.gllw[i] * m.gllw[j];
        gr *= w;
        gs *= w;
      }
      Gqr[j * Nq + i] = gr;
      Gqs[j * Nq + i] = gs;
    }
  for (int j = 0; j < Nq; ++j)
    for (int i = 0; i < Nq; ++i) {
      double ap;
      if (m.affine) ap = sq[j * Nq + i] * lambda * m.wJ[e] * (m.gllw[i] * m.gllw[j]);
      else ap = sq[j * Nq + i] * lambda * m.wJ[(size_t)e * Np + i + j * Nq];
      for (int mm = 0; mm < Nq; ++mm) {
        ap += D[mm * Nq + i] * Gqr[j * Nq + mm];
        ap += D[mm * Nq + j] * Gqs[mm * Nq + i];
      }
      AqL[lbase + i + j * Nq] = ap;
    }
}

extern "C" void bpo_mesh_free(bpo_mesh* m) { delete m; }

extern "C" int64_t bpo_mesh_int(const bpo_mesh* m, const char* name) {
  std::string s(name);
  if (s == "N") return m->N;
  if (s == "dim") return m->dim;
  if (s == "Nq") return m->Nq;
  if (s == "Np") return m->Np;
  if (s == "E") return m->E;
  if (s == "Nfields") return m->Nfields;
  if (s == "affine") return m->affine;
  if (s == "Ngather") return m->Ngather;
  if (s == "nnz") return m->nnz;
  if (s == "NblockRows") return (int64_t)m->blockRowStarts.size() - 1;
  return -1;
}

static void ensure_cubature(bpo_mesh& m);

/* Returns a pointer to a named array and its length (elements).  Asking for a
   cubature array sets the cubature up. */
extern "C" const void* bpo_mesh_array(const bpo_mesh* m, const char* name, int64_t* len) {
  std::string s(name);
  if (s.rfind("cub", 0) == 0 || s == "invV") ensure_cubature(*const_cast<bpo_mesh*>(m));
#define RET(vec) do { *len = (int64_t)(vec).size(); return (const void*)(vec).data(); } while (0)
  if (s == "gllz") RET(m->gllz);
  if (s == "gllw") RET(m->gllw);
  if (s == "D") RET(m->D);
  if (s == "MM") RET(m->MM);
  if (s == "EToV") RET(m->EToV);
  if (s == "EX") RET(m->EX);
  if (s == "EY") RET(m->EY);
  if (s == "EZ") RET(m->EZ);
  if (s == "EToE") RET(m->EToE);
  if (s == "globalIds") RET(m->globalIds);
  if (s == "x") RET(m->x);
  if (s == "y") RET(m->y);
  if (s == "z") RET(m->z);
  if (s == "wJ") RET(m->wJ);
  if (s == "ggeo") RET(m->ggeo);
  if (s == "maskedIds") RET(m->maskedIds);
  if (s == "rowStarts") RET(m->rowStarts);
  if (s == "colIds") RET(m->colIds);
  if (s == "G2L") RET(m->G2L);
  if (s == "blockRowStarts") RET(m->blockRowStarts);
  if (s == "elementList") RET(m->elementList);
  if (s == "cubr") RET(m->cubr);
  if (s == "cubw") RET(m->cubw);
  if (s == "cubInterp") RET(m->cubInterp);
  if (s == "cubD") RET(m->cubD);
  if (s == "invV") RET(m->invV);
  if (s == "cubwJ") RET(m->cubwJ);
  if (s == "cubggeo") RET(m->cubggeo);
#undef RET
  *len = -1;   // unknown name
  return nullptr;
}

/* ------------------------------------------------------------------------ */
/* operators                                                                  */
/* ------------------------------------------------------------------------ */

/* bp5AxHex3D, 3D-shared-memory variant (okl/bp5AxHex3D.okl:415-569), in its
   arithmetic order.  Used for p<=8 (the reference's own switch, :27-31). */
static void ax_bp5_e_3d(const bpo_mesh& m, dlong e, const dlong* G2L, double lambda,
                        const double* q, double* AqL, int f) {
  const int Nq = m.Nq, Np = m.Np, Nf = m.Nfields;
  const double* D = m.D.data();
  thread_local std::vector<double> sq, Gqr, Gqs, Gqt, wJl;
  sq.resize(Np); Gqr.resize(Np); Gqs.resize(Np); Gqt.resize(Np); wJl.resize(Np);
  const size_t lbase = (size_t)e * Np * Nf + (size_t)f * Np;
  for (int n = 0; n < Np; ++n) {
    dlong id = G2L[lbase + n];
    sq[n] = (id != -1) ? q[id] : 0.0;
  }
  for (int k = 0; k < Nq; ++k)
    for (int j = 0; j < Nq; ++j)
      for (int i = 0; i < Nq; ++i) {
        const int n = i + j * Nq + k * Nq * Nq;
        double G00, G01, G02, G11, G12, G22, wJ;
        if (m.affine) {
          const double* g = &m.ggeo[6 * (size_t)e];
          G00 = g[0]; G01 = g[1]; G02 = g[2]; G11 = g[3]; G12 = g[4]; G22 = g[5]; wJ = m.wJ[e];
        } else {
          const size_t gb = (size_t)e * Np + n;
          const double* g = &m.ggeo[6 * gb];
          G00 = g[0]; G01 = g[1]; G02 = g[2]; G11 = g[3]; G12 = g[4]; G22 = g[5]; wJ = m.wJ[gb];
        }
        double tmp = 0.0;
        for (int mm = 0; mm < Nq; ++mm) tmp += D[k * Nq + mm] * sq[mm * Nq * Nq + j * Nq + i];
        double gr = G02 * tmp, gs = G12 * tmp, gt = G22 * tmp;
        tmp = 0;
        for (int mm = 0; mm < Nq; ++mm) tmp += D[i * Nq + mm] * sq[k * Nq * Nq + j * Nq + mm];
        gr += G00 * tmp; gs += G01 * tmp; gt += G02 * tmp;
        tmp = 0;
        for (int mm = 0; mm < Nq; ++mm) tmp += D[j * Nq + mm] * sq[k * Nq * Nq + mm * Nq + i];
        gr += G01 * tmp; gs += G11 * tmp; gt += G12 * tmp;
        if (m.affine) {
          const double w = m.gllw[i] * m.gllw[j] * m.gllw[k];
          gr *= w; gs *= w; gt *= w; wJ *= w;
        }
        Gqr[n] = gr; Gqs[n] = gs; Gqt[n] = gt; wJl[n] = wJ;
      }
  for (int k = 0; k < Nq; ++k)
    for (int j = 0; j < Nq; ++j)
      for (int i = 0; i < Nq; ++i) {
        const int n = i + j * Nq + k * Nq * Nq;
        double ap = sq[n] * lambda * wJl[n];
        for (int mm = 0; mm < Nq; ++mm) {
          ap += D[mm * Nq + i] * Gqr[k * Nq * Nq + j * Nq + mm];
          ap += D[mm * Nq + j] * Gqs[k * Nq * Nq + mm * Nq + i];
        }
        for (int mm = 0; mm < Nq; ++mm) ap += D[mm * Nq + k] * Gqt[mm * Nq * Nq + j * Nq + i];
        AqL[lbase + n] = ap;
      }
}

/* bp5AxHex3D, register-pencil variant (okl/bp5AxHex3D.okl:50-185), in its
   arithmetic order.  Used for p>8, as the reference's CUDA build does. */
static void ax_bp5_e_pencil(const bpo_mesh& m, dlong e, const dlong* G2L, double lambda,
                            const double* q, double* AqL, int f) {
  const int Nq = m.Nq, Np = m.Np, Nf = m.Nfields;
  const double* D = m.D.data();
  const size_t lbase = (size_t)e * Np * Nf + (size_t)f * Np;
  thread_local std::vector<double> ru, rAu, sq, sv, sw, GDut, Auk;
  ru.resize(Np); rAu.assign(Np, 0.0); sq.resize(Nq * Nq); sv.resize(Nq * Nq); sw.resize(Nq * Nq);
  GDut.resize(Nq * Nq); Auk.resize(Nq * Nq);
  for (int n = 0; n < Np; ++n) {
    dlong id = G2L[lbase + n];
    ru[n] = (id != -1) ? q[id] : 0.0;
  }
  for (int k = 0; k < Nq; ++k) {
    for (int n = 0; n < Nq * Nq; ++n) sq[n] = ru[k * Nq * Nq + n];
    for (int j = 0; j < Nq; ++j)
      for (int i = 0; i < Nq; ++i) {
        const int n = i + j * Nq + k * Nq * Nq;
        double G00, G01, G02, G11, G12, G22, wJ;
        if (m.affine) {
          const double* g = &m.ggeo[6 * (size_t)e];
          const double w = m.gllw[i] * m.gllw[j] * m.gllw[k];
          G00 = g[0] * w; G01 = g[1] * w; G02 = g[2] * w; G11 = g[3] * w; G12 = g[4] * w; G22 = g[5] * w;
          wJ = m.wJ[e] * w;
        } else {
          const size_t gb = (size_t)e * Np + n;
          const double* g = &m.ggeo[6 * gb];
          G00 = g[0]; G01 = g[1]; G02 = g[2]; G11 = g[3]; G12 = g[4]; G22 = g[5]; wJ = m.wJ[gb];
        }
        double ur = 0, us = 0, ut = 0;
        for (int mm = 0; mm < Nq; ++mm) ut += D[k * Nq + mm] * ru[mm * Nq * Nq + j * Nq + i];
        for (int mm = 0; mm < Nq; ++mm) {
          ur += D[i * Nq + mm] * sq[j * Nq + mm];
          us += D[j * Nq + mm] * sq[mm * Nq + i];
        }
        sw[j * Nq + i] = G01 * ur + G11 * us + G12 * ut;
        sv[j * Nq + i] = G00 * ur + G01 * us + G02 * ut;
        GDut[j * Nq + i] = G02 * ur + G12 * us + G22 * ut;
        Auk[j * Nq + i] = wJ * lambda * ru[n];
      }
    for (int j = 0; j < Nq; ++j)
      for (int i = 0; i < Nq; ++i) {
        for (int mm = 0; mm < Nq; ++mm) rAu[mm * Nq * Nq + j * Nq + i] += D[k * Nq + mm] * GDut[j * Nq + i];
        double a = Auk[j * Nq + i];
        for (int mm = 0; mm < Nq; ++mm) {
          a += D[mm * Nq + j] * sw[mm * Nq + i];
          a += D[mm * Nq + i] * sv[j * Nq + mm];
        }
        rAu[k * Nq * Nq + j * Nq + i] += a;
      }
  }
  for (int n = 0; n < Np; ++n) AqL[lbase + n] = rAu[n];
}

/* Element-local BP5 (BP6 when Nfields==3) operator: AqL = A_e q[G2L] */
extern "C" void bpo_ax_bp5(const bpo_mesh* m, double lambda, const double* q, double* AqL) {
  const bool pencil = m->N > 8;
#pragma omp parallel for schedule(static)
  for (dlong e = 0; e < m->E; ++e)
    for (int f = 0; f < m->Nfields; ++f) {
      if (m->dim == 2) ax_bp5_e_2d(*m, e, m->G2L.data(), lambda, q, AqL, f);
      else if (pencil) ax_bp5_e_pencil(*m, e, m->G2L.data(), lambda, q, AqL, f);
      else ax_bp5_e_3d(*m, e, m->G2L.data(), lambda, q, AqL, f);
    }
}

/* ogs Gather(Add, Trans), ogsOperator.cpp:61-98: gv[r] = 0 + sum of v over the row, in column order */
extern "C" void bpo_gather(const bpo_mesh* m, const double* v, double* gv) {
#pragma omp parallel for
  for (dlong r = 0; r < m->Ngather; ++r) {
    double s = 0.0;
    for (dlong j = m->rowStarts[r]; j < m->rowStarts[r + 1]; ++j) s += v[m->colIds[j]];
    gv[r] = s;
  }
}

/* ogs Scatter(NoTrans), ogsOperator.cpp:207-239: every local copy gets its row's value; masked entries untouched */
extern "C" void bpo_scatter(const bpo_mesh* m, const double* gv, double* v) {
#pragma omp parallel for
  for (dlong r = 0; r < m->Ngather; ++r)
    for (dlong j = m->rowStarts[r]; j < m->rowStarts[r + 1]; ++j) v[m->colIds[j]] = gv[r];
}

/* bp5_t::Operator (BP/BP5/src/bp5Operator.cpp:29-85) at one rank: Ax over all elements, then Trans gather */
extern "C" void bpo_operator_bp5(const bpo_mesh* m, double lambda, const double* q, double* Aq) {
  std::vector<double> AqL((size_t)m->E * m->Np * m->Nfields);
  bpo_ax_bp5(m, lambda, q, AqL.data());
  bpo_gather(m, AqL.data(), Aq);
}

static const double kPi = 3.14159265358979323846;

/* rhsHex3D / rhsAffineHex3D (okl/rhsHex3D.okl:29-128), element-local forcing */
extern "C" void bpo_rhs_analytic(const bpo_mesh* m, double lambda, double* rL) {
  const int Nq = m->Nq, Np = m->Np, Nf = m->Nfields;
  if (m->dim == 2) {   // rhsQuad2D / rhsAffineQuad2D, okl/rhsQuad2D.okl
    for (dlong e = 0; e < m->E; ++e)
      for (int j = 0; j < Nq; ++j)
        for (int i = 0; i < Nq; ++i) {
          const int n = i + j * Nq;
          const size_t id = (size_t)e * Np + n;
          const double x = m->x[id], y = m->y[id];
          const double wJ = m->affine ? m->wJ[e] * m->gllw[i] * m->gllw[j] : m->wJ[id];
          if (Nf == 1) {
            rL[id] = wJ * ((2 * kPi * kPi + lambda) * std::sin(kPi * x) * std::sin(kPi * y));
          } else {
            const size_t base = (size_t)e * Np * Nf + n;
            rL[base + 0 * Np] = wJ * ((3 * kPi * kPi + lambda) * std::sin(2.0 * kPi * x) * std::sin(kPi * y));
            rL[base + 1 * Np] = wJ * ((3 * kPi * kPi + lambda) * std::sin(kPi * x) * std::sin(2.0 * kPi * y));
          }
        }
    return;
  }
#pragma omp parallel for
  for (dlong e = 0; e < m->E; ++e)
    for (int k = 0; k < Nq; ++k)
      for (int j = 0; j < Nq; ++j)
        for (int i = 0; i < Nq; ++i) {
          const int n = i + j * Nq + k * Nq * Nq;
          const size_t id = (size_t)e * Np + n;
          const double x = m->x[id], y = m->y[id], z = m->z[id];
          const double wJ = m->affine ? m->wJ[e] * m->gllw[i] * m->gllw[j] * m->gllw[k] : m->wJ[id];
          if (Nf == 1) {
            double f = (3 * kPi * kPi + lambda) * std::sin(kPi * x) * std::sin(kPi * y) * std::sin(kPi * z);
            rL[id] = wJ * f;
          } else {
            double f = (4 * kPi * kPi + lambda) * std::sin(2.0 * kPi * x) * std::sin(kPi * y) * std::sin(kPi * z);
            double g = (4 * kPi * kPi + lambda) * std::sin(kPi * x) * std::sin(2.0 * kPi * y) * std::sin(kPi * z);
            double h = (4 * kPi * kPi + lambda) * std::sin(kPi * x) * std::sin(kPi * y) * std::sin(2.0 * kPi * z);
            const size_t base = (size_t)e * Np * Nf + n;
            rL[base + 0 * Np] = wJ * f; rL[base + 1 * Np] = wJ * g; rL[base + 2 * Np] = wJ * h;
          }
        }
}

/* Seeded nodal forcing (extension): f[r] = 2u_r - 1 for the Ngather rows in
   row order (one LCG stream, seed), then b = M f with the lumped mass M:
   rL = wJ * f[G2L] on every local copy, and b = Trans-gather(rL). */
extern "C" void bpo_rhs_random(const bpo_mesh* m, uint64_t seed, double* f, double* b) {
  const int Nq = m->Nq, Np = m->Np, Nf = m->Nfields;
  bpo_random(seed, m->Ngather, f);
  for (dlong r = 0; r < m->Ngather; ++r) f[r] = 2 * f[r] - 1;
  std::vector<double> rL((size_t)m->E * Np * Nf);
#pragma omp parallel for
  for (dlong e = 0; e < m->E; ++e)
    for (int fl = 0; fl < Nf; ++fl)
      for (int n = 0; n < Np; ++n) {
        const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
        const double w = m->dim == 2 ? m->gllw[i] * m->gllw[j] : m->gllw[i] * m->gllw[j] * m->gllw[k];
        const double wJ = m->affine ? m->wJ[e] * w : m->wJ[(size_t)e * Np + n];
        const size_t l = (size_t)e * Np * Nf + (size_t)fl * Np + n;
        const dlong id = m->G2L[l];
        rL[l] = (id != -1) ? wJ * f[id] : 0.0;
      }
  bpo_gather(m, rL.data(), b);
}

/* Assembled diagonal of the BP5 operator (extension for Jacobi CG):
   diag(A_e)[n] = sum_m Gqq-weighted D^2 terms + 2 cross terms + lambda wJ,
   then Trans-gathered. */
extern "C" void bpo_jacobi_diag_bp5(const bpo_mesh* m, double lambda, double* diag) {
  const int Nq = m->Nq, Np = m->Np, Nf = m->Nfields;
  const double* D = m->D.data();
  std::vector<double> dL((size_t)m->E * Np * Nf);
  if (m->dim == 2) {
    for (dlong e = 0; e < m->E; ++e)
      for (int j = 0; j < Nq; ++j)
        for (int i = 0; i < Nq; ++i) {
          auto G = [&](int ii, int jj, int c) -> double {
            if (m->affine) return m->ggeo[3 * (size_t)e + c] * m->gllw[ii] * m->gllw[jj];
            return m->ggeo[3 * ((size_t)e * Np + ii + jj * Nq) + c];
          };
          const int n = i + j * Nq;
          double d = 0.0;
          for (int mm = 0; mm < Nq; ++mm) {
            d += G(mm, j, 0) * D[mm * Nq + i] * D[mm * Nq + i];
            d += G(i, mm, 2) * D[mm * Nq + j] * D[mm * Nq + j];
          }
          d += 2 * G(i, j, 1) * D[i * Nq + i] * D[j * Nq + j];
          const double wJ = m->affine ? m->wJ[e] * m->gllw[i] * m->gllw[j] : m->wJ[(size_t)e * Np + n];
          d += lambda * wJ;
          for (int f = 0; f < Nf; ++f) dL[(size_t)e * Np * Nf + (size_t)f * Np + n] = d;
        }
    bpo_gather(m, dL.data(), diag);
    return;
  }
#pragma omp parallel for
  for (dlong e = 0; e < m->E; ++e)
    for (int k = 0; k < Nq; ++k)
      for (int j = 0; j < Nq; ++j)
        for (int i = 0; i < Nq; ++i) {
          auto G = [&](int ii, int jj, int kk, int c) -> double {
            if (m->affine) return m->ggeo[6 * (size_t)e + c] * m->gllw[ii] * m->gllw[jj] * m->gllw[kk];
            return m->ggeo[6 * ((size_t)e * Np + ii + jj * Nq + kk * Nq * Nq) + c];
          };
          const int n = i + j * Nq + k * Nq * Nq;
          double d = 0.0;
          for (int mm = 0; mm < Nq; ++mm) {
            d += G(mm, j, k, 0) * D[mm * Nq + i] * D[mm * Nq + i];
            d += G(i, mm, k, 3) * D[mm * Nq + j] * D[mm * Nq + j];
            d += G(i, j, mm, 5) * D[mm * Nq + k] * D[mm * Nq + k];
          }
          d += 2 * G(i, j, k, 1) * D[i * Nq + i] * D[j * Nq + j];
          d += 2 * G(i, j, k, 2) * D[i * Nq + i] * D[k * Nq + k];
          d += 2 * G(i, j, k, 4) * D[j * Nq + j] * D[k * Nq + k];
          const double wJ = m->affine ? m->wJ[e] * m->gllw[i] * m->gllw[j] * m->gllw[k] : m->wJ[(size_t)e * Np + n];
          d += lambda * wJ;
          for (int f = 0; f < Nf; ++f) dL[(size_t)e * Np * Nf + (size_t)f * Np + n] = d;
        }
  bpo_gather(m, dL.data(), diag);
}

/* ------------------------------------------------------------------------ */
/* cubature and the over-integrated operators (BP1-BP4)                       */
/* ------------------------------------------------------------------------ */

/* CubatureSetupHex3D, libs/mesh/meshCubatureSetupHex3D.cpp:31-258.
   cubNq = N+2 Gauss points (JacobiGQ(0,0,N+1)) and the GLL->Gauss
   interpolation cubInterp [cubNq x Nq].
   Affine mesh: the reference's affine kernels work in the orthonormal
   Legendre (modal) basis instead: invV = V^-1 [Nq x Nq] and the modal
   differentiation matrix cubD = invV * Vr [Nq x Nq]; cubwJ and cubggeo are the
   per-element wJ and ggeo (no weights: the modal mass matrix is I).
   Curved mesh: cubD differentiates on the Gauss points [cubNq x cubNq]; the
   nine GLL-node derivatives of x, y, z are interpolated to the Gauss points
   (i, then j, then k) and cubwJ, cubggeo formed there with the Gauss weights. */
static void ensure_cubature(bpo_mesh& m) {
  if (m.cubNq) return;
  const int Nq = m.Nq, Np = m.Np, cNq = m.N + 2, cNp = cNq * cNq * cNq;
  m.cubr.resize(cNq); m.cubw.resize(cNq);
  bpo_jacobi_gq(0, 0, m.N + 1, m.cubr.data(), m.cubw.data());
  m.cubInterp.resize(cNq * Nq);
  bpo_interp_matrix1d(m.N, m.gllz.data(), cNq, m.cubr.data(), m.cubInterp.data());
  if (m.affine) {
    std::vector<double> Vr;
    grad_vandermonde1d(m.N, m.gllz, Vr);
    vandermonde1d(m.N, m.gllz, m.invV);
    dense_inverse(Nq, m.invV);
    m.cubD.assign(Nq * Nq, 0.0);
    for (int n = 0; n < Nq; ++n)
      for (int mm = 0; mm < Nq; ++mm) {
        double acc = 0;
        for (int k = 0; k < Nq; ++k) acc += m.invV[n * Nq + k] * Vr[k * Nq + mm];
        m.cubD[n * Nq + mm] = acc;
      }
    m.cubwJ = m.wJ;
    m.cubggeo = m.ggeo;
    m.cubNp = cNp; m.cubNq = cNq;
    return;
  }
  m.cubD.resize(cNq * cNq);
  bpo_dmatrix1d(m.N + 1, m.cubr.data(), cNq, m.cubr.data(), m.cubD.data());
  m.cubwJ.assign((size_t)m.E * cNp, 0.0);
  m.cubggeo.assign((size_t)6 * m.E * cNp, 0.0);
  const double* I = m.cubInterp.data();
  const int n1 = Nq * Nq * cNq, n2 = Nq * cNq * cNq;
#pragma omp parallel
  {
    std::vector<double> d(9 * (size_t)Np), d1(9 * (size_t)n1), d2(9 * (size_t)n2);
    const std::vector<double>* X[3] = {&m.x, &m.y, &m.z};
#pragma omp for
    for (dlong e = 0; e < m.E; ++e) {
      // d[comp][n], comp = 3*coordinate + direction: xr xs xt yr ys yt zr zs zt
      for (int k = 0; k < Nq; ++k)
        for (int j = 0; j < Nq; ++j)
          for (int i = 0; i < Nq; ++i) {
            const int n = i + j * Nq + k * Nq * Nq;
            for (int c = 0; c < 3; ++c) {
              const double* xe = X[c]->data() + (size_t)e * Np;
              double r = 0, sd = 0, t = 0;
              for (int mm = 0; mm < Nq; ++mm) {
                r += m.D[i * Nq + mm] * xe[k * Nq * Nq + j * Nq + mm];
                sd += m.D[j * Nq + mm] * xe[k * Nq * Nq + mm * Nq + i];
                t += m.D[k * Nq + mm] * xe[mm * Nq * Nq + j * Nq + i];
              }
              d[(3 * c + 0) * Np + n] = r;
              d[(3 * c + 1) * Np + n] = sd;
              d[(3 * c + 2) * Np + n] = t;
            }
          }
      for (int comp = 0; comp < 9; ++comp) {
        const double* f = &d[(size_t)comp * Np];
        double* f1 = &d1[(size_t)comp * n1];
        double* f2 = &d2[(size_t)comp * n2];
        for (int k = 0; k < Nq; ++k)
          for (int j = 0; j < Nq; ++j)
            for (int i = 0; i < cNq; ++i) {
              double acc = 0;
              for (int n = 0; n < Nq; ++n) acc += I[i * Nq + n] * f[k * Nq * Nq + j * Nq + n];
              f1[k * Nq * cNq + j * cNq + i] = acc;
            }
        for (int k = 0; k < Nq; ++k)
          for (int j = 0; j < cNq; ++j)
            for (int i = 0; i < cNq; ++i) {
              double acc = 0;
              for (int n = 0; n < Nq; ++n) acc += I[j * Nq + n] * f1[k * Nq * cNq + n * cNq + i];
              f2[k * cNq * cNq + j * cNq + i] = acc;
            }
      }
      for (int k = 0; k < cNq; ++k)
        for (int j = 0; j < cNq; ++j)
          for (int i = 0; i < cNq; ++i) {
            double v[9];
            for (int comp = 0; comp < 9; ++comp) {
              double acc = 0;
              for (int n = 0; n < Nq; ++n) acc += I[k * Nq + n] * d2[(size_t)comp * n2 + n * cNq * cNq + j * cNq + i];
              v[comp] = acc;
            }
            const double xr = v[0], xs = v[1], xt = v[2], yr = v[3], ys = v[4], yt = v[5];
            const double zr = v[6], zs = v[7], zt = v[8];
            const double J = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt);
            const double rx = (ys * zt - zs * yt) / J, ry = -(xs * zt - zs * xt) / J, rz = (xs * yt - ys * xt) / J;
            const double sx = -(yr * zt - zr * yt) / J, sy = (xr * zt - zr * xt) / J, sz = -(xr * yt - yr * xt) / J;
            const double tx = (yr * zs - zr * ys) / J, ty = -(xr * zs - zr * xs) / J, tz = (xr * ys - yr * xs) / J;
            const double JW = J * m.cubw[i] * m.cubw[j] * m.cubw[k];
            const size_t id = (size_t)e * cNp + i + j * cNq + k * cNq * cNq;
            m.cubwJ[id] = JW;
            double* g = &m.cubggeo[6 * id];
            g[0] = JW * (rx * rx + ry * ry + rz * rz);
            g[1] = JW * (rx * sx + ry * sy + rz * sz);
            g[2] = JW * (rx * tx + ry * ty + rz * tz);
            g[3] = JW * (sx * sx + sy * sy + sz * sz);
            g[4] = JW * (sx * tx + sy * ty + sz * tz);
            g[5] = JW * (tx * tx + ty * ty + tz * tz);
          }
    }
  }
  m.cubNp = cNp; m.cubNq = cNq;
}

/* Apply a 1D matrix A [no x ni] along one direction of a 3D field
   in[n2][n1][n0] (n0 fastest): dir 0 maps n0 -> no, 1 maps n1, 2 maps n2.
   out(...,o,...) = sum_i A[o*ni + i] * in(...,i,...) (AT: A[i*no + o]). */
static void apply1d(const double* A, bool AT, int no, int ni, int dir, const int dims[3], const double* in,
                    double* out) {
  int od[3] = {dims[0], dims[1], dims[2]};
  od[dir] = no;
  for (int c = 0; c < od[2]; ++c)
    for (int b = 0; b < od[1]; ++b)
      for (int a = 0; a < od[0]; ++a) {
        const int o = dir == 0 ? a : dir == 1 ? b : c;
        double acc = 0;
        for (int i = 0; i < ni; ++i) {
          const int ia = dir == 0 ? i : a, ib = dir == 1 ? i : b, ic = dir == 2 ? i : c;
          acc += (AT ? A[i * no + o] : A[o * ni + i]) * in[(ic * dims[1] + ib) * dims[0] + ia];
        }
        out[(c * od[1] + b) * od[0] + a] = acc;
      }
}

/* Three 1D applications in the order b (dir 1), a (dir 0), c (dir 2), the
   order of the reference's interpolation and projection stages
   (okl/bp3AxHex3D.okl:77-161 and :258-338). */
static void apply3d(const double* A, bool AT, int no, int ni, const double* in, double* out) {
  std::vector<double> t1((size_t)ni * no * ni), t2((size_t)ni * no * no);
  const int d0[3] = {ni, ni, ni};
  apply1d(A, AT, no, ni, 1, d0, in, t1.data());
  const int d1[3] = {ni, no, ni};
  apply1d(A, AT, no, ni, 0, d1, t1.data(), t2.data());
  const int d2[3] = {no, no, ni};
  apply1d(A, AT, no, ni, 2, d2, t2.data(), out);
}

/* Stiffness (plus lambda*mass) on a tensor grid of n^3 points with the 1D
   differentiation matrix Dm: gradient, the symmetric factor G (6 per point
   or per element), lambda*wJ*q, weak divergence with Dm^T; the loop
   structure of okl/bp3AxHex3D.okl:164-245. */
static void stiffness_grid(int n, const double* Dm, const double* G, const double* wJ, bool per_point,
                           double lambda, const double* q, double* r) {
  std::vector<double> qr(n * n * n), qs(n * n * n), qt(n * n * n);
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        const int id = i + j * n + k * n * n;
        const double* g = per_point ? &G[6 * id] : G;
        const double w = per_point ? wJ[id] : wJ[0];
        double dr = 0, ds = 0, dt = 0;
        for (int l = 0; l < n; ++l) {
          dr += Dm[i * n + l] * q[k * n * n + j * n + l];
          ds += Dm[j * n + l] * q[k * n * n + l * n + i];
          dt += Dm[k * n + l] * q[l * n * n + j * n + i];
        }
        qr[id] = g[0] * dr + g[1] * ds + g[2] * dt;
        qs[id] = g[1] * dr + g[3] * ds + g[4] * dt;
        qt[id] = g[2] * dr + g[4] * ds + g[5] * dt;
        r[id] = lambda * w * q[id];
      }
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        double acc = 0;
        for (int l = 0; l < n; ++l) {
          acc += Dm[l * n + i] * qr[k * n * n + j * n + l];
          acc += Dm[l * n + j] * qs[k * n * n + l * n + i];
          acc += Dm[l * n + k] * qt[l * n * n + j * n + i];
        }
        r[i + j * n + k * n * n] += acc;
      }
}

/* Element operators of BP1/BP2 (mass) and BP3/BP4 (stiffness + lambda mass)
   with over-integration, one field:
   - curved, BP3 (okl/bp3AxHex3D.okl:29-340): q -> Gauss points (I in b, a, c),
     stiffness_grid on cubNq^3 with cubD, cubggeo, cubwJ, project with I^T;
   - curved, BP1 (okl/bp1AxHex3D.okl): the same with cubwJ*q only;
   - affine, BP3 (okl/bp3AxAffineHex3D.okl:29-258): q -> modal (invV in b, a, c),
     stiffness_grid on Nq^3 with the modal cubD and the per-element ggeo,
     wJ, back with invV^T;
   - affine, BP1 (okl/bp1AxAffineHex3D.okl:29-135): wJ * (MM x MM x MM) q,
     applied in r, s, t order. */
static void ax_cub_e(const bpo_mesh& m, dlong e, bool stiff, double lambda, const double* q, double* AqL, int f) {
  const int Nq = m.Nq, Np = m.Np, Nf = m.Nfields, cNq = m.cubNq, cNp = m.cubNp;
  const size_t lbase = (size_t)e * Np * Nf + (size_t)f * Np;
  std::vector<double> qn(Np), rn(Np);
  for (int n = 0; n < Np; ++n) {
    const dlong id = m.G2L[lbase + n];
    qn[n] = (id != -1) ? q[id] : 0.0;
  }
  if (m.affine && !stiff) {
    std::vector<double> t1(Np), t2(Np);
    const int dims[3] = {Nq, Nq, Nq};
    apply1d(m.MM.data(), true, Nq, Nq, 0, dims, qn.data(), t1.data());
    apply1d(m.MM.data(), true, Nq, Nq, 1, dims, t1.data(), t2.data());
    apply1d(m.MM.data(), true, Nq, Nq, 2, dims, t2.data(), rn.data());
    for (int n = 0; n < Np; ++n) AqL[lbase + n] = m.cubwJ[e] * rn[n];
    return;
  }
  if (m.affine) {
    std::vector<double> qh(Np), rh(Np);
    apply3d(m.invV.data(), false, Nq, Nq, qn.data(), qh.data());
    stiffness_grid(Nq, m.cubD.data(), &m.cubggeo[6 * (size_t)e], &m.cubwJ[e], false, lambda, qh.data(), rh.data());
    apply3d(m.invV.data(), true, Nq, Nq, rh.data(), rn.data());
    for (int n = 0; n < Np; ++n) AqL[lbase + n] = rn[n];
    return;
  }
  std::vector<double> qc(cNp), rc(cNp);
  apply3d(m.cubInterp.data(), false, cNq, Nq, qn.data(), qc.data());
  if (stiff) {
    stiffness_grid(cNq, m.cubD.data(), &m.cubggeo[6 * (size_t)e * cNp], &m.cubwJ[(size_t)e * cNp], true, lambda,
                   qc.data(), rc.data());
  } else {
    for (int n = 0; n < cNp; ++n) rc[n] = m.cubwJ[(size_t)e * cNp + n] * qc[n];
  }
  apply3d(m.cubInterp.data(), true, Nq, cNq, rc.data(), rn.data());
  for (int n = 0; n < Np; ++n) AqL[lbase + n] = rn[n];
}

/* Element-local operator of benchmark problem bp (1..6) on every field of the
   mesh: BP1/BP2 mass, BP3/BP4 over-integrated stiffness, BP5/BP6 collocated
   stiffness (bpo_ax_bp5).  BP1/BP2 ignore lambda, as bp1AxHex3D has none. */
extern "C" void bpo_ax(bpo_mesh* m, int bp, double lambda, const double* q, double* AqL) {
  if (bp >= 5) { bpo_ax_bp5(m, lambda, q, AqL); return; }
  ensure_cubature(*m);
  const bool stiff = bp >= 3;
#pragma omp parallel for schedule(static)
  for (dlong e = 0; e < m->E; ++e)
    for (int f = 0; f < m->Nfields; ++f) ax_cub_e(*m, e, stiff, lambda, q, AqL, f);
}

/* bpN_t::Operator (BP/BP3/src/bp3Operator.cpp:29-85 and its siblings) at one
   rank: the element operator, then the Trans gather. */
extern "C" void bpo_operator(bpo_mesh* m, int bp, double lambda, const double* q, double* Aq) {
  std::vector<double> AqL((size_t)m->E * m->Np * m->Nfields);
  bpo_ax(m, bp, lambda, q, AqL.data());
  bpo_gather(m, AqL.data(), Aq);
}

/* Assembled diagonal of the BP1-BP4 operators (extension for Jacobi CG).  The
   element matrix is B^T W B with B a tensor product of 1D matrices, so the
   diagonal entry at node (a,b,c) is a sum over the quadrature grid of W times
   products of one 1D column per direction:
   curved:  columns of I (value) and DI = cubD I (derivative) over cubNq points;
   affine:  BP1 exact, wJ MM[a][a] MM[b][b] MM[c][c]; BP3 over the modal grid
            with columns of invV and cubD invV. */
static void jacobi_diag_cub(bpo_mesh& m, int bp, double lambda, double* diag) {
  ensure_cubature(m);
  const int Nq = m.Nq, Np = m.Np, Nf = m.Nfields;
  const bool stiff = bp >= 3;
  const bool aff = m.affine != 0;
  const int n = aff ? Nq : m.cubNq;   // quadrature grid points per direction
  const double* V = aff ? m.invV.data() : m.cubInterp.data();   // [n x Nq]
  std::vector<double> DV(n * Nq, 0.0);
  for (int i = 0; i < n; ++i)
    for (int a = 0; a < Nq; ++a) {
      double acc = 0;
      for (int l = 0; l < n; ++l) acc += m.cubD[i * n + l] * V[l * Nq + a];
      DV[i * Nq + a] = acc;
    }
  std::vector<double> dL((size_t)m.E * Np * Nf);
#pragma omp parallel for
  for (dlong e = 0; e < m.E; ++e)
    for (int c = 0; c < Nq; ++c)
      for (int b = 0; b < Nq; ++b)
        for (int a = 0; a < Nq; ++a) {
          double d = 0.0;
          if (aff && !stiff) {
            d = m.cubwJ[e] * m.MM[a * Nq + a] * m.MM[b * Nq + b] * m.MM[c * Nq + c];
          } else {
            for (int k = 0; k < n; ++k)
              for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                  const size_t id = aff ? (size_t)e : (size_t)e * m.cubNp + i + j * n + k * n * n;
                  const double Vi = V[i * Nq + a], Vj = V[j * Nq + b], Vk = V[k * Nq + c];
                  const double mass = m.cubwJ[id] * Vi * Vi * Vj * Vj * Vk * Vk;
                  if (!stiff) { d += mass; continue; }
                  const double gr = DV[i * Nq + a] * Vj * Vk, gs = Vi * DV[j * Nq + b] * Vk;
                  const double gt = Vi * Vj * DV[k * Nq + c];
                  const double* g = &m.cubggeo[6 * id];
                  d += g[0] * gr * gr + g[3] * gs * gs + g[5] * gt * gt + 2 * g[1] * gr * gs + 2 * g[2] * gr * gt +
                       2 * g[4] * gs * gt + lambda * mass;
                }
          }
          for (int f = 0; f < Nf; ++f) dL[(size_t)e * Np * Nf + (size_t)f * Np + a + b * Nq + c * Nq * Nq] = d;
        }
  bpo_gather(&m, dL.data(), diag);
}

extern "C" void bpo_jacobi_diag(bpo_mesh* m, int bp, double lambda, double* diag) {
  if (bp >= 5) bpo_jacobi_diag_bp5(m, lambda, diag);
  else jacobi_diag_cub(*m, bp, lambda, diag);
}

/* ------------------------------------------------------------------------ */
/* reductions in the reference's device order                                 */
/* ------------------------------------------------------------------------ */
/* Two-stage block tree: stage 1 as innerProd_1/norm2_1/updateCG_1
   (linAlgInnerProd.okl:29-69, linearSolverUpdateCG.okl:29-68), stage 2 as
   innerProd_2/updateCG_2.  bs is 256 (linAlg) or 512 (CG update). */
template <class F>
static double tree_reduce(dlong N, int bs, F term) {
  dlong Nblocks = (N + bs - 1) / bs;
  if (Nblocks > bs) Nblocks = bs;
  std::vector<double> partial(Nblocks);
  auto tree = [&](std::vector<double>& s) -> double {
    for (int h = bs / 2; h >= 2; h /= 2)
      for (int t = 0; t < h; ++t) s[t] += s[t + h];
    return s[0] + s[1];
  };
#pragma omp parallel for
  for (dlong b = 0; b < Nblocks; ++b) {
    std::vector<double> s(bs);
    for (int t = 0; t < bs; ++t) {
      double acc = 0.0;
      for (dlong id = t + b * bs; id < N; id += bs * Nblocks) acc += term(id);
      s[t] = acc;
    }
    partial[b] = tree(s);
  }
  std::vector<double> s(bs);
  for (int t = 0; t < bs; ++t) {
    double acc = 0.0;
    for (dlong id = t; id < Nblocks; id += bs) acc += partial[id];
    s[t] = acc;
  }
  return tree(s);
}

/* cg::Solve (linearSolverCG.cpp:62-129) with UpdateCG (:131-156).  precon=1
   switches to Jacobi-preconditioned CG with the relative stop rule
   ||r|| <= tol ||b|| (extension); precon=0 keeps the reference's plain CG and
   its stop rule rdotr <= max(tol^2 rdotr0, tol^2).  r holds b on entry and the
   final residual on exit.  hist_rnorm/hist_alpha (length >= maxit) receive
   sqrt(rdotr) and alpha of every iteration; returns the iteration count. */
extern "C" int bpo_cg_bp(bpo_mesh* m, int bp, double lambda, double* x, double* r, double tol, int maxit,
                         int precon, const double* invDiag, double* hist_rnorm, double* hist_alpha) {
  const dlong N = m->Ngather;
  auto op = [m, bp, lambda](const double* q, double* Aq) { bpo_operator(m, bp, lambda, q, Aq); };
  std::vector<double> p(N, 0.0), Ap(N, 0.0), z;
  if (precon) z.assign(N, 0.0);
  op(x, Ap.data());
#pragma omp parallel for
  for (dlong n = 0; n < N; ++n) r[n] = -1.0 * Ap[n] + 1.0 * r[n];
  if (!precon) {
    double rdotr = std::sqrt(tree_reduce(N, 256, [&](dlong i) { return r[i] * r[i]; }));
    rdotr = rdotr * rdotr;
    const double TOL = std::max(tol * tol * rdotr, tol * tol);
    double rdotr1 = 0.0, rdotr2 = 0.0;
    int iter;
    for (iter = 0; iter < maxit; ++iter) {
      if (rdotr <= TOL) break;
      rdotr2 = rdotr1;
      rdotr1 = rdotr;
      const double beta = (iter == 0) ? 0.0 : rdotr1 / rdotr2;
#pragma omp parallel for
      for (dlong n = 0; n < N; ++n) p[n] = 1.0 * r[n] + beta * p[n];
      op(p.data(), Ap.data());
      const double pAp = tree_reduce(N, 256, [&](dlong i) { return p[i] * Ap[i]; });
      const double alpha = rdotr1 / pAp;
      rdotr = tree_reduce(N, 512, [&](dlong i) {
        const double rn = r[i] - alpha * Ap[i];
        r[i] = rn;
        return rn * rn;
      });
#pragma omp parallel for
      for (dlong n = 0; n < N; ++n) x[n] = alpha * p[n] + 1.0 * x[n];
      if (hist_rnorm) hist_rnorm[iter] = std::sqrt(rdotr);
      if (hist_alpha) hist_alpha[iter] = alpha;
    }
    return iter;
  }
  /* Jacobi PCG */
  const double rr0 = tree_reduce(N, 256, [&](dlong i) { return r[i] * r[i]; });
  const double TOL = tol * tol * rr0;
  double rz = tree_reduce(N, 512, [&](dlong i) { z[i] = invDiag[i] * r[i]; return r[i] * z[i]; });
  double rr = rr0, rz_old = 0.0;
  int iter;
  for (iter = 0; iter < maxit; ++iter) {
    if (rr <= TOL) break;
    const double beta = (iter == 0) ? 0.0 : rz / rz_old;
#pragma omp parallel for
    for (dlong n = 0; n < N; ++n) p[n] = z[n] + beta * p[n];
    op(p.data(), Ap.data());
    const double pAp = tree_reduce(N, 256, [&](dlong i) { return p[i] * Ap[i]; });
    const double alpha = rz / pAp;
#pragma omp parallel for
    for (dlong n = 0; n < N; ++n) { x[n] += alpha * p[n]; r[n] -= alpha * Ap[n]; z[n] = invDiag[n] * r[n]; }
    rz_old = rz;
    rz = tree_reduce(N, 512, [&](dlong i) { return r[i] * z[i]; });
    rr = tree_reduce(N, 512, [&](dlong i) { return r[i] * r[i]; });
    if (hist_rnorm) hist_rnorm[iter] = std::sqrt(rr);
    if (hist_alpha) hist_alpha[iter] = alpha;
  }
  return iter;
}

/* BP5/BP6 CG (the operator by the mesh's field count) */
extern "C" int bpo_cg(bpo_mesh* m, double lambda, double* x, double* r, double tol, int maxit, int precon,
                      const double* invDiag, double* hist_rnorm, double* hist_alpha) {
  return bpo_cg_bp(m, 5, lambda, x, r, tol, maxit, precon, invDiag, hist_rnorm, hist_alpha);
}

extern "C" int bpo_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
