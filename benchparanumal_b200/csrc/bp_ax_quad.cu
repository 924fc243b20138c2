// Quad2D (2D tensor-product element) forms of the BP5/BP6 path: the element
// operator, the forcing, the lumped mass and the Jacobi diagonal.
//
//   Aq_e = Dr^T (G00 ur + G01 us) + Ds^T (G01 ur + G11 us) + lambda wJ q,
//   (ur, us) = (Dr, Ds) q
// (okl/bp5AxQuad2D.okl, okl/bp5AxAffineQuad2D.okl, okl/bp6AxQuad2D.okl with
// Nfields = dim = 2).  Stored factors carry the GLL weights; affine factors are
// per element and the weights w_i w_j are applied here.  One thread per node
// (i, j) of an element slot, EPB element slots per block; q, the fluxes and D
// go through shared memory (rows padded by one word), which the Nq^2 nodes of
// a 2D element fill in one pass.
#include <cuda_runtime.h>

#include <cstdint>

#include "bp_cg_device.cuh"
#include "bp_internal.hpp"

namespace bp {
namespace {

template <int NQ>
struct QuadShape {
  static constexpr int EPB0 = 256 / (NQ * NQ);
  static constexpr int EPB = EPB0 < 1 ? 1 : (EPB0 > 16 ? 16 : EPB0);   // element slots per block
  static constexpr int RS = NQ + 1;                                     // padded row
  static constexpr int THREADS = NQ * NQ * EPB;
};

template <int NQ, int NF, bool AFFINE, bool DOT, class F>
__global__ void __launch_bounds__(QuadShape<NQ>::THREADS)
ax_quad_kernel(int Nelements, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
               const F* __restrict__ wJ, const F* __restrict__ ggeo, const F* __restrict__ gllw,
               const F* __restrict__ Dg, F lambda, const F* __restrict__ q, F* __restrict__ Aq,
               const int* __restrict__ skip, CgFuse fuse) {
  if (skip && *skip) return;
  using Sh = QuadShape<NQ>;
  constexpr int EPB = Sh::EPB, RS = Sh::RS, NP = NQ * NQ;
  __shared__ F s_D[NQ][RS];
  __shared__ F s_w[NQ];
  __shared__ F s_q[EPB][NF][NQ][RS];
  __shared__ F s_Gr[EPB][NF][NQ][RS];
  __shared__ F s_Gs[EPB][NF][NQ][RS];
  __shared__ double s_red[Sh::THREADS];

  const int i = threadIdx.x, j = threadIdx.y, es = threadIdx.z;
  const int t = i + NQ * (j + NQ * es);
  const int eidx = blockIdx.x * EPB + es;
  const bool active = eidx < Nelements;
  const int e = active ? elementList[eidx] : 0;
  for (int n = t; n < NP; n += Sh::THREADS) s_D[n / NQ][n % NQ] = Dg[n];
  if (AFFINE && t < NQ) s_w[t] = gllw[t];
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    const int32_t id = active ? G2L[((size_t)e * NF + f) * NP + j * NQ + i] : -1;
    s_q[es][f][j][i] = (id != -1) ? q[id] : F(0);
  }
  __syncthreads();

  F G00, G01, G11, GwJ;
  if (AFFINE) {
    const F w = s_w[i] * s_w[j];
    G00 = active ? ggeo[3 * (size_t)e + 0] * w : F(0);
    G01 = active ? ggeo[3 * (size_t)e + 1] * w : F(0);
    G11 = active ? ggeo[3 * (size_t)e + 2] * w : F(0);
    GwJ = active ? wJ[e] * w : F(0);
  } else {
    const size_t gb = (size_t)e * NP + j * NQ + i;
    G00 = active ? ggeo[3 * gb + 0] : F(0);
    G01 = active ? ggeo[3 * gb + 1] : F(0);
    G11 = active ? ggeo[3 * gb + 2] : F(0);
    GwJ = active ? wJ[gb] : F(0);
  }
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    F ur = 0, us = 0;
#pragma unroll
    for (int m = 0; m < NQ; ++m) {
      ur += s_D[i][m] * s_q[es][f][j][m];
      us += s_D[j][m] * s_q[es][f][m][i];
    }
    s_Gr[es][f][j][i] = G00 * ur + G01 * us;
    s_Gs[es][f][j][i] = G01 * ur + G11 * us;
  }
  __syncthreads();
  double pdot = 0.0;
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    const F qn = s_q[es][f][j][i];
    F ap = qn * lambda * GwJ;
#pragma unroll
    for (int m = 0; m < NQ; ++m) {
      ap += s_D[m][i] * s_Gr[es][f][j][m];
      ap += s_D[m][j] * s_Gs[es][f][m][i];
    }
    if (active) Aq[((size_t)e * NF + f) * NP + j * NQ + i] = ap;
    if (DOT) pdot += (double)qn * (double)ap;
  }
  if (DOT) fuse_pap(pdot, fuse, s_red);
}

// Column form (affine factors, NQ <= kQuadColMax): one thread per column i of
// an element, holding the column's q values and s-fluxes in registers and row
// and column i of D; shared memory carries only what crosses columns (the rows
// of q and of the r-flux), and the other reads of D use a slice index that is
// the same for every lane (broadcasts).  The sums run in the node form's
// order.  Measured on 800x800 boxes (the same box, two alternating runs): BK5
// affine p=3 3.59 -> 4.96, p=5 4.34 -> 5.10, p=7 4.77 -> 5.87, p=9 4.61 ->
// 5.04 TFLOP/s, 100 CG iterations at p=7 123.0 -> 107.1 ms; with stored
// factors it lost (p=7 3.03 -> 2.48 TB/s: 88-102 registers leave two blocks
// per SM to wait on the per-node factor loads), so those keep the node form;
// staging each slot's stored factors in shared memory first (coalesced loads,
// 12 slots per block for the space, 142 registers) was slower still: p=7 1.55
// TB/s.
constexpr int kQuadColMax = 10;

template <int NQ>
struct QuadColShape {
  static constexpr int EPB = (NQ <= 8 ? 256 : 160) / NQ;   // element slots per block
  static constexpr int RS = NQ + 1;
  static constexpr int THREADS = NQ * EPB;
};

template <int NQ, int NF, bool AFFINE, bool DOT, class F>
__global__ void __launch_bounds__(QuadColShape<NQ>::THREADS)
ax_quad_col_kernel(int Nelements, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
                   const F* __restrict__ wJ, const F* __restrict__ ggeo, const F* __restrict__ gllw,
                   const F* __restrict__ Dg, F lambda, const F* __restrict__ q, F* __restrict__ Aq,
                   const int* __restrict__ skip, CgFuse fuse) {
  if (skip && *skip) return;
  using Sh = QuadColShape<NQ>;
  constexpr int EPB = Sh::EPB, RS = Sh::RS, NP = NQ * NQ;
  __shared__ F s_D[NQ][NQ];
  __shared__ F s_w[NQ];
  __shared__ F s_q[EPB][NQ][RS];   // rows of q (one field at a time)
  __shared__ F s_r[EPB][NQ][RS];   // rows of the r-flux
  __shared__ double s_red[Sh::THREADS];

  const int i = threadIdx.x, es = threadIdx.y;
  const int t = i + NQ * es;
  const int eidx = blockIdx.x * EPB + es;
  const bool active = eidx < Nelements;
  const int e = active ? elementList[eidx] : 0;
  for (int n = t; n < NP; n += Sh::THREADS) s_D[n / NQ][n % NQ] = Dg[n];
  if (AFFINE && t < NQ) s_w[t] = gllw[t];
  __syncthreads();
  F Di[NQ], Dci[NQ];   // row i and column i of D
#pragma unroll
  for (int m = 0; m < NQ; ++m) {
    Di[m] = s_D[i][m];
    Dci[m] = s_D[m][i];
  }
  F A00 = 0, A01 = 0, A11 = 0, AJ = 0;   // affine factors (the weights w_i w_j applied per node)
  if (AFFINE && active) {
    A00 = ggeo[3 * (size_t)e + 0];
    A01 = ggeo[3 * (size_t)e + 1];
    A11 = ggeo[3 * (size_t)e + 2];
    AJ = wJ[e];
  }
  double pdot = 0.0;
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    const size_t lb = ((size_t)e * NF + f) * NP + i;
    F qc[NQ];
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
      const int32_t id = active ? G2L[lb + j * NQ] : -1;
      qc[j] = (id != -1) ? q[id] : F(0);
      s_q[es][j][i] = qc[j];
    }
    __syncthreads();
    F fs[NQ];
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
      F ur = 0, us = 0;
#pragma unroll
      for (int m = 0; m < NQ; ++m) {
        ur += Di[m] * s_q[es][j][m];
        us += s_D[j][m] * qc[m];
      }
      F G00, G01, G11;
      if (AFFINE) {
        const F w = s_w[i] * s_w[j];
        G00 = A00 * w;
        G01 = A01 * w;
        G11 = A11 * w;
      } else {
        const size_t gb = (size_t)e * NP + j * NQ + i;
        G00 = active ? ggeo[3 * gb + 0] : F(0);
        G01 = active ? ggeo[3 * gb + 1] : F(0);
        G11 = active ? ggeo[3 * gb + 2] : F(0);
      }
      s_r[es][j][i] = G00 * ur + G01 * us;
      fs[j] = G01 * ur + G11 * us;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
      const F GwJ = AFFINE ? AJ * (s_w[i] * s_w[j]) : (active ? wJ[(size_t)e * NP + j * NQ + i] : F(0));
      F ap = qc[j] * lambda * GwJ;
#pragma unroll
      for (int m = 0; m < NQ; ++m) {
        ap += Dci[m] * s_r[es][j][m];
        ap += s_D[m][j] * fs[m];
      }
      if (active) Aq[lb + j * NQ] = ap;
      if (DOT) pdot += (double)qc[j] * (double)ap;
    }
    if (NF > 1) __syncthreads();   // the next field reuses s_q and s_r
  }
  if (DOT) fuse_pap(pdot, fuse, s_red);
}

// element slots per block of the form that runs (the column form exists for NQ <= kQuadColMax)
template <int NQ>
int quad_epb(bool col) {
  if constexpr (NQ <= kQuadColMax)
    return col ? QuadColShape<NQ>::EPB : QuadShape<NQ>::EPB;
  else
    return QuadShape<NQ>::EPB;
}

template <int NQ, class F>
static int launch_quad_nq(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                          const F* wJ, const F* ggeo, const F* gllw, const F* D, F lambda, const F* q, F* Aq,
                          const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  constexpr bool COL = NQ <= kQuadColMax;
  const bool col = COL && d.affine;
  const int epb = quad_epb<NQ>(col);
  const dim3 block = col ? dim3(NQ, epb) : dim3(NQ, NQ, epb);
  const dim3 grid((Nelements + epb - 1) / epb);
  if (nblocks) *nblocks = (int)grid.x;
  const CgFuse Fz = fuse ? *fuse : CgFuse{};
#define BP_QUAD(NF, AFF, DOT)                                                                                        \
  do {                                                                                                               \
    if constexpr (COL && AFF)                                                                                        \
      ax_quad_col_kernel<NQ, NF, AFF, DOT, F><<<grid, block, 0, s>>>(Nelements, elementList, G2L, wJ, ggeo, gllw, D, \
                                                                    lambda, q, Aq, skip, Fz);                        \
    else                                                                                                             \
      ax_quad_kernel<NQ, NF, AFF, DOT, F><<<grid, block, 0, s>>>(Nelements, elementList, G2L, wJ, ggeo, gllw, D,     \
                                                                lambda, q, Aq, skip, Fz);                            \
  } while (0)
  const bool dot = fuse != nullptr;
  if (d.Nfields == 1) {
    if (d.affine) { if (dot) BP_QUAD(1, true, true); else BP_QUAD(1, true, false); }
    else { if (dot) BP_QUAD(1, false, true); else BP_QUAD(1, false, false); }
  } else {
    if (d.affine) { if (dot) BP_QUAD(2, true, true); else BP_QUAD(2, true, false); }
    else { if (dot) BP_QUAD(2, false, true); else BP_QUAD(2, false, false); }
  }
#undef BP_QUAD
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

template <class F>
static int launch_quad_t(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                         const F* wJ, const F* ggeo, const F* gllw, const F* D, F lambda, const F* q, F* Aq,
                         const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  if (nblocks) *nblocks = 0;
  if (d.Nfields != 1 && d.Nfields != 2) return fail(BP_ERROR_ARG, "Quad2D operator: Nfields must be 1 or 2");
  if (fuse && fuse->dir) return 1;
  if (Nelements == 0) return BP_SUCCESS;
  switch (d.N + 1) {
#define BP_QUAD_CASE(nq) \
  case nq:               \
    return launch_quad_nq<nq, F>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, fuse, s, nblocks);
    BP_QUAD_CASE(2) BP_QUAD_CASE(3) BP_QUAD_CASE(4) BP_QUAD_CASE(5) BP_QUAD_CASE(6) BP_QUAD_CASE(7)
    BP_QUAD_CASE(8) BP_QUAD_CASE(9) BP_QUAD_CASE(10) BP_QUAD_CASE(11) BP_QUAD_CASE(12) BP_QUAD_CASE(13)
    BP_QUAD_CASE(14) BP_QUAD_CASE(15) BP_QUAD_CASE(16)
#undef BP_QUAD_CASE
    default:
      return fail(BP_ERROR_ARG, "Quad2D operator: degree N must be in 1..15");
  }
}

// Forcing of okl/rhsQuad2D.okl (rhsQuad2D, rhsAffineQuad2D) at the GLL nodes
// of the bilinear map (meshPhysicalNodesQuad2D.cpp)
__global__ void rhs_analytic_quad_kernel(int Nq, int affine, int Nfields, int E, const double* __restrict__ EX,
                                         const double* __restrict__ EY, const double* __restrict__ gllz,
                                         const double* __restrict__ gllw, const double* __restrict__ wJ,
                                         double lambda, double* __restrict__ rL) {
  const int Np = Nq * Nq;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)E * Np) return;
  const int e = (int)(gid / Np), n = (int)(gid % Np);
  const int i = n % Nq, j = n / Nq;
  const double r = gllz[i], s = gllz[j];
  const double* ex = EX + 4 * (size_t)e;
  const double* ey = EY + 4 * (size_t)e;
  const double x = 0.25 * (1 - r) * (1 - s) * ex[0] + 0.25 * (1 + r) * (1 - s) * ex[1] +
                   0.25 * (1 + r) * (1 + s) * ex[2] + 0.25 * (1 - r) * (1 + s) * ex[3];
  const double y = 0.25 * (1 - r) * (1 - s) * ey[0] + 0.25 * (1 + r) * (1 - s) * ey[1] +
                   0.25 * (1 + r) * (1 + s) * ey[2] + 0.25 * (1 - r) * (1 + s) * ey[3];
  const double w = affine ? wJ[e] * gllw[i] * gllw[j] : wJ[gid];
  const double pi = 3.14159265358979323846;
  if (Nfields == 1) {
    rL[gid] = w * ((2 * pi * pi + lambda) * sin(pi * x) * sin(pi * y));
  } else {
    const size_t base = (size_t)e * Np * 2 + n;
    rL[base] = w * ((3 * pi * pi + lambda) * sin(2.0 * pi * x) * sin(pi * y));
    rL[base + Np] = w * ((3 * pi * pi + lambda) * sin(pi * x) * sin(2.0 * pi * y));
  }
}

// rL[l] = wJ_l f[G2L[l]] (0 on masked nodes), Quad2D weights
__global__ void mass_local_quad_kernel(int Nq, int affine, int Nfields, int E, const int32_t* __restrict__ G2L,
                                       const double* __restrict__ gllw, const double* __restrict__ wJ,
                                       const double* __restrict__ f, double* __restrict__ rL) {
  const int Np = Nq * Nq;
  const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= (long long)E * Np * Nfields) return;
  const int e = (int)(l / ((long long)Np * Nfields));
  const int n = (int)(l % Np);
  const double w = affine ? wJ[e] * gllw[n % Nq] * gllw[n / Nq] : wJ[(size_t)e * Np + n];
  const int32_t id = G2L[l];
  rL[l] = (id != -1) ? w * f[id] : 0.0;
}

// Element diagonal of the Quad2D operator (Jacobi): the two 1D stiffness
// directions, the mixed term at the node and lambda wJ
__global__ void diag_local_quad_kernel(int Nq, int affine, int Nfields, int E, const double* __restrict__ ggeo,
                                       const double* __restrict__ wJ, const double* __restrict__ gllw,
                                       const double* __restrict__ D, double lambda, double* __restrict__ dL) {
  const int Np = Nq * Nq;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)E * Np) return;
  const int e = (int)(gid / Np), n = (int)(gid % Np);
  const int i = n % Nq, j = n / Nq;
  auto G = [&](int ii, int jj, int c) -> double {
    if (affine) return ggeo[3 * (size_t)e + c] * gllw[ii] * gllw[jj];
    return ggeo[3 * ((size_t)e * Np + ii + jj * Nq) + c];
  };
  double d = 0.0;
  for (int m = 0; m < Nq; ++m) {
    d += G(m, j, 0) * D[m * Nq + i] * D[m * Nq + i];
    d += G(i, m, 2) * D[m * Nq + j] * D[m * Nq + j];
  }
  d += 2 * G(i, j, 1) * D[i * Nq + i] * D[j * Nq + j];
  d += lambda * (affine ? wJ[e] * gllw[i] * gllw[j] : wJ[gid]);
  for (int f = 0; f < Nfields; ++f) dL[(size_t)e * Np * Nfields + (size_t)f * Np + n] = d;
}

}  // namespace

int launch_ax_quad(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                   const double* wJ, const double* ggeo, const double* gllw, const double* D, double lambda,
                   const double* q, double* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  return launch_quad_t<double>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, fuse, s,
                               nblocks);
}

int launch_ax_quad(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                   const float* wJ, const float* ggeo, const float* gllw, const float* D, float lambda,
                   const float* q, float* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  return launch_quad_t<float>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, fuse, s,
                              nblocks);
}

int launch_rhs_analytic_quad(int N, int affine, int Nfields, int E, const double* EX, const double* EY,
                             const double* gllz, const double* gllw, const double* wJ, double lambda, double* rL,
                             cudaStream_t s) {
  const int Nq = N + 1;
  const long long tot = (long long)E * Nq * Nq;
  if (tot == 0) return BP_SUCCESS;
  rhs_analytic_quad_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(Nq, affine, Nfields, E, EX, EY, gllz, gllw,
                                                                           wJ, lambda, rL);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

int launch_mass_local_quad(int N, int affine, int Nfields, int E, const int32_t* G2L, const double* gllw,
                           const double* wJ, const double* f, double* rL, cudaStream_t s) {
  const int Nq = N + 1;
  const long long tot = (long long)E * Nq * Nq * Nfields;
  if (tot == 0) return BP_SUCCESS;
  mass_local_quad_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(Nq, affine, Nfields, E, G2L, gllw, wJ, f,
                                                                         rL);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

int launch_diag_local_quad(int N, int affine, int Nfields, int E, const double* ggeo, const double* wJ,
                           const double* gllw, const double* D, double lambda, double* dL, cudaStream_t s) {
  const int Nq = N + 1;
  const long long tot = (long long)E * Nq * Nq;
  if (tot == 0) return BP_SUCCESS;
  diag_local_quad_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(Nq, affine, Nfields, E, ggeo, wJ, gllw, D,
                                                                         lambda, dL);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

}  // namespace bp
