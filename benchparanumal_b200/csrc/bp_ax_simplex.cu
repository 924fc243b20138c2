// Simplex (affine Tri2D and Tet3D) BP5 element operator, forcings and Jacobi
// diagonal.
//
// The reference's affine simplex operators (okl/bp5AxAffineTri2D.okl:27-89,
// okl/bp5AxAffineTet3D.okl) apply dense Np x Np reference matrices per element:
//   Aq_e = sum_ab G_ab S_ab q_e + lambda J MM q_e
// over ab = rr, rs, ss (triangles: NSM = 3) or rr, rs, rt, ss, st, tt
// (tetrahedra: NSM = 6), with per-element factors G_ab and J.  Np is not a
// tensor product, so there is no sum factorisation: a batched product of the
// four stacked matrices with the elements' gathered values (in shared memory),
// the matrices read with node-fastest layout (X[k*Np + n] is the weight of
// node k in output n: the reference's device copies o_S and o_MM), so the
// threads of a node group read consecutive words for every k.  The matrices (4*Np^2
// doubles, 41 KB at p = 7) are shared by all elements and stay in L1/L2.
// Sums over k run in increasing k, the output combines the four sums in the
// reference's order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "bp_cg_device.cuh"
#include "bp_internal.hpp"

namespace bp {
namespace {

constexpr int kTriThreads = 256;

// nodes of the degree-N triangle (dim 2) or tetrahedron (dim 3)
int simplex_np(int dim, int N) { return dim == 2 ? (N + 1) * (N + 2) / 2 : (N + 1) * (N + 2) * (N + 3) / 6; }

// node groups per block (element slots for the forcing) and threads per block
// (whole warps, at most kTriThreads + 32: tetrahedra of degree 11..15 have
// 364..816 nodes, and their threads walk the nodes of the element in strides)
static void tri_shape(int Np, int* epb, int* threads) {
  *epb = Np >= kTriThreads ? 1 : kTriThreads / Np;
  *threads = std::min((*epb * Np + 31) / 32 * 32, kTriThreads + 32);
}

// Thread (n, g) of a block computes node n of the kTriElems elements of group
// g, so every matrix entry it loads serves kTriElems elements (four FMAs per
// element).  Measured on 400x400 boxes (320,000 triangles): one element per
// thread 6.1 TFLOP/s (reference flop model) at p=7 and 36.7 ms for 100 CG
// iterations at p=5; four 7.3 TFLOP/s and 26.2 ms; eight 7.8 TFLOP/s but
// 43.4 ms (132 registers in the CG form with the p.Ap sum).
constexpr int kTriElems = 4;

// Triangles are held to three blocks per SM (72 registers instead of 82,
// a few words of spills): ncu showed two blocks (16 warps) waiting on the
// matrix loads (long scoreboard); three gave BK5 p=5 5.29 -> 6.18 and p=7
// 7.46 -> 8.14 TFLOP/s and 100 CG iterations at p=5 32.1 -> 29.4 ms (400x400,
// the same box).  Tetrahedra need their 110 registers (seven sums of four
// elements).
template <class F, int NSM, bool DOT>
__global__ void __launch_bounds__(kTriThreads + 32, NSM == 3 ? 3 : 1)
ax_simplex_kernel(int Nelements, int Np, int groups, const int32_t* __restrict__ elementList,
              const int32_t* __restrict__ G2L, const F* __restrict__ wJ, const F* __restrict__ ggeo,
              const F* __restrict__ S, const F* __restrict__ MM, F lambda, const F* __restrict__ q,
              F* __restrict__ Aq, const int* __restrict__ skip, double* __restrict__ partials) {
  pdl_wait();
  pdl_release();
  if (skip && *skip) return;
  // [groups*kTriElems][Np] values; the block sum reuses it (sized for doubles)
  extern __shared__ __align__(16) double s_raw[];
  F* const s_q = reinterpret_cast<F*>(s_raw);
  const int t = threadIdx.x;
  const int slots = groups * kTriElems;
  const int e0 = blockIdx.x * slots;
  for (int i = t; i < slots * Np; i += blockDim.x) {
    const int j = i / Np, m = i - j * Np;
    F v = 0;
    if (e0 + j < Nelements) {
      const int32_t id = G2L[(size_t)elementList[e0 + j] * Np + m];
      if (id >= 0) v = q[id];
    }
    s_q[i] = v;
  }
  __syncthreads();
  // one node per thread; with more nodes than threads (one group), the
  // threads take the element's nodes in strides of the block
  const int g = t / Np;
  double pdot = 0.0;
  for (int n = t - g * Np; g < groups && n < Np; n += blockDim.x) {
    const F* sq = s_q + (size_t)g * kTriElems * Np;
    const size_t NP2 = (size_t)Np * Np;
    F acc[NSM + 1][kTriElems];   // the S_ab sums, then the mass sum
#pragma unroll
    for (int a = 0; a <= NSM; ++a)
#pragma unroll
      for (int j = 0; j < kTriElems; ++j) acc[a][j] = 0;
    for (int k = 0; k < Np; ++k) {
      const size_t o = (size_t)k * Np + n;
      F w[NSM + 1];
#pragma unroll
      for (int a = 0; a < NSM; ++a) w[a] = __ldg(S + a * NP2 + o);
      w[NSM] = __ldg(MM + o);
#pragma unroll
      for (int j = 0; j < kTriElems; ++j) {
        const F qk = sq[j * Np + k];
#pragma unroll
        for (int a = 0; a <= NSM; ++a) acc[a][j] += w[a] * qk;
      }
    }
#pragma unroll
    for (int j = 0; j < kTriElems; ++j) {
      const int eidx = e0 + g * kTriElems + j;
      if (eidx < Nelements) {
        const int element = elementList[eidx];
        const F* gg = ggeo + NSM * (size_t)element;
        F out = gg[0] * acc[0][j];
#pragma unroll
        for (int a = 1; a < NSM; ++a) out += gg[a] * acc[a][j];
        out += wJ[element] * lambda * acc[NSM][j];
        Aq[(size_t)element * Np + n] = out;
        if (DOT) pdot += (double)sq[j * Np + n] * (double)out;
      }
    }
  }
  if (DOT) {
    const double bs = fuse_block_sum(pdot, s_raw);
    if (t == 0) partials[blockIdx.x] = bs;
  }
}

// b_e = J_e MM f_e with f scattered through GlobalToLocal (masked nodes 0)
__global__ void __launch_bounds__(kTriThreads + 32)
tri_mass_local_kernel(int Nelements, int Np, int epb, const int32_t* __restrict__ G2L,
                      const double* __restrict__ wJ, const double* __restrict__ MM, const double* __restrict__ f,
                      double* __restrict__ bL) {
  extern __shared__ __align__(16) double s_f[];
  for (int i = threadIdx.x; i < epb * Np; i += blockDim.x) {
    const int es = i / Np, n = i - es * Np, e = blockIdx.x * epb + es;
    if (e < Nelements) {
      const int32_t id = G2L[(size_t)e * Np + n];
      s_f[i] = id >= 0 ? f[id] : 0.0;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < epb * Np; i += blockDim.x) {
    const int es = i / Np, n = i - es * Np, e = blockIdx.x * epb + es;
    if (e >= Nelements) continue;
    double acc = 0.0;
    for (int k = 0; k < Np; ++k) acc += __ldg(MM + (size_t)k * Np + n) * s_f[es * Np + k];
    bL[(size_t)e * Np + n] = wJ[e] * acc;
  }
}

// diagonal of A_e: sum_ab G_ab S_ab(n,n) + lambda J MM(n,n)
__global__ void simplex_diag_local_kernel(int Nelements, int Np, int nsm, const double* __restrict__ wJ,
                                          const double* __restrict__ ggeo, const double* __restrict__ S,
                                          const double* __restrict__ MM, double lambda, double* __restrict__ dL) {
  const size_t NP2 = (size_t)Np * Np;
  const size_t total = (size_t)Nelements * Np;
  for (size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x; l < total; l += (size_t)blockDim.x * gridDim.x) {
    const size_t e = l / Np, n = l - e * Np;
    const size_t dn = n * Np + n;
    const double* g = ggeo + nsm * e;
    double d = g[0] * S[dn];
    for (int a = 1; a < nsm; ++a) d += g[a] * S[a * NP2 + dn];
    dL[l] = d + lambda * wJ[e] * MM[dn];
  }
}

// rhsAffineTri2D / rhsAffineTet3D (okl/rhsTri2D.okl, okl/rhsTet3D.okl):
// b_e = MM (J_e f) with f = (2 pi^2 + lambda) sin(pi x) sin(pi y) on triangles,
// (3 pi^2 + lambda) sin(pi x) sin(pi y) sin(pi z) on tetrahedra (z given)
__global__ void __launch_bounds__(kTriThreads + 32)
simplex_rhs_analytic_kernel(int Nelements, int Np, int epb, const double* __restrict__ wJ,
                            const double* __restrict__ MM, const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, double lambda, double* __restrict__ bL) {
  extern __shared__ __align__(16) double s_f[];
  const double pi = 3.14159265358979323846;
  for (int i = threadIdx.x; i < epb * Np; i += blockDim.x) {
    const int es = i / Np, e = blockIdx.x * epb + es;
    if (e < Nelements) {
      const size_t id = (size_t)e * Np + (i - es * Np);
      const double f = z ? (3 * pi * pi + lambda) * sin(pi * x[id]) * sin(pi * y[id]) * sin(pi * z[id])
                         : (2 * pi * pi + lambda) * sin(pi * x[id]) * sin(pi * y[id]);
      s_f[i] = wJ[e] * f;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < epb * Np; i += blockDim.x) {
    const int es = i / Np, n = i - es * Np, e = blockIdx.x * epb + es;
    if (e >= Nelements) continue;
    double acc = 0.0;
    for (int m = 0; m < Np; ++m) acc += __ldg(MM + (size_t)m * Np + n) * s_f[es * Np + m];
    bL[(size_t)e * Np + n] = acc;
  }
}

}  // namespace

int launch_rhs_analytic_simplex(int dim, int N, int32_t Nelements, const double* wJ, const double* MM,
                                const double* x, const double* y, const double* z, double lambda, double* bL,
                                cudaStream_t s) {
  if (Nelements == 0) return BP_SUCCESS;
  const int Np = simplex_np(dim, N);
  int epb = 0, threads = 0;
  tri_shape(Np, &epb, &threads);
  const int grid = (Nelements + epb - 1) / epb;
  simplex_rhs_analytic_kernel<<<grid, threads, sizeof(double) * epb * Np, s>>>(Nelements, Np, epb, wJ, MM, x, y,
                                                                              dim == 3 ? z : nullptr, lambda, bL);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

template <class F, int NSM>
static int launch_ax_simplex_t(int N, int32_t Nelements, const int32_t* elementList, const int32_t* G2L, const F* wJ,
                               const F* ggeo, const F* S, const F* MM, F lambda, const F* q, F* Aq, const int* skip,
                               cudaStream_t s, double* partials, int* nblocks) {
  if (nblocks) *nblocks = 0;
  if (N < 1 || N > 15) return fail(BP_ERROR_ARG, "simplex operator: degree N must be in 1..15");
  if (Nelements == 0) return BP_SUCCESS;
  const int Np = simplex_np(NSM == 3 ? 2 : 3, N);
  int groups = 0, threads = 0;
  tri_shape(Np, &groups, &threads);
  const int slots = groups * kTriElems;
  const int grid = (Nelements + slots - 1) / slots;
  if (nblocks) *nblocks = grid;
  const size_t smem = sizeof(double) * (size_t)(slots * Np > threads ? slots * Np : threads);
  if (partials)
    BP_CUDA_TRY(launch_pdl(ax_simplex_kernel<F, NSM, true>, grid, threads, smem, s, (int)Nelements, Np, groups, elementList,
                           G2L, wJ, ggeo, S, MM, lambda, q, Aq, skip, partials));
  else
    BP_CUDA_TRY(launch_pdl(ax_simplex_kernel<F, NSM, false>, grid, threads, smem, s, (int)Nelements, Np, groups, elementList,
                           G2L, wJ, ggeo, S, MM, lambda, q, Aq, skip, (double*)nullptr));
  return BP_SUCCESS;
}

template <class F>
static int launch_ax_simplex_any(int dim, int N, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                                 const F* wJ, const F* ggeo, const F* S, const F* MM, F lambda, const F* q, F* Aq,
                                 const int* skip, cudaStream_t s, double* partials, int* nblocks) {
  if (dim == 2)
    return launch_ax_simplex_t<F, 3>(N, Nelements, elementList, G2L, wJ, ggeo, S, MM, lambda, q, Aq, skip, s,
                                     partials, nblocks);
  return launch_ax_simplex_t<F, 6>(N, Nelements, elementList, G2L, wJ, ggeo, S, MM, lambda, q, Aq, skip, s, partials,
                                   nblocks);
}

int launch_ax_simplex(int dim, int N, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                      const double* wJ, const double* ggeo, const double* S, const double* MM, double lambda,
                      const double* q, double* Aq, const int* skip, cudaStream_t s, double* partials, int* nblocks) {
  return launch_ax_simplex_any<double>(dim, N, Nelements, elementList, G2L, wJ, ggeo, S, MM, lambda, q, Aq, skip, s,
                                       partials, nblocks);
}

int launch_ax_simplex(int dim, int N, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                      const float* wJ, const float* ggeo, const float* S, const float* MM, float lambda,
                      const float* q, float* Aq, const int* skip, cudaStream_t s, double* partials, int* nblocks) {
  return launch_ax_simplex_any<float>(dim, N, Nelements, elementList, G2L, wJ, ggeo, S, MM, lambda, q, Aq, skip, s,
                                      partials, nblocks);
}

int launch_mass_local_simplex(int dim, int N, int32_t Nelements, const int32_t* G2L, const double* wJ,
                              const double* MM, const double* f, double* bL, cudaStream_t s) {
  if (Nelements == 0) return BP_SUCCESS;
  const int Np = simplex_np(dim, N);
  int epb = 0, threads = 0;
  tri_shape(Np, &epb, &threads);
  const int grid = (Nelements + epb - 1) / epb;
  tri_mass_local_kernel<<<grid, threads, sizeof(double) * epb * Np, s>>>(Nelements, Np, epb, G2L, wJ, MM, f, bL);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

int launch_diag_local_simplex(int dim, int N, int32_t Nelements, const double* wJ, const double* ggeo,
                              const double* S, const double* MM, double lambda, double* dL, cudaStream_t s) {
  if (Nelements == 0) return BP_SUCCESS;
  const int Np = simplex_np(dim, N);
  const size_t total = (size_t)Nelements * Np;
  const int grid = (int)((total + 255) / 256 < 65535 ? (total + 255) / 256 : 65535);
  simplex_diag_local_kernel<<<grid, 256, 0, s>>>(Nelements, Np, dim == 2 ? 3 : 6, wJ, ggeo, S, MM, lambda, dL);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

}  // namespace bp
