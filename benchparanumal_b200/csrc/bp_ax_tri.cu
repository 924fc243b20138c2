// Tri2D (affine triangles) BP5 element operator, forcing mass and Jacobi
// diagonal.
//
// The reference's affine triangle operator (okl/bp5AxAffineTri2D.okl:27-89)
// applies four dense Np x Np reference matrices per element:
//   Aq_e = G00 Srr q_e + G01 Srs q_e + G11 Sss q_e + lambda J MM q_e
// with the per-element factors (G00, G01, G11, J).  Np = (N+1)(N+2)/2 is not a
// tensor product, so there is no sum factorisation: one thread per node of an
// element slot, the element's gathered values in shared memory, and the
// matrices read with node-fastest layout (X[k*Np + n] is the weight of node k
// in output n: the reference's device copies o_S and o_MM), so the threads of
// an element read consecutive words for every k.  The matrices (4*Np^2
// doubles, 41 KB at p = 7) are shared by all elements and stay in L1/L2.
// Sums over k run in increasing k, the output combines the four sums in the
// reference's order.
#include <cuda_runtime.h>

#include <cstdint>

#include "bp_cg_device.cuh"
#include "bp_internal.hpp"

namespace bp {
namespace {

constexpr int kTriThreads = 256;

// element slots per block and threads per block (whole warps)
static void tri_shape(int Np, int* epb, int* threads) {
  *epb = Np >= kTriThreads ? 1 : kTriThreads / Np;
  *threads = (*epb * Np + 31) / 32 * 32;
}

template <bool DOT>
__global__ void __launch_bounds__(kTriThreads + 32)
ax_tri_kernel(int Nelements, int Np, int epb, const int32_t* __restrict__ elementList,
              const int32_t* __restrict__ G2L, const double* __restrict__ wJ, const double* __restrict__ ggeo,
              const double* __restrict__ S, const double* __restrict__ MM, double lambda,
              const double* __restrict__ q, double* __restrict__ Aq, const int* __restrict__ skip,
              double* __restrict__ partials) {
  pdl_wait();
  pdl_release();
  if (skip && *skip) return;
  extern __shared__ __align__(16) double s_q[];   // [epb*Np]; the block sum reuses it
  const int t = threadIdx.x;
  const int es = t / Np, n = t - es * Np;
  const int eidx = blockIdx.x * epb + es;
  const bool active = es < epb && eidx < Nelements;
  const int element = active ? elementList[eidx] : 0;
  if (active) {
    const int32_t id = G2L[(size_t)element * Np + n];
    s_q[es * Np + n] = id >= 0 ? q[id] : 0.0;
  }
  __syncthreads();
  double pdot = 0.0;
  double out = 0.0;
  if (active) {
    const double* sq = s_q + es * Np;
    const size_t NP2 = (size_t)Np * Np;
    double qrr = 0.0, qrs = 0.0, qss = 0.0, qM = 0.0;
    for (int k = 0; k < Np; ++k) {
      const double qk = sq[k];
      const size_t o = (size_t)k * Np + n;
      qrr += __ldg(S + o) * qk;
      qrs += __ldg(S + NP2 + o) * qk;
      qss += __ldg(S + 2 * NP2 + o) * qk;
      qM += __ldg(MM + o) * qk;
    }
    const double* g = ggeo + 3 * (size_t)element;
    out = g[0] * qrr + g[1] * qrs + g[2] * qss + wJ[element] * lambda * qM;
    Aq[(size_t)element * Np + n] = out;
    if (DOT) pdot = sq[n] * out;
  }
  if (DOT) {
    const double bs = fuse_block_sum(pdot, s_q);
    if (t == 0) partials[blockIdx.x] = bs;
  }
}

// b_e = J_e MM f_e with f scattered through GlobalToLocal (masked nodes 0)
__global__ void __launch_bounds__(kTriThreads + 32)
tri_mass_local_kernel(int Nelements, int Np, int epb, const int32_t* __restrict__ G2L,
                      const double* __restrict__ wJ, const double* __restrict__ MM, const double* __restrict__ f,
                      double* __restrict__ bL) {
  extern __shared__ __align__(16) double s_f[];
  const int t = threadIdx.x;
  const int es = t / Np, n = t - es * Np;
  const int e = blockIdx.x * epb + es;
  const bool active = es < epb && e < Nelements;
  if (active) {
    const int32_t id = G2L[(size_t)e * Np + n];
    s_f[es * Np + n] = id >= 0 ? f[id] : 0.0;
  }
  __syncthreads();
  if (!active) return;
  double acc = 0.0;
  for (int k = 0; k < Np; ++k) acc += __ldg(MM + (size_t)k * Np + n) * s_f[es * Np + k];
  bL[(size_t)e * Np + n] = wJ[e] * acc;
}

// diagonal of A_e: G00 Srr(n,n) + G01 Srs(n,n) + G11 Sss(n,n) + lambda J MM(n,n)
__global__ void tri_diag_local_kernel(int Nelements, int Np, const double* __restrict__ wJ,
                                      const double* __restrict__ ggeo, const double* __restrict__ S,
                                      const double* __restrict__ MM, double lambda, double* __restrict__ dL) {
  const size_t NP2 = (size_t)Np * Np;
  const size_t total = (size_t)Nelements * Np;
  for (size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x; l < total; l += (size_t)blockDim.x * gridDim.x) {
    const size_t e = l / Np, n = l - e * Np;
    const size_t dn = n * Np + n;
    const double* g = ggeo + 3 * e;
    dL[l] = g[0] * S[dn] + g[1] * S[NP2 + dn] + g[2] * S[2 * NP2 + dn] + lambda * wJ[e] * MM[dn];
  }
}

}  // namespace

int launch_ax_tri(int N, int32_t Nelements, const int32_t* elementList, const int32_t* G2L, const double* wJ,
                  const double* ggeo, const double* S, const double* MM, double lambda, const double* q, double* Aq,
                  const int* skip, cudaStream_t s, double* partials, int* nblocks) {
  if (nblocks) *nblocks = 0;
  if (N < 1 || N > 15) return fail(BP_ERROR_ARG, "Tri2D operator: degree N must be in 1..15");
  if (Nelements == 0) return BP_SUCCESS;
  const int Np = (N + 1) * (N + 2) / 2;
  int epb = 0, threads = 0;
  tri_shape(Np, &epb, &threads);
  const int grid = (Nelements + epb - 1) / epb;
  if (nblocks) *nblocks = grid;
  const size_t smem = sizeof(double) * (size_t)(epb * Np > threads ? epb * Np : threads);
  if (partials)
    BP_CUDA_TRY(launch_pdl(ax_tri_kernel<true>, grid, threads, smem, s, (int)Nelements, Np, epb, elementList, G2L, wJ,
                           ggeo, S, MM, lambda, q, Aq, skip, partials));
  else
    BP_CUDA_TRY(launch_pdl(ax_tri_kernel<false>, grid, threads, smem, s, (int)Nelements, Np, epb, elementList, G2L,
                           wJ, ggeo, S, MM, lambda, q, Aq, skip, (double*)nullptr));
  return BP_SUCCESS;
}

int launch_mass_local_tri(int N, int32_t Nelements, const int32_t* G2L, const double* wJ, const double* MM,
                          const double* f, double* bL, cudaStream_t s) {
  if (Nelements == 0) return BP_SUCCESS;
  const int Np = (N + 1) * (N + 2) / 2;
  int epb = 0, threads = 0;
  tri_shape(Np, &epb, &threads);
  const int grid = (Nelements + epb - 1) / epb;
  tri_mass_local_kernel<<<grid, threads, sizeof(double) * epb * Np, s>>>(Nelements, Np, epb, G2L, wJ, MM, f, bL);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

int launch_diag_local_tri(int N, int32_t Nelements, const double* wJ, const double* ggeo, const double* S,
                          const double* MM, double lambda, double* dL, cudaStream_t s) {
  if (Nelements == 0) return BP_SUCCESS;
  const int Np = (N + 1) * (N + 2) / 2;
  const size_t total = (size_t)Nelements * Np;
  const int grid = (int)((total + 255) / 256 < 65535 ? (total + 255) / 256 : 65535);
  tri_diag_local_kernel<<<grid, 256, 0, s>>>(Nelements, Np, wJ, ggeo, S, MM, lambda, dL);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

}  // namespace bp
