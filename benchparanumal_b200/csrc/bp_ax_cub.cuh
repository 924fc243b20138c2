// Over-integrated element operators of BP1-BP4 (mass, and stiffness + lambda
// mass, evaluated at N+2 Gauss points per direction), templated on the degree,
// the operator form and the arithmetic type.  Instantiated by bp_ax_cub64.cu
// (FP64) and bp_ax_cub32.cu (FP32, the mixed-precision CG).
//
// Forms (reference kernels):
//   CUB_MASS_AFFINE   wJ_e (MM x MM x MM) q                  okl/bp1AxAffineHex3D.okl:29-135
//   CUB_MASS          I^T (cubwJ . (I q))                     okl/bp1AxHex3D.okl
//   CUB_STIFF_AFFINE  invV^T (S_modal + lambda wJ_e) invV q   okl/bp3AxAffineHex3D.okl:29-258
//   CUB_STIFF         I^T (S_cub + lambda cubwJ) I q          okl/bp3AxHex3D.okl:29-340
// with S = Dr^T(G00 Dr + G01 Ds + G02 Dt) + Ds^T(...) + Dt^T(...) on the
// quadrature grid.  BP2/BP4 apply the same operator to each of the 3 fields.
//
// Layout of one element slot es (threads (i, j) of a G x G plane, G the grid
// points per direction): the field lives in shared memory s_q[G][G][G] while
// it is transformed one direction at a time (b, then a, then c, in place);
// after the c transform thread (i, j) also holds its column q(i, j, 0:G-1) in
// registers, so the t-derivative and the t-part of the weak divergence stay in
// registers and only the r/s fluxes of the current k-slice go through shared
// memory.  The projection back runs b, a, c again, the c step from registers
// of the node thread (i, j), which also holds its q column for the q.Aq sum of
// the fused CG.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "bp_cg_device.cuh"
#include "bp_internal.hpp"

namespace bp {

enum CubForm { CUB_MASS_AFFINE = 0, CUB_MASS = 1, CUB_STIFF_AFFINE = 2, CUB_STIFF = 3 };

template <int NQ, int FORM>
struct CubShape {
  static constexpr bool CURVED = (FORM == CUB_MASS || FORM == CUB_STIFF);
  static constexpr bool STIFF = (FORM == CUB_STIFF_AFFINE || FORM == CUB_STIFF);
  static constexpr int G = CURVED ? NQ + 1 : NQ;   // quadrature points per direction
  static constexpr int G2 = G * G;
  static constexpr int GP = G * G * G;
  static constexpr int EPB0 = 256 / G2 < 1 ? 1 : 256 / G2;
  static constexpr int EPB = EPB0 > 16 ? 16 : EPB0;   // element slots per block
  static constexpr int THREADS = G2 * EPB;
};

template <int NQ, int FORM, class F>
__global__ void __launch_bounds__(CubShape<NQ, FORM>::THREADS)
ax_cub_kernel(int Nelements, int Nfields, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
              const F* __restrict__ wJ, const F* __restrict__ ggeo, const F* __restrict__ Dg,
              const F* __restrict__ Tg, F lambda, const F* __restrict__ q, F* __restrict__ Aq,
              const int* __restrict__ skip, double* __restrict__ partials, int vec) {
  if (skip && *skip) return;
  using Sh = CubShape<NQ, FORM>;
  using V2 = typename std::conditional<sizeof(F) == 8, double2, float2>::type;
  constexpr int G = Sh::G, G2 = Sh::G2, GP = Sh::GP, EPB = Sh::EPB;
  constexpr int NQ2 = NQ * NQ, NP = NQ * NQ * NQ;
  constexpr int GS = Sh::STIFF ? G : 1;
  __shared__ F s_T[G][NQ];                 // 1D transform, row = output point
  __shared__ F s_D[GS][GS + 1];            // differentiation on the grid
  __shared__ __align__(16) F s_q[EPB][G][G][G];   // the field of each element slot (also the
                                                  // double scratch of the q.Aq block sum)
  __shared__ F s_qr[EPB][GS][GS + 1];      // r-flux of the current k-slice
  __shared__ F s_qs[EPB][GS][GS + 1];      // s-flux of the current k-slice

  const int i = threadIdx.x, j = threadIdx.y, es = threadIdx.z;
  const int tid = i + G * (j + G * es);
  for (int t = tid; t < G * NQ; t += Sh::THREADS) {
    // BP1 affine multiplies by MM^T (okl/bp1AxAffineHex3D.okl: s_MM[m][i])
    if (FORM == CUB_MASS_AFFINE) s_T[t / NQ][t % NQ] = Tg[(t % NQ) * NQ + t / NQ];
    else s_T[t / NQ][t % NQ] = Tg[t];
  }
  if (Sh::STIFF)
    for (int t = tid; t < G * G; t += Sh::THREADS) s_D[t / G][t % G] = Dg[t];

  const int eidx = blockIdx.x * EPB + es;
  const bool valid = eidx < Nelements;
  const int element = valid ? elementList[eidx] : 0;
  const bool node = (i < NQ) && (j < NQ);   // owns the GLL column (i, j, :)
  double pdot = 0.0;

  // affine factors are per element
  F wa = 0, ga[6] = {0, 0, 0, 0, 0, 0};
  if (!Sh::CURVED) {
    wa = wJ[element];
    if (Sh::STIFF)
#pragma unroll
      for (int c = 0; c < 6; ++c) ga[c] = ggeo[6 * (size_t)element + c];
  }

  for (int f = 0; f < Nfields; ++f) {
    const size_t lbase = ((size_t)element * Nfields + f) * NP;
    F qcol[NQ];
    __syncthreads();   // s_T/s_D loaded; the previous field's reads of s_q are done
    if (node) {
#pragma unroll
      for (int c = 0; c < NQ; ++c) {
        F v = 0;
        if (valid) {
          const int32_t id = G2L[lbase + c * NQ2 + j * NQ + i];
          v = (id >= 0) ? q[id] : F(0);
        }
        qcol[c] = v;
        s_q[es][c][j][i] = v;
      }
    }
    __syncthreads();
    // transform in b: thread (a = i, c = j), column s_q[c][:][a]
    if (node) {
      F r[NQ];
#pragma unroll
      for (int b = 0; b < NQ; ++b) r[b] = s_q[es][j][b][i];
#pragma unroll
      for (int jj = 0; jj < G; ++jj) {
        F t = 0;
#pragma unroll
        for (int b = 0; b < NQ; ++b) t += s_T[jj][b] * r[b];
        s_q[es][j][jj][i] = t;
      }
    }
    __syncthreads();
    // transform in a: thread (jj = i, c = j), row s_q[c][jj][:]
    if (j < NQ) {
      F r[NQ];
#pragma unroll
      for (int a = 0; a < NQ; ++a) r[a] = s_q[es][j][i][a];
#pragma unroll
      for (int ii = 0; ii < G; ++ii) {
        F t = 0;
#pragma unroll
        for (int a = 0; a < NQ; ++a) t += s_T[ii][a] * r[a];
        s_q[es][j][i][ii] = t;
      }
    }
    __syncthreads();
    // transform in c: thread (ii = i, jj = j), column kept in registers
    F qk[G];
    {
      F r[NQ];
#pragma unroll
      for (int c = 0; c < NQ; ++c) r[c] = s_q[es][c][j][i];
#pragma unroll
      for (int k = 0; k < G; ++k) {
        F t = 0;
#pragma unroll
        for (int c = 0; c < NQ; ++c) t += s_T[k][c] * r[c];
        qk[k] = t;
      }
    }
    if (FORM == CUB_MASS_AFFINE) {
      // G == NQ: thread (i, j) is the node thread and holds the result column
      if (valid) {
#pragma unroll
        for (int k = 0; k < NQ; ++k) {
          const F out = wa * qk[k];
          Aq[lbase + k * NQ2 + j * NQ + i] = out;
          pdot += (double)qcol[k] * (double)out;
        }
      }
      continue;
    }
    F acc[G];
    if (FORM == CUB_MASS) {
      const size_t gb = (size_t)element * GP + j * G + i;
#pragma unroll
      for (int k = 0; k < G; ++k) acc[k] = wJ[gb + k * G2] * qk[k];
    } else {
#pragma unroll
      for (int k = 0; k < G; ++k) {
        acc[k] = 0;
        s_q[es][k][j][i] = qk[k];   // own column: every read of it above is this thread's
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < G; ++k) {
        F dr = 0, ds = 0, dt = 0;
#pragma unroll
        for (int n = 0; n < G; ++n) {
          dr += s_D[i][n] * s_q[es][k][j][n];
          ds += s_D[j][n] * s_q[es][k][n][i];
          dt += s_D[k][n] * qk[n];
        }
        F g0, g1, g2, g3, g4, g5, w;
        if (Sh::CURVED) {
          const size_t gb = (size_t)element * GP + k * G2 + j * G + i;
          if (vec) {
            const V2* gv = reinterpret_cast<const V2*>(ggeo + 6 * gb);
            const V2 a0 = gv[0], a1 = gv[1], a2 = gv[2];
            g0 = a0.x; g1 = a0.y; g2 = a1.x; g3 = a1.y; g4 = a2.x; g5 = a2.y;
          } else {
            const F* gp = ggeo + 6 * gb;
            g0 = gp[0]; g1 = gp[1]; g2 = gp[2]; g3 = gp[3]; g4 = gp[4]; g5 = gp[5];
          }
          w = wJ[gb];
        } else {
          g0 = ga[0]; g1 = ga[1]; g2 = ga[2]; g3 = ga[3]; g4 = ga[4]; g5 = ga[5];
          w = wa;
        }
        s_qr[es][j][i] = g0 * dr + g1 * ds + g2 * dt;
        s_qs[es][j][i] = g1 * dr + g3 * ds + g4 * dt;
        const F qt = g2 * dr + g4 * ds + g5 * dt;
        acc[k] += lambda * w * qk[k];
        __syncthreads();
        F a = 0;
#pragma unroll
        for (int n = 0; n < G; ++n) {
          a += s_D[n][i] * s_qr[es][j][n];
          a += s_D[n][j] * s_qs[es][n][i];
          acc[n] += s_D[k][n] * qt;
        }
        acc[k] += a;
        __syncthreads();
      }
    }
    // project: the grid field back to s_q, then b, a (shared) and c (registers)
#pragma unroll
    for (int k = 0; k < G; ++k) s_q[es][k][j][i] = acc[k];
    __syncthreads();
    // back in b: thread (ii = i, k = j), column s_q[k][:][ii]
    {
      F r[G];
#pragma unroll
      for (int jj = 0; jj < G; ++jj) r[jj] = s_q[es][j][jj][i];
#pragma unroll
      for (int b = 0; b < NQ; ++b) {
        F t = 0;
#pragma unroll
        for (int jj = 0; jj < G; ++jj) t += s_T[jj][b] * r[jj];
        s_q[es][j][b][i] = t;
      }
    }
    __syncthreads();
    // back in a: thread (b = i, k = j), row s_q[k][b][:]
    if (i < NQ) {
      F r[G];
#pragma unroll
      for (int ii = 0; ii < G; ++ii) r[ii] = s_q[es][j][i][ii];
#pragma unroll
      for (int a = 0; a < NQ; ++a) {
        F t = 0;
#pragma unroll
        for (int ii = 0; ii < G; ++ii) t += s_T[ii][a] * r[ii];
        s_q[es][j][i][a] = t;
      }
    }
    __syncthreads();
    // back in c: node thread (a = i, b = j), column s_q[:][b][a]
    if (node && valid) {
      F r[G];
#pragma unroll
      for (int k = 0; k < G; ++k) r[k] = s_q[es][k][j][i];
#pragma unroll
      for (int c = 0; c < NQ; ++c) {
        F t = 0;
#pragma unroll
        for (int k = 0; k < G; ++k) t += s_T[k][c] * r[k];
        Aq[lbase + c * NQ2 + j * NQ + i] = t;
        pdot += (double)qcol[c] * (double)t;
      }
    }
  }
  if (partials) {
    // s_q as the block-sum scratch: at least one double per thread
    static_assert(sizeof(F) * EPB * GP >= sizeof(double) * Sh::THREADS, "scratch too small");
    const double bs = fuse_block_sum(pdot, reinterpret_cast<double*>(&s_q[0][0][0][0]));
    if (tid == 0) partials[blockIdx.x] = bs;
  }
}

template <int NQ, int FORM, class F>
static int launch_cub_form(int32_t Nelements, int Nfields, const int32_t* elementList, const int32_t* G2L,
                           const CubOperands<F>& o, F lambda, const F* q, F* Aq, const int* skip,
                           cudaStream_t s, double* partials, int* nblocks) {
  using Sh = CubShape<NQ, FORM>;
  const dim3 block(Sh::G, Sh::G, Sh::EPB);
  const dim3 grid((Nelements + Sh::EPB - 1) / Sh::EPB);
  if (nblocks) *nblocks = (int)grid.x;
  const int vec = (reinterpret_cast<uintptr_t>(o.ggeo) % (2 * sizeof(F))) == 0;
  ax_cub_kernel<NQ, FORM, F><<<grid, block, 0, s>>>(Nelements, Nfields, elementList, G2L, o.wJ, o.ggeo, o.D, o.T,
                                                    lambda, q, Aq, skip, partials, vec);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

template <int NQ, class F>
static int launch_cub_nq(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                         const CubOperands<F>& o, F lambda, const F* q, F* Aq, const int* skip, cudaStream_t s,
                         double* partials, int* nblocks) {
  const bool stiff = d.bp >= 3;
#define BP_CUB(FORM) \
  return launch_cub_form<NQ, FORM, F>(Nelements, d.Nfields, elementList, G2L, o, lambda, q, Aq, skip, s, partials, nblocks)
  if (d.affine) {
    if (stiff) BP_CUB(CUB_STIFF_AFFINE);
    BP_CUB(CUB_MASS_AFFINE);
  }
  if (stiff) BP_CUB(CUB_STIFF);
  BP_CUB(CUB_MASS);
#undef BP_CUB
}

template <class F>
int launch_ax_cub_t(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                    const CubOperands<F>& o, F lambda, const F* q, F* Aq, const int* skip, cudaStream_t s,
                    const CgFuse* fuse, int* nblocks) {
  if (nblocks) *nblocks = 0;
  if (d.bp < 1 || d.bp > 4) return fail(BP_ERROR_ARG, "over-integrated operator: bp must be 1..4");
  if (d.Nfields != ((d.bp % 2) ? 1 : 3)) return fail(BP_ERROR_ARG, "over-integrated operator: BP1/BP3 take 1 field, BP2/BP4 3");
  if (Nelements == 0) return BP_SUCCESS;
  double* partials = fuse ? fuse->partials : nullptr;
  switch (d.N + 1) {
#define BP_CUB_CASE(nq) \
  case nq:              \
    return launch_cub_nq<nq, F>(d, Nelements, elementList, G2L, o, lambda, q, Aq, skip, s, partials, nblocks);
    BP_CUB_CASE(2) BP_CUB_CASE(3) BP_CUB_CASE(4) BP_CUB_CASE(5) BP_CUB_CASE(6) BP_CUB_CASE(7) BP_CUB_CASE(8)
    BP_CUB_CASE(9) BP_CUB_CASE(10) BP_CUB_CASE(11) BP_CUB_CASE(12) BP_CUB_CASE(13) BP_CUB_CASE(14)
    BP_CUB_CASE(15) BP_CUB_CASE(16)
#undef BP_CUB_CASE
    default:
      return fail(BP_ERROR_ARG, "over-integrated operator: degree N must be in 1..15");
  }
}

}  // namespace bp
