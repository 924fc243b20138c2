// Over-integrated element operators of BP1-BP4 (mass, and stiffness + lambda
// mass, evaluated at N+2 Gauss points per direction).  Included once by
// bp_ax_cub64.cu (BP_CUB_REAL = double) and once by bp_ax_cub32.cu
// (BP_CUB_REAL = float, the mixed-precision CG); each inclusion is its own
// CUDA module with its own constant bank.
//
// Forms (reference kernels):
//   CUB_MASS_AFFINE   wJ_e (MM x MM x MM) q                  okl/bp1AxAffineHex3D.okl:29-135
//   CUB_MASS          I^T (cubwJ . (I q))                     okl/bp1AxHex3D.okl
//   CUB_STIFF_AFFINE  invV^T (S_modal + lambda wJ_e) invV q   okl/bp3AxAffineHex3D.okl:29-258
//   CUB_STIFF         I^T (S_cub + lambda cubwJ) I q          okl/bp3AxHex3D.okl:29-340
// with S = Dr^T(G00 Dr + G01 Ds + G02 Dt) + Ds^T(...) + Dt^T(...) on the
// quadrature grid.  BP2/BP4 apply the same operator to each of the 3 fields.
//
// Work mapping.  Every 1D step (interpolation, derivative, projection, weak
// derivative) is a small matrix applied along lines of the element's grid.
// A thread owns whole lines: it reads one line into registers and writes all
// of that line's outputs, so the matrix index of every multiply-add is the
// same in all threads of the warp.  The matrices therefore live in the
// constant bank (c_cub below), read uniformly through the constant cache;
// shared memory only carries the field between steps whose line direction
// changes.
// The G x G threads of an element slot take the roles
//   (b-line of node a, c) -> (a-line of point j, c) -> (c-line of point i, j)
// through the interpolation, keep the c-line (the t-direction) in registers
// for the t-derivative and the t-part of the weak divergence, and run the
// r- and s-parts as row/column roles over shared memory.  The projection runs
// the same roles backwards and ends on b-lines of node (a, c), the lines the
// thread loaded q along; its q.Aq sum for the fused CG re-reads q there.
#pragma once

#ifndef BP_CUB_REAL
#error "define BP_CUB_REAL (double or float) before including bp_ax_cub.cuh"
#endif

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "bp_cg_device.cuh"
#include "bp_internal.hpp"

namespace bp {
namespace {

using CubReal = BP_CUB_REAL;

// Outer (output) loops of the line steps.  Fully unrolled, every matrix index
// is a compile-time constant, but the unrolled FP64 steps need more registers
// than two resident blocks allow; measured at p=7 (BK3 40^3 curved): FP64
// 1.4 ms rolled against 2.1-2.2 ms unrolled, FP32 (mixed BP3 CG to 1e-8)
// 1.57 s unrolled against 1.81 s rolled.  So FP64 keeps them rolled and FP32
// unrolls them.
#ifndef BP_CUB_OUTER
#define BP_CUB_OUTER _Pragma("unroll 1")
#endif

enum CubForm { CUB_MASS_AFFINE = 0, CUB_MASS = 1, CUB_STIFF_AFFINE = 2, CUB_STIFF = 3 };

// Constant-bank table, three groups of one slot per degree: the curved forms
// (T = cubInterp [G x NQ], then cubD [G x G]; mass and stiffness share the
// slot, both write the mesh's cubInterp), the affine stiffness forms of
// BP3/BP4 (T = invV [NQ x NQ], then the modal cubD [NQ x NQ]) and the affine
// mass forms of BP1/BP2 (T = MM [NQ x NQ]).  Each launch first copies its
// operands into its slot on the launch stream (once per slot and source in a
// stream capture: const_slot_copy), so two launches of the same
// degree and group on different streams must pass the same matrices (every
// caller that passes its mesh's own matrices does); operators of different
// groups never share a slot.
__host__ __device__ constexpr int cub_curved_size(int nq) { return (nq + 1) * nq + (nq + 1) * (nq + 1); }
__host__ __device__ constexpr int cub_affine_size(int nq) { return 2 * nq * nq; }
__host__ __device__ constexpr int cub_mass_affine_size(int nq) { return nq * nq; }
__host__ __device__ constexpr int cub_slot(int nq, int form) {
  const int group = (form == CUB_MASS || form == CUB_STIFF) ? 0 : form == CUB_STIFF_AFFINE ? 1 : 2;
  int off = 0;
  for (int n = 2; n < (group == 0 ? nq : 17); ++n) off += cub_curved_size(n);
  if (group >= 1)
    for (int n = 2; n < (group == 1 ? nq : 17); ++n) off += cub_affine_size(n);
  if (group == 2)
    for (int n = 2; n < nq; ++n) off += cub_mass_affine_size(n);
  return off;
}
constexpr int kCubTable = cub_slot(17, CUB_MASS_AFFINE);
static_assert(kCubTable * sizeof(double) <= 64 * 1024, "constant table exceeds the 64 KB bank");

static __constant__ CubReal c_cub[kCubTable];

template <int NQ, int FORM>
struct CubShape {
  static constexpr bool CURVED = (FORM == CUB_MASS || FORM == CUB_STIFF);
  static constexpr bool STIFF = (FORM == CUB_STIFF_AFFINE || FORM == CUB_STIFF);
  static constexpr int G = CURVED ? NQ + 1 : NQ;   // quadrature points per direction
  static constexpr int G2 = G * G;
  static constexpr int RS = (G % 2) ? G : G + 1;   // row stride: odd, so rows of a warp spread over banks
  static constexpr int PLANE = G * RS;
  static constexpr int FIELD = G * PLANE;           // one G^3 field in shared memory
  static constexpr int NBUF = STIFF ? 3 : 1;        // u, and the r/s buffers of the stiffness
  // words between consecutive element slots' buffers beyond NBUF fields: the
  // warps that straddle two slots then spread their shared-memory accesses
  // over more banks (padding chosen per Nq by counting the wavefronts of every
  // access pattern of the FP32 kernels: 12-25% fewer at Nq = 2, 4, 5, 6, 8)
  static constexpr int SPAD = sizeof(CubReal) != 4 ? 0
                              : NQ == 2 ? 10 : NQ == 4 ? 2 : NQ == 5 ? 8 : NQ == 6 ? 12 : NQ == 8 ? 6 : NQ == 9 ? 8 : 0;
  static constexpr int SLOTW = NBUF * FIELD + SPAD;   // words per element slot
  static constexpr int EPB0 = 256 / G2 < 1 ? 1 : 256 / G2;
  static constexpr int EPB = EPB0 > 8 ? 8 : EPB0;   // element slots per block
  static constexpr int THREADS = G2 * EPB;
  // resident blocks per SM the register budget must allow (caps registers per thread)
  static constexpr int MINB = G <= 12 ? 2 : 1;
  static constexpr int SLOT = cub_slot(NQ, FORM);
  static constexpr int TSIZE = G * NQ;              // T rows = output points
  static constexpr int DSIZE = STIFF ? G * G : 0;
  // FP32 curved forms stage each element's Gauss-point factors in shared memory
  // with cp.async at the element's start, so their latency overlaps the gather
  // and the interpolation (the FP64 factors would halve the resident blocks)
  static constexpr bool STAGE = CURVED && sizeof(CubReal) == 4;
  static constexpr int GP = G * G * G;
  static constexpr size_t FIELDS = sizeof(CubReal) * (size_t)SLOTW * EPB;
  static constexpr size_t GOFF = (FIELDS + 15) & ~(size_t)15;                        // [EPB][GP*6] ggeo
  static constexpr size_t WOFF = GOFF + (STAGE && STIFF ? sizeof(CubReal) * (size_t)EPB * GP * 6 : 0);   // [EPB][GP] wJ
  static constexpr size_t SMEM = STAGE ? WOFF + sizeof(CubReal) * (size_t)EPB * GP : FIELDS;
  // The pipelined FP32 form (ax_cub_pipe_kernel): the element groups' indices
  // and gathered q, double-buffered, and a ring of element ids behind the
  // staged factors.
  static constexpr int NP = NQ * NQ * NQ;
  static constexpr size_t IOFF = (SMEM + 15) & ~(size_t)15;                 // [EPB][NP] GlobalToLocal
  static constexpr size_t QOFF = IOFF + sizeof(int32_t) * (size_t)EPB * NP;   // [2][EPB][NP] q
  static constexpr size_t EOFF = QOFF + sizeof(CubReal) * 2 * (size_t)EPB * NP;   // [4][EPB] element ids
  static constexpr size_t PSMEM = EOFF + sizeof(int32_t) * 4 * (size_t)EPB;
  // blocks per SM that shared memory allows (228 KB per SM, 1 KB reserved per
  // block); the pipelined form is used only where it keeps the slot kernel's
  // residency (Nq = 10 would fall from two blocks to one, Nq = 16 not fit)
  static constexpr int smem_blocks(size_t bytes) { return (int)((228 * 1024) / (bytes + 1024)); }
  static constexpr int min_(int a, int b) { return a < b ? a : b; }
  static constexpr bool PIPE_OK =
      PSMEM <= 227 * 1024 && min_(smem_blocks(PSMEM), MINB) >= min_(smem_blocks(SMEM), MINB);
};

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The 1D matrices of a form in the constant bank: T(o, i) maps NQ nodes to G
// points (MASS_AFFINE applies MM^T), D(a, b) is G x G; AT indexes a G^3 field.
#define CUB_T(o, i)                                                          \
  (FORM == CUB_MASS_AFFINE ? c_cub[CubShape<NQ, FORM>::SLOT + (i) * NQ + (o)] \
                           : c_cub[CubShape<NQ, FORM>::SLOT + (o) * NQ + (i)])
#define CUB_D(a, b) c_cub[CubShape<NQ, FORM>::SLOT + CubShape<NQ, FORM>::TSIZE + (a) * CubShape<NQ, FORM>::G + (b)]
#define CUB_AT(B, z, y, x) B[(z) * CubShape<NQ, FORM>::PLANE + (y) * CubShape<NQ, FORM>::RS + (x)]

// Interpolation of one element slot to its G^3 points: along b from the
// q-line qb of node (a, c) = (tx, ty) (threads tx, ty < NQ), along a over
// shared memory (rows (j, c) = (tx, ty)), along c into the register column qk
// of point (i, j) = (tx, ty).  Reads of U after the call are the thread's own
// column.
template <int NQ, int FORM>
__device__ __forceinline__ void cub_interp(const CubReal (&qb)[NQ], CubReal* U,
                                           CubReal (&qk)[CubShape<NQ, FORM>::G], int tx, int ty) {
  using F = CubReal;
  constexpr int G = CubShape<NQ, FORM>::G;
  if (tx < NQ && ty < NQ) {
BP_CUB_OUTER
    for (int jj = 0; jj < G; ++jj) {
      F t = 0;
#pragma unroll
      for (int b = 0; b < NQ; ++b) t += CUB_T(jj, b) * qb[b];
      CUB_AT(U, ty, jj, tx) = t;
    }
  }
  __syncthreads();
  if (ty < NQ) {
    F r[NQ];
#pragma unroll
    for (int a = 0; a < NQ; ++a) r[a] = CUB_AT(U, ty, tx, a);
BP_CUB_OUTER
    for (int ii = 0; ii < G; ++ii) {
      F t = 0;
#pragma unroll
      for (int a = 0; a < NQ; ++a) t += CUB_T(ii, a) * r[a];
      CUB_AT(U, ty, tx, ii) = t;
    }
  }
  __syncthreads();
  F r[NQ];
#pragma unroll
  for (int c = 0; c < NQ; ++c) r[c] = CUB_AT(U, c, ty, tx);
#pragma unroll
  for (int k = 0; k < G; ++k) {
    F t = 0;
#pragma unroll
    for (int c = 0; c < NQ; ++c) t += CUB_T(k, c) * r[c];
    qk[k] = t;
  }
}

// Factors at the points of column (tx, ty), three sources.  ready() runs before
// the barrier ahead of the flux loop, released() after the barrier behind it
// (no thread reads factors after that).
template <class F>
struct CubStagedFactors {   // staged in shared memory by cp.async at the element's start
  const F* sG;
  const F* sW;
  __device__ __forceinline__ void ready() const { cp_async_wait_all(); }
  __device__ __forceinline__ void released() const {}
  __device__ __forceinline__ void get(int pt, F (&g)[6], F& w) const {
    using V2 = typename std::conditional<sizeof(F) == 8, double2, float2>::type;
    const V2* gv = reinterpret_cast<const V2*>(sG + 6 * pt);
    const V2 a0 = gv[0], a1 = gv[1], a2 = gv[2];
    g[0] = a0.x; g[1] = a0.y; g[2] = a1.x; g[3] = a1.y; g[4] = a2.x; g[5] = a2.y;
    w = sW[pt];
  }
};
template <class F>
struct CubGlobalFactors {   // read from global memory at the flux loop
  const F* ggeo;              // the element's block
  const F* wJ;
  __device__ __forceinline__ void ready() const {}
  __device__ __forceinline__ void released() const {}
  __device__ __forceinline__ void get(int pt, F (&g)[6], F& w) const {
    using V2 = typename std::conditional<sizeof(F) == 8, double2, float2>::type;
    const V2* gv = reinterpret_cast<const V2*>(ggeo + 6 * pt);
    const V2 a0 = gv[0], a1 = gv[1], a2 = gv[2];
    g[0] = a0.x; g[1] = a0.y; g[2] = a1.x; g[3] = a1.y; g[4] = a2.x; g[5] = a2.y;
    w = wJ[pt];
  }
};
template <class F>
struct CubAffineFactors {   // one set per element, in registers
  F ga[6];
  F wa;
  __device__ __forceinline__ void ready() const {}
  __device__ __forceinline__ void released() const {}
  __device__ __forceinline__ void get(int, F (&g)[6], F& w) const {
#pragma unroll
    for (int c = 0; c < 6; ++c) g[c] = ga[c];
    w = wa;
  }
};

// Stiffness plus lambda mass at the points of column (i, j) = (tx, ty):
// acc = Dr^T(G00 dr + G01 ds + G02 dt) + Ds^T(...) + Dt^T(...) + lambda w qk.
// The r- and s-parts run over shared memory (U, R, S), the t-part in
// registers; U's own column receives qk first.
template <int NQ, int FORM, class Fac>
__device__ __forceinline__ void cub_stiff(const CubReal (&qk)[CubShape<NQ, FORM>::G],
                                          CubReal (&acc)[CubShape<NQ, FORM>::G], CubReal* U, CubReal* R,
                                          CubReal* S, int tx, int ty, CubReal lambda, const Fac& fac) {
  using F = CubReal;
  constexpr int G = CubShape<NQ, FORM>::G;
  // own column: every earlier read of it was this thread's
#pragma unroll
  for (int k = 0; k < G; ++k) CUB_AT(U, k, ty, tx) = qk[k];
  __syncthreads();
  // r-derivative on the row (y, z) = (tx, ty); s-derivative on the column (x, z) = (tx, ty)
  {
    F r[G];
#pragma unroll
    for (int n = 0; n < G; ++n) r[n] = CUB_AT(U, ty, tx, n);
BP_CUB_OUTER
    for (int i = 0; i < G; ++i) {
      F t = 0;
#pragma unroll
      for (int n = 0; n < G; ++n) t += CUB_D(i, n) * r[n];
      CUB_AT(R, ty, tx, i) = t;
    }
#pragma unroll
    for (int n = 0; n < G; ++n) r[n] = CUB_AT(U, ty, n, tx);
BP_CUB_OUTER
    for (int j = 0; j < G; ++j) {
      F t = 0;
#pragma unroll
      for (int n = 0; n < G; ++n) t += CUB_D(j, n) * r[n];
      CUB_AT(S, ty, j, tx) = t;
    }
  }
  // t-derivative on the column (x, y) = (tx, ty) in registers, from U's own
  // column (which keeps qk until the projection) rather than from registers
  // held through the r/s phase
  F gt[G];
  {
    F u[G];
#pragma unroll
    for (int n = 0; n < G; ++n) u[n] = CUB_AT(U, n, ty, tx);
#pragma unroll
    for (int k = 0; k < G; ++k) {
      F t = 0;
#pragma unroll
      for (int n = 0; n < G; ++n) t += CUB_D(k, n) * u[n];
      gt[k] = t;
    }
  }
  fac.ready();   // this thread's copies; the barrier below makes all visible
  __syncthreads();
  // fluxes at the points of column (tx, ty)
#pragma unroll
  for (int k = 0; k < G; ++k) {
    F g[6], w;
    fac.get(k * G * G + ty * G + tx, g, w);
    const F dr = CUB_AT(R, k, ty, tx), ds = CUB_AT(S, k, ty, tx), dt = gt[k];
    CUB_AT(R, k, ty, tx) = g[0] * dr + g[1] * ds + g[2] * dt;
    CUB_AT(S, k, ty, tx) = g[1] * dr + g[3] * ds + g[4] * dt;
    gt[k] = g[2] * dr + g[4] * ds + g[5] * dt;
    acc[k] = lambda * w * CUB_AT(U, k, ty, tx);
  }
  // t-part of the weak divergence, in registers
#pragma unroll
  for (int n = 0; n < G; ++n) {
    F t = acc[n];
#pragma unroll
    for (int k = 0; k < G; ++k) t += CUB_D(k, n) * gt[k];
    acc[n] = t;
  }
  __syncthreads();
  fac.released();
  // r-part on rows, s-part on columns, in place
  {
    F r[G];
#pragma unroll
    for (int n = 0; n < G; ++n) r[n] = CUB_AT(R, ty, tx, n);
BP_CUB_OUTER
    for (int i = 0; i < G; ++i) {
      F t = 0;
#pragma unroll
      for (int n = 0; n < G; ++n) t += CUB_D(n, i) * r[n];
      CUB_AT(R, ty, tx, i) = t;
    }
#pragma unroll
    for (int n = 0; n < G; ++n) r[n] = CUB_AT(S, ty, n, tx);
BP_CUB_OUTER
    for (int j = 0; j < G; ++j) {
      F t = 0;
#pragma unroll
      for (int n = 0; n < G; ++n) t += CUB_D(n, j) * r[n];
      CUB_AT(S, ty, j, tx) = t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < G; ++k) acc[k] += CUB_AT(R, k, ty, tx) + CUB_AT(S, k, ty, tx);
}

// Projection to the nodes along c (from the register column acc of point
// (i, j) = (tx, ty)) and along a (rows (j, c) = (tx, ty)); the caller
// finishes along b from U: node (a, c) = (tx, ty) reads U(c, :, a).
template <int NQ, int FORM>
__device__ __forceinline__ void cub_project_ca(const CubReal (&acc)[CubShape<NQ, FORM>::G], CubReal* U, int tx,
                                               int ty) {
  using F = CubReal;
  constexpr int G = CubShape<NQ, FORM>::G;
  // own column of U
BP_CUB_OUTER
  for (int c = 0; c < NQ; ++c) {
    F t = 0;
#pragma unroll
    for (int k = 0; k < G; ++k) t += CUB_T(k, c) * acc[k];
    CUB_AT(U, c, ty, tx) = t;
  }
  __syncthreads();
  if (ty < NQ) {
    F r[G];
#pragma unroll
    for (int ii = 0; ii < G; ++ii) r[ii] = CUB_AT(U, ty, tx, ii);
BP_CUB_OUTER
    for (int a = 0; a < NQ; ++a) {
      F t = 0;
#pragma unroll
      for (int ii = 0; ii < G; ++ii) t += CUB_T(ii, a) * r[ii];
      CUB_AT(U, ty, tx, a) = t;
    }
  }
  __syncthreads();
}

template <int NQ, int FORM>
__global__ void __launch_bounds__(CubShape<NQ, FORM>::THREADS, CubShape<NQ, FORM>::MINB)
ax_cub_kernel(int Nelements, int Nfields, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
              const CubReal* __restrict__ wJ, const CubReal* __restrict__ ggeo, CubReal lambda,
              const CubReal* __restrict__ q, CubReal* __restrict__ Aq, const int* __restrict__ skip,
              double* __restrict__ partials) {
  pdl_wait();
  pdl_release();
  if (skip && *skip) return;
  using F = CubReal;
  using Sh = CubShape<NQ, FORM>;
  constexpr int G = Sh::G, GP = Sh::GP, EPB = Sh::EPB;
  constexpr int NQ2 = NQ * NQ, NP = NQ * NQ * NQ;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  F* const sbase = reinterpret_cast<F*>(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y, es = threadIdx.z;
  F* const U = sbase + (size_t)es * Sh::SLOTW;   // the field
  F* const R = U + Sh::FIELD;                                // r-derivative / r-flux
  F* const S = R + Sh::FIELD;                                // s-derivative / s-flux

  const int eidx = blockIdx.x * EPB + es;
  const bool valid = eidx < Nelements;
  const int element = valid ? elementList[eidx] : 0;
  double pdot = 0.0;

  // the element's factors into shared memory, in flight while q is gathered and interpolated
  F* const sG = reinterpret_cast<F*>(smem_raw + Sh::GOFF) + (size_t)es * GP * 6;
  F* const sW = reinterpret_cast<F*>(smem_raw + Sh::WOFF) + (size_t)es * GP;
  if (Sh::STAGE && valid) {
    const int tl = tx + G * ty;
    if (Sh::STIFF) {
      const F* src = ggeo + 6 * (size_t)element * GP;   // 8-byte aligned: 24 bytes per point
      for (int c = tl; c < GP * 3; c += G * G) cp_async8(sG + 2 * c, src + 2 * c);
    }
    const F* srcw = wJ + (size_t)element * GP;
    for (int c = tl; c < GP; c += G * G) cp_async4(sW + c, srcw + c);
  }

  for (int f = 0; f < Nfields; ++f) {
    const size_t lbase = ((size_t)element * Nfields + f) * NP;
    if (f > 0) __syncthreads();   // the previous field's last reads of U are done
    // q[c][b][a] along b of node (a, c) = (tx, ty)
    F qb[NQ];
#pragma unroll
    for (int b = 0; b < NQ; ++b) {
      F v = 0;
      if (valid && tx < NQ && ty < NQ) {
        const int32_t id = G2L[lbase + ty * NQ2 + b * NQ + tx];
        v = (id >= 0) ? q[id] : F(0);
      }
      qb[b] = v;
    }
    F qk[G];
    cub_interp<NQ, FORM>(qb, U, qk, tx, ty);
    if (FORM == CUB_MASS_AFFINE) {
      // G == NQ: the result column of node (tx, ty) is wJ_e * qk
      if (valid) {
        const F wa = wJ[element];
#pragma unroll
        for (int k = 0; k < NQ; ++k) {
          const F out = wa * qk[k];
          const size_t l = lbase + k * NQ2 + ty * NQ + tx;
          Aq[l] = out;
          if (partials) {
            const int32_t id = G2L[l];
            pdot += (double)(id >= 0 ? q[id] : F(0)) * (double)out;
          }
        }
      }
      continue;
    }
    F acc[G];
    if (FORM == CUB_MASS) {
      if (Sh::STAGE) {
        cp_async_wait_all();
        __syncthreads();
#pragma unroll
        for (int k = 0; k < G; ++k) acc[k] = sW[k * G * G + ty * G + tx] * qk[k];
      } else {
        const size_t gb = (size_t)element * GP + ty * G + tx;
#pragma unroll
        for (int k = 0; k < G; ++k) acc[k] = wJ[gb + k * G * G] * qk[k];
      }
    } else if (Sh::STAGE) {
      cub_stiff<NQ, FORM>(qk, acc, U, R, S, tx, ty, lambda, CubStagedFactors<F>{sG, sW});
    } else if (Sh::CURVED) {
      cub_stiff<NQ, FORM>(qk, acc, U, R, S, tx, ty, lambda,
                          CubGlobalFactors<F>{ggeo + 6 * (size_t)element * GP, wJ + (size_t)element * GP});
    } else {
      CubAffineFactors<F> fa;
#pragma unroll
      for (int c = 0; c < 6; ++c) fa.ga[c] = ggeo[6 * (size_t)element + c];
      fa.wa = wJ[element];
      cub_stiff<NQ, FORM>(qk, acc, U, R, S, tx, ty, lambda, fa);
    }
    cub_project_ca<NQ, FORM>(acc, U, tx, ty);
    // along b: node (a, c) = (tx, ty), the line q was loaded along
    if (tx < NQ && ty < NQ && valid) {
      F r[G];
#pragma unroll
      for (int jj = 0; jj < G; ++jj) r[jj] = CUB_AT(U, ty, jj, tx);
#pragma unroll
      for (int b = 0; b < NQ; ++b) {
        F t = 0;
#pragma unroll
        for (int jj = 0; jj < G; ++jj) t += CUB_T(jj, b) * r[jj];
        const size_t l = lbase + ty * NQ2 + b * NQ + tx;
        Aq[l] = t;
        if (partials) {   // q again (a cache hit) rather than a line held in registers throughout
          const int32_t id = G2L[l];
          pdot += (double)(id >= 0 ? q[id] : F(0)) * (double)t;
        }
      }
    }
  }
  if (partials) {
    static_assert(Sh::FIELDS >= sizeof(double) * Sh::THREADS, "scratch too small");
    const double bs = fuse_block_sum(pdot, reinterpret_cast<double*>(sbase));
    if (tx == 0 && ty == 0 && es == 0) partials[blockIdx.x] = bs;
  }
}

// Curved stiffness (BP3, one field, even Nq) with the memory traffic of the
// next element groups in flight while a group computes.  A resident grid of
// blocks loops over groups of EPB elements; with iteration i of a block on
// group h_i = blockIdx.x + i gridDim.x, the pipeline holds
//   element ids of h_{i+3}  -> sEl[(i+3) & 3]   (4-byte copies)
//   GlobalToLocal of h_{i+2} -> sIdx            (16-byte copies)
//   q of h_{i+1}             -> sQ[(i+1) & 1]   (gathers through sIdx)
// issued as one commit group at the start of iteration i; in FP32 the factors
// of h_{i+1} -> sG, sW follow as the next group once iteration i's flux loop
// is done with h_i's (FP64 reads its factors at the flux loop: staging them
// would halve the resident blocks).  A thread gathers the nodes of the same
// 16-byte index chunks it copies, so sIdx needs no barrier; q, the ids and the
// factors are read by other threads after a wait and a barrier.  The q.Aq
// partial reads q from sQ instead of gathering it again.
template <int NQ>
__global__ void __launch_bounds__(CubShape<NQ, CUB_STIFF>::THREADS, CubShape<NQ, CUB_STIFF>::MINB)
ax_cub_pipe_kernel(int Nelements, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
                   const CubReal* __restrict__ wJ, const CubReal* __restrict__ ggeo, CubReal lambda,
                   const CubReal* __restrict__ q, CubReal* __restrict__ Aq, const int* __restrict__ skip,
                   double* __restrict__ partials) {
  constexpr int FORM = CUB_STIFF;
  using F = CubReal;
  using Sh = CubShape<NQ, FORM>;
  static_assert(NQ % 2 == 0, "whole 16-byte index chunks");
  constexpr bool STG = Sh::STAGE;   // FP32 stages the factors; FP64 reads them at the flux loop
  constexpr int G = Sh::G, GP = Sh::GP, EPB = Sh::EPB, NP = Sh::NP, NQ2 = NQ * NQ;
  constexpr int CH = NP / 4;   // 16-byte chunks of an element's GlobalToLocal
  pdl_wait();
  pdl_release();
  if (skip && *skip) return;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  F* const sbase = reinterpret_cast<F*>(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y, es = threadIdx.z;
  const int tid = tx + G * (ty + G * es);
  F* const U = sbase + (size_t)es * Sh::SLOTW;
  F* const R = U + Sh::FIELD;
  F* const S = R + Sh::FIELD;
  F* const sG0 = reinterpret_cast<F*>(smem_raw + Sh::GOFF);
  F* const sW0 = reinterpret_cast<F*>(smem_raw + Sh::WOFF);
  int32_t* const sIdx = reinterpret_cast<int32_t*>(smem_raw + Sh::IOFF);
  F* const sQ = reinterpret_cast<F*>(smem_raw + Sh::QOFF);
  int32_t* const sEl = reinterpret_cast<int32_t*>(smem_raw + Sh::EOFF);

  const int ngroups = (Nelements + EPB - 1) / EPB;
  auto group = [&](int i) { return blockIdx.x + i * gridDim.x; };
  // element ids of iteration i's group (-1 past the end) into sEl[i & 3]
  auto issue_ids = [&](int i, bool async) {
    if (tid < EPB) {
      const int e = group(i) * EPB + tid;
      int32_t* dst = sEl + (i & 3) * EPB + tid;
      if (group(i) < ngroups && e < Nelements) {
        if (async) cp_async4(dst, elementList + e);
        else *dst = elementList[e];
      } else {
        *dst = -1;
      }
    }
  };
  // GlobalToLocal of iteration i's group into sIdx (ids in sEl[i & 3] visible)
  auto issue_idx = [&](int i) {
    for (int w = tid; w < EPB * CH; w += Sh::THREADS) {
      const int s = w / CH, c = w - s * CH;
      const int32_t e = sEl[(i & 3) * EPB + s];
      if (e >= 0) cp_async16(sIdx + s * NP + 4 * c, G2L + (size_t)e * NP + 4 * c);
    }
  };
  // q of iteration i's group into sQ[i & 1] through this thread's chunks of sIdx
  auto issue_q = [&](int i) {
    F* dstq = sQ + (size_t)(i & 1) * EPB * NP;
    for (int w = tid; w < EPB * CH; w += Sh::THREADS) {
      const int s = w / CH, c = w - s * CH;
      const bool live = sEl[(i & 3) * EPB + s] >= 0;
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        const int pos = s * NP + 4 * c + n;
        const int32_t id = live ? sIdx[pos] : -1;
        if (id < 0) dstq[pos] = F(0);
        else if constexpr (sizeof(F) == 8) cp_async8(dstq + pos, q + id);
        else cp_async4(dstq + pos, q + id);
      }
    }
  };
  // factors of iteration i's group into sG, sW
  auto issue_factors = [&](int i) {
    const int32_t e = sEl[(i & 3) * EPB + es];
    if (e >= 0) {
      const int tl = tx + G * ty;
      const F* src = ggeo + 6 * (size_t)e * GP;   // 8-byte aligned: 24 bytes per point
      F* sG = sG0 + (size_t)es * GP * 6;
      for (int c = tl; c < GP * 3; c += G * G) cp_async8(sG + 2 * c, src + 2 * c);
      const F* srcw = wJ + (size_t)e * GP;
      F* sW = sW0 + (size_t)es * GP;
      for (int c = tl; c < GP; c += G * G) cp_async4(sW + c, srcw + c);
    }
  };
  struct PipeFactors {
    CubStagedFactors<F> st;
    const decltype(issue_factors)* next;
    int i;
    __device__ __forceinline__ void ready() const { cp_async_wait_group<1>(); }
    __device__ __forceinline__ void released() const {
      (*next)(i + 1);
      cp_async_commit();
    }
    __device__ __forceinline__ void get(int pt, F (&g)[6], F& w) const { st.get(pt, g, w); }
  };

  // prologue: ids of iterations 0 and 1, indices of 0; then q of 0, indices
  // of 1 and ids of 2 as one group, the factors of 0 as the next
  issue_ids(0, false);
  issue_ids(1, false);
  __syncthreads();
  issue_idx(0);
  cp_async_commit();
  cp_async_wait_group<0>();   // this thread's index chunks
  issue_q(0);
  issue_idx(1);
  issue_ids(2, true);
  cp_async_commit();
  if (STG) {
    issue_factors(0);
    cp_async_commit();
  }

  double pdot = 0.0;
  for (int i = 0; group(i) < ngroups; ++i) {
    if (STG) cp_async_wait_group<1>();   // all but the factors of this group
    else cp_async_wait_group<0>();
    __syncthreads();
    const F* qg = sQ + (size_t)(i & 1) * EPB * NP + (size_t)es * NP;
    const int32_t element = sEl[(i & 3) * EPB + es];
    F qb[NQ];
#pragma unroll
    for (int b = 0; b < NQ; ++b) qb[b] = (tx < NQ && ty < NQ) ? qg[ty * NQ2 + b * NQ + tx] : F(0);
    // the next groups' ids, indices and q
    issue_q(i + 1);
    issue_idx(i + 2);
    issue_ids(i + 3, true);
    cp_async_commit();

    F qk[G], acc[G];
    cub_interp<NQ, FORM>(qb, U, qk, tx, ty);
    if constexpr (STG) {
      const PipeFactors fac{CubStagedFactors<F>{sG0 + (size_t)es * GP * 6, sW0 + (size_t)es * GP}, &issue_factors,
                            i};
      cub_stiff<NQ, FORM>(qk, acc, U, R, S, tx, ty, lambda, fac);
    } else {
      const size_t e = element >= 0 ? (size_t)element : 0;
      cub_stiff<NQ, FORM>(qk, acc, U, R, S, tx, ty, lambda, CubGlobalFactors<F>{ggeo + 6 * e * GP, wJ + e * GP});
    }
    cub_project_ca<NQ, FORM>(acc, U, tx, ty);
    if (tx < NQ && ty < NQ && element >= 0) {
      F r[G];
#pragma unroll
      for (int jj = 0; jj < G; ++jj) r[jj] = CUB_AT(U, ty, jj, tx);
      const size_t lbase = (size_t)element * NP;
#pragma unroll
      for (int b = 0; b < NQ; ++b) {
        F t = 0;
#pragma unroll
        for (int jj = 0; jj < G; ++jj) t += CUB_T(jj, b) * r[jj];
        Aq[lbase + ty * NQ2 + b * NQ + tx] = t;
        if (partials) pdot += (double)qg[ty * NQ2 + b * NQ + tx] * (double)t;
      }
    }
  }
  cp_async_wait_all();   // nothing is left in flight (groups past the end issue no copies)
  if (partials) {
    static_assert(Sh::FIELDS >= sizeof(double) * Sh::THREADS, "scratch too small");
    const double bs = fuse_block_sum(pdot, reinterpret_cast<double*>(sbase));
    if (tid == 0) partials[blockIdx.x] = bs;
  }
}
#undef CUB_AT
#undef CUB_D
#undef CUB_T

// The pipelined stiffness kernel is the default where it applies;
// BP_CUB_PIPE=0, read at every launch, keeps the one-element-per-slot kernel
// (for comparisons and tests).
static bool cub_pipe_enabled() {
  const char* e = getenv("BP_CUB_PIPE");
  return !(e && e[0] == '0');
}

// device address of the constant table on the current device
static CubReal* cub_table_address() {
  static DeviceSymbol sym(c_cub);
  return static_cast<CubReal*>(sym.address());
}

template <int NQ, int FORM>
static int launch_cub_form(int32_t Nelements, int Nfields, const int32_t* elementList, const int32_t* G2L,
                           const CubOperands<CubReal>& o, CubReal lambda, const CubReal* q, CubReal* Aq,
                           const int* skip, cudaStream_t s, double* partials, int* nblocks) {
  using Sh = CubShape<NQ, FORM>;
  if (Sh::CURVED && Sh::STIFF && (reinterpret_cast<uintptr_t>(o.ggeo) % (2 * sizeof(CubReal))))
    return fail(BP_ERROR_ARG, "over-integrated operator: cubggeo must be aligned to two elements");
  CubReal* tab = cub_table_address();
  if (!tab) return fail(BP_ERROR_CUDA, "over-integrated operator: constant table address lookup failed");
  // this launch's 1D operands into its slot of the constant bank, in stream order
  BP_TRY(const_slot_copy(tab + Sh::SLOT, o.T, sizeof(CubReal) * Sh::TSIZE, s));
  if (Sh::STIFF)
    BP_TRY(const_slot_copy(tab + Sh::SLOT + Sh::TSIZE, o.D, sizeof(CubReal) * Sh::DSIZE, s));
  const dim3 block(Sh::G, Sh::G, Sh::EPB);
  if constexpr (FORM == CUB_STIFF && NQ % 2 == 0 && Sh::PIPE_OK) {
    if (Nfields == 1 && !(reinterpret_cast<uintptr_t>(G2L) & 15) && cub_pipe_enabled()) {
      static DeviceOnce configured;
      static int resident[kMaxDevices] = {};
      BP_TRY(once_per_device(configured, []() -> int {
        BP_CUDA_TRY(cudaFuncSetAttribute(ax_cub_pipe_kernel<NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)Sh::PSMEM));
        int dev = 0, nb = 0;
        BP_TRY(current_device(&dev));
        BP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ax_cub_pipe_kernel<NQ>, Sh::THREADS,
                                                                  Sh::PSMEM));
        resident[dev] = nb > 0 ? nb * sm_count() : 1;
        return BP_SUCCESS;
      }));
      int dev = 0;
      BP_TRY(current_device(&dev));
      const int ngroups = (Nelements + Sh::EPB - 1) / Sh::EPB;
      const dim3 grid(ngroups < resident[dev] ? ngroups : resident[dev]);
      if (nblocks) *nblocks = (int)grid.x;
      BP_CUDA_TRY(launch_pdl(ax_cub_pipe_kernel<NQ>, grid, block, Sh::PSMEM, s, Nelements, elementList, G2L, o.wJ,
                             o.ggeo, lambda, q, Aq, skip, partials));
      return BP_SUCCESS;
    }
  }
  if (Sh::SMEM > 48 * 1024)
    BP_CUDA_TRY(cudaFuncSetAttribute(ax_cub_kernel<NQ, FORM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)Sh::SMEM));
  const dim3 grid((Nelements + Sh::EPB - 1) / Sh::EPB);
  if (nblocks) *nblocks = (int)grid.x;
  BP_CUDA_TRY(launch_pdl(ax_cub_kernel<NQ, FORM>, grid, block, Sh::SMEM, s, Nelements, Nfields, elementList, G2L, o.wJ,
                         o.ggeo, lambda, q, Aq, skip, partials));
  return BP_SUCCESS;
}

template <int NQ>
static int launch_cub_nq(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                         const CubOperands<CubReal>& o, CubReal lambda, const CubReal* q, CubReal* Aq,
                         const int* skip, cudaStream_t s, double* partials, int* nblocks) {
  const bool stiff = d.bp >= 3;
#define BP_CUB(FORM) \
  return launch_cub_form<NQ, FORM>(Nelements, d.Nfields, elementList, G2L, o, lambda, q, Aq, skip, s, partials, nblocks)
  if (d.affine) {
    if (stiff) BP_CUB(CUB_STIFF_AFFINE);
    BP_CUB(CUB_MASS_AFFINE);
  }
  if (stiff) BP_CUB(CUB_STIFF);
  BP_CUB(CUB_MASS);
#undef BP_CUB
}

int launch_ax_cub_impl(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                       const CubOperands<CubReal>& o, CubReal lambda, const CubReal* q, CubReal* Aq,
                       const int* skip, cudaStream_t s, const CgFuse* fuse, int* nblocks) {
  if (nblocks) *nblocks = 0;
  if (d.bp < 1 || d.bp > 4) return fail(BP_ERROR_ARG, "over-integrated operator: bp must be 1..4");
  if (d.Nfields != ((d.bp % 2) ? 1 : 3))
    return fail(BP_ERROR_ARG, "over-integrated operator: BP1/BP3 take 1 field, BP2/BP4 3");
  if (Nelements == 0) return BP_SUCCESS;
  double* partials = fuse ? fuse->partials : nullptr;
  switch (d.N + 1) {
#define BP_CUB_CASE(nq) \
  case nq:              \
    return launch_cub_nq<nq>(d, Nelements, elementList, G2L, o, lambda, q, Aq, skip, s, partials, nblocks);
    BP_CUB_CASE(2) BP_CUB_CASE(3) BP_CUB_CASE(4) BP_CUB_CASE(5) BP_CUB_CASE(6) BP_CUB_CASE(7) BP_CUB_CASE(8)
    BP_CUB_CASE(9) BP_CUB_CASE(10) BP_CUB_CASE(11) BP_CUB_CASE(12) BP_CUB_CASE(13) BP_CUB_CASE(14)
    BP_CUB_CASE(15) BP_CUB_CASE(16)
#undef BP_CUB_CASE
    default:
      return fail(BP_ERROR_ARG, "over-integrated operator: degree N must be in 1..15");
  }
}

}  // namespace
}  // namespace bp
