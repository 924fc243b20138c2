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
// operands into its slot on the launch stream, so two launches of the same
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
  static constexpr size_t FIELDS = sizeof(CubReal) * (size_t)NBUF * FIELD * EPB;
  static constexpr size_t GOFF = (FIELDS + 15) & ~(size_t)15;                        // [EPB][GP*6] ggeo
  static constexpr size_t WOFF = GOFF + (STAGE && STIFF ? sizeof(CubReal) * (size_t)EPB * GP * 6 : 0);   // [EPB][GP] wJ
  static constexpr size_t SMEM = STAGE ? WOFF + sizeof(CubReal) * (size_t)EPB * GP : FIELDS;
};

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <int NQ, int FORM>
__global__ void __launch_bounds__(CubShape<NQ, FORM>::THREADS, CubShape<NQ, FORM>::MINB)
ax_cub_kernel(int Nelements, int Nfields, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
              const CubReal* __restrict__ wJ, const CubReal* __restrict__ ggeo, CubReal lambda,
              const CubReal* __restrict__ q, CubReal* __restrict__ Aq, const int* __restrict__ skip,
              double* __restrict__ partials) {
  if (skip && *skip) return;
  using F = CubReal;
  using Sh = CubShape<NQ, FORM>;
  using V2 = typename std::conditional<sizeof(F) == 8, double2, float2>::type;
  constexpr int G = Sh::G, GP = Sh::GP, RS = Sh::RS, PLANE = Sh::PLANE, EPB = Sh::EPB;
  constexpr int NQ2 = NQ * NQ, NP = NQ * NQ * NQ;
  constexpr int SLOT = Sh::SLOT, DOFF = Sh::SLOT + Sh::TSIZE;
  // T(o, i): 1D transform from NQ nodes to G points; MASS_AFFINE applies MM^T
#define T_(o, i) (FORM == CUB_MASS_AFFINE ? c_cub[SLOT + (i) * NQ + (o)] : c_cub[SLOT + (o) * NQ + (i)])
#define D_(a, b) c_cub[DOFF + (a) * G + (b)]

  extern __shared__ __align__(16) unsigned char smem_raw[];
  F* const sbase = reinterpret_cast<F*>(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y, es = threadIdx.z;
  const int tid = tx + G * (ty + G * es);
  F* const U = sbase + (size_t)es * Sh::NBUF * Sh::FIELD;   // the field
  F* const R = U + Sh::FIELD;                                // r-derivative / r-flux
  F* const S = R + Sh::FIELD;                                // s-derivative / s-flux
#define AT(B, z, y, x) B[(z) * PLANE + (y) * RS + (x)]

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

  F wa = 0, ga[6] = {0, 0, 0, 0, 0, 0};
  if (!Sh::CURVED) {
    wa = wJ[element];
    if (Sh::STIFF)
#pragma unroll
      for (int c = 0; c < 6; ++c) ga[c] = ggeo[6 * (size_t)element + c];
  }

  for (int f = 0; f < Nfields; ++f) {
    const size_t lbase = ((size_t)element * Nfields + f) * NP;
    if (f > 0) __syncthreads();   // the previous field's last reads of U are done
    // load q[c][b][a] along b and interpolate along b in registers
    if (tx < NQ && ty < NQ) {
      F qb[NQ];   // q along b of node (a, c) = (tx, ty)
#pragma unroll
      for (int b = 0; b < NQ; ++b) {
        F v = 0;
        if (valid) {
          const int32_t id = G2L[lbase + ty * NQ2 + b * NQ + tx];
          v = (id >= 0) ? q[id] : F(0);
        }
        qb[b] = v;
      }
BP_CUB_OUTER
      for (int jj = 0; jj < G; ++jj) {
        F t = 0;
#pragma unroll
        for (int b = 0; b < NQ; ++b) t += T_(jj, b) * qb[b];
        AT(U, ty, jj, tx) = t;
      }
    }
    __syncthreads();
    // along a: thread (jj, c) = (tx, ty)
    if (ty < NQ) {
      F r[NQ];
#pragma unroll
      for (int a = 0; a < NQ; ++a) r[a] = AT(U, ty, tx, a);
BP_CUB_OUTER
      for (int ii = 0; ii < G; ++ii) {
        F t = 0;
#pragma unroll
        for (int a = 0; a < NQ; ++a) t += T_(ii, a) * r[a];
        AT(U, ty, tx, ii) = t;
      }
    }
    __syncthreads();
    // along c: thread (ii, jj) = (tx, ty); the grid column stays in registers
    F qk[G];
    {
      F r[NQ];
#pragma unroll
      for (int c = 0; c < NQ; ++c) r[c] = AT(U, c, ty, tx);
#pragma unroll
      for (int k = 0; k < G; ++k) {
        F t = 0;
#pragma unroll
        for (int c = 0; c < NQ; ++c) t += T_(k, c) * r[c];
        qk[k] = t;
      }
    }
    if (FORM == CUB_MASS_AFFINE) {
      // G == NQ: the result column of node (tx, ty) is wJ_e * qk
      if (valid) {
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
    } else {
      // own column: every earlier read of it was this thread's
#pragma unroll
      for (int k = 0; k < G; ++k) AT(U, k, ty, tx) = qk[k];
      __syncthreads();
      // r-derivative on the row (y, z) = (tx, ty); s-derivative on the column (x, z) = (tx, ty)
      {
        F r[G];
#pragma unroll
        for (int n = 0; n < G; ++n) r[n] = AT(U, ty, tx, n);
BP_CUB_OUTER
        for (int i = 0; i < G; ++i) {
          F t = 0;
#pragma unroll
          for (int n = 0; n < G; ++n) t += D_(i, n) * r[n];
          AT(R, ty, tx, i) = t;
        }
#pragma unroll
        for (int n = 0; n < G; ++n) r[n] = AT(U, ty, n, tx);
BP_CUB_OUTER
        for (int j = 0; j < G; ++j) {
          F t = 0;
#pragma unroll
          for (int n = 0; n < G; ++n) t += D_(j, n) * r[n];
          AT(S, ty, j, tx) = t;
        }
      }
      // t-derivative on the column (x, y) = (tx, ty) in registers
      F gt[G];
#pragma unroll
      for (int k = 0; k < G; ++k) {
        F t = 0;
#pragma unroll
        for (int n = 0; n < G; ++n) t += D_(k, n) * qk[n];
        gt[k] = t;
      }
      if (Sh::STAGE) cp_async_wait_all();   // this thread's copies; the barrier below makes all visible
      __syncthreads();
      // fluxes at the points of column (tx, ty)
#pragma unroll
      for (int k = 0; k < G; ++k) {
        F g0, g1, g2, g3, g4, g5, w;
        if (Sh::STAGE) {
          const int pt = k * G * G + ty * G + tx;
          const V2* gv = reinterpret_cast<const V2*>(sG + 6 * pt);
          const V2 a0 = gv[0], a1 = gv[1], a2 = gv[2];
          g0 = a0.x; g1 = a0.y; g2 = a1.x; g3 = a1.y; g4 = a2.x; g5 = a2.y;
          w = sW[pt];
        } else if (Sh::CURVED) {
          const size_t gb = (size_t)element * GP + k * G * G + ty * G + tx;
          const V2* gv = reinterpret_cast<const V2*>(ggeo + 6 * gb);
          const V2 a0 = gv[0], a1 = gv[1], a2 = gv[2];
          g0 = a0.x; g1 = a0.y; g2 = a1.x; g3 = a1.y; g4 = a2.x; g5 = a2.y;
          w = wJ[gb];
        } else {
          g0 = ga[0]; g1 = ga[1]; g2 = ga[2]; g3 = ga[3]; g4 = ga[4]; g5 = ga[5];
          w = wa;
        }
        const F dr = AT(R, k, ty, tx), ds = AT(S, k, ty, tx), dt = gt[k];
        AT(R, k, ty, tx) = g0 * dr + g1 * ds + g2 * dt;
        AT(S, k, ty, tx) = g1 * dr + g3 * ds + g4 * dt;
        gt[k] = g2 * dr + g4 * ds + g5 * dt;
        acc[k] = lambda * w * qk[k];
      }
      // t-part of the weak divergence, in registers
#pragma unroll
      for (int n = 0; n < G; ++n) {
        F t = acc[n];
#pragma unroll
        for (int k = 0; k < G; ++k) t += D_(k, n) * gt[k];
        acc[n] = t;
      }
      __syncthreads();
      // r-part on rows, s-part on columns, in place
      {
        F r[G];
#pragma unroll
        for (int n = 0; n < G; ++n) r[n] = AT(R, ty, tx, n);
BP_CUB_OUTER
        for (int i = 0; i < G; ++i) {
          F t = 0;
#pragma unroll
          for (int n = 0; n < G; ++n) t += D_(n, i) * r[n];
          AT(R, ty, tx, i) = t;
        }
#pragma unroll
        for (int n = 0; n < G; ++n) r[n] = AT(S, ty, n, tx);
BP_CUB_OUTER
        for (int j = 0; j < G; ++j) {
          F t = 0;
#pragma unroll
          for (int n = 0; n < G; ++n) t += D_(n, j) * r[n];
          AT(S, ty, j, tx) = t;
        }
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < G; ++k) acc[k] += AT(R, k, ty, tx) + AT(S, k, ty, tx);
    }
    // projection along c in registers: column (ii, jj) = (tx, ty); own column of U
BP_CUB_OUTER
    for (int c = 0; c < NQ; ++c) {
      F t = 0;
#pragma unroll
      for (int k = 0; k < G; ++k) t += T_(k, c) * acc[k];
      AT(U, c, ty, tx) = t;
    }
    __syncthreads();
    // along a: row (jj, c) = (tx, ty)
    if (ty < NQ) {
      F r[G];
#pragma unroll
      for (int ii = 0; ii < G; ++ii) r[ii] = AT(U, ty, tx, ii);
BP_CUB_OUTER
      for (int a = 0; a < NQ; ++a) {
        F t = 0;
#pragma unroll
        for (int ii = 0; ii < G; ++ii) t += T_(ii, a) * r[ii];
        AT(U, ty, tx, a) = t;
      }
    }
    __syncthreads();
    // along b: node (a, c) = (tx, ty), the line q was loaded along
    if (tx < NQ && ty < NQ && valid) {
      F r[G];
#pragma unroll
      for (int jj = 0; jj < G; ++jj) r[jj] = AT(U, ty, jj, tx);
#pragma unroll
      for (int b = 0; b < NQ; ++b) {
        F t = 0;
#pragma unroll
        for (int jj = 0; jj < G; ++jj) t += T_(jj, b) * r[jj];
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
    if (tid == 0) partials[blockIdx.x] = bs;
  }
#undef AT
#undef D_
#undef T_
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
  BP_CUDA_TRY(cudaMemcpyAsync(tab + Sh::SLOT, o.T, sizeof(CubReal) * Sh::TSIZE, cudaMemcpyDeviceToDevice, s));
  if (Sh::STIFF)
    BP_CUDA_TRY(cudaMemcpyAsync(tab + Sh::SLOT + Sh::TSIZE, o.D, sizeof(CubReal) * Sh::DSIZE,
                                cudaMemcpyDeviceToDevice, s));
  if (Sh::SMEM > 48 * 1024)
    BP_CUDA_TRY(cudaFuncSetAttribute(ax_cub_kernel<NQ, FORM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)Sh::SMEM));
  const dim3 block(Sh::G, Sh::G, Sh::EPB);
  const dim3 grid((Nelements + Sh::EPB - 1) / Sh::EPB);
  if (nblocks) *nblocks = (int)grid.x;
  ax_cub_kernel<NQ, FORM><<<grid, block, Sh::SMEM, s>>>(Nelements, Nfields, elementList, G2L, o.wJ, o.ggeo, lambda,
                                                         q, Aq, skip, partials);
  BP_CUDA_TRY(cudaGetLastError());
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
