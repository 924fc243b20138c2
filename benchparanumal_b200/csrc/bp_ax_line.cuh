// BP5/BP6 element operator (GLL collocation) in the line-per-thread form of
// bp_ax_cub.cuh: every 1D derivative is a constant-bank matrix applied along
// whole lines owned by single threads.  Included once by bp_ax_line64.cu
// (BP_LINE_REAL = double) and once by bp_ax_line32.cu (float).
//
//   Aq_e = Dr^T(G00 ur + G01 us + G02 ut) + Ds^T(G01 ur + G11 us + G12 ut)
//        + Dt^T(G02 ur + G12 us + G22 ut) + lambda wJ q,  (ur,us,ut) = (Dr,Ds,Dt) q
// (okl/bp5AxHex3D.okl:415-569, okl/bp5AxAffineHex3D.okl:419-579,
// okl/bp6AxHex3D.okl:50-255).  Stored factors carry the GLL weights; affine
// factors are per element and the weights w_i w_j w_k are applied here.
//
// Thread (x, y) of an element slot owns the t-line of point (x, y): it loads
// q along t, keeps it and the t-derivative in registers, and writes its
// result line along t (coalesced over x).  The r-derivative runs on rows
// (y, z) and the s-derivative on columns (x, z) of shared memory, and their
// weak forms the same way after the fluxes.
#pragma once

#ifndef BP_LINE_REAL
#error "define BP_LINE_REAL (double or float) before including bp_ax_line.cuh"
#endif

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "bp_cg_device.cuh"
#include "bp_internal.hpp"
#include "bp_pack.cuh"

// Outer loops of the line products (one output per pass) are unrolled up to
// Nq = BP_LINE_UNROLL_MAX and rolled above: unrolled FP64 needs more registers
// than two blocks allow; FP32 unrolls them all (rolled at Nq = 16: BK6 p=15
// 5.6 against 4.0 ms).
#ifndef BP_LINE_UNROLL_MAX
#define BP_LINE_UNROLL_MAX 0
#endif

namespace bp {
namespace {

using LineReal = BP_LINE_REAL;

// constant table: per degree D [NQ x NQ] then gllw [NQ]
__host__ __device__ constexpr int line_slot(int nq) {
  int off = 0;
  for (int n = 2; n < nq; ++n) off += n * n + n;
  return off;
}
constexpr int kLineTable = line_slot(17);
static __constant__ LineReal c_line[kLineTable];

// Elements per block: about 256 threads, but one element for four packed lanes
// at NQ >= 9, whose 3 x 16-byte fields take 35-83 KB per element: small blocks
// let two to four of them share an SM.
template <int NQ, class T = LineReal>
struct LineShape {
  static constexpr int G2 = NQ * NQ;
  static constexpr int RS = (NQ % 2) ? NQ : NQ + 1;
  static constexpr int PLANE = NQ * RS;
  static constexpr int FIELD = NQ * PLANE;
  static constexpr int EPB0 = 256 / G2 < 1 ? 1 : 256 / G2;
  static constexpr int EPB = (sizeof(T) >= 16 && NQ >= 9) ? 1 : (EPB0 > 8 ? 8 : EPB0);
  static constexpr int THREADS = G2 * EPB;
  static constexpr int SLOT = line_slot(NQ);
  static constexpr size_t smem() { return sizeof(T) * (size_t)3 * FIELD * EPB; }
};

// Blocks per SM the registers are sized for: two up to NQ = 13 (one element
// of NQ^2 <= 169 threads per block leaves two blocks 170 registers a thread:
// FP32 affine BK6 p=11 1.3 ms against 2.4 ms with one block), one above
// (NQ = 16 at two blocks spills: p=15 5.8 against 4.0 ms).  Four packed lanes
// at NQ >= 9 (one element per block) get about 168 registers a thread (NQ =
// 11: 936 bytes of spills at 128; BK5 four rhs p=10 6.0 -> 9.3, p=8 8.3 -> 9.1
// x 10^10 DOF/s).
template <int NQ, class T>
struct LineMinBlocks {
  static constexpr int ALLOC = (NQ * NQ + 31) / 32 * 32;
  static constexpr int WIDE = 65536 / (ALLOC * 168) > 0 ? 65536 / (ALLOC * 168) : 1;
  static constexpr int V = (PackTraits<T>::R >= 4 && NQ >= 9) ? WIDE : (NQ <= 13 ? 2 : 1);
};

// T: the value type of q and Aq, LineReal or Pack<LineReal, PK> (PK right-hand
// sides of one mesh in lockstep, one pack per node); p.Ap partials per lane at
// partials[lane * gridDim.x + blockIdx.x].
//
// The body works on element block `blk` of `nblk` (partials[lane * nblk +
// blk]) in the dynamic shared memory smem_raw: the kernel below and the
// persistent CG step share it.
template <int NQ, bool AFFINE, class T>
__device__ __forceinline__ void ax_line_body(int blk, int nblk, int Nelements, int Nfields,
                                             const int32_t* __restrict__ elementList,
                                             const int32_t* __restrict__ G2L, const LineReal* __restrict__ wJ,
                                             const LineReal* __restrict__ ggeo, const LineReal* __restrict__ gllw,
                                             LineReal lambda, const T* __restrict__ q, T* __restrict__ Aq,
                                             double* __restrict__ partials, unsigned char* smem_raw) {
  using F = LineReal;
  using Sh = LineShape<NQ, T>;
  using V2 = typename std::conditional<sizeof(F) == 8, double2, float2>::type;
  constexpr int RS = Sh::RS, PLANE = Sh::PLANE, EPB = Sh::EPB, NQ2 = NQ * NQ, NP = NQ * NQ * NQ;
  constexpr int SLOT = Sh::SLOT, LANES = PackTraits<T>::R;
  constexpr int OUTER = NQ <= BP_LINE_UNROLL_MAX ? NQ : 1;
#define D_(a, b) c_line[SLOT + (a) * NQ + (b)]
#define W_(a) c_line[SLOT + NQ * NQ + (a)]
#define AT(B, z, y, x) B[(z) * PLANE + (y) * RS + (x)]

  __syncthreads();   // a previous call's last uses of this shared memory are done (persistent use)
  T* const sbase = reinterpret_cast<T*>(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y, es = threadIdx.z;
  const int tid = tx + NQ * (ty + NQ * es);
  T* const U = sbase + (size_t)es * 3 * Sh::FIELD;
  T* const R = U + Sh::FIELD;
  T* const S = R + Sh::FIELD;

  const int eidx = blk * EPB + es;
  const bool valid = eidx < Nelements;
  const int element = valid ? elementList[eidx] : 0;
  double pdot[LANES];
#pragma unroll
  for (int l = 0; l < LANES; ++l) pdot[l] = 0.0;

  F wa = 0, ga[6] = {0, 0, 0, 0, 0, 0}, wxy = 0;
  if (AFFINE) {
    wxy = gllw[tx] * gllw[ty];
    wa = wJ[element];
#pragma unroll
    for (int c = 0; c < 6; ++c) ga[c] = ggeo[6 * (size_t)element + c];
  }

  for (int f = 0; f < Nfields; ++f) {
    const size_t lbase = ((size_t)element * Nfields + f) * NP;
    if (f > 0) __syncthreads();   // the previous field's last reads of U, R, S are done
    T qk[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      T v = pack_zero<T>();
      if (valid) {
        const int32_t id = G2L[lbase + k * NQ2 + ty * NQ + tx];
        if (id >= 0) v = q[id];
      }
      qk[k] = v;
      AT(U, k, ty, tx) = v;
    }
    T gt[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      T t = pack_zero<T>();
#pragma unroll
      for (int n = 0; n < NQ; ++n) t += D_(k, n) * qk[n];
      gt[k] = t;
    }
    __syncthreads();
    {
      T r[NQ];
#pragma unroll
      for (int n = 0; n < NQ; ++n) r[n] = AT(U, ty, tx, n);
#pragma unroll OUTER
      for (int i = 0; i < NQ; ++i) {
        T t = pack_zero<T>();
#pragma unroll
        for (int n = 0; n < NQ; ++n) t += D_(i, n) * r[n];
        AT(R, ty, tx, i) = t;
      }
#pragma unroll
      for (int n = 0; n < NQ; ++n) r[n] = AT(U, ty, n, tx);
#pragma unroll OUTER
      for (int j = 0; j < NQ; ++j) {
        T t = pack_zero<T>();
#pragma unroll
        for (int n = 0; n < NQ; ++n) t += D_(j, n) * r[n];
        AT(S, ty, j, tx) = t;
      }
    }
    __syncthreads();
    T acc[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      if (AFFINE) {
        // the element's G applied first, the node weight after: scaling G by
        // the weight per k let the compiler form all 7*NQ scaled factors up
        // front (Nq = 16: 380 bytes of spills at 255 registers; BK6 p=15 FP32
        // 4.5 -> 4.0 ms)
        const F wk = wxy * W_(k);
        const T dr = AT(R, k, ty, tx), ds = AT(S, k, ty, tx), dt = gt[k];
        AT(R, k, ty, tx) = wk * (ga[0] * dr + ga[1] * ds + ga[2] * dt);
        AT(S, k, ty, tx) = wk * (ga[1] * dr + ga[3] * ds + ga[4] * dt);
        gt[k] = wk * (ga[2] * dr + ga[4] * ds + ga[5] * dt);
        acc[k] = (lambda * (wa * wk)) * AT(U, k, ty, tx);
        continue;
      }
      F g0, g1, g2, g3, g4, g5, w;
      {
        const size_t gb = (size_t)element * NP + k * NQ2 + ty * NQ + tx;
        const V2* gv = reinterpret_cast<const V2*>(ggeo + 6 * gb);
        const V2 a0 = gv[0], a1 = gv[1], a2 = gv[2];
        g0 = a0.x; g1 = a0.y; g2 = a1.x; g3 = a1.y; g4 = a2.x; g5 = a2.y;
        w = wJ[gb];
      }
      const T dr = AT(R, k, ty, tx), ds = AT(S, k, ty, tx), dt = gt[k];
      AT(R, k, ty, tx) = g0 * dr + g1 * ds + g2 * dt;
      AT(S, k, ty, tx) = g1 * dr + g3 * ds + g4 * dt;
      gt[k] = g2 * dr + g4 * ds + g5 * dt;
      // q again from the slice copy (the same value as qk[k]): the pencil qk
      // then dies after the t-gradient, 8 packs of registers fewer through the
      // r/s phases (NQ = 8, four lanes: 128 registers with spills before)
      acc[k] = (lambda * w) * AT(U, k, ty, tx);
    }
#pragma unroll
    for (int n = 0; n < NQ; ++n) {
      T t = acc[n];
#pragma unroll
      for (int k = 0; k < NQ; ++k) t += D_(k, n) * gt[k];
      acc[n] = t;
    }
    __syncthreads();
    {
      T r[NQ];
#pragma unroll
      for (int n = 0; n < NQ; ++n) r[n] = AT(R, ty, tx, n);
#pragma unroll OUTER
      for (int i = 0; i < NQ; ++i) {
        T t = pack_zero<T>();
#pragma unroll
        for (int n = 0; n < NQ; ++n) t += D_(n, i) * r[n];
        AT(R, ty, tx, i) = t;
      }
#pragma unroll
      for (int n = 0; n < NQ; ++n) r[n] = AT(S, ty, n, tx);
#pragma unroll OUTER
      for (int j = 0; j < NQ; ++j) {
        T t = pack_zero<T>();
#pragma unroll
        for (int n = 0; n < NQ; ++n) t += D_(n, j) * r[n];
        AT(S, ty, j, tx) = t;
      }
    }
    __syncthreads();
    if (valid) {
#pragma unroll
      for (int k = 0; k < NQ; ++k) {
        const T out = acc[k] + AT(R, k, ty, tx) + AT(S, k, ty, tx);
        Aq[lbase + k * NQ2 + ty * NQ + tx] = out;
        lane_dot(pdot, AT(U, k, ty, tx), out);
      }
    }
  }
  if (partials) {
    double bs[LANES];
    if (LANES == 1) {
      bs[0] = fuse_block_sum(pdot[0], reinterpret_cast<double*>(sbase));
    } else {
      static_assert(sizeof(T) * 3 * Sh::FIELD >= sizeof(double) * LANES * NQ2 &&
                        sizeof(T) * 3 * Sh::FIELD * EPB >= sizeof(double) * LANES * 32,
                    "block-sum scratch too small");
      fuse_block_sum_lanes<LANES>(pdot, reinterpret_cast<double*>(sbase), bs);
    }
    if (tid == 0)
#pragma unroll
      for (int l = 0; l < LANES; ++l) partials[(size_t)l * nblk + blk] = bs[l];
  }
#undef AT
#undef W_
#undef D_
}

template <int NQ, bool AFFINE, class T>
__global__ void __launch_bounds__(LineShape<NQ, T>::THREADS, (LineMinBlocks<NQ, T>::V))
ax_line_kernel(int Nelements, int Nfields, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
               const LineReal* __restrict__ wJ, const LineReal* __restrict__ ggeo,
               const LineReal* __restrict__ gllw, LineReal lambda, const T* __restrict__ q,
               T* __restrict__ Aq, const int* __restrict__ skip, double* __restrict__ partials) {
  pdl_wait();
  pdl_release();
  if (skip && *skip) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ax_line_body<NQ, AFFINE, T>(blockIdx.x, gridDim.x, Nelements, Nfields, elementList, G2L, wJ, ggeo, gllw, lambda, q,
                              Aq, partials, smem_raw);
}

// device address of the constant table on the current device
static LineReal* line_table_address() {
  static DeviceSymbol sym(c_line);
  return static_cast<LineReal*>(sym.address());
}

template <int NQ, class T = LineReal>
static int launch_line_nq(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                          const LineReal* wJ, const LineReal* ggeo, const LineReal* gllw, const LineReal* D,
                          LineReal lambda, const T* q, T* Aq, const int* skip, cudaStream_t s,
                          double* partials, int* nblocks) {
  using Sh = LineShape<NQ, T>;
  constexpr size_t SMEM = Sh::smem();
  if (!d.affine && (reinterpret_cast<uintptr_t>(ggeo) % (2 * sizeof(LineReal))))
    return fail(BP_ERROR_ARG, "element operator: ggeo must be aligned to two elements");
  LineReal* tab = line_table_address();
  if (!tab) return fail(BP_ERROR_CUDA, "element operator: constant table address lookup failed");
  BP_TRY(const_slot_copy(tab + Sh::SLOT, D, sizeof(LineReal) * NQ * NQ, s));
  if (d.affine)
    BP_TRY(const_slot_copy(tab + Sh::SLOT + NQ * NQ, gllw, sizeof(LineReal) * NQ, s));
  const dim3 block(NQ, NQ, Sh::EPB);
  const dim3 grid((Nelements + Sh::EPB - 1) / Sh::EPB);
  if (nblocks) *nblocks = (int)grid.x;
  if (d.affine) {
    if (SMEM > 48 * 1024)
      BP_CUDA_TRY(cudaFuncSetAttribute(ax_line_kernel<NQ, true, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)SMEM));
    BP_CUDA_TRY(launch_pdl(ax_line_kernel<NQ, true, T>, grid, block, SMEM, s, Nelements, d.Nfields, elementList, G2L,
                           wJ, ggeo, gllw, lambda, q, Aq, skip, partials));
  } else {
    if (SMEM > 48 * 1024)
      BP_CUDA_TRY(cudaFuncSetAttribute(ax_line_kernel<NQ, false, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)SMEM));
    BP_CUDA_TRY(launch_pdl(ax_line_kernel<NQ, false, T>, grid, block, SMEM, s, Nelements, d.Nfields, elementList,
                           G2L, wJ, ggeo, gllw, lambda, q, Aq, skip, partials));
  }
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

int launch_ax_line_impl(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                        const LineReal* wJ, const LineReal* ggeo, const LineReal* gllw, const LineReal* D,
                        LineReal lambda, const LineReal* q, LineReal* Aq, const int* skip, cudaStream_t s,
                        const CgFuse* fuse, int* nblocks) {
  if (nblocks) *nblocks = 0;
  if (Nelements == 0) return BP_SUCCESS;
  double* partials = fuse ? fuse->partials : nullptr;
  switch (d.N + 1) {
#define BP_LINE_CASE(nq) \
  case nq:               \
    return launch_line_nq<nq>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, s, partials, nblocks);
    BP_LINE_CASE(2) BP_LINE_CASE(3) BP_LINE_CASE(4) BP_LINE_CASE(5) BP_LINE_CASE(6) BP_LINE_CASE(7)
    BP_LINE_CASE(8) BP_LINE_CASE(9) BP_LINE_CASE(10) BP_LINE_CASE(11) BP_LINE_CASE(12) BP_LINE_CASE(13)
    BP_LINE_CASE(14) BP_LINE_CASE(15) BP_LINE_CASE(16)
#undef BP_LINE_CASE
    default:
      return fail(BP_ERROR_ARG, "element operator: degree N must be in 1..15");
  }
}

// the same operator on PK right-hand sides packed per node (one field)
template <int PK>
int launch_ax_line_pk(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                      const LineReal* wJ, const LineReal* ggeo, const LineReal* gllw, const LineReal* D,
                      LineReal lambda, const LineReal* q, LineReal* Aq, const int* skip, cudaStream_t s,
                      const CgFuse* fuse, int* nblocks) {
  using T = Pack<LineReal, PK>;
  if (nblocks) *nblocks = 0;
  if (d.Nfields != 1) return fail(BP_ERROR_ARG, "packed element operator: one field only");
  if (Nelements == 0) return BP_SUCCESS;
  double* partials = fuse ? fuse->partials : nullptr;
  const T* qp = reinterpret_cast<const T*>(q);
  T* ap = reinterpret_cast<T*>(Aq);
  switch (d.N + 1) {
#define BP_LINE_PK_CASE(nq) \
  case nq:                  \
    return launch_line_nq<nq, T>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, qp, ap, skip, s, partials, nblocks);
    BP_LINE_PK_CASE(2) BP_LINE_PK_CASE(3) BP_LINE_PK_CASE(4) BP_LINE_PK_CASE(5) BP_LINE_PK_CASE(6)
    BP_LINE_PK_CASE(7) BP_LINE_PK_CASE(8) BP_LINE_PK_CASE(9) BP_LINE_PK_CASE(10) BP_LINE_PK_CASE(11)
    BP_LINE_PK_CASE(12)
#undef BP_LINE_PK_CASE
    default:
      return fail(BP_ERROR_ARG, "packed element operator: degree N must be in 1..11");
  }
}

}  // namespace
}  // namespace bp
