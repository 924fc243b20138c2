// Affine BP5/BP6 element operator on the tensor cores, for high degree.
//
// At Nq = 16 every 1D contraction of the sum-factorised operator is a dense
// product D (16 x 16) x slab (16 x 256): the element's values along one axis
// times the 256 lines along the other two.  The scalar kernels pay for these
// with one shared-memory load per multiply-add (BK6 p=15: 7.6 ms FP64, 4.0 ms
// FP32 for 24^3 elements, about 12% of the FP64 peak); here they run as warp
// MMAs whose operands are reused from registers:
//   FP64  mma.sync m8n8k4 f64 (DMMA, the FP64 tensor-core instruction),
//   FP32  mma.sync m16n8k8 tf32 with both operands split in two TF32 parts
//         (a = a_hi + a_lo; a.b ~ a_hi b_hi + a_hi b_lo + a_lo b_hi, FP32
//         accumulation), about 2^-21 relative per product, what the FP32
//         inner solve of the mixed-precision CG needs.
// The operator is the reference's affine one (okl/bp5AxAffineHex3D.okl:419-579,
// okl/bp6AxAffineHex3D.okl for three fields):
//   Aq = lambda wJ w q + Dr^T Vr + Ds^T Vs + Dt^T Vt,
//   (Vr, Vs, Vt) = w G (Dr q, Ds q, Dt q),  w = gllw_i gllw_j gllw_k,
// G the element's six factors.  One element per block; per field the values go
// through shared memory in four arrays of NQ^3 (q, then the lambda-term and the
// divergence sums; the three gradients, then the three fluxes), with padded
// strides that keep the FP64 fragment loads of all three axes free of bank
// conflicts.
#include <cuda_runtime.h>

#include <cstdint>

#include "bp_cg_device.cuh"
#include "bp_internal.hpp"

namespace bp {
namespace {

template <int NQ>
struct MmaShape {
  static constexpr int S1 = NQ + 4;            // stride of the j index (words of F)
  static constexpr int S2 = NQ * S1 + 4;       // stride of the k index
  static constexpr int ARR = NQ * S2;          // one NQ^3 array, padded
  static constexpr int NP = NQ * NQ * NQ;
  static constexpr int NCOL = NQ * NQ;         // columns of a slab
  static constexpr int THREADS = 256;
  static constexpr int WARPS = THREADS / 32;
  static constexpr int NTILES = NCOL / 8;      // n-tiles of 8 columns
  static constexpr int PER = NP / THREADS;     // nodes per thread in the pointwise phases
  template <class F>
  static constexpr size_t smem() { return sizeof(F) * 4 * (size_t)ARR; }
  static_assert(NQ % 8 == 0 && NCOL % (8 * WARPS) == 0 && NP % THREADS == 0, "shape");
};

// offset of the node whose index along axis `d` is x and whose other two
// indices, in (i, j, k) order with d left out, are (a, b)
template <int NQ>
__device__ __forceinline__ int mma_off(int d, int x, int a, int b) {
  using Sh = MmaShape<NQ>;
  return d == 0 ? b * Sh::S2 + a * Sh::S1 + x : d == 1 ? b * Sh::S2 + x * Sh::S1 + a : x * Sh::S2 + b * Sh::S1 + a;
}

// ---- FP64: DMMA m8n8k4 --------------------------------------------------
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// ---- FP32: TF32 m16n8k8, split operands ----------------------------------
__device__ __forceinline__ uint32_t tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void tf32_split(float x, uint32_t& hi, uint32_t& lo) {
  hi = tf32_hi(x);
  lo = tf32_hi(x - __uint_as_float(hi));
}
__device__ __forceinline__ void tmma(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Register fragments of the 1D matrix used as the A operand (NQ x NQ): M = NQ
// rows (outputs along the axis), K = NQ (inputs).  TRANS: A[x][m] = D[m][x]
// (the divergence), else A[x][m] = D[x][m] (the gradient).
template <int NQ, class F>
struct AFrag;

template <int NQ>
struct AFrag<NQ, double> {
  static constexpr int MT = NQ / 8, KT = NQ / 4;   // m-tiles of 8, k-steps of 4
  double a[MT][KT];
  template <bool TRANS>
  __device__ void load(const double* sD, int lane) {
    const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int kt = 0; kt < KT; ++kt) {
        const int x = mt * 8 + g, m = kt * 4 + t4;
        a[mt][kt] = TRANS ? sD[m * NQ + x] : sD[x * NQ + m];
      }
  }
};

template <int NQ>
struct AFrag<NQ, float> {
  static constexpr int MT = NQ / 16, KT = NQ / 8;  // m-tiles of 16, k-steps of 8
  uint32_t hi[MT][KT][4], lo[MT][KT][4];
  template <bool TRANS>
  __device__ void load(const float* sD, int lane) {
    const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int kt = 0; kt < KT; ++kt)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int x = mt * 16 + g + ((r & 1) ? 8 : 0), m = kt * 8 + t4 + ((r & 2) ? 4 : 0);
          tf32_split(TRANS ? sD[m * NQ + x] : sD[x * NQ + m], hi[mt][kt][r], lo[mt][kt][r]);
        }
  }
};

// One axis of the element: out(x, n) = sum_m A[x][m] in(m, n) for the NCOL
// columns n = a + NQ b, the columns spread over the warps in tiles of 8.
// ACC: out += (the divergence sums), else out = (the gradients).
template <int NQ, bool ACC>
__device__ __forceinline__ void axis_mma(int d, const AFrag<NQ, double>& A, const double* in, double* out, int warp,
                                         int lane) {
  using Sh = MmaShape<NQ>;
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll 1
  for (int nt = warp; nt < Sh::NTILES; nt += Sh::WARPS) {
    double c[AFrag<NQ, double>::MT][2];
#pragma unroll
    for (int mt = 0; mt < AFrag<NQ, double>::MT; ++mt) c[mt][0] = c[mt][1] = 0.0;
    const int nb = nt * 8 + g;                   // this thread's B column
    const int ab = nb % NQ, bb = nb / NQ;
#pragma unroll
    for (int kt = 0; kt < AFrag<NQ, double>::KT; ++kt) {
      const double b = in[mma_off<NQ>(d, kt * 4 + t4, ab, bb)];
#pragma unroll
      for (int mt = 0; mt < AFrag<NQ, double>::MT; ++mt) dmma(c[mt][0], c[mt][1], A.a[mt][kt], b);
    }
#pragma unroll
    for (int mt = 0; mt < AFrag<NQ, double>::MT; ++mt)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int n = nt * 8 + 2 * t4 + e;
        const int o = mma_off<NQ>(d, mt * 8 + g, n % NQ, n / NQ);
        out[o] = ACC ? out[o] + c[mt][e] : c[mt][e];
      }
  }
}

template <int NQ, bool ACC>
__device__ __forceinline__ void axis_mma(int d, const AFrag<NQ, float>& A, const float* in, float* out, int warp,
                                         int lane) {
  using Sh = MmaShape<NQ>;
  using AF = AFrag<NQ, float>;
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll 1
  for (int nt = warp; nt < Sh::NTILES; nt += Sh::WARPS) {
    float c[AF::MT][4];
#pragma unroll
    for (int mt = 0; mt < AF::MT; ++mt) c[mt][0] = c[mt][1] = c[mt][2] = c[mt][3] = 0.f;
    const int nb = nt * 8 + g;
    const int ab = nb % NQ, bb = nb / NQ;
#pragma unroll
    for (int kt = 0; kt < AF::KT; ++kt) {
      uint32_t b0h, b0l, b1h, b1l;
      tf32_split(in[mma_off<NQ>(d, kt * 8 + t4, ab, bb)], b0h, b0l);
      tf32_split(in[mma_off<NQ>(d, kt * 8 + t4 + 4, ab, bb)], b1h, b1l);
#pragma unroll
      for (int mt = 0; mt < AF::MT; ++mt) {   // small terms first
        tmma(c[mt], A.lo[mt][kt], b0h, b1h);
        tmma(c[mt], A.hi[mt][kt], b0l, b1l);
        tmma(c[mt], A.hi[mt][kt], b0h, b1h);
      }
    }
#pragma unroll
    for (int mt = 0; mt < AF::MT; ++mt)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int n = nt * 8 + 2 * t4 + (r & 1);
        const int o = mma_off<NQ>(d, mt * 16 + g + ((r & 2) ? 8 : 0), n % NQ, n / NQ);
        out[o] = ACC ? out[o] + c[mt][r] : c[mt][r];
      }
  }
}

template <int NQ, int NF, bool DOT, class F>
__global__ void __launch_bounds__(MmaShape<NQ>::THREADS, 1)
ax_mma_affine_kernel(int Nelements, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
                     const F* __restrict__ wJ, const F* __restrict__ ggeo, const F* __restrict__ gllw,
                     const F* __restrict__ Dg, F lambda, const F* __restrict__ q, F* __restrict__ Aq,
                     const int* __restrict__ skip, CgFuse fuse) {
  if (skip && *skip) return;
  using Sh = MmaShape<NQ>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  F* sA = reinterpret_cast<F*>(smem_raw);   // q, then the lambda term and the divergence sums
  F* sU0 = sA + Sh::ARR;                    // gradients, then fluxes (r, s, t)
  F* sU1 = sU0 + Sh::ARR;
  F* sU2 = sU1 + Sh::ARR;
  __shared__ F sD[NQ * NQ];
  __shared__ F sW[NQ];

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int e = elementList[blockIdx.x];
  for (int n = t; n < NQ * NQ; n += Sh::THREADS) sD[n] = Dg[n];
  if (t < NQ) sW[t] = gllw[t];
  F G[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) G[c] = ggeo[6 * (size_t)e + c];
  const F eJ = wJ[e];
  __syncthreads();
  AFrag<NQ, F> Dgrad, Ddiv;
  Dgrad.template load<false>(sD, lane);
  Ddiv.template load<true>(sD, lane);

  double pdot = 0.0;
#pragma unroll 1
  for (int f = 0; f < NF; ++f) {
    const size_t lbase = ((size_t)e * NF + f) * Sh::NP;
    F rq[Sh::PER];
#pragma unroll
    for (int c = 0; c < Sh::PER; ++c) {
      const int n = t + c * Sh::THREADS;
      const int id = __ldg(G2L + lbase + n);
      rq[c] = id >= 0 ? q[id] : F(0);
      const int i = n % NQ, j = (n / NQ) % NQ, k = n / (NQ * NQ);
      sA[k * Sh::S2 + j * Sh::S1 + i] = rq[c];
    }
    __syncthreads();
    // gradients along r, s, t
    axis_mma<NQ, false>(0, Dgrad, sA, sU0, warp, lane);
    axis_mma<NQ, false>(1, Dgrad, sA, sU1, warp, lane);
    axis_mma<NQ, false>(2, Dgrad, sA, sU2, warp, lane);
    __syncthreads();
    // fluxes w G (ur, us, ut) and the lambda term, node by node
#pragma unroll
    for (int c = 0; c < Sh::PER; ++c) {
      const int n = t + c * Sh::THREADS;
      const int i = n % NQ, j = (n / NQ) % NQ, k = n / (NQ * NQ);
      const int o = k * Sh::S2 + j * Sh::S1 + i;
      const F w = sW[i] * sW[j] * sW[k];
      const F ur = sU0[o], us = sU1[o], ut = sU2[o];
      sU0[o] = w * (G[0] * ur + G[1] * us + G[2] * ut);
      sU1[o] = w * (G[1] * ur + G[3] * us + G[4] * ut);
      sU2[o] = w * (G[2] * ur + G[4] * us + G[5] * ut);
      sA[o] = lambda * eJ * w * rq[c];
    }
    __syncthreads();
    // divergence: the three transposed contractions, summed into sA in turn
    axis_mma<NQ, true>(0, Ddiv, sU0, sA, warp, lane);
    __syncthreads();
    axis_mma<NQ, true>(1, Ddiv, sU1, sA, warp, lane);
    __syncthreads();
    axis_mma<NQ, true>(2, Ddiv, sU2, sA, warp, lane);
    __syncthreads();
#pragma unroll
    for (int c = 0; c < Sh::PER; ++c) {
      const int n = t + c * Sh::THREADS;
      const int i = n % NQ, j = (n / NQ) % NQ, k = n / (NQ * NQ);
      const F v = sA[k * Sh::S2 + j * Sh::S1 + i];
      Aq[lbase + n] = v;
      if (DOT) pdot += (double)rq[c] * (double)v;
    }
    __syncthreads();   // sA is rewritten by the next field
  }
  if (DOT) fuse_pap(pdot, fuse, reinterpret_cast<double*>(sU0));
}

template <int NQ, class F>
int launch_mma_nq(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const F* wJ, const F* ggeo, const F* gllw, const F* D, F lambda, const F* q, F* Aq,
                  const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  using Sh = MmaShape<NQ>;
  const size_t smem = Sh::template smem<F>();
  const CgFuse Fz = fuse ? *fuse : CgFuse{};
  if (nblocks) *nblocks = Nelements;
#define BP_MMA_LAUNCH(NF, DOT)                                                                                  \
  do {                                                                                                          \
    static DeviceOnce configured;                                                                               \
    BP_TRY(once_per_device(configured, [smem]() -> int {                                                        \
      BP_CUDA_TRY(cudaFuncSetAttribute(ax_mma_affine_kernel<NQ, NF, DOT, F>,                                    \
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));               \
      return BP_SUCCESS;                                                                                        \
    }));                                                                                                        \
    ax_mma_affine_kernel<NQ, NF, DOT, F><<<Nelements, Sh::THREADS, smem, s>>>(Nelements, elementList, G2L, wJ,  \
                                                                             ggeo, gllw, D, lambda, q, Aq,    \
                                                                             skip, Fz);                        \
  } while (0)
  if (d.Nfields == 3) {
    if (fuse) BP_MMA_LAUNCH(3, true); else BP_MMA_LAUNCH(3, false);
  } else {
    if (fuse) BP_MMA_LAUNCH(1, true); else BP_MMA_LAUNCH(1, false);
  }
#undef BP_MMA_LAUNCH
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

template <class F>
int launch_ax_mma_t(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                    const F* wJ, const F* ggeo, const F* gllw, const F* D, F lambda, const F* q, F* Aq,
                    const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  if (!d.affine || (d.Nfields != 1 && d.Nfields != 3)) return 1;
  switch (d.N + 1) {
    case 16:
      return launch_mma_nq<16, F>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, fuse, s,
                                  nblocks);
    default:
      return 1;
  }
}

}  // namespace

int launch_ax_mma(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const double* wJ, const double* ggeo, const double* gllw, const double* D, double lambda,
                  const double* q, double* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  return launch_ax_mma_t<double>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, fuse, s,
                                 nblocks);
}

int launch_ax_mma(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const float* wJ, const float* ggeo, const float* gllw, const float* D, float lambda,
                  const float* q, float* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  return launch_ax_mma_t<float>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, fuse, s,
                                nblocks);
}

}  // namespace bp
