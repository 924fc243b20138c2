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
// through shared memory in three arrays of NQ^3 with padded strides that keep
// the FP64 fragment loads of all three axes free of bank conflicts.  A warp's
// n-tile reads and writes the same 8 columns of a slab, so a contraction may
// overwrite its own input: the s and t gradients go to two arrays, then the r
// gradient replaces q, the fluxes replace the gradients, and each divergence
// contraction replaces its flux; the sum and the mass term are formed at the
// end, q coming from registers.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>

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
  static constexpr size_t smem() { return sizeof(F) * 3 * (size_t)ARR; }
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
// columns n = a + NQ b, the columns spread over the warps in tiles of 8.  out
// may be in: a tile's loads all precede its stores.
template <int NQ, int TERMS = 1>
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
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < AFrag<NQ, double>::MT; ++mt)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int n = nt * 8 + 2 * t4 + e;
        out[mma_off<NQ>(d, mt * 8 + g, n % NQ, n / NQ)] = c[mt][e];
      }
  }
}

// TERMS = 3: the split product; 1: plain TF32 (a_hi b_hi only), kept for the
// precision experiment behind BP_MMA_TF32_TERMS=1
template <int NQ, int TERMS = 3>
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
        if (TERMS == 3) {
          tmma(c[mt], A.lo[mt][kt], b0h, b1h);
          tmma(c[mt], A.hi[mt][kt], b0l, b1l);
        }
        tmma(c[mt], A.hi[mt][kt], b0h, b1h);
      }
    }
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < AF::MT; ++mt)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int n = nt * 8 + 2 * t4 + (r & 1);
        out[mma_off<NQ>(d, mt * 16 + g + ((r & 2) ? 8 : 0), n % NQ, n / NQ)] = c[mt][r];
      }
  }
}

template <int NQ, int NF, bool DOT, class F, int TERMS = 3>
__global__ void __launch_bounds__(MmaShape<NQ>::THREADS, sizeof(F) == 4 ? 2 : 1)
ax_mma_affine_kernel(int Nelements, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
                     const F* __restrict__ wJ, const F* __restrict__ ggeo, const F* __restrict__ gllw,
                     const F* __restrict__ Dg, F lambda, const F* __restrict__ q, F* __restrict__ Aq,
                     const int* __restrict__ skip, CgFuse fuse) {
  if (skip && *skip) return;
  using Sh = MmaShape<NQ>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  F* sA = reinterpret_cast<F*>(smem_raw);   // q, then the r gradient, flux and divergence
  F* sU1 = sA + Sh::ARR;                    // the s gradient, flux and divergence
  F* sU2 = sU1 + Sh::ARR;                   // the t ones
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
    // gradients: s and t from q, then r over q itself
    axis_mma<NQ, TERMS>(1, Dgrad, sA, sU1, warp, lane);
    axis_mma<NQ, TERMS>(2, Dgrad, sA, sU2, warp, lane);
    __syncthreads();
    axis_mma<NQ, TERMS>(0, Dgrad, sA, sA, warp, lane);
    __syncthreads();
    // fluxes w G (ur, us, ut), node by node
#pragma unroll
    for (int c = 0; c < Sh::PER; ++c) {
      const int n = t + c * Sh::THREADS;
      const int i = n % NQ, j = (n / NQ) % NQ, k = n / (NQ * NQ);
      const int o = k * Sh::S2 + j * Sh::S1 + i;
      const F w = sW[i] * sW[j] * sW[k];
      const F ur = sA[o], us = sU1[o], ut = sU2[o];
      sA[o] = w * (G[0] * ur + G[1] * us + G[2] * ut);
      sU1[o] = w * (G[1] * ur + G[3] * us + G[4] * ut);
      sU2[o] = w * (G[2] * ur + G[4] * us + G[5] * ut);
    }
    __syncthreads();
    // divergence: each transposed contraction over its own flux
    axis_mma<NQ, TERMS>(0, Ddiv, sA, sA, warp, lane);
    axis_mma<NQ, TERMS>(1, Ddiv, sU1, sU1, warp, lane);
    axis_mma<NQ, TERMS>(2, Ddiv, sU2, sU2, warp, lane);
    __syncthreads();
#pragma unroll
    for (int c = 0; c < Sh::PER; ++c) {
      const int n = t + c * Sh::THREADS;
      const int i = n % NQ, j = (n / NQ) % NQ, k = n / (NQ * NQ);
      const int o = k * Sh::S2 + j * Sh::S1 + i;
      const F w = sW[i] * sW[j] * sW[k];
      const F v = lambda * eJ * w * rq[c] + sA[o] + sU1[o] + sU2[o];
      Aq[lbase + n] = v;
      if (DOT) pdot += (double)rq[c] * (double)v;
    }
    __syncthreads();   // sA is rewritten by the next field
  }
  if (DOT) fuse_pap(pdot, fuse, reinterpret_cast<double*>(sU1));
}

// ---------------------------------------------------------------------------
// Stored-factor FP32 operator on PK = 4 right-hand sides packed per node, at
// Nq = 8 (the mixed-precision BP5 inner operator of a packed group): each
// direction is 256 lines (the two other node indices x 4 lanes) times the
// 8 x 8 matrix, m16n8k8 TF32 MMAs with the data as the A operand (16 lines per
// tile, both parts of its TF32 split) and D^T (gradient) or D (divergence) as
// the constant B operand.  A warp's tile reads and writes the same 16 lines,
// so each divergence contraction runs in place, with no barrier between the
// three directions.  Factors of the thread's nodes are loaded into registers
// while the gradients run.
// ---------------------------------------------------------------------------
template <int NQ>
struct Pk4Shape {
  static_assert(NQ == 8, "packed tensor-core operator: Nq = 8");
  static constexpr int S1 = 12;                // node stride of j: i- and k-lines load conflict-free
  static constexpr int S2 = 98;                // node stride of k
  static constexpr int NODES = NQ * S2;        // padded nodes of one array (float4 each)
  static constexpr int NP = NQ * NQ * NQ;
  static constexpr int THREADS = 128;
  static constexpr int WARPS = THREADS / 32;
  static constexpr int MTILES = NQ * NQ * 4 / 16;   // tiles of 16 lines per direction
  static constexpr int PER = NP / THREADS;     // nodes per thread in the pointwise phases
  static constexpr size_t SMEM = sizeof(float4) * 4 * (size_t)NODES;
};

template <int NQ>
__device__ __forceinline__ int pk_off(int d, int x, int a, int b) {
  using Sh = Pk4Shape<NQ>;
  return d == 0 ? b * Sh::S2 + a * Sh::S1 + x : d == 1 ? b * Sh::S2 + x * Sh::S1 + a : x * Sh::S2 + b * Sh::S1 + a;
}

__device__ __forceinline__ float lane_of(const float4& v, int l) {
  return l == 0 ? v.x : l == 1 ? v.y : l == 2 ? v.z : v.w;
}

// one direction d over this warp's tiles: out(line, x) = sum_m in(line, m) B[m][x]
// (in and out may be the same array: a tile touches only its own lines)
template <int NQ>
__device__ __forceinline__ void pk_axis(int d, const uint32_t (&bh)[2], const uint32_t (&bl)[2], const float* in,
                                        float* out, int warp, int lane) {
  using Sh = Pk4Shape<NQ>;
  const int g = lane >> 2, t4 = lane & 3, l = g & 3;
#pragma unroll 1
  for (int T = warp; T < Sh::MTILES; T += Sh::WARPS) {
    const int b = T >> 1, a = (T & 1) * 4 + (g >> 2);   // rows g (a) and g + 8 (a + 2)
    uint32_t ah[4], al[4];
    tf32_split(in[4 * pk_off<NQ>(d, t4, a, b) + l], ah[0], al[0]);
    tf32_split(in[4 * pk_off<NQ>(d, t4, a + 2, b) + l], ah[1], al[1]);
    tf32_split(in[4 * pk_off<NQ>(d, t4 + 4, a, b) + l], ah[2], al[2]);
    tf32_split(in[4 * pk_off<NQ>(d, t4 + 4, a + 2, b) + l], ah[3], al[3]);
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    tmma(c, al, bh[0], bh[1]);   // small terms first
    tmma(c, ah, bl[0], bl[1]);
    tmma(c, ah, bh[0], bh[1]);
    __syncwarp();                // every lane's loads of this tile are done before any store
    out[4 * pk_off<NQ>(d, 2 * t4, a, b) + l] = c[0];
    out[4 * pk_off<NQ>(d, 2 * t4 + 1, a, b) + l] = c[1];
    out[4 * pk_off<NQ>(d, 2 * t4, a + 2, b) + l] = c[2];
    out[4 * pk_off<NQ>(d, 2 * t4 + 1, a + 2, b) + l] = c[3];
  }
}

template <int NQ, bool DOT>
__global__ void __launch_bounds__(Pk4Shape<NQ>::THREADS, 4)
ax_mma_pk4_kernel(int Nelements, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
                  const float* __restrict__ wJ, const float* __restrict__ ggeo, const float* __restrict__ Dg,
                  float lambda, const float4* __restrict__ q, float4* __restrict__ Aq, const int* __restrict__ skip,
                  CgFuse fuse) {
  if (skip && *skip) return;
  using Sh = Pk4Shape<NQ>;
  extern __shared__ __align__(16) float4 smem4[];
  float4* sQ = smem4;
  float4* sU0 = sQ + Sh::NODES;   // the three directions' arrays follow, NODES apart
  float4* sU1 = sU0 + Sh::NODES;
  float4* sU2 = sU1 + Sh::NODES;
  __shared__ float sD[NQ * NQ];

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int e = elementList[blockIdx.x];
  const size_t ebase = (size_t)e * Sh::NP;
  if (t < NQ * NQ) sD[t] = Dg[t];
  float4 rq[Sh::PER];
#pragma unroll
  for (int c = 0; c < Sh::PER; ++c) {
    const int n = t + c * Sh::THREADS;
    const int id = __ldg(G2L + ebase + n);
    rq[c] = id >= 0 ? q[id] : make_float4(0.f, 0.f, 0.f, 0.f);
    sQ[pk_off<NQ>(0, n % NQ, (n / NQ) % NQ, n / (NQ * NQ))] = rq[c];
  }
  __syncthreads();
  // B operands: gradient B[m][x] = D[x][m], divergence B[m][x] = D[m][x]
  const int g = lane >> 2, t4 = lane & 3;
  uint32_t gh[2], gl[2], vh[2], vl[2];
  tf32_split(sD[g * NQ + t4], gh[0], gl[0]);
  tf32_split(sD[g * NQ + t4 + 4], gh[1], gl[1]);
  tf32_split(sD[t4 * NQ + g], vh[0], vl[0]);
  tf32_split(sD[(t4 + 4) * NQ + g], vh[1], vl[1]);
  const float* fQ = reinterpret_cast<const float*>(sQ);
#pragma unroll 1
  for (int d = 0; d < 3; ++d) pk_axis<NQ>(d, gh, gl, fQ, reinterpret_cast<float*>(sU0 + d * Sh::NODES), warp, lane);
  // the factors of this thread's nodes (in flight while the gradients ran)
  float G[Sh::PER][6], J[Sh::PER];
#pragma unroll
  for (int c = 0; c < Sh::PER; ++c) {
    const int n = t + c * Sh::THREADS;
    const float2* g2 = reinterpret_cast<const float2*>(ggeo + 6 * (ebase + n));
    const float2 x0 = __ldg(g2), x1 = __ldg(g2 + 1), x2 = __ldg(g2 + 2);
    G[c][0] = x0.x; G[c][1] = x0.y; G[c][2] = x1.x; G[c][3] = x1.y; G[c][4] = x2.x; G[c][5] = x2.y;
    J[c] = __ldg(wJ + ebase + n);
  }
  __syncthreads();
  // fluxes G (ur, us, ut), node by node (G00 G01 G02 G11 G12 G22)
#pragma unroll
  for (int c = 0; c < Sh::PER; ++c) {
    const int n = t + c * Sh::THREADS;
    const int o = pk_off<NQ>(0, n % NQ, (n / NQ) % NQ, n / (NQ * NQ));
    const float4 ur = sU0[o], us = sU1[o], ut = sU2[o];
    const float* Gc = G[c];
    sU0[o] = make_float4(Gc[0] * ur.x + Gc[1] * us.x + Gc[2] * ut.x, Gc[0] * ur.y + Gc[1] * us.y + Gc[2] * ut.y,
                           Gc[0] * ur.z + Gc[1] * us.z + Gc[2] * ut.z, Gc[0] * ur.w + Gc[1] * us.w + Gc[2] * ut.w);
    sU1[o] = make_float4(Gc[1] * ur.x + Gc[3] * us.x + Gc[4] * ut.x, Gc[1] * ur.y + Gc[3] * us.y + Gc[4] * ut.y,
                           Gc[1] * ur.z + Gc[3] * us.z + Gc[4] * ut.z, Gc[1] * ur.w + Gc[3] * us.w + Gc[4] * ut.w);
    sU2[o] = make_float4(Gc[2] * ur.x + Gc[4] * us.x + Gc[5] * ut.x, Gc[2] * ur.y + Gc[4] * us.y + Gc[5] * ut.y,
                           Gc[2] * ur.z + Gc[4] * us.z + Gc[5] * ut.z, Gc[2] * ur.w + Gc[4] * us.w + Gc[5] * ut.w);
  }
  __syncthreads();
  // divergence, each direction in place
#pragma unroll 1
  for (int d = 0; d < 3; ++d) {
    float* u = reinterpret_cast<float*>(sU0 + d * Sh::NODES);
    pk_axis<NQ>(d, vh, vl, u, u, warp, lane);
  }
  __syncthreads();
  double v[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int c = 0; c < Sh::PER; ++c) {
    const int n = t + c * Sh::THREADS;
    const int o = pk_off<NQ>(0, n % NQ, (n / NQ) % NQ, n / (NQ * NQ));
    const float4 a = sU0[o], b = sU1[o], cc = sU2[o];
    const float m = lambda * J[c];
    const float4 r = make_float4(m * rq[c].x + a.x + b.x + cc.x, m * rq[c].y + a.y + b.y + cc.y,
                                 m * rq[c].z + a.z + b.z + cc.z, m * rq[c].w + a.w + b.w + cc.w);
    Aq[ebase + n] = r;
    if (DOT) {
      v[0] += (double)rq[c].x * r.x;
      v[1] += (double)rq[c].y * r.y;
      v[2] += (double)rq[c].z * r.z;
      v[3] += (double)rq[c].w * r.w;
    }
  }
  if (DOT) {
    double bs[4];
    fuse_block_sum_lanes<4>(v, reinterpret_cast<double*>(smem4), bs);
    if (t == 0)
#pragma unroll
      for (int l = 0; l < 4; ++l) fuse.partials[(size_t)l * gridDim.x + blockIdx.x] = bs[l];
  }
}

template <int NQ, class F>
int launch_mma_nq(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const F* wJ, const F* ggeo, const F* gllw, const F* D, F lambda, const F* q, F* Aq,
                  const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  using Sh = MmaShape<NQ>;
  const size_t smem = Sh::template smem<F>();
  const CgFuse Fz = fuse ? *fuse : CgFuse{};
  if (nblocks) *nblocks = Nelements;
  // BP_MMA_TF32_TERMS=1 (FP32 only): plain TF32 products instead of the split
  // ones, an experiment on how much operator precision the mixed CG needs
  const char* terms_env = getenv("BP_MMA_TF32_TERMS");
  const bool plain = sizeof(F) == 4 && terms_env && terms_env[0] == '1';
#define BP_MMA_LAUNCH(NF, DOT, TERMS)                                                                           \
  do {                                                                                                          \
    static DeviceOnce configured;                                                                               \
    BP_TRY(once_per_device(configured, [smem]() -> int {                                                        \
      BP_CUDA_TRY(cudaFuncSetAttribute(ax_mma_affine_kernel<NQ, NF, DOT, F, TERMS>,                             \
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));               \
      return BP_SUCCESS;                                                                                        \
    }));                                                                                                        \
    ax_mma_affine_kernel<NQ, NF, DOT, F, TERMS><<<Nelements, Sh::THREADS, smem, s>>>(                          \
        Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, Fz);                               \
  } while (0)
  if (plain) {
    if (d.Nfields == 3) {
      if (fuse) BP_MMA_LAUNCH(3, true, 1); else BP_MMA_LAUNCH(3, false, 1);
    } else {
      if (fuse) BP_MMA_LAUNCH(1, true, 1); else BP_MMA_LAUNCH(1, false, 1);
    }
  } else if (d.Nfields == 3) {
    if (fuse) BP_MMA_LAUNCH(3, true, 3); else BP_MMA_LAUNCH(3, false, 3);
  } else {
    if (fuse) BP_MMA_LAUNCH(1, true, 3); else BP_MMA_LAUNCH(1, false, 3);
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

int launch_ax_mma_packed(int pk, const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList,
                         const int32_t* G2L, const float* wJ, const float* ggeo, const float* D, float lambda,
                         const float* q, float* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s,
                         int* nblocks) {
  if (pk != 4 || d.affine || d.Nfields != 1 || d.N + 1 != 8 ||
      ((reinterpret_cast<uintptr_t>(q) | reinterpret_cast<uintptr_t>(Aq)) & 15) || (reinterpret_cast<uintptr_t>(ggeo) & 7))
    return 1;
  using Sh = Pk4Shape<8>;
  const CgFuse Fz = fuse ? *fuse : CgFuse{};
  if (nblocks) *nblocks = Nelements;
  if (Nelements == 0) return BP_SUCCESS;
  const float4* q4 = reinterpret_cast<const float4*>(q);
  float4* a4 = reinterpret_cast<float4*>(Aq);
#define BP_PK_LAUNCH(DOT)                                                                                      \
  do {                                                                                                         \
    static DeviceOnce configured;                                                                              \
    BP_TRY(once_per_device(configured, []() -> int {                                                           \
      BP_CUDA_TRY(cudaFuncSetAttribute(ax_mma_pk4_kernel<8, DOT>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                       (int)Sh::SMEM));                                                        \
      return BP_SUCCESS;                                                                                       \
    }));                                                                                                       \
    ax_mma_pk4_kernel<8, DOT><<<Nelements, Sh::THREADS, Sh::SMEM, s>>>(Nelements, elementList, G2L, wJ, ggeo, D, \
                                                                      lambda, q4, a4, skip, Fz);              \
  } while (0)
  if (fuse) BP_PK_LAUNCH(true); else BP_PK_LAUNCH(false);
#undef BP_PK_LAUNCH
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

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
