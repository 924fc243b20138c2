// Device kernels of the BK/BP Hex3D hot path for sm_100a (FP64).
//
//  - ax_pencil_kernel   element-local stiffness + lambda*mass operator
//                       (reference: okl/bp5AxHex3D.okl, okl/bp5AxAffineHex3D.okl,
//                        okl/bp6AxHex3D.okl)
//  - gather_kernel      CSR Trans gather, one row per thread, column order kept
//                       (reference: libs/ogs/okl/ogsKernels.okl:86-122)
//  - geometry_kernel    geometric factors from the trilinear vertex map
//                       (reference: libs/mesh/meshGeometricFactorsHex3D.cpp:31-153)
//  - forcing / mass / diagonal kernels used by the problem setup
//  - vector and deterministic reduction kernels (linAlg / updateCG)
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <string>
#include <type_traits>

#include "bp_cg_device.cuh"
#include "bp_internal.hpp"

namespace bp {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 1184;   // fixed so reductions are reproducible run to run

int reduction_blocks() { return kRedBlocks; }

// ---------------------------------------------------------------------------
// Element-local operator, register-pencil form.
//
// Thread (i,j) of element slot es holds the pencil q(i,j,0:NQ-1) and the
// accumulators Aq(i,j,0:NQ-1) in registers and walks the k-slices; the (i,j)
// slice of q and the r/s fluxes go through shared memory.  Geometric factors of
// slice k+1 are prefetched while slice k is computed.  Each element is the sum
//   Aq = Dr^T(G00 ur + G01 us + G02 ut) + Ds^T(G01 ur + G11 us + G12 ut)
//      + Dt^T(G02 ur + G12 us + G22 ut) + lambda wJ q,
// (ur,us,ut) = (Dr q, Ds q, Dt q), the same operator as the reference kernels.
// ---------------------------------------------------------------------------
template <int NQ>
struct AxShape {
  static constexpr int EPB = NQ <= 2 ? 32 : NQ <= 3 ? 16 : NQ <= 4 ? 16 : NQ <= 5 ? 8 : NQ <= 8 ? 4 : NQ <= 11 ? 2 : 1;
  static constexpr bool DREG = NQ <= 12;   // keep the D rows of i and j in registers
  static constexpr int MINB = NQ <= 8 ? 2 : 1; // resident blocks per SM the register budget must allow
};

template <int NQ, int NF, bool AFFINE, bool VEC, bool DOT, class F>
__global__ void __launch_bounds__(NQ * NQ * AxShape<NQ>::EPB, AxShape<NQ>::MINB)
ax_pencil_kernel(int Nelements, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
                 const F* __restrict__ wJ, const F* __restrict__ ggeo, const F* __restrict__ gllw,
                 const F* __restrict__ Dg, F lambda, const F* __restrict__ q, F* __restrict__ Aq,
                 const int* __restrict__ skip, CgFuse fuse) {
  pdl_wait();
  pdl_release();
  if (skip && *skip) return;
  using V2 = typename std::conditional<sizeof(F) == 8, double2, float2>::type;
  constexpr int EPB = AxShape<NQ>::EPB;
  constexpr int NP = NQ * NQ * NQ;
  constexpr int NQ2 = NQ * NQ;
  constexpr int PAD = (NQ % 2 == 0) ? 1 : 0;
  __shared__ F s_D[NQ][NQ + 1];
  __shared__ F s_gw[NQ];
  __shared__ F s_q[EPB][NQ][NQ + PAD];
  __shared__ F s_v[EPB][NQ][NQ + PAD];
  __shared__ F s_w[EPB][NQ][NQ + PAD];
  // one double per thread for the p.Ap block sum (DOT)
  __shared__ double s_red[DOT ? NQ * NQ * EPB : 1];

  const int i = threadIdx.x, j = threadIdx.y, es = threadIdx.z;
  const int t = i + NQ * (j + NQ * es);
  for (int n = t; n < NQ2; n += NQ2 * EPB) s_D[n / NQ][n % NQ] = Dg[n];
  if (AFFINE)
    for (int n = t; n < NQ; n += NQ2 * EPB) s_gw[n] = gllw[n];
  const int eIdx = blockIdx.x * EPB + es;
  const bool active = eIdx < Nelements;
  const int e = active ? elementList[eIdx] : 0;
  __syncthreads();

  F Di[AxShape<NQ>::DREG ? NQ : 1], Dj[AxShape<NQ>::DREG ? NQ : 1];
  if (AxShape<NQ>::DREG) {
#pragma unroll
    for (int m = 0; m < NQ; ++m) {
      Di[m] = s_D[i][m];
      Dj[m] = s_D[j][m];
    }
  }

  F aG[6] = {0, 0, 0, 0, 0, 0}, aJ = 0, wij = 0;
  if (AFFINE) {
    if (active) {
#pragma unroll
      for (int c = 0; c < 6; ++c) aG[c] = ggeo[6 * (size_t)e + c];
      aJ = wJ[e];
    }
    wij = s_gw[i] * s_gw[j];
  }

  double pdot = 0.0;   // sum of q*Aq over this thread's nodes (DOT)
#pragma unroll 1
  for (int f = 0; f < NF; ++f) {
    const size_t lbase = ((size_t)e * NF + f) * NP + j * NQ + i;
    const size_t gbase = (size_t)e * NP + j * NQ + i;
    F r_u[NQ], r_Au[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      const int id = active ? __ldg(G2L + lbase + k * NQ2) : -1;
      r_u[k] = (id >= 0) ? __ldg(q + id) : F(0);
      r_Au[k] = F(0);
    }

    // prefetch slice 0 of the geometric factors
    F n00 = 0, n01 = 0, n02 = 0, n11 = 0, n12 = 0, n22 = 0, nJ = 0;
    auto load_factors = [&](size_t gb) {
      if (VEC) {
        const V2* g2 = reinterpret_cast<const V2*>(ggeo + 6 * gb);
        const V2 a = g2[0], b = g2[1], c = g2[2];
        n00 = a.x; n01 = a.y; n02 = b.x; n11 = b.y; n12 = c.x; n22 = c.y;
      } else {
        const F* g = ggeo + 6 * gb;
        n00 = __ldg(g); n01 = __ldg(g + 1); n02 = __ldg(g + 2);
        n11 = __ldg(g + 3); n12 = __ldg(g + 4); n22 = __ldg(g + 5);
      }
      nJ = __ldg(wJ + gb);
    };
    if (!AFFINE && active) load_factors(gbase);

#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      F G00, G01, G02, G11, G12, G22, GwJ;
      if (AFFINE) {
        const F w = wij * s_gw[k];
        G00 = aG[0] * w; G01 = aG[1] * w; G02 = aG[2] * w;
        G11 = aG[3] * w; G12 = aG[4] * w; G22 = aG[5] * w;
        GwJ = aJ * w;
      } else {
        G00 = n00; G01 = n01; G02 = n02; G11 = n11; G12 = n12; G22 = n22; GwJ = nJ;
        if (k + 1 < NQ && active) load_factors(gbase + (size_t)(k + 1) * NQ2);
      }

      s_q[es][j][i] = r_u[k];
      __syncthreads();

      F ur = 0, us = 0, ut = 0;
#pragma unroll
      for (int m = 0; m < NQ; ++m) ut += s_D[k][m] * r_u[m];
#pragma unroll
      for (int m = 0; m < NQ; ++m) {
        const F dim = AxShape<NQ>::DREG ? Di[m] : s_D[i][m];
        const F djm = AxShape<NQ>::DREG ? Dj[m] : s_D[j][m];
        ur += dim * s_q[es][j][m];
        us += djm * s_q[es][m][i];
      }
      s_w[es][j][i] = G01 * ur + G11 * us + G12 * ut;
      s_v[es][j][i] = G00 * ur + G01 * us + G02 * ut;
      const F GDut = G02 * ur + G12 * us + G22 * ut;
      F Auk = GwJ * lambda * r_u[k];
      __syncthreads();

#pragma unroll
      for (int m = 0; m < NQ; ++m) r_Au[m] += s_D[k][m] * GDut;
#pragma unroll
      for (int m = 0; m < NQ; ++m) {
        Auk += s_D[m][j] * s_w[es][m][i];
        Auk += s_D[m][i] * s_v[es][j][m];
      }
      r_Au[k] += Auk;
    }
    if (active) {
#pragma unroll
      for (int k = 0; k < NQ; ++k) Aq[lbase + k * NQ2] = r_Au[k];
      if (DOT) {
#pragma unroll
        for (int k = 0; k < NQ; ++k) pdot += (double)r_u[k] * (double)r_Au[k];
      }
    }
  }
  if (DOT) fuse_pap(pdot, fuse, s_red);
}

// Kernel variant of the element operator: stored factors use the TMA-staged
// kernel where it applies and the line-per-thread kernel (bp_ax_line.cuh)
// elsewhere; affine factors the tensor-core kernel at Nq = 16 (bp_ax_mma.cu),
// else the line kernel in FP32 and the register-pencil kernel in FP64.
// BP_AX_VARIANT=pencil, =line, =tma or =mma in the environment selects that
// kernel wherever it applies (for comparisons).
int ax_variant() {   // read at every launch, so a process (a test) can switch forms
  const char* e = getenv("BP_AX_VARIANT");
  if (!e) return AX_AUTO;
  const std::string s = e;
  return s == "pencil" ? AX_PENCIL : s == "line" ? AX_LINE : s == "mma" ? AX_MMA : s == "tma" ? AX_TMA :
         s == "rb" ? AX_RB : AX_AUTO;
}

// The register-pencil form (FP64 affine default; any configuration)
template <int NQ, class F>
static int launch_pencil(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                         const F* wJ, const F* ggeo, const F* gllw, const F* D, F lambda, const F* q, F* Aq,
                         const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  constexpr int EPB = AxShape<NQ>::EPB;
  const dim3 block(NQ, NQ, EPB);
  const dim3 grid((Nelements + EPB - 1) / EPB);
  if (nblocks) *nblocks = (int)grid.x;
  const bool vec = ((reinterpret_cast<uintptr_t>(ggeo) & (2 * sizeof(F) - 1)) == 0);
  const CgFuse Fz = fuse ? *fuse : CgFuse{};
#define BP_PENCIL(NF, AFF, VEC, DOT)                                                                             \
  BP_CUDA_TRY(launch_pdl(ax_pencil_kernel<NQ, NF, AFF, VEC, DOT, F>, grid, block, 0, s, Nelements, elementList, G2L, \
                         wJ, ggeo, gllw, D, lambda, q, Aq, skip, Fz))
  if (fuse) {
    if (!d.affine && !vec) return fail(BP_ERROR_ARG, "CG operator needs aligned geometric factors");
    if (d.Nfields == 1) {
      if (d.affine) BP_PENCIL(1, true, true, true); else BP_PENCIL(1, false, true, true);
    } else {
      if (d.affine) BP_PENCIL(3, true, true, true); else BP_PENCIL(3, false, true, true);
    }
  } else if (d.Nfields == 1) {
    if (d.affine) BP_PENCIL(1, true, true, false);
    else if (vec) BP_PENCIL(1, false, true, false);
    else BP_PENCIL(1, false, false, false);
  } else {
    if (d.affine) BP_PENCIL(3, true, true, false);
    else if (vec) BP_PENCIL(3, false, true, false);
    else BP_PENCIL(3, false, false, false);
  }
#undef BP_PENCIL
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

// One form of the element operator; 1 when it does not apply to d
template <int NQ, class F>
static int launch_ax_form(int form, const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList,
                          const int32_t* G2L, const F* wJ, const F* ggeo, const F* gllw, const F* D, F lambda,
                          const F* q, F* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  switch (form) {
    case FORM_MMA:
      return launch_ax_mma(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, fuse, s, nblocks);
    case FORM_TMA:
      return d.affine ? 1
                      : launch_ax_tma(d, Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, fuse, s,
                                      nblocks);
    case FORM_LINE:
      return launch_ax_line(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, s, fuse, nblocks);
    default:
      return launch_pencil<NQ, F>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, fuse, s,
                                  nblocks);
  }
}

// The forms that may serve d, the measured static choice first (40^3 or 24^3
// boxes): stored factors the TMA kernel where it applies (even Nq), else the
// line kernel (FP32 mixed BP5 p=10: 0.61 vs 1.15 s pencil; FP64 BK5 p=6 0.6
// vs 0.7 ms); affine factors the tensor-core kernel at Nq = 16 (BK6 p=15 FP64
// 2.3 vs 7.5 ms, FP32 1.4 vs 4.0 ms), else the line kernel in FP32 and the
// pencil kernel in FP64 (BK5 p=7 0.6 vs 0.8 ms).  The autotuner measures them
// all on first use and keeps the fastest.
template <int NQ, class F>
static std::vector<int> ax_forms(const bp_ax_desc_t& d) {
  std::vector<int> f;
  if (d.affine) {
    if (NQ == 16) f.push_back(FORM_MMA);
    if (sizeof(F) == 4) {
      f.push_back(FORM_LINE);
      f.push_back(FORM_PENCIL);
    } else {
      f.push_back(FORM_PENCIL);
      f.push_back(FORM_LINE);
    }
  } else {
    f = {FORM_TMA, FORM_LINE, FORM_PENCIL};
  }
  return f;
}

template <int NQ, class F>
static int launch_ax_nq(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList,
                        const int32_t* G2L, const F* wJ, const F* ggeo, const F* gllw, const F* D, F lambda,
                        const F* q, F* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  const std::vector<int> forms = ax_forms<NQ, F>(d);
  auto run = [&](int f, const int* sk) {
    return launch_ax_form<NQ, F>(f, d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, sk, fuse, s,
                                 nblocks);
  };
  int form = forms[0];
  const int v = ax_variant();
  if (v != AX_AUTO) {
    form = v == AX_MMA ? FORM_MMA : v == AX_TMA ? FORM_TMA : v == AX_LINE ? FORM_LINE : FORM_PENCIL;
  } else {
    const TuneConfig cfg{0, NQ, d.Nfields, d.affine, (int)sizeof(F), 1, fuse != nullptr, element_class(Nelements)};
    BP_TRY(tuned_form(cfg, forms, [&](int f) { return run(f, nullptr); }, s, &form));
  }
  int rc = run(form, skip);
  for (size_t k = 0; rc == 1 && k < forms.size(); ++k) rc = run(forms[k], skip);   // a forced form that does not apply
  return rc == 1 ? fail(BP_ERROR_ARG, "element operator: no kernel form covers this configuration") : rc;
}

// The packed FP32 operator (pk right-hand sides per node, stored or affine
// factors, one field) in its tuned form: TMA-staged (even Nq >= 8, the static
// choice), line-per-thread (Nq <= 12), or tensor-core (Nq = 8, four lanes).
int launch_ax_packed(int pk, const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList,
                     const int32_t* G2L, const float* wJ, const float* ggeo, const float* gllw, const float* D,
                     float lambda, const float* q, float* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s,
                     int* nblocks) {
  if (d.dim == 2) return fail(BP_ERROR_ARG, "packed element operator: Hex3D only");
  auto run = [&](int f, const int* sk) -> int {
    switch (f) {
      case FORM_MMA:
        return launch_ax_mma_packed(pk, d, Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, sk, fuse, s,
                                    nblocks);
      case FORM_TMA:
        return launch_ax_tma_packed(pk, d, Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, sk, fuse, s,
                                    nblocks);
      case FORM_RB:
        return launch_ax_rb_packed(pk, d, Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, sk, fuse, s,
                                   nblocks);
      default:
        if (d.N + 1 > 12) return 1;
        return launch_ax_line_packed(pk, d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, sk, fuse,
                                     s, nblocks);
    }
  };
  const std::vector<int> forms = {FORM_TMA, FORM_RB, FORM_LINE, FORM_MMA};
  int form = forms[0];
  const int v = ax_variant();
  if (v != AX_AUTO) {
    form = v == AX_MMA ? FORM_MMA : v == AX_TMA ? FORM_TMA : v == AX_RB ? FORM_RB : FORM_LINE;
  } else {
    const TuneConfig cfg{1, d.N + 1, d.Nfields, d.affine, 4, pk, fuse != nullptr, element_class(Nelements)};
    BP_TRY(tuned_form(cfg, forms, [&](int f) { return run(f, nullptr); }, s, &form));
  }
  int rc = run(form, skip);
  for (size_t k = 0; rc == 1 && k < forms.size(); ++k) rc = run(forms[k], skip);
  return rc == 1 ? fail(BP_ERROR_ARG, "packed element operator: no kernel form covers this configuration") : rc;
}

int ax_current_form(const bp_ax_desc_t& d, int bytes, int lanes, int32_t Nelements) {
  const int v = ax_variant();
  if (lanes > 1) {
    if (v != AX_AUTO) return v == AX_MMA ? FORM_MMA : v == AX_TMA ? FORM_TMA : v == AX_RB ? FORM_RB : FORM_LINE;
  } else if (v != AX_AUTO) {
    return v == AX_MMA ? FORM_MMA : v == AX_TMA ? FORM_TMA : v == AX_LINE ? FORM_LINE : FORM_PENCIL;
  }
  const TuneConfig cfg{lanes > 1 ? 1 : 0, d.N + 1, d.Nfields, d.affine, bytes, lanes, 1, element_class(Nelements)};
  int form = -1, n = 0, forms[8];
  float ms[8];
  if (tuned_report(cfg, &form, &n, forms, ms, 8) == BP_SUCCESS && form >= 0) return form;
  // the static choice (first of the candidate lists above)
  if (lanes > 1 || !d.affine) return FORM_TMA;
  return d.N + 1 == 16 ? FORM_MMA : (bytes == 4 ? FORM_LINE : FORM_PENCIL);
}

template <class F>
static int launch_ax_t(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                       const F* wJ, const F* ggeo, const F* gllw, const F* D, F lambda, const F* q, F* Aq,
                       const int* skip, cudaStream_t s, const CgFuse* fuse, int* nblocks) {
  if (nblocks) *nblocks = 0;
  if (d.dim == 2) {
    const int rc = launch_ax_quad(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, fuse, s,
                                  nblocks);
    return rc == 1 ? fail(BP_ERROR_ARG, "Quad2D operator: no fused direction update") : rc;
  }
  if (Nelements == 0) return BP_SUCCESS;
  switch (d.N + 1) {
#define BP_AX_CASE(nq) \
  case nq:             \
    return launch_ax_nq<nq, F>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, fuse, s, nblocks);
    BP_AX_CASE(2) BP_AX_CASE(3) BP_AX_CASE(4) BP_AX_CASE(5) BP_AX_CASE(6) BP_AX_CASE(7) BP_AX_CASE(8)
    BP_AX_CASE(9) BP_AX_CASE(10) BP_AX_CASE(11) BP_AX_CASE(12) BP_AX_CASE(13) BP_AX_CASE(14)
    BP_AX_CASE(15) BP_AX_CASE(16)
#undef BP_AX_CASE
    default:
      return fail(BP_ERROR_ARG, "bp_ax_hex3d: degree N must be in 1..15");
  }
}

int launch_ax_skip(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                   const double* wJ, const double* ggeo, const double* gllw, const double* D, double lambda,
                   const double* q, double* Aq, const int* skip, cudaStream_t s, const CgFuse* fuse,
                   int* nblocks) {
  return launch_ax_t<double>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, s, fuse,
                             nblocks);
}

int launch_ax_skip(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                   const float* wJ, const float* ggeo, const float* gllw, const float* D, float lambda,
                   const float* q, float* Aq, const int* skip, cudaStream_t s, const CgFuse* fuse,
                   int* nblocks) {
  return launch_ax_t<float>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, s, fuse,
                            nblocks);
}

int launch_ax(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
              const double* wJ, const double* ggeo, const double* gllw, const double* D, double lambda,
              const double* q, double* Aq, cudaStream_t s) {
  return launch_ax_skip(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, nullptr, s);
}

// ---------------------------------------------------------------------------
// Block reduction helpers (fixed order: warp shuffle tree, then warp partials)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* s_tmp) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) s_tmp[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = (lane < NT / 32) ? s_tmp[lane] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;   // valid in thread 0
}

// Writes this block's partial sums, and in the last block to finish returns
// true with the column sums of all partials in tot[0..NS) (thread 0 only).
template <int NT, int NS>
__device__ __forceinline__ bool grid_sum(const double (&v)[NS], double* partials, unsigned int* counter,
                                         double (&tot)[NS]) {
  __shared__ double s_tmp[NT / 32];
  __shared__ bool s_last;
  for (int c = 0; c < NS; ++c) {
    const double b = block_sum<NT>(v[c], s_tmp);
    if (threadIdx.x == 0) partials[c * gridDim.x + blockIdx.x] = b;
  }
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int done = atomicAdd(counter, 1u);
    s_last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  for (int c = 0; c < NS; ++c) {
    double acc = 0.0;
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += NT)
      acc += *((volatile double*)&partials[c * gridDim.x + b]);
    tot[c] = block_sum<NT>(acc, s_tmp);
  }
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

// ---------------------------------------------------------------------------
// ogs gather / scatter
// ---------------------------------------------------------------------------
__global__ void gather_kernel(int32_t Nrows, const int32_t* __restrict__ rowStarts,
                              const int32_t* __restrict__ colIds, const double* __restrict__ v,
                              double* __restrict__ gv) {
  const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= Nrows) return;
  const int32_t start = rowStarts[r], end = rowStarts[r + 1];
  double s = 0.0;
  for (int32_t c = start; c < end; ++c) s += __ldg(v + __ldg(colIds + c));
  gv[r] = s;
}

int launch_gather(int32_t Nrows, const int32_t* rowStarts, const int32_t* colIds, const double* v, double* gv,
                  cudaStream_t s) {
  if (Nrows <= 0) return BP_SUCCESS;
  gather_kernel<<<(Nrows + 255) / 256, 256, 0, s>>>(Nrows, rowStarts, colIds, v, gv);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

__global__ void scatter_kernel(int32_t Nrows, const int32_t* __restrict__ rowStarts,
                               const int32_t* __restrict__ colIds, const double* __restrict__ gv,
                               double* __restrict__ v) {
  const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= Nrows) return;
  const double g = gv[r];
  for (int32_t c = rowStarts[r]; c < rowStarts[r + 1]; ++c) v[colIds[c]] = g;
}

int launch_scatter(int32_t Nrows, const int32_t* rowStarts, const int32_t* colIds, const double* gv, double* v,
                   cudaStream_t s) {
  if (Nrows <= 0) return BP_SUCCESS;
  scatter_kernel<<<(Nrows + 255) / 256, 256, 0, s>>>(Nrows, rowStarts, colIds, gv, v);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

// ---------------------------------------------------------------------------
// Geometry: trilinear map of the 8 vertices, analytic derivatives at the GLL
// nodes, J and the symmetric G = J (grad r)(grad r)^T times the GLL weights.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void trilinear_jacobian(const double* ex, const double* ey, const double* ez, double r,
                                                   double s, double t, double (&Jm)[3][3]) {
  // d/dr, d/ds, d/dt of the 8 trilinear shape functions
  const double rm = 1 - r, rp = 1 + r, sm = 1 - s, sp = 1 + s, tm = 1 - t, tp = 1 + t;
  const double dr[8] = {-sm * tm, sm * tm, sp * tm, -sp * tm, -sm * tp, sm * tp, sp * tp, -sp * tp};
  const double ds[8] = {-rm * tm, -rp * tm, rp * tm, rm * tm, -rm * tp, -rp * tp, rp * tp, rm * tp};
  const double dt[8] = {-rm * sm, -rp * sm, -rp * sp, -rm * sp, rm * sm, rp * sm, rp * sp, rm * sp};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) Jm[a][b] = 0.0;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    Jm[0][0] += dr[v] * ex[v]; Jm[0][1] += ds[v] * ex[v]; Jm[0][2] += dt[v] * ex[v];
    Jm[1][0] += dr[v] * ey[v]; Jm[1][1] += ds[v] * ey[v]; Jm[1][2] += dt[v] * ey[v];
    Jm[2][0] += dr[v] * ez[v]; Jm[2][1] += ds[v] * ez[v]; Jm[2][2] += dt[v] * ez[v];
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) Jm[a][b] *= 0.125;
}

__device__ __forceinline__ void factors_from_jacobian(const double (&Jm)[3][3], double scale, double (&g)[6],
                                                      double& JW, bool& bad, double minJ) {
  const double xr = Jm[0][0], xs = Jm[0][1], xt = Jm[0][2];
  const double yr = Jm[1][0], ys = Jm[1][1], yt = Jm[1][2];
  const double zr = Jm[2][0], zs = Jm[2][1], zt = Jm[2][2];
  const double J = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt);
  bad = !(J >= minJ);
  const double iJ = 1.0 / J;
  const double rx = (ys * zt - zs * yt) * iJ, ry = -(xs * zt - zs * xt) * iJ, rz = (xs * yt - ys * xt) * iJ;
  const double sx = -(yr * zt - zr * yt) * iJ, sy = (xr * zt - zr * xt) * iJ, sz = -(xr * yt - yr * xt) * iJ;
  const double tx = (yr * zs - zr * ys) * iJ, ty = -(xr * zs - zr * xs) * iJ, tz = (xr * ys - yr * xs) * iJ;
  JW = J * scale;
  g[0] = JW * (rx * rx + ry * ry + rz * rz);
  g[1] = JW * (rx * sx + ry * sy + rz * sz);
  g[2] = JW * (rx * tx + ry * ty + rz * tz);
  g[3] = JW * (sx * sx + sy * sy + sz * sz);
  g[4] = JW * (sx * tx + sy * ty + sz * tz);
  g[5] = JW * (tx * tx + ty * ty + tz * tz);
}

__global__ void geometry_kernel(int Nq, int E, const double* __restrict__ EX, const double* __restrict__ EY,
                                const double* __restrict__ EZ, const double* __restrict__ gllz,
                                const double* __restrict__ gllw, double* __restrict__ wJ,
                                double* __restrict__ ggeo, int* __restrict__ bad) {
  const int Np = Nq * Nq * Nq;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)E * Np) return;
  const int e = (int)(gid / Np), n = (int)(gid % Np);
  const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
  double ex[8], ey[8], ez[8];
  for (int v = 0; v < 8; ++v) { ex[v] = EX[8 * e + v]; ey[v] = EY[8 * e + v]; ez[v] = EZ[8 * e + v]; }
  double Jm[3][3];
  trilinear_jacobian(ex, ey, ez, gllz[i], gllz[j], gllz[k], Jm);
  double g[6], JW;
  bool b;
  factors_from_jacobian(Jm, gllw[i] * gllw[j] * gllw[k], g, JW, b, 1e-12);
  if (b) atomicOr(bad, 1);
  wJ[gid] = JW;
  double2* o = reinterpret_cast<double2*>(ggeo + 6 * gid);
  o[0] = make_double2(g[0], g[1]);
  o[1] = make_double2(g[2], g[3]);
  o[2] = make_double2(g[4], g[5]);
}

// affine: constant Jacobian from vertices 0,1,3,4 (meshGeometricFactorsHex3D.cpp:42-80)
__global__ void geometry_affine_kernel(int E, const double* __restrict__ EX, const double* __restrict__ EY,
                                       const double* __restrict__ EZ, double* __restrict__ wJ,
                                       double* __restrict__ ggeo, int* __restrict__ bad) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const double* ex = EX + 8 * e;
  const double* ey = EY + 8 * e;
  const double* ez = EZ + 8 * e;
  double Jm[3][3] = {{0.5 * (ex[1] - ex[0]), 0.5 * (ex[3] - ex[0]), 0.5 * (ex[4] - ex[0])},
                     {0.5 * (ey[1] - ey[0]), 0.5 * (ey[3] - ey[0]), 0.5 * (ey[4] - ey[0])},
                     {0.5 * (ez[1] - ez[0]), 0.5 * (ez[3] - ez[0]), 0.5 * (ez[4] - ez[0])}};
  double g[6], JW;
  bool b;
  factors_from_jacobian(Jm, 1.0, g, JW, b, 0.0);
  if (b) atomicOr(bad, 1);
  wJ[e] = JW;
  for (int c = 0; c < 6; ++c) ggeo[6 * e + c] = g[c];
}

int launch_geometry(int N, int affine, int E, const double* EX, const double* EY, const double* EZ,
                    const double* gllz, const double* gllw, double* wJ, double* ggeo, int* bad, cudaStream_t s) {
  if (E == 0) return BP_SUCCESS;
  if (affine) {
    geometry_affine_kernel<<<(E + 127) / 128, 128, 0, s>>>(E, EX, EY, EZ, wJ, ggeo, bad);
  } else {
    const int Nq = N + 1;
    const long long tot = (long long)E * Nq * Nq * Nq;
    geometry_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(Nq, E, EX, EY, EZ, gllz, gllw, wJ, ggeo, bad);
  }
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

// ---------------------------------------------------------------------------
// Masked gathered numbering of the box on the device (the host form is
// box_numbering in bp_mesh.cpp; reference: ogsSetup.cpp:87-290, 492-579,
// 833-849, meshMaskedGatherScatterSetup.cpp:31-77).  Along each axis of n
// elements of degree N a lattice point L = a*N + i lies on the Dirichlet
// boundary (L = 0 or n*N) or is shared by count(L) elements (2 on an interior
// element face, else 1), the first of which represents it.  Rows follow the
// representative element, then the field, then (k, j, i) inside it, and every
// prefix sum of that order -- row numbers and CSR row starts -- has a closed
// form, so each local node finds its row, its row's first column and its
// position in the row (members in ascending element order) by itself.
// ---------------------------------------------------------------------------
struct BoxAxis {
  int n, N;
  __device__ bool boundary(int L) const { return L == 0 || L == n * N; }
  __device__ int first(int L) const { return (L > 0 && L % N == 0) ? L / N - 1 : min(L / N, n - 1); }
  __device__ int count(int L) const { return (L > 0 && L < n * N && L % N == 0) ? 2 : 1; }
  __device__ int reps(int a) const { return N - 1 + (a < n - 1 ? 1 : 0); }                 // rows of element a
  __device__ long long reps_before(int a) const { return (long long)a * (N - 1) + min(a, n - 1); }
  __device__ int mult(int a) const { return N - 1 + (a < n - 1 ? 2 : 0); }                 // columns of element a
  __device__ long long mult_before(int a) const { return (long long)a * (N - 1) + 2LL * min(a, n - 1); }
};

__global__ void box_numbering_kernel(int nx, int ny, int nz, int N, int Nf, long long NL, int32_t* __restrict__ G2L,
                                     int32_t* __restrict__ rowStarts, int32_t* __restrict__ colIds) {
  const BoxAxis ax{nx, N}, ay{ny, N}, az{nz, N};
  const int Nq = N + 1, Np = Nq * Nq * Nq;
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < NL;
       l += (long long)gridDim.x * blockDim.x) {
    const int n = (int)(l % Np);
    const long long ef = l / Np;
    const int f = (int)(ef % Nf);
    const int e = (int)(ef / Nf);
    const int ex = e % nx, ey = (e / nx) % ny, ez = e / (nx * ny);
    const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
    const int LI = ex * N + i, LJ = ey * N + j, LK = ez * N + k;
    if (ax.boundary(LI) || ay.boundary(LJ) || az.boundary(LK)) {
      G2L[l] = -1;
      continue;
    }
    const int rx = ax.first(LI), ry = ay.first(LJ), rz = az.first(LK);
    const int li = LI - rx * N, lj = LJ - ry * N, lk = LK - rz * N;   // 1..reps
    const long long Tx = ax.reps_before(nx), Ty = ay.reps_before(ny);
    const int ci = ax.reps(rx), cj = ay.reps(ry), ck = az.reps(rz);
    const long long rowBase =
        (long long)Nf * (Tx * Ty * az.reps_before(rz) + Tx * ay.reps_before(ry) * ck + ax.reps_before(rx) * cj * ck);
    const long long row = rowBase + (long long)f * ci * cj * ck + ((long long)(lk - 1) * cj + (lj - 1)) * ci + (li - 1);
    const long long TMx = ax.mult_before(nx), TMy = ay.mult_before(ny);
    const int mi = ax.mult(rx), mj = ay.mult(ry), mk = az.mult(rz);
    const int cx = ax.count(LI), cy = ay.count(LJ), cz = az.count(LK);
    const long long nnzBase = (long long)Nf * (TMx * TMy * az.mult_before(rz) + TMx * ay.mult_before(ry) * mk +
                                               ax.mult_before(rx) * mj * mk);
    const long long start = nnzBase + (long long)f * mi * mj * mk + (long long)(lk - 1) * mj * mi +
                            (long long)cz * (lj - 1) * mi + (long long)cz * cy * (li - 1);
    const int pos = ((ez - rz) * cy + (ey - ry)) * cx + (ex - rx);
    G2L[l] = (int32_t)row;
    colIds[start + pos] = (int32_t)l;
    if (pos == 0) rowStarts[row] = (int32_t)start;
  }
}

// rows and columns of the box numbering (closed forms of the kernel's prefix sums)
void box_numbering_counts(int nx, int ny, int nz, int N, int Nf, int64_t* Ngather, int64_t* nnz) {
  auto T = [N](int n) { return (int64_t)n * N - 1; };                          // interior lattice points
  auto TM = [N](int n) { return (int64_t)n * (N - 1) + 2 * (int64_t)(n - 1); };  // their element memberships
  *Ngather = (int64_t)Nf * T(nx) * T(ny) * T(nz);
  *nnz = (int64_t)Nf * TM(nx) * TM(ny) * TM(nz);
}

int launch_box_numbering(int nx, int ny, int nz, int N, int Nf, int32_t* G2L, int32_t* rowStarts, int32_t* colIds,
                         cudaStream_t s) {
  const long long NL = (long long)nx * ny * nz * (N + 1) * (N + 1) * (N + 1) * Nf;
  int64_t ng = 0, nnz = 0;
  box_numbering_counts(nx, ny, nz, N, Nf, &ng, &nnz);
  const int32_t last = (int32_t)nnz;   // pageable source: staged before the call returns
  BP_CUDA_TRY(cudaMemcpyAsync(rowStarts + ng, &last, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  if (NL == 0) return BP_SUCCESS;
  long long g = (NL + 255) / 256;
  if (g > 65536) g = 65536;
  box_numbering_kernel<<<(unsigned)g, 256, 0, s>>>(nx, ny, nz, N, Nf, NL, G2L, rowStarts, colIds);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

// Factors of a curved mesh at any tensor grid of points r (weights w), e.g.
// the N+2 Gauss points of the over-integrated operators.  The reference
// interpolates the GLL-node derivatives of x, y, z to the Gauss points
// (meshCubatureSetupHex3D.cpp:104-225); for the trilinear element map those
// derivatives are exactly representable, so the analytic Jacobian at the
// points is the same quantity.
int launch_geometry_at(int Nq, int E, const double* EX, const double* EY, const double* EZ, const double* r,
                       const double* w, double* wJ, double* ggeo, int* bad, cudaStream_t s) {
  if (E == 0) return BP_SUCCESS;
  const long long tot = (long long)E * Nq * Nq * Nq;
  geometry_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(Nq, E, EX, EY, EZ, r, w, wJ, ggeo, bad);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

// ---------------------------------------------------------------------------
// Forcing (okl/rhsHex3D.okl:29-128) on the fly from the vertex map
// ---------------------------------------------------------------------------
__global__ void rhs_analytic_kernel(int Nq, int affine, int Nfields, int E, const double* __restrict__ EX,
                                    const double* __restrict__ EY, const double* __restrict__ EZ,
                                    const double* __restrict__ gllz, const double* __restrict__ gllw,
                                    const double* __restrict__ wJ, double lambda, double* __restrict__ rL) {
  const int Np = Nq * Nq * Nq;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)E * Np) return;
  const int e = (int)(gid / Np), n = (int)(gid % Np);
  const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
  const double r = gllz[i], s = gllz[j], t = gllz[k];
  const double x = trilinear(EX + 8 * e, r, s, t), y = trilinear(EY + 8 * e, r, s, t),
               z = trilinear(EZ + 8 * e, r, s, t);
  const double w = affine ? wJ[e] * gllw[i] * gllw[j] * gllw[k] : wJ[gid];
  const double pi = 3.14159265358979323846;
  if (Nfields == 1) {
    rL[gid] = w * ((3 * pi * pi + lambda) * sin(pi * x) * sin(pi * y) * sin(pi * z));
  } else {
    const size_t base = (size_t)e * Np * 3 + n;
    rL[base] = w * ((4 * pi * pi + lambda) * sin(2.0 * pi * x) * sin(pi * y) * sin(pi * z));
    rL[base + Np] = w * ((4 * pi * pi + lambda) * sin(pi * x) * sin(2.0 * pi * y) * sin(pi * z));
    rL[base + 2 * Np] = w * ((4 * pi * pi + lambda) * sin(pi * x) * sin(pi * y) * sin(2.0 * pi * z));
  }
}

int launch_rhs_analytic(int N, int affine, int Nfields, int E, const double* EX, const double* EY, const double* EZ,
                        const double* gllz, const double* gllw, const double* wJ, double lambda, double* rL,
                        cudaStream_t s) {
  const int Nq = N + 1;
  const long long tot = (long long)E * Nq * Nq * Nq;
  if (tot == 0) return BP_SUCCESS;
  rhs_analytic_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(Nq, affine, Nfields, E, EX, EY, EZ, gllz, gllw,
                                                                      wJ, lambda, rL);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

// Seeded nodal forcing: f[r] = 2 u_r - 1 with u_r the r-th value of the
// reference's LCG stream (libs/primitives/random.cpp:29-170), computed with a
// per-thread jump-ahead so the stream is identical to the sequential one.
__global__ void rhs_random_kernel(int32_t N, uint64_t seed, double* __restrict__ f) {
  const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  const uint64_t A = 6364136223846793005ULL, C = 1ULL;
  uint64_t x = A * (~seed) + C;            // initial state
  // apply the affine map x -> A x + C, r times, by binary powering
  uint64_t pa = A, pc = C;                 // map for 2^bit steps
  uint32_t rr = (uint32_t)r;
  while (rr) {
    if (rr & 1u) x = pa * x + pc;
    pc = pa * pc + pc;
    pa = pa * pa;
    rr >>= 1;
  }
  const double u = __ull2double_rn(x) * (1.0 / 18446744073709551615.0);
  f[r] = 2 * u - 1;
}

int launch_rhs_random(int32_t Ngather, uint64_t seed, double* f, cudaStream_t s) {
  if (Ngather <= 0) return BP_SUCCESS;
  rhs_random_kernel<<<(Ngather + 255) / 256, 256, 0, s>>>(Ngather, seed, f);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

// rL[l] = wJ_l * f[G2L[l]] (0 on masked nodes): local lumped mass times f
__global__ void mass_local_kernel(int Nq, int affine, int Nfields, int E, const int32_t* __restrict__ G2L,
                                  const double* __restrict__ gllw, const double* __restrict__ wJ,
                                  const double* __restrict__ f, double* __restrict__ rL) {
  const int Np = Nq * Nq * Nq;
  const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= (long long)E * Np * Nfields) return;
  const int e = (int)(l / ((long long)Np * Nfields));
  const int n = (int)(l % Np);
  const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
  const double w = affine ? wJ[e] * gllw[i] * gllw[j] * gllw[k] : wJ[(size_t)e * Np + n];
  const int32_t id = G2L[l];
  rL[l] = (id != -1) ? w * f[id] : 0.0;
}

int launch_mass_local(int N, int affine, int Nfields, int E, const int32_t* G2L, const double* gllw,
                      const double* wJ, const double* f, double* rL, cudaStream_t s) {
  const int Nq = N + 1;
  const long long tot = (long long)E * Nq * Nq * Nq * Nfields;
  if (tot == 0) return BP_SUCCESS;
  mass_local_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(Nq, affine, Nfields, E, G2L, gllw, wJ, f, rL);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

// Element diagonal of the operator (for Jacobi): sum over the three 1D
// stiffness directions of G_dd D^2, the three mixed terms at the node, and
// lambda wJ.
__global__ void diag_local_kernel(int Nq, int affine, int Nfields, int E, const double* __restrict__ ggeo,
                                  const double* __restrict__ wJ, const double* __restrict__ gllw,
                                  const double* __restrict__ D, double lambda, double* __restrict__ dL) {
  const int Np = Nq * Nq * Nq;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)E * Np) return;
  const int e = (int)(gid / Np), n = (int)(gid % Np);
  const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
  auto G = [&](int ii, int jj, int kk, int c) -> double {
    if (affine) return ggeo[6 * (size_t)e + c] * gllw[ii] * gllw[jj] * gllw[kk];
    return ggeo[6 * ((size_t)e * Np + ii + jj * Nq + kk * Nq * Nq) + c];
  };
  double d = 0.0;
  for (int m = 0; m < Nq; ++m) {
    d += G(m, j, k, 0) * D[m * Nq + i] * D[m * Nq + i];
    d += G(i, m, k, 3) * D[m * Nq + j] * D[m * Nq + j];
    d += G(i, j, m, 5) * D[m * Nq + k] * D[m * Nq + k];
  }
  d += 2 * G(i, j, k, 1) * D[i * Nq + i] * D[j * Nq + j];
  d += 2 * G(i, j, k, 2) * D[i * Nq + i] * D[k * Nq + k];
  d += 2 * G(i, j, k, 4) * D[j * Nq + j] * D[k * Nq + k];
  const double w = affine ? wJ[e] * gllw[i] * gllw[j] * gllw[k] : wJ[gid];
  d += lambda * w;
  for (int f = 0; f < Nfields; ++f) dL[(size_t)e * Np * Nfields + (size_t)f * Np + n] = d;
}

int launch_diag_local(int N, int affine, int Nfields, int E, const double* ggeo, const double* wJ,
                      const double* gllw, const double* D, double lambda, double* dL, cudaStream_t s) {
  const int Nq = N + 1;
  const long long tot = (long long)E * Nq * Nq * Nq;
  if (tot == 0) return BP_SUCCESS;
  diag_local_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(Nq, affine, Nfields, E, ggeo, wJ, gllw, D, lambda,
                                                                    dL);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

// ---------------------------------------------------------------------------
// linAlg vector kernels
// ---------------------------------------------------------------------------
__global__ void set_kernel(int32_t N, double alpha, double* __restrict__ x) {
  const int32_t n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < N) x[n] = alpha;
}

__global__ void axpy_kernel(int32_t N, double alpha, const double* __restrict__ x, double beta,
                            double* __restrict__ y) {
  const int32_t n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < N) y[n] = alpha * x[n] + beta * y[n];
}

__global__ void reciprocal_kernel(int32_t N, double* __restrict__ x) {
  const int32_t n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < N) x[n] = 1.0 / x[n];
}

int launch_set(int32_t N, double alpha, double* x, cudaStream_t s) {
  if (N <= 0) return BP_SUCCESS;
  set_kernel<<<(N + 255) / 256, 256, 0, s>>>(N, alpha, x);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

int launch_axpy(int32_t N, double alpha, const double* x, double beta, double* y, cudaStream_t s) {
  if (N <= 0) return BP_SUCCESS;
  axpy_kernel<<<(N + 255) / 256, 256, 0, s>>>(N, alpha, x, beta, y);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

int launch_reciprocal(int32_t N, double* x, cudaStream_t s) {
  if (N <= 0) return BP_SUCCESS;
  reciprocal_kernel<<<(N + 255) / 256, 256, 0, s>>>(N, x);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

__global__ void sqrt1_kernel(double* v) { v[0] = sqrt(v[0]); }

int launch_sqrt1(double* v, cudaStream_t s) {
  sqrt1_kernel<<<1, 1, 0, s>>>(v);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

static inline int red_grid(int32_t N) {
  int g = (N + kRedThreads - 1) / kRedThreads;
  if (g > kRedBlocks) g = kRedBlocks;
  if (g < 1) g = 1;
  return g;
}

__global__ void __launch_bounds__(kRedThreads)
dot_kernel(int32_t N, const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ result,
           double* partials, unsigned int* counter) {
  double acc[1] = {0.0};
  for (int32_t n = blockIdx.x * kRedThreads + threadIdx.x; n < N; n += kRedThreads * gridDim.x)
    acc[0] += x[n] * y[n];
  double tot[1];
  if (grid_sum<kRedThreads, 1>(acc, partials, counter, tot) && threadIdx.x == 0) result[0] = tot[0];
}

int launch_dot(int32_t N, const double* x, const double* y, double* result, double* partials, unsigned int* counter,
               cudaStream_t s) {
  dot_kernel<<<red_grid(N), kRedThreads, 0, s>>>(N, x, y, result, partials, counter);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

__global__ void __launch_bounds__(kRedThreads)
update_cg_kernel(int32_t N, const double* __restrict__ Ap, double alpha, double* __restrict__ r,
                 double* __restrict__ result, double* partials, unsigned int* counter) {
  double acc[1] = {0.0};
  for (int32_t n = blockIdx.x * kRedThreads + threadIdx.x; n < N; n += kRedThreads * gridDim.x) {
    const double rn = r[n] - alpha * Ap[n];
    r[n] = rn;
    acc[0] += rn * rn;
  }
  double tot[1];
  if (grid_sum<kRedThreads, 1>(acc, partials, counter, tot) && threadIdx.x == 0) result[0] = tot[0];
}

int launch_update_cg(int32_t N, const double* Ap, double alpha, double* r, double* result, double* partials,
                     unsigned int* counter, cudaStream_t s) {
  update_cg_kernel<<<red_grid(N), kRedThreads, 0, s>>>(N, Ap, alpha, r, result, partials, counter);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

}  // namespace bp
