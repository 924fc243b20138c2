// Element operator with the geometric-factor stream moved by the TMA engine.
//
// The stored-factor BP5/BP6 operator reads 56 bytes of geometric factors per
// node (6 symmetric G entries + wJ), about 75% of its traffic.  Here every
// k-slice of an element's factors (Nq^2 nodes: 48*Nq^2 bytes of ggeo and
// 8*Nq^2 bytes of wJ, both contiguous in the reference layout) is fetched by
// one-dimensional bulk copies (cp.async.bulk, no tensor map) into a ring of R
// shared-memory slots, completing on one mbarrier per slot.  One thread
// issues the copies; the compute threads only wait on the slot's mbarrier, so
// many slices stay in flight without holding registers, and the slot of slice
// k is refilled with slice k+R as soon as slice k has been consumed.
//
// Block = S slots of Nq x Nq threads; slot s works on element s / NF, field
// s % NF, so the three fields of a BP6 element share one copy of the factors.
// Compute per slot follows the register-pencil scheme of ax_pencil_kernel
// (reference operator: okl/bp5AxHex3D.okl, okl/bp6AxHex3D.okl).
//
// Waits are bounded: a wait that gives up records BP_ERROR_TIMEOUT in the
// library's device error word and the block stops writing results.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>

#include "bp_cg_device.cuh"
#include "bp_internal.hpp"

namespace bp {

__device__ int g_device_error = 0;

int* device_error_word() {
  static int* p = nullptr;
  if (!p) {
    if (cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_device_error) != cudaSuccess) p = nullptr;
  }
  return p;
}

int check_device_error() {
  int h = 0;
  BP_CUDA_TRY(cudaMemcpyFromSymbol(&h, g_device_error, sizeof(int)));
  if (h) {
    const int zero = 0;
    cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int));
    return fail(BP_ERROR_TIMEOUT, "a bounded device-side wait gave up (TMA copy did not complete)");
  }
  return BP_SUCCESS;
}

namespace {

constexpr uint32_t kWaitLimit = 1u << 22;   // try_wait rounds before a wait gives up

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// bounded wait for the phase with the given parity; false if it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_addr(bar);
  for (uint32_t it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 1D bulk copy global -> shared, completion counted on the mbarrier (bytes % 16 == 0,
// both addresses 16-byte aligned)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

template <int NQ>
struct TmaShape {
  static constexpr int NQ2 = NQ * NQ;
  static constexpr int SLICE_G = NQ2 * 6;          // doubles of ggeo per slice
  static constexpr int SLICE_BYTES = NQ2 * 56;     // ggeo + wJ bytes per slice
  // ring depth: whole element up to p=5, four slices above (measured faster at p=7)
  static constexpr int R = NQ <= 6 ? NQ : (NQ <= 12 ? 4 : 4);
  static constexpr int EPB = NQ <= 4 ? 8 : (NQ <= 6 ? 2 : 1);   // elements per block
};

}  // namespace

template <int NQ, int NF, bool DOT, int R>
__global__ void __launch_bounds__(NQ * NQ * TmaShape<NQ>::EPB * NF)
ax_tma_kernel(int Nelements, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
              const double* __restrict__ wJ, const double* __restrict__ ggeo, const double* __restrict__ Dg,
              double lambda, const double* __restrict__ q, double* __restrict__ Aq, const int* __restrict__ skip,
              CgFuse fuse) {
  if (skip && *skip) return;
  using T = TmaShape<NQ>;
  constexpr int NQ2 = T::NQ2, NP = NQ2 * NQ, EPB = T::EPB, S = EPB * NF;
  constexpr int PAD = (NQ % 2 == 0) ? 1 : 0;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // layout: [EPB][R] slots of ggeo slices, [EPB][R] slots of wJ slices, D, q/v/w scratch, barriers
  double* s_g = reinterpret_cast<double*>(smem_raw);
  double* s_J = s_g + EPB * R * T::SLICE_G;
  double* s_D = s_J + EPB * R * NQ2;                     // [NQ][NQ] row-major, rows 16-byte aligned
  double* s_q = s_D + NQ * (NQ + 1);                     // [S][NQ][NQ+PAD]
  double* s_v = s_q + S * NQ * (NQ + PAD);
  double* s_w = s_v + S * NQ * (NQ + PAD);
  uint64_t* s_bar = reinterpret_cast<uint64_t*>(s_w + S * NQ * (NQ + PAD));   // [R]

  const int i = threadIdx.x, j = threadIdx.y, slot = threadIdx.z;
  const int t = i + NQ * (j + NQ * slot);
  const int el = slot / NF, f = slot % NF;
  const int e0 = blockIdx.x * EPB;
  const int nact = min(EPB, Nelements - e0);
  const bool active = el < nact;
  const int e = active ? elementList[e0 + el] : 0;

  if (t == 0) {
    for (int r = 0; r < R; ++r) mbar_init(&s_bar[r], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // producer: first R slices of every active element
  if (t == 0) {
    for (int k = 0; k < R; ++k) {
      mbar_expect_tx(&s_bar[k], nact * T::SLICE_BYTES);
      for (int a = 0; a < nact; ++a) {
        const size_t eb = (size_t)elementList[e0 + a] * NP + (size_t)k * NQ2;
        bulk_g2s(s_g + (a * R + k) * T::SLICE_G, ggeo + 6 * eb, NQ2 * 48, &s_bar[k]);
        bulk_g2s(s_J + (a * R + k) * NQ2, wJ + eb, NQ2 * 8, &s_bar[k]);
      }
    }
  }
  for (int n = t; n < NQ2; n += NQ2 * S) s_D[n] = Dg[n];

  // the pencil of q and the D rows of this thread, while the copies fly
  const size_t lbase = ((size_t)e * NF + f) * NP + j * NQ + i;
  double r_u[NQ], r_Au[NQ];
  {
    int id[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) id[k] = active ? __ldg(G2L + lbase + k * NQ2) : -1;
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      r_u[k] = (id[k] >= 0) ? __ldg(q + id[k]) : 0.0;
      r_Au[k] = 0.0;
    }
  }
  __syncthreads();   // s_D
  // rows i, j of D and (up to Nq=10) columns i, j in registers; row k per slice
  // comes from shared memory as 16-byte broadcasts
  constexpr bool DTREG = false;   // columns i, j from shared memory: registers buy more occupancy
  double Di[NQ], Dj[NQ], DTi[DTREG ? NQ : 1], DTj[DTREG ? NQ : 1];
#pragma unroll
  for (int m = 0; m < NQ; ++m) {
    Di[m] = s_D[i * NQ + m];
    Dj[m] = s_D[j * NQ + m];
    if (DTREG) {
      DTi[m] = s_D[m * NQ + i];
      DTj[m] = s_D[m * NQ + j];
    }
  }
  double* sq = s_q + slot * NQ * (NQ + PAD);
  double* sv = s_v + slot * NQ * (NQ + PAD);
  double* sw = s_w + slot * NQ * (NQ + PAD);
  bool ok = true;

#pragma unroll
  for (int k = 0; k < NQ; ++k) {
    const int rs = k % R;
    ok = mbar_wait(&s_bar[rs], (uint32_t)((k / R) & 1)) && ok;
    const double2* g2 = reinterpret_cast<const double2*>(s_g + ((el < EPB ? el : 0) * R + rs) * T::SLICE_G +
                                                         6 * (j * NQ + i));
    const double2 ga = g2[0], gb = g2[1], gc = g2[2];
    const double G00 = ga.x, G01 = ga.y, G02 = gb.x, G11 = gb.y, G12 = gc.x, G22 = gc.y;
    const double GwJ = s_J[((el < EPB ? el : 0) * R + rs) * NQ2 + j * NQ + i];

    sq[j * (NQ + PAD) + i] = r_u[k];
    __syncthreads();
    double Dk[NQ];
#pragma unroll
    for (int m = 0; m < NQ; m += 2) {
      const double2 d2 = *reinterpret_cast<const double2*>(s_D + k * NQ + m);
      Dk[m] = d2.x;
      Dk[m + 1] = d2.y;
    }
    double ur = 0.0, us = 0.0, ut = 0.0;
#pragma unroll
    for (int m = 0; m < NQ; ++m) ut += Dk[m] * r_u[m];
#pragma unroll
    for (int m = 0; m < NQ; ++m) {
      ur += Di[m] * sq[j * (NQ + PAD) + m];
      us += Dj[m] * sq[m * (NQ + PAD) + i];
    }
    sw[j * (NQ + PAD) + i] = G01 * ur + G11 * us + G12 * ut;
    sv[j * (NQ + PAD) + i] = G00 * ur + G01 * us + G02 * ut;
    const double GDut = G02 * ur + G12 * us + G22 * ut;
    double Auk = GwJ * lambda * r_u[k], Auk2 = 0.0;
    __syncthreads();
    // slot rs is free again: refill it with slice k+R
    if (R < NQ && k + R < NQ && t == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&s_bar[rs], nact * T::SLICE_BYTES);
      for (int a = 0; a < nact; ++a) {
        const size_t eb = (size_t)elementList[e0 + a] * NP + (size_t)(k + R) * NQ2;
        bulk_g2s(s_g + (a * R + rs) * T::SLICE_G, ggeo + 6 * eb, NQ2 * 48, &s_bar[rs]);
        bulk_g2s(s_J + (a * R + rs) * NQ2, wJ + eb, NQ2 * 8, &s_bar[rs]);
      }
    }
#pragma unroll
    for (int m = 0; m < NQ; ++m) r_Au[m] += Dk[m] * GDut;
#pragma unroll
    for (int m = 0; m < NQ; ++m) {
      Auk += (DTREG ? DTj[m] : s_D[m * NQ + j]) * sw[m * (NQ + PAD) + i];
      Auk2 += (DTREG ? DTi[m] : s_D[m * NQ + i]) * sv[j * (NQ + PAD) + m];
    }
    r_Au[k] += Auk + Auk2;
  }
  if (!__syncthreads_and(ok)) {   // block-uniform: every thread leaves together
    if (t == 0) atomicExch(&g_device_error, 1);
    return;
  }
  if (active) {
#pragma unroll
    for (int k = 0; k < NQ; ++k) Aq[lbase + k * NQ2] = r_Au[k];
  }
  if (DOT) {
    double v = 0.0;
    if (active) {
#pragma unroll
      for (int k = 0; k < NQ; ++k) v += r_u[k] * r_Au[k];
    }
    fuse_pap(v, fuse, s_g);   // the factor ring is free now and holds >= one double per thread
  }
}

template <int NQ, int NF, int R>
static size_t tma_smem_bytes() {
  using T = TmaShape<NQ>;
  constexpr int S = T::EPB * NF, PAD = (NQ % 2 == 0) ? 1 : 0;
  return sizeof(double) * ((size_t)T::EPB * R * (T::SLICE_G + T::NQ2) + NQ * (NQ + 1) + 3 * S * NQ * (NQ + PAD)) +
         sizeof(uint64_t) * R;
}

template <int NQ, int NF, bool DOT, int R>
static int launch_tma_r(int32_t Nelements, const int32_t* elementList, const int32_t* G2L, const double* wJ,
                        const double* ggeo, const double* D, double lambda, const double* q, double* Aq,
                        const int* skip, const CgFuse& fuse, cudaStream_t s, int* nblocks) {
  using T = TmaShape<NQ>;
  const size_t smem = tma_smem_bytes<NQ, NF, R>();
  static bool configured = false;
  if (!configured) {
    BP_CUDA_TRY(
        cudaFuncSetAttribute(ax_tma_kernel<NQ, NF, DOT, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured = true;
  }
  const dim3 block(NQ, NQ, T::EPB * NF);
  const dim3 grid((Nelements + T::EPB - 1) / T::EPB);
  if (nblocks) *nblocks = (int)grid.x;
  ax_tma_kernel<NQ, NF, DOT, R><<<grid, block, smem, s>>>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq,
                                                          skip, fuse);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

// ring depth: BP_TMA_RING=half in the environment halves the default ring
// (for tuning runs)
static bool tma_half_ring() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("BP_TMA_RING");
    v = (e && e[0] == 'h') ? 1 : 0;
  }
  return v == 1;
}

template <int NQ, int NF, bool DOT>
static int launch_tma_dot(int32_t Nelements, const int32_t* elementList, const int32_t* G2L, const double* wJ,
                          const double* ggeo, const double* D, double lambda, const double* q, double* Aq,
                          const int* skip, const CgFuse& fuse, cudaStream_t s, int* nblocks) {
  constexpr int R = TmaShape<NQ>::R, RH = R / 2 > 0 ? R / 2 : 1;
  if (tma_half_ring())
    return launch_tma_r<NQ, NF, DOT, RH>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, fuse, s,
                                         nblocks);
  return launch_tma_r<NQ, NF, DOT, R>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, fuse, s,
                                      nblocks);
}

template <int NQ, int NF>
static int launch_tma(int32_t Nelements, const int32_t* elementList, const int32_t* G2L, const double* wJ,
                      const double* ggeo, const double* D, double lambda, const double* q, double* Aq,
                      const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  if (fuse)
    return launch_tma_dot<NQ, NF, true>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, *fuse, s,
                                        nblocks);
  return launch_tma_dot<NQ, NF, false>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, CgFuse{}, s,
                                       nblocks);
}

// Stored-factor operator through the TMA path.  Returns 1 (and launches
// nothing) when the configuration is not covered: odd Nq (slices not a
// multiple of 16 bytes), affine factors, or factor arrays not 16-byte aligned.
int launch_ax_tma(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const double* wJ, const double* ggeo, const double* D, double lambda, const double* q, double* Aq,
                  const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  const int NQ = d.N + 1;
  if (d.affine || (NQ % 2) != 0 || ((reinterpret_cast<uintptr_t>(ggeo) | reinterpret_cast<uintptr_t>(wJ)) & 15))
    return 1;
  const bool three = d.Nfields == 3;
  if (three && NQ > 10) return 1;   // 3 slots of Nq^2 threads exceed the register file
  switch (NQ) {
#define BP_TMA_CASE(nq)                                                                                         \
  case nq:                                                                                                      \
    return three ? launch_tma<nq, 3>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, fuse, s, nblocks)          \
                 : launch_tma<nq, 1>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, fuse, s, nblocks);
#define BP_TMA_CASE1(nq) \
  case nq:               \
    return launch_tma<nq, 1>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, fuse, s, nblocks);
    BP_TMA_CASE(2) BP_TMA_CASE(4) BP_TMA_CASE(6) BP_TMA_CASE(8) BP_TMA_CASE(10) BP_TMA_CASE1(12)
    BP_TMA_CASE1(14) BP_TMA_CASE1(16)
#undef BP_TMA_CASE
#undef BP_TMA_CASE1
    default:
      return 1;
  }
}

}  // namespace bp
