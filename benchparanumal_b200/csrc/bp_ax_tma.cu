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

#include "bp_cg_device.cuh"
#include "bp_cg_persist.cuh"
#include "bp_internal.hpp"
#include "bp_pack.cuh"

namespace bp {

__device__ int g_device_error = 0;

int* device_error_word() {
  static DeviceSymbol sym(&g_device_error);
  return static_cast<int*>(sym.address());
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

// A wait gives up after about one second of SM clocks (2^31 cycles at
// 1.965 GHz); the test-only instantiation below uses a short limit.
constexpr long long kWaitCycles = 1ll << 31;
constexpr long long kTestWaitCycles = 1ll << 21;

// D of every degree in the constant bank (slot of NQ: sum of n^2 for n < NQ):
// row k of the slice being processed is the same for every thread, so its
// entries enter the FMAs as constant operands instead of shared-memory loads.
// D depends on the degree only, so launches on any mesh write the same values.
__host__ __device__ constexpr int tma_d_slot(int nq) {
  int off = 0;
  for (int n = 2; n < nq; ++n) off += n * n;
  return off;
}
constexpr int kTmaDTable = tma_d_slot(17);
__constant__ double c_tma_d64[kTmaDTable];
__constant__ float c_tma_d32[kTmaDTable];

template <class F>
__device__ __forceinline__ F tma_d(int idx);
template <>
__device__ __forceinline__ double tma_d<double>(int idx) { return c_tma_d64[idx]; }
template <>
__device__ __forceinline__ float tma_d<float>(int idx) { return c_tma_d32[idx]; }

template <class F>
F* tma_d_table() {
  static DeviceSymbol sym(sizeof(F) == 8 ? static_cast<const void*>(c_tma_d64) : static_cast<const void*>(c_tma_d32));
  return static_cast<F*>(sym.address());
}

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

__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(a), "r"(parity)
      : "memory");
  return done != 0;
}

// bounded wait for the phase with the given parity; false if it gave up after
// `limit` SM cycles (the clock is read only once the first try has failed)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit) {
  const uint32_t a = smem_addr(bar);
  if (mbar_try(a, parity)) return true;
  const long long t0 = clock64();
  while (clock64() - t0 < limit)
    if (mbar_try(a, parity)) return true;
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

template <class F>
struct Vec2;
template <>
struct Vec2<double> { using type = double2; };
template <>
struct Vec2<float> { using type = float2; };

template <int NQ, class F>
struct TmaShape {
  static constexpr int NQ2 = NQ * NQ;
  static constexpr int SLICE_G = NQ2 * 6;                        // values of ggeo per slice
  static constexpr int SLICE_BYTES = NQ2 * 7 * (int)sizeof(F);    // ggeo + wJ bytes per slice
  // ring depth: whole element up to p=5, four slices above (measured faster at p=7)
  static constexpr int R = NQ <= 6 ? NQ : 4;
  static constexpr int EPB = NQ <= 4 ? 8 : (NQ <= 6 ? 2 : 1);    // elements per block
};

}  // namespace

// Shared-memory layout of ax_tma_kernel: [EPB][R] slots of ggeo slices, [EPB][R]
// slots of wJ slices, D, then the q/v/w scratch of the S slots (values of type
// T, 16-byte aligned), then R mbarriers.
template <int NQ, int NF, int R, class F, class T>
struct TmaSmem {
  using Sh = TmaShape<NQ, F>;
  static constexpr int S = Sh::EPB * NF;
  static constexpr int PAD = 1;   // rows of NQ+1: conflict-free row and column walks
  static constexpr size_t FACT = sizeof(F) * ((size_t)Sh::EPB * R * (Sh::SLICE_G + Sh::NQ2) + NQ * (NQ + 2));
  static constexpr size_t QOFF = (FACT + 15) & ~(size_t)15;
  static constexpr size_t QVALS = (size_t)S * NQ * (NQ + PAD);
  static constexpr size_t BAR = (QOFF + 3 * QVALS * sizeof(T) + 7) & ~(size_t)7;
  static constexpr size_t BYTES = BAR + sizeof(uint64_t) * R;
};

// F is the arithmetic and storage type of the factors (double, or float for the
// inner solve of the mixed-precision CG); T the type of the q and Aq values: F,
// or Pack<F, PK> for PK right-hand sides of one mesh in lockstep (then NF = 1
// and the q/Aq arrays hold one pack per node).  p.Ap partials are summed in
// double, one per lane: fuse.partials[lane * gridDim.x + blockIdx.x].
// Packed values: a thread holds 2*NQ packs of R values (its pencil of q and
// of A q) and two rows of D, about REGS = max(128, 2*NQ*R + 2*NQ + 40)
// registers.  The second launch bound caps them there, so 65536 / (REGS *
// threads rounded up to whole warps) blocks stay resident (NQ=8, R=4: 8 blocks
// of 64 threads instead of 6 at 133 registers, 4 bytes of spills; NQ=10, R=4:
// 3 blocks without spills instead of 5 at 96 registers with 1.5 KB).
template <int NQ, int NF, class F, class T>
struct TmaMinBlocks {
  static constexpr int THREADS = NQ * NQ * TmaShape<NQ, F>::EPB * NF;
  static constexpr int ALLOC = (THREADS + 31) / 32 * 32;
  static constexpr int R = PackTraits<T>::R;
  static constexpr int WANT = 2 * NQ * R + 2 * NQ + 40;
  static constexpr int REGS = WANT > 128 ? WANT : 128;
  // One system: FP64 at Nq = 8, 10, 12 is capped to 128 registers too (Nq = 8:
  // 140 uncapped, 7 blocks of two warps per SM; capped, 8 blocks with no
  // spills: BK5 40^3 0.501 -> 0.475 ms, FP64 CG 100 iterations 90.7 -> 87.2
  // ms, while a 96-register cap spilled and lost, 0.520 ms; Nq = 10 on 24^3
  // 0.276 -> 0.263 ms, Nq = 12 on 20^3 0.481 -> 0.315 ms).  FP32 single-system
  // shapes need fewer registers and stay uncapped.
  static constexpr int V = R > 1 ? (65536 / (ALLOC * REGS) > 0 ? 65536 / (ALLOC * REGS) : 1)
                                 : (sizeof(F) == 8 && (NQ == 8 || NQ == 10 || NQ == 12) ? 65536 / (ALLOC * 128) : 1);
};

// WITHHOLD >= 0 builds the test-only form: the producer arms the mbarrier of
// that slice but issues none of its copies, so the wait on it runs out (after
// the short test limit) with nothing in flight.
//
// DIR builds the form with the CG direction update fused in (CgFuse::dir): q
// is not read, the pencil is p_k formed from p_{k-1}, r and invD, and the
// owners of the element's nodes write p_k and the deferred x update.
//
// The body works on element block `blk` of `nblk` (the block sums of p.Ap go
// to partials[lane * nblk + blk]) in the dynamic shared memory smem_raw, so the
// same code serves the kernel below (blk = blockIdx.x) and the persistent CG
// step (bp_solver.cu), whose blocks walk over the element blocks.
template <int NQ, int NF, bool DOT, int R, class F, class T, int WITHHOLD = -1, bool DIR = false>
__device__ __forceinline__ void ax_tma_body(int blk, int nblk, int Nelements, const int32_t* __restrict__ elementList,
                                            const int32_t* __restrict__ G2L, const F* __restrict__ wJ,
                                            const F* __restrict__ ggeo, const F* __restrict__ Dg, F lambda,
                                            const T* __restrict__ q, T* __restrict__ Aq, const CgFuse& fuse,
                                            unsigned char* smem_raw) {
  DirStep<PackTraits<T>::R, F> ds;
  if (DIR) {
    ds.load(fuse);
    if (!ds.any) return;   // every lane has finished (grid-uniform)
  }
  using Sh = TmaShape<NQ, F>;
  using Lay = TmaSmem<NQ, NF, R, F, T>;
  using V2 = typename Vec2<F>::type;
  constexpr int NQ2 = Sh::NQ2, NP = NQ2 * NQ, EPB = Sh::EPB, S = EPB * NF, LANES = PackTraits<T>::R;
  constexpr int PAD = Lay::PAD;
  F* s_g = reinterpret_cast<F*>(smem_raw);
  F* s_J = s_g + EPB * R * Sh::SLICE_G;
  F* s_D = s_J + EPB * R * NQ2;                     // [NQ][NQ] row-major, rows 8-byte aligned
  T* s_q = reinterpret_cast<T*>(smem_raw + Lay::QOFF);   // [S][NQ][NQ+PAD]
  T* s_v = s_q + Lay::QVALS;
  T* s_w = s_v + Lay::QVALS;
  uint64_t* s_bar = reinterpret_cast<uint64_t*>(smem_raw + Lay::BAR);   // [R]

  const int i = threadIdx.x, j = threadIdx.y, slot = threadIdx.z;
  const int t = i + NQ * (j + NQ * slot);
  const int el = slot / NF, f = slot % NF;
  const int e0 = blk * EPB;
  const int nact = min(EPB, Nelements - e0);
  const bool active = el < nact;
  const int e = active ? elementList[e0 + el] : 0;

  __syncthreads();   // a previous call's last uses of this shared memory are done (persistent use)
  if (t == 0) {
    for (int r = 0; r < R; ++r) mbar_init(&s_bar[r], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic accesses before the bulk copies
  }
  __syncthreads();
  constexpr long long LIMIT = WITHHOLD >= 0 ? kTestWaitCycles : kWaitCycles;
  int armed = R;   // slices whose mbarrier phase the producer (t == 0) has armed: 0 .. armed-1
  // producer: first R slices of every active element
  if (t == 0) {
    for (int k = 0; k < R; ++k) {
      mbar_expect_tx(&s_bar[k], nact * Sh::SLICE_BYTES);
      if (k == WITHHOLD) continue;
      for (int a = 0; a < nact; ++a) {
        const size_t eb = (size_t)elementList[e0 + a] * NP + (size_t)k * NQ2;
        bulk_g2s(s_g + (a * R + k) * Sh::SLICE_G, ggeo + 6 * eb, NQ2 * 6 * sizeof(F), &s_bar[k]);
        bulk_g2s(s_J + (a * R + k) * NQ2, wJ + eb, NQ2 * sizeof(F), &s_bar[k]);
      }
    }
  }
  for (int n = t; n < NQ2; n += NQ2 * S) s_D[n] = Dg[n];

  // the pencil of q and the D rows of this thread, while the copies fly
  const size_t lbase = ((size_t)e * NF + f) * NP + j * NQ + i;
  T r_u[NQ], r_Au[NQ];
  if (DIR) {
    const bool odd = (ds.gen & 1) != 0;   // selects, not indexes: no local-memory copy of the parameters
    const T* pold = static_cast<const T*>(odd ? fuse.pbuf[1] : fuse.pbuf[0]);
    T* pnew = static_cast<T*>(odd ? fuse.pbuf[0] : fuse.pbuf[1]);
    const T* rv = static_cast<const T*>(fuse.r);
    const F* dv = static_cast<const F*>(fuse.invD);
    T* xv = static_cast<T*>(fuse.x);
    int id[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) id[k] = active ? __ldg(G2L + lbase + k * NQ2) : -1;
    // every load of the pencil is issued before any store: p_old, r and invD
    // are read-only here (non-coherent loads), x is read at owned nodes only
    T po[NQ], xo[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      const int g = id[k] & kIdMask;
      po[k] = id[k] >= 0 ? ldg_val(pold + g) : pack_zero<T>();
      r_u[k] = id[k] >= 0 ? ldg_val(rv + g) : pack_zero<T>();
    }
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      const int g = id[k] & kIdMask;
      const F d = (dv && id[k] >= 0) ? ldg_val(dv + g) : F(1);
#pragma unroll
      for (int l = 0; l < PackTraits<T>::R; ++l) {
        const F z = d * lane(r_u[k], l);
        lane_set(r_u[k], l, ds.act[l] ? (ds.first[l] ? z : z + ds.beta[l] * lane(po[k], l)) : lane(po[k], l));
      }
      r_Au[k] = pack_zero<T>();
    }
    if (ds.anyx) {
#pragma unroll
      for (int k = 0; k < NQ; ++k)
        xo[k] = (id[k] >= 0 && (id[k] & kOwnerBit)) ? xv[id[k] & kIdMask] : pack_zero<T>();
#pragma unroll
      for (int k = 0; k < NQ; ++k) {
        if (id[k] < 0 || !(id[k] & kOwnerBit)) continue;
#pragma unroll
        for (int l = 0; l < PackTraits<T>::R; ++l)
          if (ds.addx[l]) lane_set(xo[k], l, ds.alpha[l] * lane(po[k], l) + F(1) * lane(xo[k], l));
        xv[id[k] & kIdMask] = xo[k];
      }
    }
#pragma unroll
    for (int k = 0; k < NQ; ++k)
      if (id[k] >= 0 && (id[k] & kOwnerBit)) pnew[id[k] & kIdMask] = r_u[k];
  } else {
    int id[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) id[k] = active ? __ldg(G2L + lbase + k * NQ2) : -1;
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      r_u[k] = (id[k] >= 0) ? q[id[k]] : pack_zero<T>();
      r_Au[k] = pack_zero<T>();
    }
  }
  __syncthreads();   // s_D
  // rows i, j of D in registers; row k per slice comes from shared memory as
  // vector broadcasts; columns i, j are read from shared memory (registers buy
  // more occupancy)
  F Di[NQ], Dj[NQ];
#pragma unroll
  for (int m = 0; m < NQ; ++m) {
    Di[m] = s_D[i * NQ + m];
    Dj[m] = s_D[j * NQ + m];
  }
  T* sq = s_q + slot * NQ * (NQ + PAD);
  T* sv = s_v + slot * NQ * (NQ + PAD);
  T* sw = s_w + slot * NQ * (NQ + PAD);
  bool ok = true;

#pragma unroll
  for (int k = 0; k < NQ; ++k) {
    const int rs = k % R;
    if (ok) ok = mbar_wait(&s_bar[rs], (uint32_t)((k / R) & 1), LIMIT);   // after a give-up, no more waits
    const V2* g2 = reinterpret_cast<const V2*>(s_g + (el * R + rs) * Sh::SLICE_G + 6 * (j * NQ + i));
    const V2 ga = g2[0], gb = g2[1], gc = g2[2];
    const F G00 = ga.x, G01 = ga.y, G02 = gb.x, G11 = gb.y, G12 = gc.x, G22 = gc.y;
    const F GwJ = s_J[(el * R + rs) * NQ2 + j * NQ + i];

    sq[j * (NQ + PAD) + i] = r_u[k];
    __syncthreads();
    constexpr int DSLOT = tma_d_slot(NQ);
    T ur = pack_zero<T>(), us = pack_zero<T>(), ut = pack_zero<T>();
#pragma unroll
    for (int m = 0; m < NQ; ++m) ut += tma_d<F>(DSLOT + k * NQ + m) * r_u[m];
#pragma unroll
    for (int m = 0; m < NQ; ++m) {
      ur += Di[m] * sq[j * (NQ + PAD) + m];
      us += Dj[m] * sq[m * (NQ + PAD) + i];
    }
    sw[j * (NQ + PAD) + i] = G01 * ur + G11 * us + G12 * ut;
    sv[j * (NQ + PAD) + i] = G00 * ur + G01 * us + G02 * ut;
    const T GDut = G02 * ur + G12 * us + G22 * ut;
    T Auk = (GwJ * lambda) * r_u[k], Auk2 = pack_zero<T>();
    __syncthreads();
    // slot rs is free again: refill it with slice k+R (never after the
    // producer's own wait gave up: the slot's phase may still be open)
    if (R < NQ && k + R < NQ && t == 0 && ok) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&s_bar[rs], nact * Sh::SLICE_BYTES);
      armed = k + R + 1;
      for (int a = 0; a < nact && k + R != WITHHOLD; ++a) {
        const size_t eb = (size_t)elementList[e0 + a] * NP + (size_t)(k + R) * NQ2;
        bulk_g2s(s_g + (a * R + rs) * Sh::SLICE_G, ggeo + 6 * eb, NQ2 * 6 * sizeof(F), &s_bar[rs]);
        bulk_g2s(s_J + (a * R + rs) * NQ2, wJ + eb, NQ2 * sizeof(F), &s_bar[rs]);
      }
    }
#pragma unroll
    for (int m = 0; m < NQ; ++m) r_Au[m] += tma_d<F>(DSLOT + k * NQ + m) * GDut;
#pragma unroll
    for (int m = 0; m < NQ; ++m) {
      Auk += s_D[m * NQ + j] * sw[m * (NQ + PAD) + i];
      Auk2 += s_D[m * NQ + i] * sv[j * (NQ + PAD) + m];
    }
    r_Au[k] += Auk + Auk2;
  }
  if (!__syncthreads_and(ok)) {   // block-uniform: every thread leaves together
    if (t == 0) {
      atomicExch(&g_device_error, 1);
      // The block must not leave while its own bulk copies may still write its
      // shared memory.  Every phase armed on a slot before its last one was
      // seen complete by the producer (a slot is re-armed only after that), so
      // wait, again bounded, for the last armed phase of each slot.
      for (int r = 0; r < R; ++r) {
        const int last = armed - 1 - ((armed - 1 - r) % R + R) % R;   // largest armed slice on slot r
        if (last >= 0) mbar_wait(&s_bar[r], (uint32_t)((last / R) & 1), LIMIT);
      }
    }
    __syncthreads();
    return;
  }
  if (active) {
#pragma unroll
    for (int k = 0; k < NQ; ++k) Aq[lbase + k * NQ2] = r_Au[k];
  }
  if (DOT) {
    double v[LANES];
#pragma unroll
    for (int l = 0; l < LANES; ++l) v[l] = 0.0;
    if (active) {
#pragma unroll
      for (int k = 0; k < NQ; ++k) lane_dot(v, r_u[k], r_Au[k]);
    }
    // the factor ring and the q/v/w scratch are free now: LANES doubles per thread
    double bs[LANES];
    if (LANES == 1) {
      bs[0] = fuse_block_sum(v[0], reinterpret_cast<double*>(s_g));
    } else {
      static_assert(Lay::BAR >= sizeof(double) * LANES * NQ2 * S && Lay::BAR >= sizeof(double) * LANES * 32,
                    "block-sum scratch too small");
      fuse_block_sum_lanes<LANES>(v, reinterpret_cast<double*>(s_g), bs);
    }
    if (t == 0)
#pragma unroll
      for (int l = 0; l < LANES; ++l) fuse.partials[(size_t)l * nblk + blk] = bs[l];
  }
}

template <int NQ, int NF, bool DOT, int R, class F, class T, int WITHHOLD = -1, bool DIR = false>
__global__ void __launch_bounds__(NQ * NQ * TmaShape<NQ, F>::EPB * NF, (TmaMinBlocks<NQ, NF, F, T>::V))
ax_tma_kernel(int Nelements, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
              const F* __restrict__ wJ, const F* __restrict__ ggeo, const F* __restrict__ Dg, F lambda,
              const T* __restrict__ q, T* __restrict__ Aq, const int* __restrict__ skip, CgFuse fuse) {
  pdl_wait();
  pdl_release();
  if (skip && *skip) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  ax_tma_body<NQ, NF, DOT, R, F, T, WITHHOLD, DIR>(blockIdx.x, gridDim.x, Nelements, elementList, G2L, wJ, ggeo, Dg,
                                                   lambda, q, Aq, fuse, smem_raw);
}

template <int NQ, int NF, bool DOT, class F, class T, bool DIR = false>
static int launch_tma_dot(int32_t Nelements, const int32_t* elementList, const int32_t* G2L, const F* wJ,
                          const F* ggeo, const F* D, F lambda, const T* q, T* Aq, const int* skip,
                          const CgFuse& fuse, cudaStream_t s, int* nblocks) {
  using Sh = TmaShape<NQ, F>;
  constexpr int R = Sh::R;
  const size_t smem = TmaSmem<NQ, NF, R, F, T>::BYTES;
  static DeviceOnce configured;   // the shared-memory attribute is set once per device
  BP_TRY(once_per_device(configured, [smem]() -> int {
    BP_CUDA_TRY(cudaFuncSetAttribute(ax_tma_kernel<NQ, NF, DOT, R, F, T, -1, DIR>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return BP_SUCCESS;
  }));
  F* tab = tma_d_table<F>();
  if (!tab) return fail(BP_ERROR_CUDA, "element operator: constant table address lookup failed");
  BP_TRY(const_slot_copy(tab + tma_d_slot(NQ), D, sizeof(F) * NQ * NQ, s));
  const dim3 block(NQ, NQ, Sh::EPB * NF);
  const dim3 grid((Nelements + Sh::EPB - 1) / Sh::EPB);
  if (nblocks) *nblocks = (int)grid.x;
  BP_CUDA_TRY(launch_pdl(ax_tma_kernel<NQ, NF, DOT, R, F, T, -1, DIR>, grid, block, smem, s, Nelements, elementList,
                         G2L, wJ, ggeo, D, lambda, q, Aq, skip, fuse));
  return BP_SUCCESS;
}

template <int NQ, int NF, class F, class T>
static int launch_tma(int32_t Nelements, const int32_t* elementList, const int32_t* G2L, const F* wJ, const F* ggeo,
                      const F* D, F lambda, const T* q, T* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s,
                      int* nblocks) {
  if (fuse && fuse->dir)
    return launch_tma_dot<NQ, NF, true, F, T, true>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip,
                                                    *fuse, s, nblocks);
  if (fuse)
    return launch_tma_dot<NQ, NF, true, F, T>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, *fuse,
                                              s, nblocks);
  return launch_tma_dot<NQ, NF, false, F, T>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip,
                                             CgFuse{}, s, nblocks);
}

// Stored-factor operator through the TMA path.  Returns 1 (and launches
// nothing) when the configuration is not covered: odd Nq (slices not a
// multiple of 16 bytes), affine factors, or factor arrays not 16-byte aligned.
template <class F>
static int launch_ax_tma_t(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                           const F* wJ, const F* ggeo, const F* D, F lambda, const F* q, F* Aq, const int* skip,
                           const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  const int NQ = d.N + 1;
  if (d.affine || (NQ % 2) != 0 || ((reinterpret_cast<uintptr_t>(ggeo) | reinterpret_cast<uintptr_t>(wJ)) & 15))
    return 1;
  const bool three = d.Nfields == 3;
  if (three && NQ > 10) return 1;   // 3 slots of Nq^2 threads exceed the register file
  switch (NQ) {
#define BP_TMA_ARGS Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, fuse, s, nblocks
#define BP_TMA_CASE(nq) \
  case nq:              \
    return three ? launch_tma<nq, 3, F, F>(BP_TMA_ARGS) : launch_tma<nq, 1, F, F>(BP_TMA_ARGS);
#define BP_TMA_CASE1(nq) \
  case nq:               \
    return launch_tma<nq, 1, F, F>(BP_TMA_ARGS);
    BP_TMA_CASE(2) BP_TMA_CASE(4) BP_TMA_CASE(6) BP_TMA_CASE(8) BP_TMA_CASE(10) BP_TMA_CASE1(12)
    BP_TMA_CASE1(14) BP_TMA_CASE1(16)
#undef BP_TMA_CASE
#undef BP_TMA_CASE1
#undef BP_TMA_ARGS
    default:
      return 1;
  }
}

int launch_ax_tma(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const double* wJ, const double* ggeo, const double* D, double lambda, const double* q, double* Aq,
                  const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  return launch_ax_tma_t<double>(d, Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, fuse, s, nblocks);
}

int launch_ax_tma(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const float* wJ, const float* ggeo, const float* D, float lambda, const float* q, float* Aq,
                  const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  return launch_ax_tma_t<float>(d, Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, fuse, s, nblocks);
}

// Test hook behind bp_test_wait_timeout: one element of the FP64 stored-factor
// operator at Nq = 8 (ring of R = 4 slots), through the instantiation that
// withholds slice `withhold` (0..7), or through the product instantiation for
// withhold = -1; then the library's device error word.  Allocates and frees
// its own small buffers.
template <int W>
static int tma_wait_test_launch(const int32_t* el, const int32_t* g2l, const double* wJ, const double* ggeo,
                                const double* D, const double* q, double* Aq, cudaStream_t s) {
  constexpr int NQ = 8, R = TmaShape<NQ, double>::R;
  const size_t smem = TmaSmem<NQ, 1, R, double, double>::BYTES;
  BP_CUDA_TRY(cudaFuncSetAttribute(ax_tma_kernel<NQ, 1, false, R, double, double, W>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ax_tma_kernel<NQ, 1, false, R, double, double, W><<<1, dim3(NQ, NQ, 1), smem, s>>>(1, el, g2l, wJ, ggeo, D, 1.0, q,
                                                                                    Aq, nullptr, CgFuse{});
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

int tma_wait_test(int withhold) {
  constexpr int NQ = 8, NP = NQ * NQ * NQ;
  if (withhold < -1 || withhold >= NQ) return fail(BP_ERROR_ARG, "bp_test_wait_timeout: slice must be -1..7");
  DeviceArray<int32_t> el, g2l;
  DeviceArray<double> wJ, ggeo, D, q, Aq;
  const cudaStream_t s = default_stream();
  BP_TRY(el.upload(std::vector<int32_t>(1, 0), s));
  BP_TRY(g2l.upload(std::vector<int32_t>(NP, 0), s));
  BP_TRY(wJ.upload(std::vector<double>(NP, 1.0), s));
  BP_TRY(ggeo.upload(std::vector<double>(6 * NP, 1.0), s));
  BP_TRY(D.upload(std::vector<double>(NQ * NQ, 0.0), s));
  BP_TRY(q.upload(std::vector<double>(1, 1.0), s));
  BP_TRY(Aq.alloc(NP));
  int rc = BP_SUCCESS;
  switch (withhold) {
#define BP_WAIT_CASE(w) \
  case w:               \
    rc = tma_wait_test_launch<w>(el.ptr, g2l.ptr, wJ.ptr, ggeo.ptr, D.ptr, q.ptr, Aq.ptr, s); \
    break;
    BP_WAIT_CASE(-1) BP_WAIT_CASE(0) BP_WAIT_CASE(3) BP_WAIT_CASE(5) BP_WAIT_CASE(7)
#undef BP_WAIT_CASE
    default:
      return fail(BP_ERROR_ARG, "bp_test_wait_timeout: slice must be one of -1, 0, 3, 5, 7");
  }
  BP_TRY(rc);
  BP_CUDA_TRY(cudaStreamSynchronize(s));
  return check_device_error();
}

// ---------------------------------------------------------------------------
// Register-blocked packed operator (FP32, L right-hand sides packed per node).
//
// The packed TMA kernel above gives each thread all L lanes of one k-pencil:
// every shared-memory value it loads (16 bytes) feeds one multiply-add per
// lane, so the r- and s-contractions cost 32 16-byte loads per node and slice
// and the kernel is bound by shared-memory wavefronts (about 126 per warp and
// slice).  Here a thread owns one lane of four k-pencils, (i, j) for i in
// {a, Nq-1-a} and j in {b, Nq-1-b}: a value of row j (or column i) of the
// slice feeds the two pencils that share it, and the four lanes of a node sit
// in consecutive threads, so a warp's 4-byte loads are broadcast-free and
// conflict-free in one wavefront each.  The gradient and the weak divergence
// then cost 16 4-byte loads per pencil pair and direction, about half the
// shared-memory traffic per node and lane.  The thread keeps rows a and b and
// columns a and b of D in registers and takes the mirrored rows and columns
// from the antisymmetry of the GLL differentiation matrix, D[Nq-1-i][Nq-1-m]
// = -D[i][m] (exact for the true matrix; the computed one, rounded to FP32,
// satisfies it to an ulp or two, far below this FP32 operator's accuracy);
// the t-direction uses the slice's row of D from the constant bank, as above.
// Factors come through the same ring of bulk-copied slices.
// ---------------------------------------------------------------------------
template <int NQ, int L>
struct RbShape {
  static constexpr int H = NQ / 2;
  static constexpr int THREADS = L * H * H;
  static constexpr int NQ2 = NQ * NQ;
  static constexpr int R = 4;                                    // ring slots
  static constexpr int SLICE_G = NQ2 * 6;
  static constexpr int SLICE_BYTES = NQ2 * 7 * (int)sizeof(float);
  // row stride (floats) of the slice arrays [j][i][lane]: rows b and b+1 (and
  // Nq-1-b) of a warp's stores fall in opposite halves of the 32 banks
  static constexpr int BASE = NQ * L;
  static constexpr int RS = BASE + ((16 - BASE % 32) + 32) % 32;
  static constexpr int SARR = NQ * RS;                           // floats per slice array
  static constexpr size_t FACT = sizeof(float) * ((size_t)R * (SLICE_G + NQ2) + NQ2);
  static constexpr size_t SOFF = (FACT + 15) & ~(size_t)15;
  static constexpr size_t BAR = (SOFF + sizeof(float) * 3 * SARR + 7) & ~(size_t)7;
  static constexpr size_t BYTES = BAR + sizeof(uint64_t) * R;
  static_assert(RS >= BASE && RS % 32 == 16, "slice row stride");
};

template <int NQ, int L, bool DOT>
__global__ void __launch_bounds__(RbShape<NQ, L>::THREADS, (L == 4 && NQ == 8) ? 8 : 1)
ax_rb_kernel(int Nelements, const int32_t* __restrict__ elementList, const int32_t* __restrict__ G2L,
             const float* __restrict__ wJ, const float* __restrict__ ggeo, const float* __restrict__ Dg,
             float lambda, const float* __restrict__ q, float* __restrict__ Aq, const int* __restrict__ skip,
             CgFuse fuse) {
  pdl_wait();
  pdl_release();
  if (skip && *skip) return;
  using Sh = RbShape<NQ, L>;
  constexpr int H = Sh::H, NQ2 = Sh::NQ2, NP = NQ2 * NQ, R = Sh::R, RS = Sh::RS;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* s_g = reinterpret_cast<float*>(smem_raw);
  float* s_J = s_g + R * Sh::SLICE_G;
  float* s_D = s_J + R * NQ2;
  float* sS = reinterpret_cast<float*>(smem_raw + Sh::SOFF);   // [NQ][RS]: q slice, [j][i][lane]
  float* sV = sS + Sh::SARR;                                    // r-fluxes
  float* sW = sV + Sh::SARR;                                    // s-fluxes
  uint64_t* s_bar = reinterpret_cast<uint64_t*>(smem_raw + Sh::BAR);

  const int t = threadIdx.x;
  const int l = t % L, a = (t / L) % H, b = t / (L * H);
  const int i0 = a, i1 = NQ - 1 - a, j0 = b, j1 = NQ - 1 - b;
  const int e = elementList[blockIdx.x];

  if (t == 0) {
    for (int r = 0; r < R; ++r) mbar_init(&s_bar[r], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  int armed = R;
  if (t == 0) {
    for (int k = 0; k < R; ++k) {
      mbar_expect_tx(&s_bar[k], Sh::SLICE_BYTES);
      const size_t eb = (size_t)e * NP + (size_t)k * NQ2;
      bulk_g2s(s_g + k * Sh::SLICE_G, ggeo + 6 * eb, NQ2 * 6 * sizeof(float), &s_bar[k]);
      bulk_g2s(s_J + k * NQ2, wJ + eb, NQ2 * sizeof(float), &s_bar[k]);
    }
  }
  for (int n = t; n < NQ2; n += Sh::THREADS) s_D[n] = Dg[n];

  // the four pencils (p = 2 * jj + ii: (i0,j0), (i1,j0), (i0,j1), (i1,j1)), lane l
  const size_t lbase = (size_t)e * NP;
  const int nodes[4] = {j0 * NQ + i0, j0 * NQ + i1, j1 * NQ + i0, j1 * NQ + i1};
  float u[4][NQ], Au[4][NQ];
  {
    int id[4][NQ];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int k = 0; k < NQ; ++k) id[p][k] = __ldg(G2L + lbase + k * NQ2 + nodes[p]);
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int k = 0; k < NQ; ++k) {
        u[p][k] = id[p][k] >= 0 ? q[(size_t)id[p][k] * L + l] : 0.0f;
        Au[p][k] = 0.0f;
      }
  }
  __syncthreads();   // s_D
  // rows a, b and columns a, b of D; the mirrored ones by antisymmetry
  float Dra[NQ], Drb[NQ], Dca[NQ], Dcb[NQ];
#pragma unroll
  for (int m = 0; m < NQ; ++m) {
    Dra[m] = s_D[a * NQ + m];
    Drb[m] = s_D[b * NQ + m];
    Dca[m] = s_D[m * NQ + a];
    Dcb[m] = s_D[m * NQ + b];
  }
  bool ok = true;
  constexpr int DSLOT = tma_d_slot(NQ);
#pragma unroll
  for (int k = 0; k < NQ; ++k) {
    const int rs = k % R;
    if (ok) ok = mbar_wait(&s_bar[rs], (uint32_t)((k / R) & 1), kWaitCycles);
    sS[j0 * RS + i0 * L + l] = u[0][k];
    sS[j0 * RS + i1 * L + l] = u[1][k];
    sS[j1 * RS + i0 * L + l] = u[2][k];
    sS[j1 * RS + i1 * L + l] = u[3][k];
    __syncthreads();
    float ur[4] = {0.f, 0.f, 0.f, 0.f}, us[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int m = 0; m < NQ; ++m) {
      const float r0 = sS[j0 * RS + m * L + l], r1 = sS[j1 * RS + m * L + l];   // rows j0, j1
      const float c0 = sS[m * RS + i0 * L + l], c1 = sS[m * RS + i1 * L + l];   // columns i0, i1
      const float da = Dra[m], da1 = -Dra[NQ - 1 - m];   // D[i0][m], D[i1][m]
      const float db = Drb[m], db1 = -Drb[NQ - 1 - m];   // D[j0][m], D[j1][m]
      ur[0] += da * r0;
      ur[1] += da1 * r0;
      ur[2] += da * r1;
      ur[3] += da1 * r1;
      us[0] += db * c0;
      us[1] += db * c1;
      us[2] += db1 * c0;
      us[3] += db1 * c1;
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      float ut = 0.0f;
#pragma unroll
      for (int m = 0; m < NQ; ++m) ut += tma_d<float>(DSLOT + k * NQ + m) * u[p][m];
      const float2* g2 = reinterpret_cast<const float2*>(s_g + rs * Sh::SLICE_G + 6 * nodes[p]);
      const float2 ga = g2[0], gb = g2[1], gc = g2[2];
      const float G00 = ga.x, G01 = ga.y, G02 = gb.x, G11 = gb.y, G12 = gc.x, G22 = gc.y;
      const float GwJ = s_J[rs * NQ2 + nodes[p]];
      const int ii = (p & 1) ? i1 : i0, jj = (p & 2) ? j1 : j0;
      sV[jj * RS + ii * L + l] = G00 * ur[p] + G01 * us[p] + G02 * ut;
      sW[jj * RS + ii * L + l] = G01 * ur[p] + G11 * us[p] + G12 * ut;
      const float GDut = G02 * ur[p] + G12 * us[p] + G22 * ut;
      Au[p][k] += (GwJ * lambda) * u[p][k];
#pragma unroll
      for (int m = 0; m < NQ; ++m) Au[p][m] += tma_d<float>(DSLOT + k * NQ + m) * GDut;
    }
    __syncthreads();
    if (k + R < NQ && t == 0 && ok) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&s_bar[rs], Sh::SLICE_BYTES);
      armed = k + R + 1;
      const size_t eb = (size_t)e * NP + (size_t)(k + R) * NQ2;
      bulk_g2s(s_g + rs * Sh::SLICE_G, ggeo + 6 * eb, NQ2 * 6 * sizeof(float), &s_bar[rs]);
      bulk_g2s(s_J + rs * NQ2, wJ + eb, NQ2 * sizeof(float), &s_bar[rs]);
    }
    float dv[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int m = 0; m < NQ; ++m) {
      const float v0 = sV[j0 * RS + m * L + l], v1 = sV[j1 * RS + m * L + l];   // V(m, j0), V(m, j1)
      const float w0 = sW[m * RS + i0 * L + l], w1 = sW[m * RS + i1 * L + l];   // W(i0, m), W(i1, m)
      const float ca = Dca[m], ca1 = -Dca[NQ - 1 - m];   // D[m][i0], D[m][i1]
      const float cb = Dcb[m], cb1 = -Dcb[NQ - 1 - m];   // D[m][j0], D[m][j1]
      dv[0] += ca * v0 + cb * w0;
      dv[1] += ca1 * v0 + cb * w1;
      dv[2] += ca * v1 + cb1 * w0;
      dv[3] += ca1 * v1 + cb1 * w1;
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) Au[p][k] += dv[p];
  }
  if (!__syncthreads_and(ok)) {   // block-uniform: every thread leaves together
    if (t == 0) {
      atomicExch(&g_device_error, 1);
      for (int r = 0; r < R; ++r) {   // the last armed phase of every slot, bounded
        const int last = armed - 1 - ((armed - 1 - r) % R + R) % R;
        if (last >= 0) mbar_wait(&s_bar[r], (uint32_t)((last / R) & 1), kWaitCycles);
      }
    }
    __syncthreads();
    return;
  }
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int k = 0; k < NQ; ++k) Aq[(lbase + k * NQ2 + nodes[p]) * L + l] = Au[p][k];
  if (DOT) {
    double v = 0.0;
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int k = 0; k < NQ; ++k) v += (double)u[p][k] * (double)Au[p][k];
    // per lane: shuffle over the threads of this lane in the warp, then the
    // warps in order (the ring is free for the warp sums)
#pragma unroll
    for (int o = 16; o >= L; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    double* ws = reinterpret_cast<double*>(s_g);
    constexpr int W = (Sh::THREADS + 31) / 32;
    if ((t & 31) < L) ws[(t >> 5) * L + (t & 31)] = v;
    __syncthreads();
    if (t < L) {
      double sum = 0.0;
#pragma unroll
      for (int w = 0; w < W; ++w) sum += ws[w * L + t];
      fuse.partials[(size_t)t * gridDim.x + blockIdx.x] = sum;
    }
  }
}

template <int NQ, int L, bool DOT>
static int launch_rb_dot(int32_t Nelements, const int32_t* elementList, const int32_t* G2L, const float* wJ,
                         const float* ggeo, const float* D, float lambda, const float* q, float* Aq, const int* skip,
                         const CgFuse& fuse, cudaStream_t s, int* nblocks) {
  using Sh = RbShape<NQ, L>;
  static_assert(Sh::THREADS % 32 == 0, "whole warps (the p.Ap sum shuffles over full warps)");
  const size_t smem = Sh::BYTES;
  static DeviceOnce configured;
  BP_TRY(once_per_device(configured, [smem]() -> int {
    BP_CUDA_TRY(cudaFuncSetAttribute(ax_rb_kernel<NQ, L, DOT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return BP_SUCCESS;
  }));
  float* tab = tma_d_table<float>();
  if (!tab) return fail(BP_ERROR_CUDA, "element operator: constant table address lookup failed");
  BP_TRY(const_slot_copy(tab + tma_d_slot(NQ), D, sizeof(float) * NQ * NQ, s));
  if (nblocks) *nblocks = Nelements;
  BP_CUDA_TRY(launch_pdl(ax_rb_kernel<NQ, L, DOT>, Nelements, Sh::THREADS, smem, s, Nelements, elementList, G2L, wJ,
                         ggeo, D, lambda, q, Aq, skip, fuse));
  return BP_SUCCESS;
}

int launch_ax_rb_packed(int pk, const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList,
                        const int32_t* G2L, const float* wJ, const float* ggeo, const float* D, float lambda,
                        const float* q, float* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s,
                        int* nblocks) {
  const int NQ = d.N + 1;
  if (d.affine || d.Nfields != 1 || pk != 4 || (fuse && fuse->dir) ||
      ((reinterpret_cast<uintptr_t>(ggeo) | reinterpret_cast<uintptr_t>(wJ)) & 15) ||
      (reinterpret_cast<uintptr_t>(q) | reinterpret_cast<uintptr_t>(Aq)) % 16)
    return 1;
  if (Nelements == 0) {
    if (nblocks) *nblocks = 0;
    return BP_SUCCESS;
  }
  switch (NQ) {
#define BP_RB_CASE(nq)                                                                                          \
  case nq:                                                                                                      \
    return fuse ? launch_rb_dot<nq, 4, true>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, *fuse, \
                                             s, nblocks)                                                         \
                : launch_rb_dot<nq, 4, false>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip,      \
                                              CgFuse{}, s, nblocks);
    BP_RB_CASE(8)
#undef BP_RB_CASE
    default:
      return 1;
  }
}

// FP32 operator on PK right-hand sides packed per node (q, Aq hold PK floats per
// node; one field).  Returns 1 when the configuration is not covered.
template <int PK>
static int launch_ax_tma_pk(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                            const float* wJ, const float* ggeo, const float* D, float lambda, const float* q,
                            float* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks) {
  using T = Pack<float, PK>;
  const int NQ = d.N + 1;
  if (d.affine || d.Nfields != 1 || (NQ % 2) != 0 ||
      ((reinterpret_cast<uintptr_t>(ggeo) | reinterpret_cast<uintptr_t>(wJ)) & 15) ||
      (reinterpret_cast<uintptr_t>(q) | reinterpret_cast<uintptr_t>(Aq)) % alignof(T))
    return 1;
  const T* qp = reinterpret_cast<const T*>(q);
  T* ap = reinterpret_cast<T*>(Aq);
  switch (NQ) {
#define BP_TMA_PK_CASE(nq) \
  case nq:                 \
    return launch_tma<nq, 1, float, T>(Nelements, elementList, G2L, wJ, ggeo, D, lambda, qp, ap, skip, fuse, s, nblocks);
    // Nq <= 6: the line form is faster with packed lanes (BK5 30^3, four rhs:
    // p=3 6.4 vs 6.0, p=5 8.6 vs 8.3 x 10^10 DOF/s; C5 batch 5.67 vs 5.70 s)
    BP_TMA_PK_CASE(8) BP_TMA_PK_CASE(10) BP_TMA_PK_CASE(12)
#undef BP_TMA_PK_CASE
    default:
      return 1;
  }
}

bool tma_covers(const bp_ax_desc_t& d, int lanes) {
  const int NQ = d.N + 1;
  if (d.dim == 2 || d.affine || NQ % 2 != 0) return false;
  if (lanes > 1) return d.Nfields == 1 && (lanes == 2 || lanes == 4) && NQ >= 8 && NQ <= 12;
  return d.Nfields == 1 ? NQ <= 16 : (d.Nfields == 3 && NQ <= 10);
}

namespace {
// the TMA body as the operator phase of the persistent CG step
template <int NQ, class T>
struct TmaStepOp {
  static constexpr int THREADS = NQ * NQ * TmaShape<NQ, float>::EPB;
  static constexpr int MINB = TmaMinBlocks<NQ, 1, float, T>::V;
  static __device__ __forceinline__ void run(int blk, const GrpStepArgs& a, unsigned char* smem) {
    CgFuse f;
    f.partials = a.parts;
    ax_tma_body<NQ, 1, true, TmaShape<NQ, float>::R, float, T>(blk, a.nblk_op, a.Nelements, a.elementList, a.G2L,
                                                                a.wJ, a.ggeo, a.D, a.lambda,
                                                                reinterpret_cast<const T*>(a.p),
                                                                reinterpret_cast<T*>(a.AqL), f, smem);
  }
};

template <int NQ, int PK>
int launch_step_tma_nq(GrpStepArgs a, int grid_cap, cudaStream_t s) {
  using T = Pack<float, PK>;
  using Sh = TmaShape<NQ, float>;
  float* tab = tma_d_table<float>();
  if (!tab) return fail(BP_ERROR_CUDA, "persistent CG step: constant table address lookup failed");
  BP_TRY(const_slot_copy(tab + tma_d_slot(NQ), a.D, sizeof(float) * NQ * NQ, s));
  a.nblk_op = (a.Nelements + Sh::EPB - 1) / Sh::EPB;
  return launch_grp_step_kernel<PK, TmaStepOp<NQ, T>>(a, dim3(NQ, NQ, Sh::EPB), TmaSmem<NQ, 1, Sh::R, float, T>::BYTES,
                                                       grid_cap, s);
}
}  // namespace

// One CG step of a packed group as one cooperative kernel with the TMA form of
// the operator (bp_cg_persist.cuh); pk = 4, stored factors, Nq 8, 10, 12
int launch_grp_step_tma(int pk, const bp_ax_desc_t& d, const GrpStepArgs& a, int grid_cap, cudaStream_t s) {
  if (pk != 4 || !tma_covers(d, pk) ||
      ((reinterpret_cast<uintptr_t>(a.ggeo) | reinterpret_cast<uintptr_t>(a.wJ)) & 15))
    return 1;
  switch (d.N + 1) {
    case 8: return launch_step_tma_nq<8, 4>(a, grid_cap, s);
    case 10: return launch_step_tma_nq<10, 4>(a, grid_cap, s);
    case 12: return launch_step_tma_nq<12, 4>(a, grid_cap, s);
    default: return 1;
  }
}

int launch_ax_tma_packed(int pk, const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList,
                         const int32_t* G2L, const float* wJ, const float* ggeo, const float* D, float lambda,
                         const float* q, float* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s,
                         int* nblocks) {
  switch (pk) {
    case 2:
      return launch_ax_tma_pk<2>(d, Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, fuse, s, nblocks);
    case 4:
      return launch_ax_tma_pk<4>(d, Nelements, elementList, G2L, wJ, ggeo, D, lambda, q, Aq, skip, fuse, s, nblocks);
    default:
      return 1;
  }
}

}  // namespace bp
