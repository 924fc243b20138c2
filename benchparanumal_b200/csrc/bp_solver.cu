// Benchmark problem object: operator, forcing, Jacobi diagonal and the CG
// solves (reference: BP/BP5/src/bp5{Setup,Operator,Run}.cpp,
// libs/core/linearSolverCG.cpp:62-156).
//
// CG runs with every scalar on the device.  One iteration is four kernels:
//   cg_direction_kernel     x += alpha_{k-1} p_{k-1} (deferred),  p = z + beta p
//   element operator        AqL = A_e p, and block partials of p.Ap = sum_e p_e.(A_e p_e)
//   cg_alpha_kernel         p.Ap from the partials, alpha = rho / p.Ap
//   cg_gather_update_kernel r -= alpha Gather(AqL), r.r (and r.z), stop test
// so A p is never stored as a gathered vector.  The reductions finish in the
// last block to arrive, so there is no host round trip per iteration.
// Iterations are captured once into a CUDA graph (kChunk iterations per graph)
// and replayed; a finished solve turns the remaining kernels into immediate
// returns through a device flag.
//
// On request (BP_FUSE_DIRECTION=1, where the element operator runs in its TMA
// form) the direction update is fused into the operator (CgFuse::dir): it
// forms p = z + beta p at the nodes it reads anyway and writes p and the x
// update at the nodes it owns, so an iteration is three kernels; p then
// alternates between two buffers (CgScalars::gen).
//
// Mixed precision: the same kernels run on FP32 vectors, FP32 factors and an
// FP32 operator (dot products accumulate in FP64).  The FP64 iterate is x_hi;
// the FP32 recursion carries a correction x_lo and residual r_lo.  When the
// FP32 residual has dropped by kReliableDrop since the last replacement (or
// reaches the tolerance), the host folds x_lo into x_hi, recomputes the FP64
// residual b - A x_hi with the FP64 operator and restarts r_lo from it while
// keeping the search direction -- a reliable update -- so the FP32 CG keeps
// its Krylov space and needs about as many iterations as FP64 CG.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <type_traits>
#include <vector>

#include "bp_cg_device.cuh"
#include "bp_cg_persist.cuh"
#include "bp_internal.hpp"
#include "bp_pack.cuh"

namespace bp {

constexpr int kThreads = 256;
constexpr int kChunk = 20;            // iterations per captured graph (divides the usual 100 and 1000)
// Iterations per graph of a batch unit.  A lane that asks for a reliable
// update idles until its chunk ends while the group's other lanes go on, so
// shorter chunks waste fewer iterations (and cost more host round trips).
constexpr int kBatchChunk = 10;

__device__ __forceinline__ double warp_sum_cg(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double block_sum_cg(double v, double* s_tmp) {
  v = warp_sum_cg(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) s_tmp[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = (lane < kThreads / 32) ? s_tmp[lane] : 0.0;
    r = warp_sum_cg(r);
  }
  __syncthreads();
  return r;
}

// NS block sums at once, each with block_sum_cg's tree (warp sums, then warp
// 0 over the warps in order), so the results are the same bits; two barriers
// for all NS values instead of two per value.  Thread 0 holds the sums.
template <int NS>
__device__ __forceinline__ void block_sum_multi_cg(double (&v)[NS], double* s_tmp) {
  constexpr int W = kThreads / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < NS; ++c) v[c] = warp_sum_cg(v[c]);
  if (lane == 0)
#pragma unroll
    for (int c = 0; c < NS; ++c) s_tmp[c * W + w] = v[c];
  __syncthreads();
  if (w == 0)
#pragma unroll
    for (int c = 0; c < NS; ++c) v[c] = warp_sum_cg(lane < W ? s_tmp[c * W + lane] : 0.0);
  __syncthreads();
}

// Deterministic grid sum: block partials in a fixed slot, the last block to
// arrive adds them in slot order.  Returns true in the last block (thread 0
// holds tot).
template <int NS>
__device__ __forceinline__ bool grid_sum_cg(const double (&v)[NS], double* partials, unsigned int* counter,
                                            double (&tot)[NS]) {
  __shared__ double s_tmp[NS * (kThreads / 32)];
  __shared__ bool s_last;
  double b[NS];
#pragma unroll
  for (int c = 0; c < NS; ++c) b[c] = v[c];
  block_sum_multi_cg<NS>(b, s_tmp);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int c = 0; c < NS; ++c) partials[c * gridDim.x + blockIdx.x] = b[c];
    __threadfence();
    s_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
#pragma unroll
  for (int c = 0; c < NS; ++c) tot[c] = 0.0;
  for (unsigned int k = threadIdx.x; k < gridDim.x; k += kThreads)
#pragma unroll
    for (int c = 0; c < NS; ++c) tot[c] += *((volatile double*)&partials[c * gridDim.x + k]);
  block_sum_multi_cg<NS>(tot, s_tmp);
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

// r <- r - Ap (Ap = A x0), then the initial residual norms and stop threshold.
__global__ void __launch_bounds__(kThreads)
cg_init_kernel(int32_t N, const double* __restrict__ Ap, double* __restrict__ r, const double* __restrict__ invD,
               CgScalars* sc, double tol, int maxit, int precon, double* partials, unsigned int* counter) {
  double acc[2] = {0.0, 0.0};
  for (int32_t n = blockIdx.x * kThreads + threadIdx.x; n < N; n += kThreads * gridDim.x) {
    const double rn = -1.0 * Ap[n] + 1.0 * r[n];
    r[n] = rn;
    acc[0] += rn * rn;
    if (precon) acc[1] += rn * invD[n] * rn;
  }
  double tot[2];
  if (grid_sum_cg<2>(acc, partials, counter, tot) && threadIdx.x == 0) {
    double rdotr;
    if (precon) {
      rdotr = tot[0];
      sc->tol2 = tol * tol * rdotr;
      sc->rz = tot[1];
    } else {
      // linAlg.norm2 then squared (linearSolverCG.cpp:84-87)
      const double nrm = sqrt(tot[0]);
      rdotr = nrm * nrm;
      sc->tol2 = fmax(tol * tol * rdotr, tol * tol);
      sc->rz = rdotr;
    }
    sc->rdotr = rdotr;
    sc->rdotr0 = rdotr;
    sc->rdotr_prev = rdotr;
    sc->rz_prev = sc->rz;
    sc->pAp = 0.0;
    sc->alpha = 0.0;
    sc->iter = 0;
    sc->maxit = maxit;
    sc->breakdown = 0;
    sc->precon = precon;
    sc->mixed = 0;
    sc->skip_x = 0;
    sc->update = 0;
    sc->done = (rdotr <= sc->tol2 || maxit <= 0) ? 1 : 0;
    // a non-finite initial residual (Inf or NaN in b or x) is a breakdown, not
    // convergence: with Inf, r.r <= tol^2 r0.r0 would hold at once
    if (!isfinite(rdotr) || !isfinite(sc->rz)) {
      sc->breakdown = 1;
      sc->done = 1;
    }
  }
}

// x += alpha p (the previous iteration's update, deferred unless a reliable
// update has applied it already), p = z + beta p
template <class V>
__global__ void __launch_bounds__(kThreads)
cg_direction_kernel(int32_t N, V* __restrict__ x, V* __restrict__ p, const V* __restrict__ r,
                    const V* __restrict__ invD, const CgScalars* __restrict__ sc) {
  pdl_wait();
  pdl_release();
  if (sc->done) return;
  const int iter = sc->iter;
  const bool addx = iter > 0 && !sc->skip_x;
  const V alpha = (V)sc->alpha;
  V beta = 0;
  if (iter > 0) beta = (V)(sc->precon ? sc->rz / sc->rz_prev : sc->rdotr / sc->rdotr_prev);
  const bool precon = sc->precon != 0;
  for (int32_t n = blockIdx.x * kThreads + threadIdx.x; n < N; n += kThreads * gridDim.x) {
    const V pn = p[n];
    if (addx) x[n] = alpha * pn + V(1) * x[n];
    const V z = precon ? invD[n] * r[n] : V(1) * r[n];
    p[n] = (iter > 0) ? z + beta * pn : z;   // p is not read at iteration 0
  }
}

// p.Ap of lanes sc[0..NL-1] from the element operator's per-lane block
// partials (parts[l * nparts + k]), then alpha.  Each block sums a strided
// share of the partials, the last block to arrive adds the block sums in slot
// order (grid_sum_cg), so the sum is reproducible; one block over 64000
// partials per lane took 36 us, most of a small problem's iteration.
template <int NL>
__global__ void __launch_bounds__(kThreads)
cg_alpha_kernel(int nparts, const double* __restrict__ parts, CgScalars* sc, double* hist_alpha, double* partials,
                unsigned int* counter) {
  pdl_wait();
  pdl_release();
  bool act[NL];
  bool any = false;
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    act[l] = !sc[l].done;   // every block reads sc before the last block changes it
    any = any || act[l];
  }
  if (!any) return;   // grid-uniform
  double acc[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) acc[l] = 0.0;
  for (int k = blockIdx.x * kThreads + threadIdx.x; k < nparts; k += kThreads * gridDim.x)
#pragma unroll
    for (int l = 0; l < NL; ++l) acc[l] += parts[(size_t)l * nparts + k];
  double tot[NL];
  if (grid_sum_cg<NL>(acc, partials, counter, tot) && threadIdx.x == 0) {
    for (int l = 0; l < NL; ++l) {
      if (!act[l]) continue;
      CgScalars& c = sc[l];
      const double pAp = tot[l];
      const double rho = c.precon ? c.rz : c.rdotr;
      const double alpha = rho / pAp;
      c.pAp = pAp;
      if (!(pAp > 0.0) || !isfinite(alpha)) {
        c.breakdown = 1;
        c.done = 1;
      } else {
        c.alpha = alpha;
        if (hist_alpha) hist_alpha[c.iter] = alpha;
      }
    }
  }
}

// blocks of cg_alpha_kernel: about four partials per thread
static int alpha_grid(int nparts) {
  int g = (nparts + 4 * kThreads - 1) / (4 * kThreads);
  if (g > reduction_blocks()) g = reduction_blocks();
  return g < 1 ? 1 : g;
}

// Grid-stride rows, RU of them in flight per thread (rows row0 + j*stride):
// each row's values are summed in column order (the reference's order, so the
// sums match its gather bit for bit), the rows' chains of dependent loads
// (rowStarts -> colIds -> AqL) interleaved.  The rows reach r.r in the same
// per-thread order as one at a time.  Measured at 40^3 p=7 (CG iteration, one
// row against four): FP32 BP3 0.929 -> 0.914 ms, BP5 0.580 -> 0.574 ms; FP64
// BP5 0.903 -> 0.949 ms, so FP64 keeps one row per thread.
// r -= alpha Gather(AqL); r.r (and r.z); stop test.  In a mixed solve the test
// also asks the host for a reliable update.
template <class V>
constexpr int kGatherRows = sizeof(V) == 4 ? 4 : 1;
template <class V, int RU>
__global__ void __launch_bounds__(kThreads)
cg_gather_update_kernel(int32_t Nrows, const int32_t* __restrict__ rowStarts, const int32_t* __restrict__ colIds,
                        const V* __restrict__ AqL, V* __restrict__ r, const V* __restrict__ invD, CgScalars* sc,
                        double* hist_rnorm, double* partials, unsigned int* counter) {
  pdl_wait();
  pdl_release();
  if (sc->done) return;
  const V alpha = (V)sc->alpha;
  const bool precon = sc->precon != 0;
  const int32_t stride = kThreads * gridDim.x;
  double acc[2] = {0.0, 0.0};
  for (int32_t row0 = blockIdx.x * kThreads + threadIdx.x; row0 < Nrows; row0 += RU * stride) {
    V rold[RU], dinv[RU], s[RU];
    int32_t c[RU], e[RU];
#pragma unroll
    for (int j = 0; j < RU; ++j) {
      const int32_t row = row0 + j * stride;
      const bool ok = row < Nrows;
      c[j] = ok ? __ldg(rowStarts + row) : 0;
      e[j] = ok ? __ldg(rowStarts + row + 1) : 0;
      rold[j] = ok ? r[row] : V(0);
      dinv[j] = ok && precon ? __ldg(invD + row) : V(0);
      s[j] = 0;
    }
    for (bool more = true; more;) {
      more = false;
#pragma unroll
      for (int j = 0; j < RU; ++j)
        if (c[j] < e[j]) {
          s[j] += __ldg(AqL + __ldg(colIds + c[j]));
          ++c[j];
          more = more || c[j] < e[j];
        }
    }
#pragma unroll
    for (int j = 0; j < RU; ++j) {
      const int32_t row = row0 + j * stride;
      if (row < Nrows) {
        const V rn = rold[j] - alpha * s[j];
        r[row] = rn;
        acc[0] += (double)rn * (double)rn;
        if (precon) acc[1] += (double)rn * (double)dinv[j] * (double)rn;
      }
    }
  }
  double tot[2];
  if (grid_sum_cg<2>(acc, partials, counter, tot) && threadIdx.x == 0) {
    sc->rdotr_prev = sc->rdotr;
    sc->rdotr = tot[0];
    if (precon) {
      sc->rz_prev = sc->rz;
      sc->rz = tot[1];
    }
    if (hist_rnorm) hist_rnorm[sc->iter] = sqrt(tot[0]);
    sc->iter += 1;
    sc->gen += 1;
    sc->skip_x = 0;
    if (!isfinite(tot[0])) {
      sc->breakdown = 1;
      sc->done = 1;
    } else if (sc->mixed) {
      if (tot[0] <= sc->tol2 || tot[0] < kReliableDrop * kReliableDrop * sc->rmax2 || sc->iter >= sc->maxit) {
        sc->update = 1;
        sc->done = 1;
      }
    } else if (tot[0] <= sc->tol2 || sc->iter >= sc->maxit) {
      sc->done = 1;
    }
  }
}

// apply the last completed iteration's x update (x and p with element stride
// `stride`: 1, or the lane count of a packed group).  With the fused direction
// update (gsc != null) p is p1 when gsc->gen is odd, else p0.
template <class V>
__global__ void __launch_bounds__(kThreads)
cg_final_kernel(int32_t N, V* __restrict__ x, const V* p0, const V* p1, const CgScalars* gsc,
                const CgScalars* __restrict__ sc, int stride = 1) {
  if (sc->iter == 0 || sc->breakdown || sc->skip_x) return;
  const V* __restrict__ p = (gsc && (gsc->gen & 1)) ? p1 : p0;
  const V alpha = (V)sc->alpha;
  for (int32_t n = blockIdx.x * kThreads + threadIdx.x; n < N; n += kThreads * gridDim.x)
    x[(size_t)n * stride] = alpha * p[(size_t)n * stride] + V(1) * x[(size_t)n * stride];
}

// mixed: x_hi += x_lo, x_lo = 0 (x_lo with element stride `stride`)
__global__ void __launch_bounds__(kThreads)
mixed_fold_kernel(int32_t N, double* __restrict__ x_hi, float* __restrict__ x_lo, int stride = 1) {
  for (int32_t n = blockIdx.x * kThreads + threadIdx.x; n < N; n += kThreads * gridDim.x) {
    x_hi[n] += (double)x_lo[(size_t)n * stride];
    x_lo[(size_t)n * stride] = 0.0f;
  }
}

// mixed: r_hi = b - Ax_hi (FP64), r_lo = (float) r_hi, and the norms that
// restart the FP32 recursion.  init != 0: first call of a solve.
__global__ void __launch_bounds__(kThreads)
mixed_replace_kernel(int32_t N, const double* __restrict__ b, const double* __restrict__ Ax, double* __restrict__ r_hi,
                     float* __restrict__ r_lo, const float* __restrict__ invD, CgScalars* sc, int init, double tol,
                     int maxit, int precon, double* partials, unsigned int* counter, int stride = 1) {
  double acc[3] = {0.0, 0.0, 0.0};
  for (int32_t n = blockIdx.x * kThreads + threadIdx.x; n < N; n += kThreads * gridDim.x) {
    const double rn = b[n] - Ax[n];
    r_hi[n] = rn;
    const float rl = (float)rn;
    r_lo[(size_t)n * stride] = rl;
    acc[0] += rn * rn;
    acc[1] += (double)rl * (double)rl;
    if (precon) acc[2] += (double)rl * (double)invD[n] * (double)rl;
  }
  double tot[3];
  if (grid_sum_cg<3>(acc, partials, counter, tot) && threadIdx.x == 0) {
    sc->rtrue2 = tot[0];
    sc->rmax2 = tot[0];
    sc->rdotr = tot[1];
    sc->rz = precon ? tot[2] : tot[1];
    if (init) {
      sc->rdotr0 = tot[0];
      sc->tol2 = tol * tol * tot[0];
      sc->rdotr_prev = tot[1];
      sc->rz_prev = sc->rz;
      sc->pAp = 0.0;
      sc->alpha = 0.0;
      sc->iter = 0;
      sc->maxit = maxit;
      sc->breakdown = 0;
      sc->precon = precon;
      sc->mixed = 1;
      sc->skip_x = 0;
    } else {
      sc->skip_x = 1;   // x_lo += alpha p of the last iteration is already folded in
    }
    sc->update = 0;
    sc->done = (tot[0] <= sc->tol2 || sc->iter >= sc->maxit) ? 1 : 0;
    if (!isfinite(tot[0]) || !isfinite(tot[1]) || !isfinite(sc->rz)) {   // Inf or NaN: breakdown
      sc->breakdown = 1;
      sc->done = 1;
    }
  }
}

// ---------------------------------------------------------------------------
// Packed groups: PK systems on one mesh advanced in lockstep.  Their FP32
// vectors hold one Pack<float, PK> per node (lane l = system l), so the
// direction update, the gather and the element operator read every index and
// factor once for all lanes.  Each lane keeps its own scalars (alpha, beta,
// norms, stop flags) in its own CgScalars slot; a finished lane stops changing
// while the others continue.
// ---------------------------------------------------------------------------
template <int PK>
__global__ void __launch_bounds__(kThreads)
grp_direction_kernel(int32_t N, Pack<float, PK>* __restrict__ x, Pack<float, PK>* __restrict__ p,
                     const Pack<float, PK>* __restrict__ r, const float* __restrict__ invD,
                     const CgScalars* __restrict__ sc) {
  pdl_wait();
  pdl_release();
  bool act[PK], addx[PK], first[PK];
  float alpha[PK], beta[PK];
  bool any = false;
#pragma unroll
  for (int l = 0; l < PK; ++l) {
    const CgScalars& c = sc[l];
    act[l] = !c.done;
    any = any || act[l];
    first[l] = c.iter == 0;
    addx[l] = c.iter > 0 && !c.skip_x;
    alpha[l] = (float)c.alpha;
    beta[l] = first[l] ? 0.0f : (float)(c.precon ? c.rz / c.rz_prev : c.rdotr / c.rdotr_prev);
  }
  if (!any) return;
  const bool precon = sc[0].precon != 0;
  for (int32_t n = blockIdx.x * kThreads + threadIdx.x; n < N; n += kThreads * gridDim.x) {
    Pack<float, PK> pn = p[n], xn = x[n];
    const Pack<float, PK> rn = r[n];
    const float d = precon ? invD[n] : 1.0f;
#pragma unroll
    for (int l = 0; l < PK; ++l) {
      if (!act[l]) continue;
      if (addx[l]) xn.v[l] = alpha[l] * pn.v[l] + 1.0f * xn.v[l];
      const float z = d * rn.v[l];
      pn.v[l] = first[l] ? z : z + beta[l] * pn.v[l];
    }
    x[n] = xn;
    p[n] = pn;
  }
}

// r -= alpha Gather(AqL) per lane, r.r and r.z per lane, each lane's stop test
template <int PK>
__global__ void __launch_bounds__(kThreads, 8)
grp_gather_update_kernel(int32_t Nrows, const int32_t* __restrict__ rowStarts, const int32_t* __restrict__ colIds,
                         const Pack<float, PK>* __restrict__ AqL, Pack<float, PK>* __restrict__ r,
                         const float* __restrict__ invD, CgScalars* sc, double* partials, unsigned int* counter) {
  pdl_wait();
  pdl_release();
  bool act[PK];
  float alpha[PK];
  bool any = false;
#pragma unroll
  for (int l = 0; l < PK; ++l) {
    act[l] = !sc[l].done;
    any = any || act[l];
    alpha[l] = (float)sc[l].alpha;
  }
  if (!any) return;
  const bool precon = sc[0].precon != 0;
  // the per-thread FP64 sums live in shared memory (one column per thread):
  // in registers they held the kernel at 48 registers, five blocks per SM
  __shared__ double s_acc[2 * PK][kThreads];
#pragma unroll
  for (int c = 0; c < 2 * PK; ++c) s_acc[c][threadIdx.x] = 0.0;
  for (int32_t row = blockIdx.x * kThreads + threadIdx.x; row < Nrows; row += kThreads * gridDim.x) {
    Pack<float, PK> rn = r[row];
    const float dinv = precon ? __ldg(invD + row) : 0.0f;
    const int32_t start = __ldg(rowStarts + row), end = __ldg(rowStarts + row + 1);
    // every row has a column; the first two (most rows have one or two) are
    // fetched side by side, the sum keeps column order (464 -> 367 us per
    // four-rhs launch at 40^3 p=7; the scalar FP64 gather is faster without it,
    // 208 vs 290 us, and keeps the plain loop)
    const bool two = start + 1 < end;
    const int32_t c0 = __ldg(colIds + start);
    const int32_t c1 = two ? __ldg(colIds + start + 1) : c0;
    const Pack<float, PK> a0 = AqL[c0];
    const Pack<float, PK> a1 = AqL[c1];
    Pack<float, PK> sum = a0;
    if (two) sum += a1;
    for (int32_t c = start + 2; c < end; ++c) sum += AqL[__ldg(colIds + c)];
#pragma unroll
    for (int l = 0; l < PK; ++l) {
      if (act[l]) rn.v[l] = rn.v[l] - alpha[l] * sum.v[l];
      s_acc[l][threadIdx.x] += (double)rn.v[l] * (double)rn.v[l];
      if (precon) s_acc[PK + l][threadIdx.x] += (double)rn.v[l] * (double)dinv * (double)rn.v[l];
    }
    r[row] = rn;
  }
  double acc[2 * PK];
#pragma unroll
  for (int c = 0; c < 2 * PK; ++c) acc[c] = s_acc[c][threadIdx.x];
  double tot[2 * PK];
  if (grid_sum_cg<2 * PK>(acc, partials, counter, tot) && threadIdx.x == 0) {
    sc[0].gen += 1;
    for (int l = 0; l < PK; ++l) {
      if (!act[l]) continue;
      CgScalars& c = sc[l];
      c.rdotr_prev = c.rdotr;
      c.rdotr = tot[l];
      if (precon) {
        c.rz_prev = c.rz;
        c.rz = tot[PK + l];
      }
      c.iter += 1;
      c.skip_x = 0;
      if (!isfinite(tot[l])) {
        c.breakdown = 1;
        c.done = 1;
      } else if (tot[l] <= c.tol2 || c.iter >= c.maxit) {
        c.update = 1;   // a packed group always runs the mixed-precision recursion
        c.done = 1;
      } else if (tot[l] < kReliableDrop * kReliableDrop * c.rmax2) {
        // the lane asks for a reliable update but keeps iterating: the group
        // runs on for its other lanes anyway, and the host replaces this lane's
        // residual when the chunk ends (stopping it here left it idle until then)
        c.update = 1;
      }
    }
  }
}

// the owner bit on the first local node (column) of every gathered row
__global__ void __launch_bounds__(kThreads)
owner_bits_kernel(int32_t Nrows, const int32_t* __restrict__ rowStarts, const int32_t* __restrict__ colIds,
                  int32_t* __restrict__ G2Lo) {
  for (int32_t row = blockIdx.x * kThreads + threadIdx.x; row < Nrows; row += kThreads * gridDim.x)
    G2Lo[colIds[rowStarts[row]]] |= kOwnerBit;
}

__global__ void d2f_kernel(size_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

static int vec_grid(int32_t N) {
  int g = (N + kThreads - 1) / kThreads;
  const int cap = reduction_blocks();
  if (g > cap) g = cap;
  return g < 1 ? 1 : g;
}

// Grid of a grid-stride kernel that needs more registers than eight resident
// blocks of kThreads allow: the blocks resident at once (one wave; a fixed
// count per kernel and device, so its reductions stay reproducible).  The
// four-lane gather at 48 registers keeps 5 blocks per SM: 1184 blocks ran as
// 1.6 waves.
static int vec_grid_wave(const void* kernel, int32_t N) {
  static std::mutex lock;
  static std::vector<std::pair<std::pair<const void*, int>, int>> cache;   // (kernel, device) -> wave
  int dev = 0, wave = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
  std::lock_guard<std::mutex> guard(lock);
  for (const auto& c : cache)
    if (c.first.first == kernel && c.first.second == dev) wave = c.second;
  if (wave == 0) {
    int sms = 0, per_sm = 0;
    if (dev < 0 || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0) != cudaSuccess)
      per_sm = 0;
    wave = per_sm > 0 && sms > 0 ? std::min(per_sm * sms, reduction_blocks()) : reduction_blocks();
    cache.push_back({{kernel, dev}, wave});
  }
  int g = (N + kThreads - 1) / kThreads;
  if (g > wave) g = wave;
  return g < 1 ? 1 : g;
}

int launch_d2f(size_t n, const double* a, float* b, cudaStream_t s) {
  if (n == 0) return BP_SUCCESS;
  size_t g = (n + 255) / 256;
  if (g > 8192) g = 8192;
  d2f_kernel<<<(unsigned)g, 256, 0, s>>>(n, a, b);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

static int to_float(const double* a, float* b, size_t n, cudaStream_t s) {
  if (n == 0) return BP_SUCCESS;
  size_t g = (n + 255) / 256;
  if (g > 8192) g = 8192;
  d2f_kernel<<<(unsigned)g, 256, 0, s>>>(n, a, b);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

}  // namespace bp

using namespace bp;

struct bp_solver_s {
  bp_mesh_s* mesh = nullptr;
  int bp = 5;
  double lambda = 1.0;
  int precon = 0;
  int mixed = 0;
  int32_t N = 0;               // Ngather
  bp_ax_desc_t ax{};
  DeviceArray<double> AqL, p, Ap, invD, xw, rw, partials, hist, fuse_partials, bcopy;
  // FP32 data of the mixed-precision solve
  DeviceArray<float> invD32, AqL32, p32, x32, r32;
  // second direction buffers of the fused direction update (allocated when used)
  DeviceArray<double> p_alt;
  DeviceArray<float> p32_alt;
  bool dir64 = false, dir32 = false;   // the captured FP64 / FP32 iterations fuse the direction update
  int family = 0;              // operator family of the FP32 data on the mesh (mesh_fp32)
  DeviceArray<unsigned int> counter;
  DeviceArray<CgScalars> sc;
  CgScalars* scal = nullptr;   // the CG scalars: sc.ptr, or a slot of a batch's array
  int64_t launches = 0;        // kernels launched (graph nodes included) since the solve began
  int hist_len = 0;
  // graph of kChunk iterations, keyed by the vectors it was captured for
  cudaGraphExec_t graph = nullptr;
  const double* g_x = nullptr;
  const double* g_r = nullptr;
  cudaGraphExec_t graph32 = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  ~bp_solver_s() {
    if (graph) cudaGraphExecDestroy(graph);
    if (graph32) cudaGraphExecDestroy(graph32);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

namespace bp {

// Operands of the element operator in one arithmetic type: BP5/BP6 use wJ,
// ggeo, gllw, D (GLL collocation); BP1-BP4 use wJ, ggeo, D and the 1D
// transform T at the quadrature points (CubOperands).
template <class V>
struct ElemOperands {
  const V* wJ;
  const V* ggeo;
  const V* gllw;
  const V* D;
  const V* T;
};

static ElemOperands<double> operands64(const bp_solver_s* S) {
  const bp_mesh_s* m = S->mesh;
  if (m->simplex) return {m->wJ.ptr, m->ggeo.ptr, nullptr, m->S.ptr, m->MM.ptr};   // Tri2D: S and MM
  if (S->bp >= 5) return {m->wJ.ptr, m->ggeo.ptr, m->gllw.ptr, m->D.ptr, nullptr};
  const double* D = m->affine ? m->cubDmodal.ptr : m->cubD.ptr;
  const double* T = !m->affine ? m->cubInterp.ptr : (S->bp >= 3 ? m->invV.ptr : m->MM.ptr);
  return {m->cubwJ(), m->cubggeo(), nullptr, D, T};
}

static ElemOperands<float> operands32(const bp_solver_s* S) {
  const bp_mesh_s::Fp32Ops& f = S->mesh->f32[S->family];
  return {f.wJ.ptr, f.ggeo.ptr, f.gllw.ptr, f.D.ptr, f.T.ptr};
}

// FP32 copies of a mesh's operator data for mixed-precision solvers, built once
// per operator family and shared by every solver on the mesh
static int mesh_fp32(bp_solver_s* S, cudaStream_t s) {
  bp_mesh_s* mesh = S->mesh;
  bp_mesh_s::Fp32Ops& f = mesh->f32[S->family];
  if (f.ready) return BP_SUCCESS;
  const ElemOperands<double> o = operands64(S);
  const bool cub = S->bp <= 4;
  const size_t ng = cub ? (mesh->affine ? (size_t)mesh->E : mesh->cubwJ_c.n) : mesh->wJ.n;
  const size_t nD = mesh->simplex ? mesh->S.n : cub ? (mesh->affine ? mesh->cubDmodal.n : mesh->cubD.n) : mesh->D.n;
  const size_t nT = mesh->simplex ? mesh->MM.n : cub ? (mesh->affine ? mesh->MM.n : mesh->cubInterp.n) : 0;
  BP_TRY(f.wJ.alloc(ng));
  const int nggeo = mesh->dim == 2 ? 3 : 6;   // factors per node (per element when affine)
  BP_TRY(f.ggeo.alloc(nggeo * ng));
  BP_TRY(f.D.alloc(nD));
  BP_TRY(f.gllw.alloc(mesh->gllw.n));
  BP_TRY(f.T.alloc(nT));
  BP_TRY(to_float(o.wJ, f.wJ.ptr, ng, s));
  BP_TRY(to_float(o.ggeo, f.ggeo.ptr, nggeo * ng, s));
  BP_TRY(to_float(o.D, f.D.ptr, nD, s));
  BP_TRY(to_float(mesh->gllw.ptr, f.gllw.ptr, mesh->gllw.n, s));
  if (nT) BP_TRY(to_float(o.T, f.T.ptr, nT, s));
  BP_CUDA_TRY(cudaStreamSynchronize(s));
  f.ready = true;
  return BP_SUCCESS;
}

template <class V>
static int elem_apply(bp_solver_s* S, const ElemOperands<V>& o, const V* q, V* AqL, const int* skip, cudaStream_t s,
                      const CgFuse* fuse = nullptr, int* nblocks = nullptr) {
  bp_mesh_s* m = S->mesh;
  if (m->simplex)   // Tri2D, Tet3D: D carries the stiffness matrices S, T the mass matrix
    return launch_ax_simplex(m->dim, m->N, m->E, m->elementList.ptr, m->G2L.ptr, o.wJ, o.ggeo, o.D, o.T, (V)S->lambda, q, AqL,
                         skip, s, fuse ? fuse->partials : nullptr, nblocks);
  if (S->bp >= 5)
    return launch_ax_skip(S->ax, m->E, m->elementList.ptr, m->G2L.ptr, o.wJ, o.ggeo, o.gllw, o.D, (V)S->lambda, q,
                          AqL, skip, s, fuse, nblocks);
  const CubOperands<V> c{o.wJ, o.ggeo, o.D, o.T};
  return launch_ax_cub(S->ax, m->E, m->elementList.ptr, m->G2L.ptr, c, (V)S->lambda, q, AqL, skip, s, fuse, nblocks);
}

static int operator_apply(bp_solver_s* S, const double* q, double* Aq, const int* skip, cudaStream_t s) {
  bp_mesh_s* m = S->mesh;
  S->launches += 2;
  BP_TRY(elem_apply<double>(S, operands64(S), q, S->AqL.ptr, skip, s));
  return launch_gather(m->Ngather, m->rowStarts.ptr, m->colIds.ptr, S->AqL.ptr, Aq, s);
}

// The fused direction update (CgFuse::dir) is used where BP_FUSE_DIRECTION=1.
// Measured on the 40^3 p=7 box it is slower than the separate direction
// kernel: the fused four-rhs launch took 1.07 ms against 0.61 ms for the
// operator alone and 0.28 ms for the direction pass (bench step 2.01 vs
// 1.82 s; FP64 Jacobi-PCG 22.5 vs 22.9 GDOF*it/s).  The gathered loads of
// p, r, invD and x, all needed before the element's first slice, lengthen
// each block's start-up latency, which the 16 resident warps per SM do not
// hide; the separate pass streams the same vectors at the HBM rate.
static bool fuse_direction_enabled() {
  const char* e = getenv("BP_FUSE_DIRECTION");
  return e && e[0] == '1';
}

int launch_owner_map(size_t NL, const int32_t* G2L, int32_t Ngather, const int32_t* rowStarts, const int32_t* colIds,
                     int32_t* G2Lo, cudaStream_t s) {
  if (NL && G2Lo != G2L)
    BP_CUDA_TRY(cudaMemcpyAsync(G2Lo, G2L, sizeof(int32_t) * NL, cudaMemcpyDeviceToDevice, s));
  if (Ngather > 0) {
    owner_bits_kernel<<<vec_grid(Ngather), kThreads, 0, s>>>(Ngather, rowStarts, colIds, G2Lo);
    BP_CUDA_TRY(cudaGetLastError());
  }
  return BP_SUCCESS;
}

// GlobalToLocal with owner bits of the mesh, built on first use
static int mesh_owner_g2l(bp_mesh_s* m, cudaStream_t s) {
  if (m->G2Lo.ptr || m->G2L.n == 0) return BP_SUCCESS;
  BP_TRY(m->G2Lo.alloc(m->G2L.n));
  BP_TRY(launch_owner_map(m->G2L.n, m->G2L.ptr, m->Ngather, m->rowStarts.ptr, m->colIds.ptr, m->G2Lo.ptr, s));
  BP_CUDA_TRY(cudaStreamSynchronize(s));
  return BP_SUCCESS;
}

// Whether the CG iterations of the element operator (d, `lanes` values per
// node, arithmetic of `bytes`) take the fused direction update: they do where
// the operator's current form is the TMA form.  Builds the owner bits.
static int want_dir(bp_mesh_s* m, const bp_ax_desc_t& d, int bytes, int lanes, bool* dir, cudaStream_t s) {
  *dir = false;
  if (!fuse_direction_enabled() || d.bp < 5 || m->Ngather >= kOwnerBit || !tma_covers(d, lanes) ||
      ax_current_form(d, bytes, lanes, m->E) != FORM_TMA)
    return BP_SUCCESS;
  BP_TRY(mesh_owner_g2l(m, s));
  *dir = true;
  return BP_SUCCESS;
}

template <class V>
static int alloc_zero(DeviceArray<V>& a, size_t n, cudaStream_t s) {
  if (a.n == n && a.ptr) return BP_SUCCESS;
  BP_TRY(a.alloc(n));
  if (n) BP_CUDA_TRY(cudaMemsetAsync(a.ptr, 0, sizeof(V) * n, s));
  return BP_SUCCESS;
}

// enqueue one CG iteration on vectors of type V (FP64, or FP32 in a mixed solve);
// dir: the operator does the direction update (p and p_alt alternate)
template <class V>
static int enqueue_iteration(bp_solver_s* S, V* x, V* r, V* p, V* p_alt, V* AqL, const V* invD,
                             const ElemOperands<V>& o, bool dir, cudaStream_t s) {
  bp_mesh_s* m = S->mesh;
  const int32_t N = S->N;
  const int g = vec_grid(N);
  double* hist_alpha = S->hist.ptr;
  double* hist_rnorm = S->hist.ptr ? S->hist.ptr + S->hist_len : nullptr;
  int nparts = 0;
  if (dir) {
    CgFuse fuse;
    fuse.partials = S->fuse_partials.ptr;
    fuse.dir = 1;
    fuse.pbuf[0] = p;
    fuse.pbuf[1] = p_alt;
    fuse.r = r;
    fuse.invD = S->precon ? invD : nullptr;
    fuse.x = x;
    fuse.sc = S->scal;
    const int rc = launch_ax_tma(S->ax, m->E, m->elementList.ptr, m->G2Lo.ptr, o.wJ, o.ggeo, o.D, (V)S->lambda,
                                 nullptr, AqL, &S->scal->done, &fuse, s, &nparts);
    if (rc == 1) return fail(BP_ERROR_ARG, "CG: the fused direction update does not cover this operator");
    BP_TRY(rc);
  } else {
    BP_CUDA_TRY(launch_pdl(cg_direction_kernel<V>, g, kThreads, 0, s, N, x, p, r, invD, S->scal));
    CgFuse fuse;
    fuse.partials = S->fuse_partials.ptr;
    BP_TRY(elem_apply<V>(S, o, p, AqL, &S->scal->done, s, &fuse, &nparts));
  }
  BP_CUDA_TRY(launch_pdl(cg_alpha_kernel<1>, alpha_grid(nparts), kThreads, 0, s, nparts, S->fuse_partials.ptr,
                         S->scal, hist_alpha, S->partials.ptr, S->counter.ptr));
  BP_CUDA_TRY(launch_pdl(cg_gather_update_kernel<V, kGatherRows<V>>, g, kThreads, 0, s, N, m->rowStarts.ptr,
                         m->colIds.ptr, AqL, r, invD, S->scal, hist_rnorm, S->partials.ptr, S->counter.ptr));
  return BP_SUCCESS;
}

static int capture(cudaGraphExec_t* out, cudaStream_t s, int (*body)(bp_solver_s*, void*, void*, cudaStream_t),
                   bp_solver_s* S, void* a, void* b) {
  if (*out) {
    cudaGraphExecDestroy(*out);
    *out = nullptr;
  }
  cudaGraph_t g;
  BP_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int rc = BP_SUCCESS;
  for (int k = 0; k < kChunk && rc == BP_SUCCESS; ++k) rc = body(S, a, b, s);
  cudaError_t ce = cudaStreamEndCapture(s, &g);
  if (rc != BP_SUCCESS) return rc;
  BP_CUDA_TRY(ce);
  ce = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  BP_CUDA_TRY(ce);
  return BP_SUCCESS;
}

static int body64(bp_solver_s* S, void* x, void* r, cudaStream_t s) {
  return enqueue_iteration<double>(S, (double*)x, (double*)r, S->p.ptr, S->p_alt.ptr, S->AqL.ptr, S->invD.ptr,
                                   operands64(S), S->dir64, s);
}

static int body32(bp_solver_s* S, void*, void*, cudaStream_t s) {
  return enqueue_iteration<float>(S, S->x32.ptr, S->r32.ptr, S->p32.ptr, S->p32_alt.ptr, S->AqL32.ptr, S->invD32.ptr,
                                  operands32(S), S->dir32, s);
}

// One launch of the iteration's element operator outside any capture, on the
// solver's scratch vectors: the autotuner measures the operator's forms here,
// so the graphs captured next use the tuned one.
template <class V>
static int tune_elem(bp_solver_s* S, const ElemOperands<V>& o, V* p, V* AqL, cudaStream_t s) {
  CgFuse fuse;
  fuse.partials = S->fuse_partials.ptr;
  int nparts = 0;
  return elem_apply<V>(S, o, p, AqL, nullptr, s, &fuse, &nparts);
}

// before capturing a solver's iterations: tune the operator, then choose
// whether the iterations fuse the direction update
static int prepare64(bp_solver_s* S, cudaStream_t s) {
  BP_TRY(tune_elem<double>(S, operands64(S), S->p.ptr, S->AqL.ptr, s));
  BP_TRY(want_dir(S->mesh, S->ax, 8, 1, &S->dir64, s));
  if (S->dir64) BP_TRY(alloc_zero(S->p_alt, S->p.n, s));
  return BP_SUCCESS;
}
static int prepare32(bp_solver_s* S, cudaStream_t s) {
  BP_TRY(tune_elem<float>(S, operands32(S), S->p32.ptr, S->AqL32.ptr, s));
  BP_TRY(want_dir(S->mesh, S->ax, 4, 1, &S->dir32, s));
  if (S->dir32) BP_TRY(alloc_zero(S->p32_alt, S->p32.n, s));
  return BP_SUCCESS;
}

static int ensure_graph(bp_solver_s* S, double* x, double* r, cudaStream_t s) {
  if (S->graph && S->g_x == x && S->g_r == r) return BP_SUCCESS;
  BP_TRY(prepare64(S, s));
  BP_TRY(capture(&S->graph, s, body64, S, x, r));
  S->g_x = x;
  S->g_r = r;
  return BP_SUCCESS;
}

static int ensure_hist(bp_solver_s* S, int maxit) {
  if (maxit <= S->hist_len) return BP_SUCCESS;
  // history buffers move: the captured graphs refer to them
  if (S->graph) {
    cudaGraphExecDestroy(S->graph);
    S->graph = nullptr;
  }
  if (S->graph32) {
    cudaGraphExecDestroy(S->graph32);
    S->graph32 = nullptr;
  }
  const int len = std::max(maxit, 128);
  BP_TRY(S->hist.alloc((size_t)2 * len));
  S->hist_len = len;
  return BP_SUCCESS;
}

static int read_scalars(bp_solver_s* S, CgScalars& h, cudaStream_t s) {
  BP_CUDA_TRY(cudaMemcpyAsync(&h, S->scal, sizeof(CgScalars), cudaMemcpyDeviceToHost, s));
  BP_CUDA_TRY(cudaStreamSynchronize(s));
  return BP_SUCCESS;
}

static int finish_solve(bp_solver_s* S, const CgScalars& h, double* hist_rnorm, double* hist_alpha,
                        bp_solve_stats_t* stats, bool record_events, int updates) {
  const int it = h.iter;
  if (hist_alpha && it > 0)
    BP_CUDA_TRY(cudaMemcpy(hist_alpha, S->hist.ptr, sizeof(double) * it, cudaMemcpyDeviceToHost));
  if (hist_rnorm && it > 0)
    BP_CUDA_TRY(cudaMemcpy(hist_rnorm, S->hist.ptr + S->hist_len, sizeof(double) * it, cudaMemcpyDeviceToHost));
  if (stats) {
    stats->iterations = it;
    stats->rdotr0 = h.rdotr0;
    stats->rdotr = S->mixed ? h.rtrue2 : h.rdotr;
    stats->updates = updates;
    stats->kernel_launches = S->launches;
    stats->elapsed_ms = 0.0;
    if (record_events) {
      float ms = 0.f;
      BP_CUDA_TRY(cudaEventElapsedTime(&ms, S->ev0, S->ev1));
      stats->elapsed_ms = ms;
    }
  }
  BP_TRY(check_device_error());
  if (h.breakdown) return fail(BP_ERROR_NUMERIC, "bp_solver_solve: CG breakdown (p.Ap <= 0 or non-finite residual)");
  return BP_SUCCESS;
}

static int solve_fp64(bp_solver_s* S, double* x, double* r, double tol, int maxit, double* hist_rnorm,
                      double* hist_alpha, bp_solve_stats_t* stats, cudaStream_t s, bool record_events) {
  const int32_t N = S->N;
  BP_TRY(ensure_hist(S, maxit));
  BP_TRY(ensure_graph(S, x, r, s));
  S->launches = 0;
  if (record_events) BP_CUDA_TRY(cudaEventRecord(S->ev0, s));
  // r = b - A x
  BP_TRY(operator_apply(S, x, S->Ap.ptr, nullptr, s));
  S->launches += 1;
  cg_init_kernel<<<vec_grid(N), kThreads, 0, s>>>(N, S->Ap.ptr, r, S->invD.ptr, S->scal, tol, maxit, S->precon,
                                                  S->partials.ptr, S->counter.ptr);
  BP_CUDA_TRY(cudaGetLastError());
  const int nchunks = (maxit + kChunk - 1) / kChunk;
  CgScalars h{};
  for (int c = 0; c < nchunks; ++c) {
    BP_CUDA_TRY(cudaGraphLaunch(S->graph, s));
    S->launches += (S->dir64 ? 3 : 4) * kChunk;
    if (tol > 0.0 && c + 1 < nchunks) {
      BP_TRY(read_scalars(S, h, s));
      if (h.done) break;
    }
  }
  S->launches += 1;
  cg_final_kernel<double><<<vec_grid(N), kThreads, 0, s>>>(N, x, S->p.ptr, S->p_alt.ptr,
                                                            S->dir64 ? S->scal : nullptr, S->scal);
  BP_CUDA_TRY(cudaGetLastError());
  if (record_events) BP_CUDA_TRY(cudaEventRecord(S->ev1, s));
  BP_TRY(read_scalars(S, h, s));
  return finish_solve(S, h, hist_rnorm, hist_alpha, stats, record_events, 0);
}

// FP64 residual r_hi = b - A x_hi and the FP32 restart (init: start of a solve)
static int mixed_replace(bp_solver_s* S, double* x, double* r, bool init, double tol, int maxit, cudaStream_t s) {
  const int32_t N = S->N;
  BP_TRY(operator_apply(S, x, S->Ap.ptr, nullptr, s));
  S->launches += 1;
  mixed_replace_kernel<<<vec_grid(N), kThreads, 0, s>>>(N, S->bcopy.ptr, S->Ap.ptr, r, S->r32.ptr, S->invD32.ptr,
                                                        S->scal, init ? 1 : 0, tol, maxit, S->precon,
                                                        S->partials.ptr, S->counter.ptr);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

// start of a mixed solve: keep b, x_lo = 0, FP64 residual and the FP32 restart
static int mixed_begin(bp_solver_s* S, double* x, double* r, double tol, int maxit, cudaStream_t s) {
  const int32_t N = S->N;
  BP_CUDA_TRY(cudaMemcpyAsync(S->bcopy.ptr, r, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  BP_CUDA_TRY(cudaMemsetAsync(S->x32.ptr, 0, sizeof(float) * N, s));
  return mixed_replace(S, x, r, true, tol, maxit, s);
}

// reliable update: fold the pending x_lo step, x_hi += x_lo, FP64 residual
static int mixed_reliable(bp_solver_s* S, double* x, double* r, double tol, int maxit, cudaStream_t s) {
  const int32_t N = S->N;
  S->launches += 2;
  cg_final_kernel<float><<<vec_grid(N), kThreads, 0, s>>>(N, S->x32.ptr, S->p32.ptr, S->p32_alt.ptr,
                                                           S->dir32 ? S->scal : nullptr, S->scal);
  BP_CUDA_TRY(cudaGetLastError());
  mixed_fold_kernel<<<vec_grid(N), kThreads, 0, s>>>(N, x, S->x32.ptr);
  BP_CUDA_TRY(cudaGetLastError());
  return mixed_replace(S, x, r, false, tol, maxit, s);
}

static int solve_mixed(bp_solver_s* S, double* x, double* r, double tol, int maxit, double* hist_rnorm,
                       double* hist_alpha, bp_solve_stats_t* stats, cudaStream_t s, bool record_events) {
  if (!(tol > 0.0)) return fail(BP_ERROR_ARG, "bp_solver_solve: a mixed-precision solve needs tol > 0");
  BP_TRY(ensure_hist(S, maxit));
  if (!S->graph32) {
    BP_TRY(prepare32(S, s));
    BP_TRY(capture(&S->graph32, s, body32, S, nullptr, nullptr));
  }
  S->launches = 0;
  if (record_events) BP_CUDA_TRY(cudaEventRecord(S->ev0, s));
  BP_TRY(mixed_begin(S, x, r, tol, maxit, s));
  CgScalars h{};
  BP_TRY(read_scalars(S, h, s));
  int updates = 0;
  while (!h.done || h.update) {
    if (h.update) {
      BP_TRY(mixed_reliable(S, x, r, tol, maxit, s));
      ++updates;
    } else {
      BP_CUDA_TRY(cudaGraphLaunch(S->graph32, s));
      S->launches += (S->dir32 ? 3 : 4) * kChunk;
    }
    BP_TRY(read_scalars(S, h, s));
    if (h.breakdown) break;
  }
  if (record_events) BP_CUDA_TRY(cudaEventRecord(S->ev1, s));
  BP_CUDA_TRY(cudaStreamSynchronize(s));
  return finish_solve(S, h, hist_rnorm, hist_alpha, stats, record_events, updates);
}

static int solve_device(bp_solver_s* S, double* x, double* r, double tol, int maxit, double* hist_rnorm,
                        double* hist_alpha, bp_solve_stats_t* stats, cudaStream_t s, bool record_events) {
  if (S->mixed) return solve_mixed(S, x, r, tol, maxit, hist_rnorm, hist_alpha, stats, s, record_events);
  return solve_fp64(S, x, r, tol, maxit, hist_rnorm, hist_alpha, stats, s, record_events);
}

}  // namespace bp

extern "C" {

int bp_solver_create(bp_mesh_t mesh, const bp_solver_desc_t* d, bp_solver_t* out) {
  if (!mesh || !d || !out) return fail(BP_ERROR_ARG, "bp_solver_create: null pointer");
  *out = nullptr;
  if (d->bp < 1 || d->bp > 6) return fail(BP_ERROR_ARG, "bp_solver_create: bp must be 1..6");
  if (mesh->simplex) {
    if (d->bp != 5) return fail(BP_ERROR_ARG, "bp_solver_create: Tri2D and Tet3D meshes take BP5");
  } else if (mesh->dim == 2) {
    if (d->bp < 5) return fail(BP_ERROR_ARG, "bp_solver_create: Quad2D meshes take BP5 and BP6 (the BP1-BP4 forms are Hex3D only)");
    if ((d->bp == 6) != (mesh->Nfields == 2))
      return fail(BP_ERROR_ARG, "bp_solver_create: Quad2D BP6 needs a 2-field mesh, BP5 a 1-field mesh");
  } else if ((d->bp % 2 == 0) != (mesh->Nfields == 3)) {
    return fail(BP_ERROR_ARG, "bp_solver_create: BP2/BP4/BP6 need a 3-field mesh, BP1/BP3/BP5 a 1-field mesh");
  }
  if (d->precon != BP_PRECON_NONE && d->precon != BP_PRECON_JACOBI)
    return fail(BP_ERROR_ARG, "bp_solver_create: unknown preconditioner");
  if (d->precision != BP_PRECISION_FP64 && d->precision != BP_PRECISION_MIXED)
    return fail(BP_ERROR_ARG, "bp_solver_create: unknown precision");
  if (d->bp <= 4) BP_TRY(bp_mesh_cubature(mesh));
  cudaStream_t s = default_stream();
  bp_solver_s* S = new bp_solver_s();
  S->mesh = mesh;
  S->bp = d->bp;
  S->lambda = d->lambda;
  S->precon = d->precon;
  S->mixed = d->precision == BP_PRECISION_MIXED;
  S->N = mesh->Ngather;
  S->ax.bp = d->bp;
  S->ax.N = mesh->N;
  S->ax.affine = mesh->affine;
  S->ax.Nfields = mesh->Nfields;
  S->ax.dim = mesh->dim;
  const size_t NL = (size_t)mesh->E * mesh->Np * mesh->Nfields;
  int rc = BP_SUCCESS;
  do {
    if ((rc = S->AqL.alloc(NL))) break;
    if ((rc = S->p.alloc(S->N))) break;
    if ((rc = S->Ap.alloc(S->N))) break;
    if ((rc = S->partials.alloc((size_t)4 * reduction_blocks()))) break;
    if ((rc = S->counter.alloc(4))) break;
    // p.Ap epilogue of the element operator: one partial per block, at most
    // one block per element
    if ((rc = S->fuse_partials.alloc((size_t)mesh->E + 1))) break;
    if ((rc = S->sc.alloc(1))) break;
    S->scal = S->sc.ptr;
    cudaError_t ce = cudaMemsetAsync(S->p.ptr, 0, sizeof(double) * S->N, s);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(S->counter.ptr, 0, sizeof(unsigned int) * 4, s);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(S->scal, 0, sizeof(CgScalars), s);
    if (ce == cudaSuccess) ce = cudaEventCreate(&S->ev0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&S->ev1);
    if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_solver_create", __FILE__, __LINE__); break; }
    if (S->precon == BP_PRECON_JACOBI) {
      if ((rc = S->invD.alloc(S->N))) break;
      if ((rc = bp_solver_diagonal(S, S->invD.ptr))) break;
      if ((rc = launch_reciprocal(S->N, S->invD.ptr, s))) break;
    }
    if (S->mixed) {
      // FP32 copies of the stored factors and the 1D operators (on the mesh), FP32 CG vectors
      S->family = S->bp >= 5 ? 0 : (S->bp >= 3 ? 1 : 2);
      if ((rc = mesh_fp32(S, s))) break;
      if ((rc = S->AqL32.alloc(NL))) break;
      if ((rc = S->p32.alloc(S->N))) break;
      if ((rc = S->x32.alloc(S->N))) break;
      if ((rc = S->r32.alloc(S->N))) break;
      if ((rc = S->bcopy.alloc(S->N))) break;
      if (S->precon == BP_PRECON_JACOBI) {
        if ((rc = S->invD32.alloc(S->N))) break;
        if ((rc = to_float(S->invD.ptr, S->invD32.ptr, S->N, s))) break;
      }
      ce = cudaMemsetAsync(S->p32.ptr, 0, sizeof(float) * S->N, s);
      if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_solver_create", __FILE__, __LINE__); break; }
    }
    ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_solver_create", __FILE__, __LINE__); break; }
  } while (0);
  if (rc != BP_SUCCESS) {
    delete S;
    return rc;
  }
  *out = S;
  return BP_SUCCESS;
}

int bp_solver_destroy(bp_solver_t S) {
  delete S;
  return BP_SUCCESS;
}

int bp_solver_size(bp_solver_t S, int32_t* n) {
  if (!S || !n) return fail(BP_ERROR_ARG, "bp_solver_size: null pointer");
  *n = S->N;
  return BP_SUCCESS;
}

int bp_solver_operator(bp_solver_t S, const double* q, double* Aq, bp_stream_t stream) {
  if (!S || !q || !Aq) return fail(BP_ERROR_ARG, "bp_solver_operator: null pointer");
  return operator_apply(S, q, Aq, nullptr, to_stream(stream));
}

int bp_solver_rhs(bp_solver_t S, int32_t mode, uint64_t seed, double* b, double* f_out) {
  if (!S || !b) return fail(BP_ERROR_ARG, "bp_solver_rhs: null pointer");
  bp_mesh_s* m = S->mesh;
  cudaStream_t s = default_stream();
  if (mode == BP_RHS_ANALYTIC) {
    // BP1/BP2 force with lambda = 0 (BP/BP1/src/bp1Run.cpp:54-62)
    const double lam = S->bp <= 2 ? 0.0 : S->lambda;
    if (m->simplex)
      BP_TRY(launch_rhs_analytic_simplex(m->dim, m->N, m->E, m->wJ.ptr, m->MM.ptr, m->x.ptr, m->y.ptr, m->z.ptr, lam,
                                         S->AqL.ptr, s));
    else if (m->dim == 2)
      BP_TRY(launch_rhs_analytic_quad(m->N, m->affine, m->Nfields, m->E, m->EX.ptr, m->EY.ptr, m->gllz.ptr,
                                      m->gllw.ptr, m->wJ.ptr, lam, S->AqL.ptr, s));
    else
      BP_TRY(launch_rhs_analytic(m->N, m->affine, m->Nfields, m->E, m->EX.ptr, m->EY.ptr, m->EZ.ptr, m->gllz.ptr,
                                 m->gllw.ptr, m->wJ.ptr, lam, S->AqL.ptr, s));
  } else if (mode == BP_RHS_RANDOM) {
    DeviceArray<double> ftmp;
    double* f = f_out;
    if (!f) {
      BP_TRY(ftmp.alloc(S->N));
      f = ftmp.ptr;
    }
    BP_TRY(launch_rhs_random(S->N, seed, f, s));
    if (m->simplex)
      BP_TRY(launch_mass_local_simplex(m->dim, m->N, m->E, m->G2L.ptr, m->wJ.ptr, m->MM.ptr, f, S->AqL.ptr, s));
    else if (m->dim == 2)
      BP_TRY(launch_mass_local_quad(m->N, m->affine, m->Nfields, m->E, m->G2L.ptr, m->gllw.ptr, m->wJ.ptr, f,
                                    S->AqL.ptr, s));
    else
      BP_TRY(launch_mass_local(m->N, m->affine, m->Nfields, m->E, m->G2L.ptr, m->gllw.ptr, m->wJ.ptr, f, S->AqL.ptr,
                               s));
    BP_TRY(launch_gather(m->Ngather, m->rowStarts.ptr, m->colIds.ptr, S->AqL.ptr, b, s));
    BP_CUDA_TRY(cudaStreamSynchronize(s));   // ftmp is released on return
    return BP_SUCCESS;
  } else {
    return fail(BP_ERROR_ARG, "bp_solver_rhs: unknown forcing mode");
  }
  BP_TRY(launch_gather(m->Ngather, m->rowStarts.ptr, m->colIds.ptr, S->AqL.ptr, b, s));
  BP_CUDA_TRY(cudaStreamSynchronize(s));
  return BP_SUCCESS;
}

int bp_solver_diagonal(bp_solver_t S, double* diag) {
  if (!S || !diag) return fail(BP_ERROR_ARG, "bp_solver_diagonal: null pointer");
  bp_mesh_s* m = S->mesh;
  cudaStream_t s = default_stream();
  if (m->simplex) {
    BP_TRY(launch_diag_local_simplex(m->dim, m->N, m->E, m->wJ.ptr, m->ggeo.ptr, m->S.ptr, m->MM.ptr, S->lambda,
                                     S->AqL.ptr, s));
  } else if (S->bp >= 5 && m->dim == 2) {
    BP_TRY(launch_diag_local_quad(m->N, m->affine, m->Nfields, m->E, m->ggeo.ptr, m->wJ.ptr, m->gllw.ptr, m->D.ptr,
                                  S->lambda, S->AqL.ptr, s));
  } else if (S->bp >= 5) {
    BP_TRY(launch_diag_local(m->N, m->affine, m->Nfields, m->E, m->ggeo.ptr, m->wJ.ptr, m->gllw.ptr, m->D.ptr,
                             S->lambda, S->AqL.ptr, s));
  } else {
    const ElemOperands<double> o = operands64(S);
    BP_TRY(launch_diag_cub(S->ax, m->E, o.wJ, o.ggeo, o.T, m->cubDV.ptr, S->lambda, S->AqL.ptr, s));
  }
  BP_TRY(launch_gather(m->Ngather, m->rowStarts.ptr, m->colIds.ptr, S->AqL.ptr, diag, s));
  BP_CUDA_TRY(cudaStreamSynchronize(s));
  return BP_SUCCESS;
}

int bp_solver_solve(bp_solver_t S, double* x, double* r, double tol, int32_t maxit, double* hist_rnorm,
                    double* hist_alpha, bp_solve_stats_t* stats) {
  if (!S || ((!x || !r) && S->N > 0)) return fail(BP_ERROR_ARG, "bp_solver_solve: null pointer");
  if (maxit < 0 || !(tol >= 0.0)) return fail(BP_ERROR_ARG, "bp_solver_solve: bad tol or maxit");
  return solve_device(S, x, r, tol, maxit, hist_rnorm, hist_alpha, stats, default_stream(), true);
}

int bp_solver_solve_host(bp_solver_t S, const double* b_host, double* x_host, double tol, int32_t maxit,
                         bp_solve_stats_t* stats) {
  if (!S || ((!b_host || !x_host) && S->N > 0)) return fail(BP_ERROR_ARG, "bp_solver_solve_host: null pointer");
  if (maxit < 0 || !(tol >= 0.0)) return fail(BP_ERROR_ARG, "bp_solver_solve_host: bad tol or maxit");
  cudaStream_t s = default_stream();
  if (!S->xw.ptr) {
    BP_TRY(S->xw.alloc(S->N));
    BP_TRY(S->rw.alloc(S->N));
  }
  const size_t bytes = sizeof(double) * S->N;
  cudaEvent_t e0, e1;
  BP_CUDA_TRY(cudaEventCreate(&e0));
  BP_CUDA_TRY(cudaEventCreate(&e1));
  int rc = BP_SUCCESS;
  do {
    cudaError_t ce = cudaEventRecord(e0, s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(S->rw.ptr, b_host, bytes, cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(S->xw.ptr, 0, bytes, s);
    if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_solver_solve_host", __FILE__, __LINE__); break; }
    // inner solve without its own events, then the copy back
    if ((rc = solve_device(S, S->xw.ptr, S->rw.ptr, tol, maxit, nullptr, nullptr, stats, s, false))) break;
    ce = cudaMemcpyAsync(x_host, S->xw.ptr, bytes, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaEventRecord(e1, s);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
    if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_solver_solve_host", __FILE__, __LINE__); break; }
    if (stats) stats->elapsed_ms = ms;
  } while (0);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched solves: many independent problems (each its own box, degree and
// element count) with several right-hand sides each.  Every (problem, rhs)
// pair is a CG system on its problem's mesh.  In a mixed-precision BP5 batch
// the right-hand sides of a problem (degree up to 11) are solved in lockstep as
// packed groups of 2 or 4 lanes (padding lanes carry b = 0 and finish at once);
// a single right-hand side and the other cases are standalone systems.  Each
// group or standalone system (a unit) has a CUDA graph of kBatchChunk iterations
// and runs on one stream of a pool; the host drives every unit on its own
// (reliable updates, next chunk, retirement) as its scalars arrive, so no unit
// waits for another.
// ---------------------------------------------------------------------------
struct CgGroup {
  int pk = 0;                                   // lanes
  bp_solver_s* base = nullptr;                  // mixed solver on the mesh: FP64 operator, invD, FP32 data
  DeviceArray<float> x32, r32, p32, AqL32;      // packed [N][pk], AqL [NL][pk]
  DeviceArray<float> p32b;                      // second direction buffer of the fused direction update
  bool dir = false;                             // the captured iterations fuse the direction update
  // one cooperative kernel per CG step (bp_cg_persist.cuh) instead of four
  bool persist = false;
  int persist_cap = 0;                          // resident blocks at most
  DeviceArray<double> step_red;                 // its block sums [3 pk + 1][persist_cap]
  DeviceArray<unsigned int> step_bar;           // its grid barrier [2]
  DeviceArray<double> parts;                    // operator p.Ap partials [pk][blocks]
  DeviceArray<double> gparts;                   // gather-update grid sums [2 pk][reduction blocks]
  DeviceArray<unsigned int> gcount;             // their arrival counter (zero between launches)
  CgScalars* sc = nullptr;                      // pk consecutive slots
  std::vector<double*> x, r, b;                 // per lane FP64 vectors
};

// A unit of a batch: one packed group, or one standalone system.  Each unit
// has its own graph of kBatchChunk iterations and is driven independently.
struct BatchUnit {
  CgGroup* G = nullptr;
  int sys = -1;                  // the standalone system (G == nullptr)
  int slot0 = 0, lanes = 1;      // its CG scalar slots
  double weight = 0.0;           // lane-nodes of element data per iteration
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t posted = nullptr;  // the host copy of its scalars has landed
  int stream = -1;               // stream of the pool while in flight
};

struct bp_batch_s {
  std::vector<bp_mesh_s*> meshes;             // owned
  std::vector<bp_solver_s*> owned;            // owned solvers (standalone systems and group bases)
  std::vector<CgGroup*> groups;               // owned
  std::vector<bp_solver_s*> sys_solver;       // per system: its solver (a group's base for grouped systems)
  std::vector<int> sys_prob, sys_group, sys_lane, sys_slot;
  std::vector<BatchUnit> units;
  std::vector<DeviceArray<double>*> x, r, b;  // per system (owned)
  std::vector<DeviceArray<double>*> pad;      // padding lanes' x, r, b (owned)
  DeviceArray<CgScalars> sc;                  // every slot's CG scalars, one array
  CgScalars* host_sc = nullptr;               // pinned host copy of sc
  int mixed = 0;
  std::vector<cudaStream_t> pool;             // the stream pool
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
  ~bp_batch_s() {
    for (auto& u : units) {
      if (u.graph) cudaGraphExecDestroy(u.graph);
      if (u.posted) cudaEventDestroy(u.posted);
    }
    if (host_sc) cudaFreeHost(host_sc);
    for (auto* G : groups) delete G;
    for (auto* S : owned) delete S;
    for (auto* m : meshes) bp_mesh_destroy(m);
    for (auto* v : x) delete v;
    for (auto* v : r) delete v;
    for (auto* v : b) delete v;
    for (auto* v : pad) delete v;
    for (auto st : pool) cudaStreamDestroy(st);
    for (auto e : joins) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

namespace bp {

// Streams of a batch's pool: units in flight at once.  Sixteen units side by
// side, each driven on its own, took 64 uneven problems from 9.1 s (one graph
// of all units with a host barrier after every chunk) to 7.1 s; 8 or 32
// streams, largest or smallest unit first, all gave 7.1 s.
constexpr int kPoolStreams = 16;

// one packed iteration of a group: direction, operator with per-lane p.Ap
// partials, alpha, gather + update
template <int PK>
static int grp_iteration(CgGroup* G, cudaStream_t s) {
  bp_solver_s* S = G->base;
  bp_mesh_s* m = S->mesh;
  const int32_t N = S->N;
  using T = Pack<float, PK>;
  const ElemOperands<float> o = operands32(S);
  CgFuse fuse;
  fuse.partials = G->parts.ptr;
  int nparts = 0;
  if (G->dir) {
    fuse.dir = 1;
    fuse.pbuf[0] = G->p32.ptr;
    fuse.pbuf[1] = G->p32b.ptr;
    fuse.r = G->r32.ptr;
    fuse.invD = S->precon ? S->invD32.ptr : nullptr;
    fuse.x = G->x32.ptr;
    fuse.sc = G->sc;
    const int rc = launch_ax_tma_packed(PK, S->ax, m->E, m->elementList.ptr, m->G2Lo.ptr, o.wJ, o.ggeo, o.D,
                                       (float)S->lambda, nullptr, G->AqL32.ptr, nullptr, &fuse, s, &nparts);
    if (rc == 1) return fail(BP_ERROR_ARG, "CG: the fused direction update does not cover this operator");
    BP_TRY(rc);
  } else {
    const int g = vec_grid_wave(reinterpret_cast<const void*>(&grp_direction_kernel<PK>), N);
    BP_CUDA_TRY(launch_pdl(grp_direction_kernel<PK>, g, kThreads, 0, s, N, reinterpret_cast<T*>(G->x32.ptr),
                           reinterpret_cast<T*>(G->p32.ptr), reinterpret_cast<const T*>(G->r32.ptr), S->invD32.ptr,
                           G->sc));
    BP_TRY(launch_ax_packed(PK, S->ax, m->E, m->elementList.ptr, m->G2L.ptr, o.wJ, o.ggeo, o.gllw, o.D,
                            (float)S->lambda, G->p32.ptr, G->AqL32.ptr, nullptr, &fuse, s, &nparts));
  }
  BP_CUDA_TRY(launch_pdl(cg_alpha_kernel<PK>, alpha_grid(nparts), kThreads, 0, s, nparts, G->parts.ptr, G->sc,
                         nullptr, G->gparts.ptr, G->gcount.ptr));
  const int gg = vec_grid_wave(reinterpret_cast<const void*>(&grp_gather_update_kernel<PK>), N);
  BP_CUDA_TRY(launch_pdl(grp_gather_update_kernel<PK>, gg, kThreads, 0, s, N, m->rowStarts.ptr, m->colIds.ptr,
                         reinterpret_cast<const T*>(G->AqL32.ptr), reinterpret_cast<T*>(G->r32.ptr), S->invD32.ptr,
                         G->sc, G->gparts.ptr, G->gcount.ptr));
  return BP_SUCCESS;
}

// one CG step of the group as one cooperative kernel (bp_cg_persist.cuh)
static int grp_step(CgGroup* G, cudaStream_t s) {
  bp_solver_s* S = G->base;
  bp_mesh_s* m = S->mesh;
  const ElemOperands<float> o = operands32(S);
  GrpStepArgs a{};
  a.N = S->N;
  a.Nelements = m->E;
  a.lambda = (float)S->lambda;
  a.precon = S->precon;
  a.elementList = m->elementList.ptr;
  a.G2L = m->G2L.ptr;
  a.rowStarts = m->rowStarts.ptr;
  a.colIds = m->colIds.ptr;
  a.wJ = o.wJ;
  a.ggeo = o.ggeo;
  a.gllw = o.gllw;
  a.D = o.D;
  a.invD = S->precon ? S->invD32.ptr : nullptr;
  a.x = G->x32.ptr;
  a.p = G->p32.ptr;
  a.r = G->r32.ptr;
  a.AqL = G->AqL32.ptr;
  a.sc = G->sc;
  a.parts = G->parts.ptr;
  a.red = G->step_red.ptr;
  a.bar = G->step_bar.ptr;
  a.err = device_error_word();
  if (!a.err) return fail(BP_ERROR_CUDA, "persistent CG step: device error word lookup failed");
  int rc = launch_grp_step_tma(G->pk, S->ax, a, G->persist_cap, s);
  if (rc == 1) rc = launch_grp_step_line(G->pk, S->ax, a, G->persist_cap, s);
  return rc == 1 ? fail(BP_ERROR_ARG, "persistent CG step: no form covers this group") : rc;
}

static int grp_body(CgGroup* G, cudaStream_t s) {
  if (G->persist) return grp_step(G, s);
  return G->pk == 4 ? grp_iteration<4>(G, s) : grp_iteration<2>(G, s);
}

// Whether a group's CG steps run as one cooperative kernel: where a form
// covers it and BP_PERSIST=1.  Measured, it does not pay: the 16^3 p=4 box
// with four right-hand sides takes 18.4 ms to 1e-8 against 18.3 ms for the
// graph of four kernels per step (the step is bound by the latency of its
// phases, the operator's above all, not by launches: 420 kernels instead of
// 1412 changed nothing), and the 64-problem batch 9.7 s against 5.5 s with it
// forced on everywhere (a cooperative grid holds the whole GPU, so the units
// on the other streams of the pool no longer overlap with it).
static bool want_persist(const CgGroup* G) {
  const bp_mesh_s* m = G->base->mesh;
  if (G->pk != 4 || m->dim == 2 || m->Nfields != 1 || m->N + 1 > 12) return false;
  const char* e = getenv("BP_PERSIST");
  return e && e[0] == '1';
}

// FP64 residual of lane l and the restart of its FP32 recursion (init: start of a solve)
static int grp_replace(CgGroup* G, int l, bool init, double tol, int maxit, cudaStream_t s) {
  bp_solver_s* S = G->base;
  const int32_t N = S->N;
  BP_TRY(operator_apply(S, G->x[l], S->Ap.ptr, nullptr, s));
  S->launches += 1;
  mixed_replace_kernel<<<vec_grid(N), kThreads, 0, s>>>(N, G->b[l], S->Ap.ptr, G->r[l], G->r32.ptr + l,
                                                        S->invD32.ptr, G->sc + l, init ? 1 : 0, tol, maxit,
                                                        S->precon, S->partials.ptr, S->counter.ptr, G->pk);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

// reliable update of lane l: the pending step, x_hi += x_lo, FP64 residual
static int grp_reliable(CgGroup* G, int l, double tol, int maxit, cudaStream_t s) {
  bp_solver_s* S = G->base;
  const int32_t N = S->N;
  S->launches += 2;
  cg_final_kernel<float><<<vec_grid(N), kThreads, 0, s>>>(N, G->x32.ptr + l, G->p32.ptr + l,
                                                           (G->dir ? G->p32b.ptr : G->p32.ptr) + l,
                                                           G->dir ? G->sc : nullptr, G->sc + l, G->pk);
  BP_CUDA_TRY(cudaGetLastError());
  mixed_fold_kernel<<<vec_grid(N), kThreads, 0, s>>>(N, G->x[l], G->x32.ptr + l, G->pk);
  BP_CUDA_TRY(cudaGetLastError());
  return grp_replace(G, l, false, tol, maxit, s);
}

// Units of the batch with their scalar slots and weights
static int batch_units(bp_batch_s* B) {
  for (auto* G : B->groups) {
    BatchUnit u;
    u.G = G;
    u.slot0 = (int)(G->sc - B->sc.ptr);
    u.lanes = G->pk;
    u.weight = (double)G->base->mesh->E * G->base->mesh->Np * G->pk;
    B->units.push_back(u);
  }
  for (size_t i = 0; i < B->sys_solver.size(); ++i) {
    if (B->sys_group[i] >= 0) continue;
    BatchUnit u;
    u.sys = (int)i;
    u.slot0 = B->sys_slot[i];
    const bp_mesh_s* m = B->sys_solver[i]->mesh;
    u.weight = (double)m->E * m->Np;
    B->units.push_back(u);
  }
  for (auto& u : B->units) BP_CUDA_TRY(cudaEventCreateWithFlags(&u.posted, cudaEventDisableTiming));
  return BP_SUCCESS;
}

// fork the stream pool off s (their work follows) and join it back
static int batch_fork(bp_batch_s* B, cudaStream_t s) {
  BP_CUDA_TRY(cudaEventRecord(B->fork, s));
  for (auto st : B->pool) BP_CUDA_TRY(cudaStreamWaitEvent(st, B->fork, 0));
  return BP_SUCCESS;
}
static int batch_join(bp_batch_s* B, cudaStream_t s) {
  for (size_t k = 0; k < B->pool.size(); ++k) {
    BP_CUDA_TRY(cudaEventRecord(B->joins[k], B->pool[k]));
    BP_CUDA_TRY(cudaStreamWaitEvent(s, B->joins[k], 0));
  }
  return BP_SUCCESS;
}

// kBatchChunk iterations of one unit as a graph
static int unit_capture(bp_batch_s* B, BatchUnit& u, cudaStream_t s) {
  if (u.graph) return BP_SUCCESS;
  // the element operator once outside the capture: the autotuner picks its form
  if (u.G) {
    CgGroup* G = u.G;
    bp_solver_s* S = G->base;
    bp_mesh_s* m = S->mesh;
    const ElemOperands<float> o = operands32(S);
    CgFuse fuse;
    fuse.partials = G->parts.ptr;
    int nparts = 0;
    BP_TRY(launch_ax_packed(G->pk, S->ax, m->E, m->elementList.ptr, m->G2L.ptr, o.wJ, o.ggeo, o.gllw, o.D,
                            (float)S->lambda, G->p32.ptr, G->AqL32.ptr, nullptr, &fuse, s, &nparts));
    BP_TRY(want_dir(m, S->ax, 4, G->pk, &G->dir, s));
    if (G->dir) BP_TRY(alloc_zero(G->p32b, G->p32.n, s));
    G->persist = !G->dir && want_persist(G);
    if (G->persist) {
      G->persist_cap = 32 * sm_count();
      BP_TRY(G->step_red.alloc((size_t)(3 * G->pk + 1) * G->persist_cap));
      BP_TRY(alloc_zero(G->step_bar, 2, s));
      BP_CUDA_TRY(cudaStreamSynchronize(s));
    }
  } else {
    bp_solver_s* S = B->sys_solver[u.sys];
    if (B->mixed) BP_TRY(prepare32(S, s));
    else BP_TRY(prepare64(S, s));
  }
  cudaGraph_t g;
  BP_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int rc = BP_SUCCESS;
  for (int k = 0; k < kBatchChunk && rc == BP_SUCCESS; ++k) {
    if (u.G) {
      rc = grp_body(u.G, s);
    } else {
      bp_solver_s* S = B->sys_solver[u.sys];
      rc = B->mixed ? body32(S, nullptr, nullptr, s) : body64(S, B->x[u.sys]->ptr, B->r[u.sys]->ptr, s);
    }
  }
  cudaError_t ce = cudaStreamEndCapture(s, &g);
  if (rc != BP_SUCCESS) return rc;
  BP_CUDA_TRY(ce);
  ce = cudaGraphInstantiate(&u.graph, g, 0);
  cudaGraphDestroy(g);
  BP_CUDA_TRY(ce);
  return BP_SUCCESS;
}

// start of a unit's solve: x = 0, r = b, the initial residuals
static int unit_start(bp_batch_s* B, BatchUnit& u, double tol, int maxit, cudaStream_t s) {
  if (u.G) {
    CgGroup* G = u.G;
    const size_t bytes = sizeof(double) * G->base->N;
    for (int l = 0; l < G->pk; ++l) {
      BP_CUDA_TRY(cudaMemsetAsync(G->x[l], 0, bytes, s));
      BP_CUDA_TRY(cudaMemcpyAsync(G->r[l], G->b[l], bytes, cudaMemcpyDeviceToDevice, s));
    }
    BP_CUDA_TRY(cudaMemsetAsync(G->x32.ptr, 0, sizeof(float) * G->x32.n, s));
    BP_CUDA_TRY(cudaMemsetAsync(G->p32.ptr, 0, sizeof(float) * G->p32.n, s));
    if (G->p32b.ptr) BP_CUDA_TRY(cudaMemsetAsync(G->p32b.ptr, 0, sizeof(float) * G->p32b.n, s));
    for (int l = 0; l < G->pk; ++l) BP_TRY(grp_replace(G, l, true, tol, maxit, s));
    return BP_SUCCESS;
  }
  const int i = u.sys;
  bp_solver_s* S = B->sys_solver[i];
  const size_t bytes = sizeof(double) * S->N;
  BP_CUDA_TRY(cudaMemsetAsync(B->x[i]->ptr, 0, bytes, s));
  BP_CUDA_TRY(cudaMemcpyAsync(B->r[i]->ptr, B->b[i]->ptr, bytes, cudaMemcpyDeviceToDevice, s));
  if (B->mixed) return mixed_begin(S, B->x[i]->ptr, B->r[i]->ptr, tol, maxit, s);
  BP_TRY(operator_apply(S, B->x[i]->ptr, S->Ap.ptr, nullptr, s));
  S->launches += 1;
  cg_init_kernel<<<vec_grid(S->N), kThreads, 0, s>>>(S->N, S->Ap.ptr, B->r[i]->ptr, S->invD.ptr, S->scal, tol, maxit,
                                                      S->precon, S->partials.ptr, S->counter.ptr);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

// copy the unit's scalars to the pinned host array, then mark the copy
static int unit_post(bp_batch_s* B, BatchUnit& u, cudaStream_t s) {
  BP_CUDA_TRY(cudaMemcpyAsync(B->host_sc + u.slot0, B->sc.ptr + u.slot0, sizeof(CgScalars) * u.lanes,
                              cudaMemcpyDeviceToHost, s));
  BP_CUDA_TRY(cudaEventRecord(u.posted, s));
  return BP_SUCCESS;
}

// Every unit runs on a stream of the pool, driven by the host without a
// global barrier: when a unit's scalars land, the host applies the reliable
// updates of its lanes, launches its next chunk, or retires it and admits the
// next unit (largest first).
static int batch_solve(bp_batch_s* B, double tol, int maxit, bp_solve_stats_t* stats, double* elapsed_ms) {
  cudaStream_t s = default_stream();
  const size_t ns = B->sys_solver.size();
  if (B->mixed && !(tol > 0.0)) return fail(BP_ERROR_ARG, "bp_batch_solve: a mixed-precision batch needs tol > 0");
  for (auto& u : B->units) BP_TRY(unit_capture(B, u, s));
  std::vector<int> updates(B->sc.n, 0);
  for (auto* S : B->owned) S->launches = 0;
  BP_CUDA_TRY(cudaEventRecord(B->ev0, s));
  BP_TRY(batch_fork(B, s));
  const int nu = (int)B->units.size();
  std::vector<int> order(nu);
  for (int k = 0; k < nu; ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return B->units[a].weight > B->units[b].weight; });
  std::vector<int> free_streams;
  for (int k = (int)B->pool.size() - 1; k >= 0; --k) free_streams.push_back(k);
  std::vector<int> inflight;
  int next = 0;   // order[next..]: not started
  auto admit = [&](int ui) -> int {
    BatchUnit& u = B->units[ui];
    u.stream = free_streams.back();
    free_streams.pop_back();
    const cudaStream_t st = B->pool[u.stream];
    BP_TRY(unit_start(B, u, tol, maxit, st));
    BP_TRY(unit_post(B, u, st));
    inflight.push_back(ui);
    return BP_SUCCESS;
  };
  auto fill = [&]() -> int {
    while (next < nu && !free_streams.empty()) BP_TRY(admit(order[next++]));
    return BP_SUCCESS;
  };
  BP_TRY(fill());
  while (!inflight.empty()) {
    bool progressed = false;
    for (size_t a = 0; a < inflight.size();) {
      BatchUnit& u = B->units[inflight[a]];
      const cudaError_t q = cudaEventQuery(u.posted);
      if (q == cudaErrorNotReady) {
        ++a;
        continue;
      }
      BP_CUDA_TRY(q);
      progressed = true;
      const cudaStream_t st = B->pool[u.stream];
      bool running = false, updated = false;
      for (int l = 0; l < u.lanes; ++l) {
        const CgScalars& c = B->host_sc[u.slot0 + l];
        if (c.breakdown) continue;
        if (B->mixed && c.update) {
          if (u.G) BP_TRY(grp_reliable(u.G, l, tol, maxit, st));
          else BP_TRY(mixed_reliable(B->sys_solver[u.sys], B->x[u.sys]->ptr, B->r[u.sys]->ptr, tol, maxit, st));
          ++updates[u.slot0 + l];
          updated = true;
        } else if (!c.done) {
          running = true;
        }
      }
      if (updated) {   // the updated lanes may have converged or resume
        BP_TRY(unit_post(B, u, st));
        ++a;
        continue;
      }
      if (running) {
        BP_CUDA_TRY(cudaGraphLaunch(u.graph, st));
        bp_solver_s* us = u.G ? u.G->base : B->sys_solver[u.sys];
        const bool ud = u.G ? u.G->dir : (B->mixed ? us->dir32 : us->dir64);
        us->launches += ((u.G && u.G->persist) ? 1 : ud ? 3 : 4) * kBatchChunk;
        BP_TRY(unit_post(B, u, st));
        ++a;
        continue;
      }
      // retired: its stream goes back to the pool (stream order keeps its tail first)
      if (!B->mixed && !u.G) {
        bp_solver_s* S = B->sys_solver[u.sys];
        S->launches += 1;
        cg_final_kernel<double><<<vec_grid(S->N), kThreads, 0, st>>>(S->N, B->x[u.sys]->ptr, S->p.ptr, S->p_alt.ptr,
                                                                     S->dir64 ? S->scal : nullptr, S->scal);
        BP_CUDA_TRY(cudaGetLastError());
      }
      free_streams.push_back(u.stream);
      u.stream = -1;
      inflight.erase(inflight.begin() + (long)a);
      BP_TRY(fill());
    }
    if (!progressed) std::this_thread::yield();
  }
  BP_TRY(batch_join(B, s));
  BP_CUDA_TRY(cudaEventRecord(B->ev1, s));
  BP_CUDA_TRY(cudaMemcpyAsync(B->host_sc, B->sc.ptr, sizeof(CgScalars) * B->sc.n, cudaMemcpyDeviceToHost, s));
  BP_CUDA_TRY(cudaStreamSynchronize(s));
  const CgScalars* h = B->host_sc;
  float ms = 0.f;
  BP_CUDA_TRY(cudaEventElapsedTime(&ms, B->ev0, B->ev1));
  if (elapsed_ms) *elapsed_ms = ms;
  BP_TRY(check_device_error());
  bool breakdown = false;
  for (size_t i = 0; i < ns; ++i) {
    const CgScalars& c = h[B->sys_slot[i]];
    if (stats) {
      stats[i].iterations = c.iter;
      stats[i].rdotr0 = c.rdotr0;
      stats[i].rdotr = B->mixed ? c.rtrue2 : c.rdotr;
      stats[i].elapsed_ms = ms;
      stats[i].updates = updates[B->sys_slot[i]];
      // a group's launches serve all its lanes: each lane reports an equal share
      const int g = B->sys_group[i];
      stats[i].kernel_launches =
          g >= 0 ? B->sys_solver[i]->launches / B->groups[g]->pk : B->sys_solver[i]->launches;
    }
    breakdown = breakdown || c.breakdown;
  }
  if (breakdown) return fail(BP_ERROR_NUMERIC, "bp_batch_solve: CG breakdown in a system (p.Ap <= 0 or non-finite)");
  return BP_SUCCESS;
}

}  // namespace bp

extern "C" {

int bp_batch_create(const bp_batch_problem_t* problems, int32_t nproblems, const bp_solver_desc_t* d,
                    bp_batch_t* out) {
  if (!problems || !d || !out || nproblems < 1) return fail(BP_ERROR_ARG, "bp_batch_create: bad arguments");
  *out = nullptr;
  if (d->bp != 1 && d->bp != 3 && d->bp != 5) return fail(BP_ERROR_ARG, "bp_batch_create: bp must be 1, 3 or 5");
  for (int j = 0; j < nproblems; ++j)
    if (problems[j].nrhs < 1 || problems[j].nrhs > 64) return fail(BP_ERROR_ARG, "bp_batch_create: nrhs must be 1..64");
  cudaStream_t s = default_stream();
  bp_batch_s* B = new bp_batch_s();
  B->mixed = d->precision == BP_PRECISION_MIXED;
  int rc = BP_SUCCESS;
  do {
    cudaError_t ce = cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaEventCreate(&B->ev0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&B->ev1);
    for (int k = 0; k < kPoolStreams && ce == cudaSuccess; ++k) {
      cudaStream_t st;
      cudaEvent_t e;
      ce = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
      if (ce != cudaSuccess) break;
      B->pool.push_back(st);
      ce = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
      if (ce != cudaSuccess) break;
      B->joins.push_back(e);
    }
    if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_batch_create", __FILE__, __LINE__); break; }
    // plan: which systems are packed into groups, and the scalar slots
    struct Unit { int prob, first_rhs, nrhs, pk; };   // pk 0: standalone system
    std::vector<Unit> units;
    int nslots = 0;
    for (int j = 0; j < nproblems; ++j) {
      const bp_batch_problem_t& P = problems[j];
      const bool packable = B->mixed && d->bp == 5 && P.N + 1 <= 12;
      // four lanes at every degree: per right-hand side the four-lane operator
      // beats the two-lane one (BK5 18^3, FP32: p=8 9.13 vs 5.63 x 10^10 DOF/s),
      // and in the C5 batch (64 uneven problems: 5.71 s, two lanes at Nq = 9
      // 6.00 s)
      const int maxpk = 4;
      for (int k = 0; k < P.nrhs;) {
        const int left = P.nrhs - k;
        const int pk = !packable || left == 1 ? 0 : (left == 2 ? 2 : maxpk);
        const int n = pk ? std::min(pk, left) : 1;
        units.push_back({j, k, n, pk});
        nslots += pk ? pk : 1;
        k += n;
      }
    }
    if ((rc = B->sc.alloc(nslots))) break;
    ce = cudaMemsetAsync(B->sc.ptr, 0, sizeof(CgScalars) * nslots, s);
    if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_batch_create", __FILE__, __LINE__); break; }
    int slot = 0, cur = -1;
    bp_mesh_t m = nullptr;
    for (const Unit& u : units) {
      const bp_batch_problem_t& P = problems[u.prob];
      if (u.prob != cur) {
        bp_box_desc_t bd{};
        bd.nx = P.nx; bd.ny = P.ny; bd.nz = P.nz; bd.N = P.N; bd.affine = P.affine ? 1 : 0; bd.Nfields = 1;
        bd.pert = P.pert; bd.pert_seed = P.pert_seed;
        m = nullptr;
        if ((rc = bp_mesh_create(&bd, &m))) break;
        B->meshes.push_back(m);
        cur = u.prob;
      }
      bp_solver_t S = nullptr;
      if ((rc = bp_solver_create(m, d, &S))) break;
      B->owned.push_back(S);
      CgGroup* G = nullptr;
      if (u.pk) {
        G = new CgGroup();
        B->groups.push_back(G);
        G->pk = u.pk;
        G->base = S;
        G->sc = B->sc.ptr + slot;
        const size_t NL = (size_t)m->E * m->Np;
        if ((rc = G->x32.alloc((size_t)S->N * u.pk))) break;
        if ((rc = G->r32.alloc((size_t)S->N * u.pk))) break;
        if ((rc = G->p32.alloc((size_t)S->N * u.pk))) break;
        if ((rc = G->AqL32.alloc(NL * u.pk))) break;
        if ((rc = G->parts.alloc(((size_t)m->E + 1) * u.pk))) break;
        if ((rc = G->gparts.alloc((size_t)2 * u.pk * reduction_blocks()))) break;
        if ((rc = G->gcount.alloc(1))) break;
        ce = cudaMemsetAsync(G->gcount.ptr, 0, sizeof(unsigned int), s);
        if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_batch_create", __FILE__, __LINE__); break; }
      } else {
        S->scal = B->sc.ptr + slot;
      }
      for (int k = 0; k < (u.pk ? u.pk : 1) && rc == BP_SUCCESS; ++k) {
        auto* xv = new DeviceArray<double>();
        auto* rv = new DeviceArray<double>();
        auto* bv = new DeviceArray<double>();
        const bool real = k < u.nrhs;
        if (real) {
          B->x.push_back(xv);
          B->r.push_back(rv);
          B->b.push_back(bv);
          B->sys_solver.push_back(S);
          B->sys_prob.push_back(u.prob);
          B->sys_group.push_back(G ? (int)B->groups.size() - 1 : -1);
          B->sys_lane.push_back(G ? k : 0);
          B->sys_slot.push_back(slot + k);
        } else {
          B->pad.push_back(xv);
          B->pad.push_back(rv);
          B->pad.push_back(bv);
        }
        if ((rc = xv->alloc(S->N))) break;
        if ((rc = rv->alloc(S->N))) break;
        if ((rc = bv->alloc(S->N))) break;
        if (G) {
          G->x.push_back(xv->ptr);
          G->r.push_back(rv->ptr);
          G->b.push_back(bv->ptr);
        }
        if (real) {
          rc = bp_solver_rhs(S, BP_RHS_RANDOM, P.rhs_seed + (uint64_t)(u.first_rhs + k), bv->ptr, nullptr);
        } else {
          // a padding lane: b = 0 converges at its first test and stays idle
          ce = cudaMemsetAsync(bv->ptr, 0, sizeof(double) * S->N, s);
          if (ce == cudaSuccess) ce = cudaMemsetAsync(xv->ptr, 0, sizeof(double) * S->N, s);
          if (ce != cudaSuccess) rc = cuda_fail(ce, "bp_batch_create", __FILE__, __LINE__);
        }
      }
      if (rc != BP_SUCCESS) break;
      slot += u.pk ? u.pk : 1;
    }
    if (rc == BP_SUCCESS) rc = batch_units(B);
    if (rc == BP_SUCCESS) {
      ce = cudaMallocHost(reinterpret_cast<void**>(&B->host_sc), sizeof(CgScalars) * B->sc.n);
      if (ce != cudaSuccess) rc = cuda_fail(ce, "bp_batch_create", __FILE__, __LINE__);
    }
    if (rc == BP_SUCCESS) {
      cudaError_t ce2 = cudaStreamSynchronize(s);
      if (ce2 != cudaSuccess) rc = cuda_fail(ce2, "bp_batch_create", __FILE__, __LINE__);
    }
  } while (0);
  if (rc != BP_SUCCESS) {
    delete B;
    return rc;
  }
  *out = B;
  return BP_SUCCESS;
}

int bp_batch_destroy(bp_batch_t B) {
  delete B;
  return BP_SUCCESS;
}

int bp_batch_systems(bp_batch_t B, int32_t* nsystems) {
  if (!B || !nsystems) return fail(BP_ERROR_ARG, "bp_batch_systems: null pointer");
  *nsystems = (int32_t)B->sys_solver.size();
  return BP_SUCCESS;
}

int bp_batch_system_info(bp_batch_t B, int32_t system, int32_t* problem, int32_t* Ngather) {
  if (!B || system < 0 || system >= (int32_t)B->sys_solver.size())
    return fail(BP_ERROR_ARG, "bp_batch_system_info: bad system index");
  if (problem) *problem = B->sys_prob[system];
  if (Ngather) *Ngather = B->sys_solver[system]->N;
  return BP_SUCCESS;
}

int bp_batch_solve(bp_batch_t B, double tol, int32_t maxit, bp_solve_stats_t* stats, double* elapsed_ms) {
  if (!B) return fail(BP_ERROR_ARG, "bp_batch_solve: null batch");
  if (maxit < 0 || !(tol >= 0.0)) return fail(BP_ERROR_ARG, "bp_batch_solve: bad tol or maxit");
  return batch_solve(B, tol, maxit, stats, elapsed_ms);
}

int bp_batch_vectors(bp_batch_t B, int32_t system, double** x, double** b) {
  if (!B || system < 0 || system >= (int32_t)B->sys_solver.size())
    return fail(BP_ERROR_ARG, "bp_batch_vectors: bad system index");
  if (x) *x = B->x[system]->ptr;
  if (b) *b = B->b[system]->ptr;
  return BP_SUCCESS;
}

int bp_batch_solver(bp_batch_t B, int32_t system, bp_solver_t* solver) {
  if (!B || !solver || system < 0 || system >= (int32_t)B->sys_solver.size())
    return fail(BP_ERROR_ARG, "bp_batch_solver: bad system index");
  *solver = B->sys_solver[system];
  return BP_SUCCESS;
}

}  // extern "C"
