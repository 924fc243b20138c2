// One CG step of a packed group (PK right-hand sides of one mesh in lockstep)
// as a single cooperative kernel.
//
// The graph form of a step is four kernels (direction, element operator with
// p.Ap partials, alpha, gather + update); on small meshes every one of them is
// mostly launch, ramp-up and tail.  Here the blocks of one resident grid run
// the four phases back to back, separated by grid barriers:
//   A  x += alpha_{k-1} p, p = z + beta p       (rows, grid-stride)
//   B  AqL = A_e p, p.Ap partials                 (element blocks, grid-stride;
//                                                  the operator's own body)
//   C  p.Ap: strided partial sums per block, then every block adds the block
//      sums in block order, so all blocks hold the same alpha
//   D  r -= alpha Gather(AqL), r.r and r.z per lane (rows, grid-stride)
//   E  block 0 adds the block sums in block order and updates the lanes'
//      scalars (the gather-update's stop test and reliable-update request)
// The sums keep a fixed order, so the step is reproducible; it is the same
// arithmetic as the graph form up to the grouping of the sums.
//
// The grid is launched cooperatively (every block resident), so the barriers
// cannot deadlock; each still waits at most kBarrierCycles and, if that runs
// out, records BP_ERROR_TIMEOUT in the library's device error word and the
// blocks leave the step.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "bp_cg_device.cuh"
#include "bp_internal.hpp"
#include "bp_pack.cuh"

namespace bp {

struct GrpStepArgs {
  int32_t N;                  // gathered rows
  int32_t Nelements;
  int nblk_op;                // element blocks of the operator body
  float lambda;
  int precon;
  const int32_t* elementList;
  const int32_t* G2L;
  const int32_t* rowStarts;
  const int32_t* colIds;
  const float* wJ;
  const float* ggeo;
  const float* gllw;
  const float* D;
  const float* invD;          // [N], null without preconditioner
  float* x;                   // packed [N][PK]
  float* p;
  float* r;
  float* AqL;                 // packed [NL][PK]
  CgScalars* sc;              // PK lanes
  double* parts;              // operator p.Ap partials [PK][nblk_op]
  double* red;                // block sums [3 PK][gridDim]
  unsigned int* bar;          // barrier: [0] arrivals, [1] generation
  int* err;                   // the library's device error word
};

constexpr long long kBarrierCycles = 1ll << 31;   // about one second of SM clocks

// Grid barrier over a cooperative grid, bounded; false when it gave up.
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, int* err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
    // the generation is read with atomics (at the L2, never a stale L1 copy)
    const unsigned int g = atomicAdd(bar + 1, 0u);
    __threadfence();
    int ok = 1;
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);   // nobody arrives again before the release below
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const long long t0 = clock64();
      while (atomicAdd(bar + 1, 0u) == g) {
        if (clock64() - t0 > kBarrierCycles) {
          ok = 0;
          atomicExch(err, 1);
          break;
        }
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Sum over the grid-stride partition of the block: valid in thread 0
template <int L>
__device__ __forceinline__ void step_block_sum(const double (&v)[L], double* scratch, double (&out)[L]) {
  fuse_block_sum_lanes<L>(v, scratch, out);
}

// Op: the operator phase, Op::run(blk, args, smem) on element block blk, with
// the block shape (Op::THREADS threads) and register budget (Op::MINB resident
// blocks per SM) of the operator's own kernel.
template <int PK, class Op>
__global__ void __launch_bounds__(Op::THREADS, Op::MINB) grp_step_kernel(GrpStepArgs a) {
  using T = Pack<float, PK>;
  extern __shared__ __align__(128) unsigned char step_smem[];
  double* scratch = reinterpret_cast<double*>(step_smem);
  __shared__ double s_alpha[PK];
  __shared__ bool s_ok[PK];   // p.Ap > 0 and alpha finite (else the lane breaks down and is left alone)
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int gt = blockIdx.x * nt + t, gstride = gridDim.x * nt;

  bool act[PK], addx[PK], first[PK];
  float alpha[PK], beta[PK];
  bool any = false;
#pragma unroll
  for (int l = 0; l < PK; ++l) {
    const CgScalars& c = a.sc[l];
    act[l] = !c.done;
    any = any || act[l];
    first[l] = c.iter == 0;
    addx[l] = c.iter > 0 && !c.skip_x;
    alpha[l] = (float)c.alpha;
    beta[l] = first[l] ? 0.0f : (float)(c.precon ? c.rz / c.rz_prev : c.rdotr / c.rdotr_prev);
  }
  if (!any) return;   // grid-uniform: the scalars change only after the last barrier

  // A: direction
  T* x = reinterpret_cast<T*>(a.x);
  T* p = reinterpret_cast<T*>(a.p);
  T* r = reinterpret_cast<T*>(a.r);
  for (int32_t n = gt; n < a.N; n += gstride) {
    T pn = p[n], xn = x[n];
    const T rn = r[n];
    const float d = a.precon ? a.invD[n] : 1.0f;
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
  if (!grid_barrier(a.bar, a.err)) return;

  // B: element operator and its p.Ap partials
  for (int blk = blockIdx.x; blk < a.nblk_op; blk += gridDim.x) Op::run(blk, a, step_smem);
  if (!grid_barrier(a.bar, a.err)) return;

  // C: p.Ap and alpha, the same in every block
  {
    double acc[PK], bs[PK];
#pragma unroll
    for (int l = 0; l < PK; ++l) acc[l] = 0.0;
    for (int k = gt; k < a.nblk_op; k += gstride)
#pragma unroll
      for (int l = 0; l < PK; ++l) acc[l] += a.parts[(size_t)l * a.nblk_op + k];
    step_block_sum<PK>(acc, scratch, bs);
    if (t == 0)
#pragma unroll
      for (int l = 0; l < PK; ++l) a.red[(size_t)l * gridDim.x + blockIdx.x] = bs[l];
  }
  if (!grid_barrier(a.bar, a.err)) return;
  {
    double acc[PK], tot[PK];
#pragma unroll
    for (int l = 0; l < PK; ++l) acc[l] = 0.0;
    for (int b = t; b < (int)gridDim.x; b += nt)
#pragma unroll
      for (int l = 0; l < PK; ++l) acc[l] += *((volatile double*)&a.red[(size_t)l * gridDim.x + b]);
    step_block_sum<PK>(acc, scratch, tot);
    if (t == 0)
#pragma unroll
      for (int l = 0; l < PK; ++l) {
        const double rho = a.sc[l].precon ? a.sc[l].rz : a.sc[l].rdotr;
        s_alpha[l] = rho / tot[l];
        s_ok[l] = tot[l] > 0.0 && isfinite(s_alpha[l]);
        if (blockIdx.x == 0) a.red[(size_t)(3 * PK) * gridDim.x + l] = tot[l];   // p.Ap for the lane's scalars
      }
    __syncthreads();
  }

  // D: gather + residual update, r.r and r.z per lane
  {
    float al[PK];
#pragma unroll
    for (int l = 0; l < PK; ++l) al[l] = (float)s_alpha[l];
    double acc[2 * PK], bs[2 * PK];
#pragma unroll
    for (int c = 0; c < 2 * PK; ++c) acc[c] = 0.0;
    const T* AqL = reinterpret_cast<const T*>(a.AqL);
    for (int32_t row = gt; row < a.N; row += gstride) {
      T rn = r[row];
      const float dinv = a.precon ? __ldg(a.invD + row) : 0.0f;
      const int32_t start = __ldg(a.rowStarts + row), end = __ldg(a.rowStarts + row + 1);
      T sum = AqL[__ldg(a.colIds + start)];
      for (int32_t c = start + 1; c < end; ++c) sum += AqL[__ldg(a.colIds + c)];
#pragma unroll
      for (int l = 0; l < PK; ++l) {
        if (act[l] && s_ok[l]) rn.v[l] = rn.v[l] - al[l] * sum.v[l];
        acc[l] += (double)rn.v[l] * (double)rn.v[l];
        if (a.precon) acc[PK + l] += (double)rn.v[l] * (double)dinv * (double)rn.v[l];
      }
      r[row] = rn;
    }
    step_block_sum<2 * PK>(acc, scratch, bs);
    if (t == 0)
#pragma unroll
      for (int c = 0; c < 2 * PK; ++c) a.red[(size_t)(PK + c) * gridDim.x + blockIdx.x] = bs[c];
  }
  if (!grid_barrier(a.bar, a.err)) return;

  // E: block 0 closes the step
  if (blockIdx.x != 0) return;
  double acc[2 * PK], tot[2 * PK];
#pragma unroll
  for (int c = 0; c < 2 * PK; ++c) acc[c] = 0.0;
  for (int b = t; b < (int)gridDim.x; b += nt)
#pragma unroll
    for (int c = 0; c < 2 * PK; ++c) acc[c] += *((volatile double*)&a.red[(size_t)(PK + c) * gridDim.x + b]);
  step_block_sum<2 * PK>(acc, scratch, tot);
  if (t != 0) return;
  for (int l = 0; l < PK; ++l) {
    if (!act[l]) continue;
    CgScalars& c = a.sc[l];
    const double pAp = a.red[(size_t)(3 * PK) * gridDim.x + l];
    const double al = s_alpha[l];
    c.pAp = pAp;
    if (!s_ok[l]) {   // the alpha kernel's breakdown test
      c.breakdown = 1;
      c.done = 1;
      continue;
    }
    c.alpha = al;
    c.rdotr_prev = c.rdotr;
    c.rdotr = tot[l];
    if (a.precon) {
      c.rz_prev = c.rz;
      c.rz = tot[PK + l];
    }
    c.iter += 1;
    c.skip_x = 0;
    if (!isfinite(tot[l])) {
      c.breakdown = 1;
      c.done = 1;
    } else if (tot[l] <= c.tol2 || c.iter >= c.maxit) {
      c.update = 1;
      c.done = 1;
    } else if (tot[l] < kReliableDrop * kReliableDrop * c.rmax2) {   // as grp_gather_update_kernel
      c.update = 1;
    }
  }
  a.sc[0].gen += 1;
}

// Resident blocks of grp_step_kernel<PK, Op> (one cooperative grid) for a
// block of `threads` threads and `smem` bytes of dynamic shared memory
template <int PK, class Op>
int grp_step_grid(int threads, size_t smem, int* blocks) {
  int dev = 0, sms = 0, per_sm = 0;
  BP_CUDA_TRY(cudaGetDevice(&dev));
  BP_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (smem > 48 * 1024)
    BP_CUDA_TRY(cudaFuncSetAttribute(grp_step_kernel<PK, Op>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  BP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grp_step_kernel<PK, Op>, threads, smem));
  *blocks = per_sm * sms;
  return *blocks > 0 ? BP_SUCCESS : fail(BP_ERROR_CUDA, "persistent CG step: no block fits on an SM");
}

template <int PK, class Op>
int launch_grp_step_kernel(const GrpStepArgs& a, dim3 block, size_t op_smem, int grid_cap, cudaStream_t s) {
  const int threads = (int)(block.x * block.y * block.z);
  // the block sums need 2 PK doubles per thread in the strided form
  const size_t smem = op_smem > sizeof(double) * 2 * PK * threads ? op_smem : sizeof(double) * 2 * PK * threads;
  int blocks = 0;
  const int rc = grp_step_grid<PK, Op>(threads, smem, &blocks);
  if (rc != BP_SUCCESS) return rc;
  if (blocks > grid_cap) blocks = grid_cap;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  BP_CUDA_TRY(cudaLaunchKernelEx(&cfg, grp_step_kernel<PK, Op>, a));
  return BP_SUCCESS;
}

}  // namespace bp
