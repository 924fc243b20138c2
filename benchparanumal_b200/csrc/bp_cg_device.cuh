// Device-side CG state and the p.Ap epilogue shared by the element-operator
// kernels and the CG kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace bp {

// A mixed-precision lane asks for a reliable update once its FP32 residual
// has dropped by this factor since the last replacement.
constexpr double kReliableDrop = 1e-2;

struct CgScalars {
  double rdotr;       // r.r after the last update (plain CG: the reference's rdotr)
  double rdotr_prev;  // r.r one update earlier
  double rz, rz_prev; // r.z for Jacobi CG
  double pAp, alpha;
  double tol2;        // stop when rdotr <= tol2 (mixed: when the FP64 residual r.r <= tol2)
  double rdotr0;
  double rtrue2;      // mixed: r.r of the FP64 residual b - A x at the last replacement
  double rmax2;       // mixed: the same, the reference level for the next replacement
  int iter;           // completed iterations
  int done;           // 1 once converged, at maxit, broken down, or (mixed) a replacement is due
  int maxit;
  int breakdown;
  int precon;
  int mixed;          // 1 in a mixed-precision solve
  int skip_x;         // 1: the last iteration's x update has been applied already
  int update;         // mixed: 1 asks the host for a reliable update
  int gen;            // completed gather-updates (never reset): the current direction p of an operator
                      // with the fused direction update lives in pbuf[gen & 1] (CgFuse)
};

// Where an element-operator launch inside CG leaves p.Ap.  Because
// A = sum_e Q_e^T A_e Q_e, p.Ap = sum_e (Q_e p).(A_e Q_e p): each block adds up
// q*Aq over its own nodes and stores the sum in partials[blockIdx.x];
// cg_alpha_kernel then adds the partials in index order and forms alpha.
//
// With `dir` set, the operator also does the CG direction update of its step
// (the work of cg_direction_kernel): it does not read q but, at every node it
// reads, forms p_k = z + beta p_{k-1} (z = invD r, or r) from p_{k-1} in
// pbuf[gen & 1], works on p_k, and at the nodes it owns -- GlobalToLocal
// entries carrying kOwnerBit, one local node per gathered node -- writes p_k
// to pbuf[(gen + 1) & 1] and applies the deferred x += alpha_{k-1} p_{k-1}.
// The two buffers keep p_{k-1} intact while other elements still read it; the
// gather-update that ends the step advances gen.  Per lane l the scalars are
// sc[l]; gen is the first lane's.
//
// Outside a CG solve (sc null) the step is given by value: lane l has
// coefficients alpha[l], beta[l] (beta[l] = 0 forms p = z, the first step;
// alpha[l] = 0 leaves x alone), p_{k-1} is pbuf[0] and p_k goes to pbuf[1].
constexpr int kMaxLanes = 4;
struct CgFuse {
  double* partials = nullptr;   // [number of blocks of the operator launch]
  int dir = 0;
  void* pbuf[2] = {nullptr, nullptr};
  const void* r = nullptr;
  const void* invD = nullptr;   // null: no preconditioner (z = r)
  void* x = nullptr;
  const CgScalars* sc = nullptr;
  double alpha[kMaxLanes] = {0, 0, 0, 0}, beta[kMaxLanes] = {0, 0, 0, 0};
};

// GlobalToLocal entries of an operator with the fused direction update:
// the gathered index in the low bits, kOwnerBit on the one local node of each
// gathered node that writes it (the first column of its CSR row); -1 masked.
constexpr int32_t kOwnerBit = 0x40000000;
constexpr int32_t kIdMask = kOwnerBit - 1;

// The step's per-lane scalars of the fused direction update (the values
// cg_direction_kernel and grp_direction_kernel use).
template <int L, class F>
struct DirStep {
  bool act[L], first[L], addx[L];
  F alpha[L], beta[L];
  bool any, anyx;
  int gen;
  __device__ __forceinline__ void load(const CgFuse& fz) {
    any = anyx = false;
    if (!fz.sc) {   // coefficients by value
      gen = 0;
      any = true;
#pragma unroll
      for (int l = 0; l < L; ++l) {
        act[l] = true;
        first[l] = fz.beta[l] == 0.0;
        addx[l] = fz.alpha[l] != 0.0;
        anyx = anyx || addx[l];
        alpha[l] = (F)fz.alpha[l];
        beta[l] = (F)fz.beta[l];
      }
      return;
    }
    const CgScalars* sc = fz.sc;
    gen = sc[0].gen;
#pragma unroll
    for (int l = 0; l < L; ++l) {
      const CgScalars& c = sc[l];
      act[l] = !c.done;
      any = any || act[l];
      first[l] = c.iter == 0;
      addx[l] = act[l] && c.iter > 0 && !c.skip_x;
      anyx = anyx || addx[l];
      alpha[l] = (F)c.alpha;
      beta[l] = first[l] ? F(0) : (F)(c.precon ? c.rz / c.rz_prev : c.rdotr / c.rdotr_prev);
    }
  }
};

// Sum of v over the block in a fixed order, valid in thread 0.  `scratch`
// holds at least one double per thread and is free for the caller to reuse
// (any block shape, partial warps included).
//
// A block of whole warps sums each warp by a shuffle tree and thread 0 adds
// the warp sums in warp order: one barrier pair and nt/32 serial additions
// (the strided form below ends in 32 dependent shared-memory reads and adds in
// thread 0, about 1000 cycles per block).
__device__ __forceinline__ double warp_tree_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double fuse_block_sum(double v, double* scratch) {
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  if ((nt & 31) == 0) {
    v = warp_tree_sum(v);
    __syncthreads();   // the caller's last reads of scratch are done
    if ((t & 31) == 0) scratch[t >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (t == 0)
      for (int w = 0; w < (nt >> 5); ++w) r += scratch[w];
    return r;
  }
  __syncthreads();   // the caller's last reads of scratch are done
  scratch[t] = v;
  __syncthreads();
  if (t < 32) {
    double r = 0.0;
    for (int k = t; k < nt; k += 32) r += scratch[k];
    scratch[t] = r;   // index t is read by this thread only
  }
  __syncthreads();
  double r = 0.0;
  if (t == 0)
    for (int k = 0; k < (nt < 32 ? nt : 32); ++k) r += scratch[k];
  return r;
}

// L sums at once (one per lane of a packed group), valid in thread 0, in a
// fixed order: four barriers for any L instead of three per sum.  `scratch`
// holds at least L doubles per thread and max(L*32, ...) doubles.
template <int L>
__device__ __forceinline__ void fuse_block_sum_lanes(const double (&v)[L], double* scratch, double (&out)[L]) {
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  if ((nt & 31) == 0) {   // whole warps: shuffle trees, then the warp sums in warp order
    double w[L];
#pragma unroll
    for (int l = 0; l < L; ++l) w[l] = warp_tree_sum(v[l]);
    __syncthreads();   // the caller's last reads of scratch are done
    if ((t & 31) == 0)
#pragma unroll
      for (int l = 0; l < L; ++l) scratch[(t >> 5) * L + l] = w[l];
    __syncthreads();
    if (t == 0)
#pragma unroll
      for (int l = 0; l < L; ++l) {
        double r = 0.0;
        for (int k = 0; k < (nt >> 5); ++k) r += scratch[k * L + l];
        out[l] = r;
      }
    return;
  }
  __syncthreads();   // the caller's last reads of scratch are done
#pragma unroll
  for (int l = 0; l < L; ++l) scratch[l * nt + t] = v[l];
  __syncthreads();
  if (nt < 32) {   // tiny blocks: thread 0 adds everything
    if (t == 0)
#pragma unroll
      for (int l = 0; l < L; ++l) {
        double r = 0.0;
        for (int k = 0; k < nt; ++k) r += scratch[l * nt + k];
        out[l] = r;
      }
    return;
  }
  // stage 1: strided partial sums, (lane, w) = (idx / 32, idx % 32), idx < 32 L
  double part[L];
#pragma unroll
  for (int it = 0; it < L; ++it) {
    const int idx = t + it * nt;
    double r = 0.0;
    if (idx < L * 32) {
      const int lane = idx >> 5, w = idx & 31;
      for (int k = w; k < nt; k += 32) r += scratch[lane * nt + k];
    }
    part[it] = r;
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < L; ++it) {
    const int idx = t + it * nt;
    if (idx < L * 32) scratch[idx] = part[it];
  }
  __syncthreads();
  if (t == 0) {
#pragma unroll
    for (int l = 0; l < L; ++l) {
      double r = 0.0;
      for (int w = 0; w < 32; ++w) r += scratch[l * 32 + w];
      out[l] = r;
    }
  }
}

// block partial of p.Ap (plain store; the next kernel reads it)
__device__ __forceinline__ void fuse_pap(double v, const CgFuse& F, double* scratch) {
  const double bs = fuse_block_sum(v, scratch);
  if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) F.partials[blockIdx.x] = bs;
}

}  // namespace bp
