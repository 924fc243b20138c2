// Benchmark problem object: operator, forcing, Jacobi diagonal and the CG
// solve (reference: BP/BP5/src/bp5{Setup,Operator,Run}.cpp,
// libs/core/linearSolverCG.cpp:62-156).
//
// CG runs with every scalar on the device.  One iteration is four kernels:
//   cg_direction_kernel     x += alpha_{k-1} p_{k-1} (deferred),  p = z + beta p
//   element operator        AqL = A_e p, and block partials of p.Ap = sum_e p_e.(A_e p_e)
//   cg_alpha_kernel         p.Ap from the partials, alpha = rho / p.Ap
//   cg_gather_update_kernel r -= alpha Gather(AqL), r.r (and r.z), stop test
// so A p is never stored as a gathered vector.  The reductions finish in the
// last block to arrive, so there is no host round trip per iteration.  Iterations are captured once into a CUDA graph
// (kChunk iterations per graph) and replayed; a finished solve turns the
// remaining kernels into immediate returns through a device flag.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "bp_cg_device.cuh"
#include "bp_internal.hpp"

namespace bp {

constexpr int kThreads = 256;
constexpr int kChunk = 20;   // iterations per captured graph (divides the usual 100 and 1000)

template <int NS>
__device__ __forceinline__ bool grid_sum_cg(const double (&v)[NS], double* partials, unsigned int* counter,
                                            double (&tot)[NS]);

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

// Deterministic grid sum: block partials in a fixed slot, the last block to
// arrive adds them in slot order.  Returns true in the last block (thread 0
// holds tot).
template <int NS>
__device__ __forceinline__ bool grid_sum_cg(const double (&v)[NS], double* partials, unsigned int* counter,
                                            double (&tot)[NS]) {
  __shared__ double s_tmp[kThreads / 32];
  __shared__ bool s_last;
  for (int c = 0; c < NS; ++c) {
    const double b = block_sum_cg(v[c], s_tmp);
    if (threadIdx.x == 0) partials[c * gridDim.x + blockIdx.x] = b;
  }
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  for (int c = 0; c < NS; ++c) {
    double acc = 0.0;
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += kThreads)
      acc += *((volatile double*)&partials[c * gridDim.x + b]);
    tot[c] = block_sum_cg(acc, s_tmp);
  }
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
    sc->done = (rdotr <= sc->tol2 || maxit <= 0) ? 1 : 0;
  }
}

// x += alpha p (the previous iteration's update, deferred), p = z + beta p
__global__ void __launch_bounds__(kThreads)
cg_direction_kernel(int32_t N, double* __restrict__ x, double* __restrict__ p, const double* __restrict__ r,
                    const double* __restrict__ invD, const CgScalars* __restrict__ sc) {
  if (sc->done) return;
  const int iter = sc->iter;
  const double alpha = sc->alpha;
  double beta = 0.0;
  if (iter > 0) beta = sc->precon ? sc->rz / sc->rz_prev : sc->rdotr / sc->rdotr_prev;
  const bool precon = sc->precon != 0;
  for (int32_t n = blockIdx.x * kThreads + threadIdx.x; n < N; n += kThreads * gridDim.x) {
    const double pn = p[n];
    if (iter > 0) x[n] = alpha * pn + 1.0 * x[n];
    const double z = precon ? invD[n] * r[n] : 1.0 * r[n];
    p[n] = (iter > 0) ? z + beta * pn : z;   // p is not read at iteration 0
  }
}

// p.Ap from the element operator's block partials (index order), then alpha
constexpr int kAlphaThreads = 1024;
__global__ void __launch_bounds__(kAlphaThreads)
cg_alpha_kernel(int nparts, const double* __restrict__ parts, CgScalars* sc, double* hist_alpha) {
  if (sc->done) return;
  __shared__ double s_w[kAlphaThreads / 32];
  double acc = 0.0;
  for (int k = threadIdx.x; k < nparts; k += kAlphaThreads) acc += parts[k];
  acc = warp_sum_cg(acc);
  if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double pAp = 0.0;
    for (int w = 0; w < kAlphaThreads / 32; ++w) pAp += s_w[w];
    const double rho = sc->precon ? sc->rz : sc->rdotr;
    const double alpha = rho / pAp;
    sc->pAp = pAp;
    if (!(pAp > 0.0) || !isfinite(alpha)) {
      sc->breakdown = 1;
      sc->done = 1;
    } else {
      sc->alpha = alpha;
      if (hist_alpha) hist_alpha[sc->iter] = alpha;
    }
  }
}

// r -= alpha Gather(AqL); r.r (and r.z); stop test.  alpha comes from the
// element operator's p.Ap epilogue.
// One row per thread: r and invD of the row are requested first, then the
// row's local values in column order (the reference's order, so the sums match
// its gather bit for bit).
__global__ void __launch_bounds__(kThreads)
cg_gather_update_kernel(int32_t Nrows, const int32_t* __restrict__ rowStarts, const int32_t* __restrict__ colIds,
                        const double* __restrict__ AqL, double* __restrict__ r, const double* __restrict__ invD,
                        CgScalars* sc, double* hist_rnorm, double* partials, unsigned int* counter) {
  if (sc->done) return;
  const double alpha = sc->alpha;
  const bool precon = sc->precon != 0;
  double acc[2] = {0.0, 0.0};
  for (int32_t row = blockIdx.x * kThreads + threadIdx.x; row < Nrows; row += kThreads * gridDim.x) {
    const double rold = r[row];
    const double dinv = precon ? __ldg(invD + row) : 0.0;
    const int32_t start = __ldg(rowStarts + row), end = __ldg(rowStarts + row + 1);
    double s = 0.0;
    for (int32_t c = start; c < end; ++c) s += __ldg(AqL + __ldg(colIds + c));
    const double rn = rold - alpha * s;
    r[row] = rn;
    acc[0] += rn * rn;
    if (precon) acc[1] += rn * dinv * rn;
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
    if (!isfinite(tot[0])) {
      sc->breakdown = 1;
      sc->done = 1;
    } else if (tot[0] <= sc->tol2 || sc->iter >= sc->maxit) {
      sc->done = 1;
    }
  }
}

// apply the last completed iteration's x update
__global__ void __launch_bounds__(kThreads)
cg_final_kernel(int32_t N, double* __restrict__ x, const double* __restrict__ p, const CgScalars* __restrict__ sc) {
  if (sc->iter == 0 || sc->breakdown) return;
  const double alpha = sc->alpha;
  for (int32_t n = blockIdx.x * kThreads + threadIdx.x; n < N; n += kThreads * gridDim.x)
    x[n] = alpha * p[n] + 1.0 * x[n];
}

static int vec_grid(int32_t N) {
  int g = (N + kThreads - 1) / kThreads;
  const int cap = reduction_blocks();
  if (g > cap) g = cap;
  return g < 1 ? 1 : g;
}

}  // namespace bp

using namespace bp;

struct bp_solver_s {
  bp_mesh_s* mesh = nullptr;
  int bp = 5;
  double lambda = 1.0;
  int precon = 0;
  int32_t N = 0;               // Ngather
  bp_ax_desc_t ax{};
  DeviceArray<double> AqL, p, Ap, invD, xw, rw, partials, hist, fuse_partials;
  DeviceArray<unsigned int> counter;
  DeviceArray<CgScalars> sc;
  int hist_len = 0;
  // graph of kChunk iterations, keyed by the vectors it was captured for
  cudaGraphExec_t graph = nullptr;
  const double* g_x = nullptr;
  const double* g_r = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  ~bp_solver_s() {
    if (graph) cudaGraphExecDestroy(graph);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

namespace bp {

static int operator_apply(bp_solver_s* S, const double* q, double* Aq, const int* skip, cudaStream_t s) {
  bp_mesh_s* m = S->mesh;
  BP_TRY(launch_ax_skip(S->ax, m->E, m->elementList.ptr, m->G2L.ptr, m->wJ.ptr, m->ggeo.ptr, m->gllw.ptr,
                        m->D.ptr, S->lambda, q, S->AqL.ptr, skip, s));
  return launch_gather(m->Ngather, m->rowStarts.ptr, m->colIds.ptr, S->AqL.ptr, Aq, s);
}

// enqueue one CG iteration
static int enqueue_iteration(bp_solver_s* S, double* x, double* r, cudaStream_t s) {
  bp_mesh_s* m = S->mesh;
  const int32_t N = S->N;
  const int g = vec_grid(N);
  double* hist_alpha = S->hist.ptr;
  double* hist_rnorm = S->hist.ptr ? S->hist.ptr + S->hist_len : nullptr;
  cg_direction_kernel<<<g, kThreads, 0, s>>>(N, x, S->p.ptr, r, S->invD.ptr, S->sc.ptr);
  BP_CUDA_TRY(cudaGetLastError());
  const CgFuse fuse{S->fuse_partials.ptr};
  int nparts = 0;
  BP_TRY(launch_ax_skip(S->ax, m->E, m->elementList.ptr, m->G2L.ptr, m->wJ.ptr, m->ggeo.ptr, m->gllw.ptr, m->D.ptr,
                        S->lambda, S->p.ptr, S->AqL.ptr, &S->sc.ptr->done, s, &fuse, &nparts));
  cg_alpha_kernel<<<1, kAlphaThreads, 0, s>>>(nparts, S->fuse_partials.ptr, S->sc.ptr, hist_alpha);
  BP_CUDA_TRY(cudaGetLastError());
  cg_gather_update_kernel<<<g, kThreads, 0, s>>>(N, m->rowStarts.ptr, m->colIds.ptr, S->AqL.ptr, r, S->invD.ptr,
                                                 S->sc.ptr, hist_rnorm, S->partials.ptr, S->counter.ptr);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

static int ensure_graph(bp_solver_s* S, double* x, double* r, cudaStream_t s) {
  if (S->graph && S->g_x == x && S->g_r == r) return BP_SUCCESS;
  if (S->graph) {
    cudaGraphExecDestroy(S->graph);
    S->graph = nullptr;
  }
  cudaGraph_t g;
  BP_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int rc = BP_SUCCESS;
  for (int k = 0; k < kChunk && rc == BP_SUCCESS; ++k) rc = enqueue_iteration(S, x, r, s);
  cudaError_t ce = cudaStreamEndCapture(s, &g);
  if (rc != BP_SUCCESS) return rc;
  BP_CUDA_TRY(ce);
  ce = cudaGraphInstantiate(&S->graph, g, 0);
  cudaGraphDestroy(g);
  BP_CUDA_TRY(ce);
  S->g_x = x;
  S->g_r = r;
  return BP_SUCCESS;
}

static int ensure_hist(bp_solver_s* S, int maxit) {
  if (maxit <= S->hist_len) return BP_SUCCESS;
  // history buffers move: the captured graph refers to them
  if (S->graph) {
    cudaGraphExecDestroy(S->graph);
    S->graph = nullptr;
  }
  const int len = std::max(maxit, 128);
  BP_TRY(S->hist.alloc((size_t)2 * len));
  S->hist_len = len;
  return BP_SUCCESS;
}

static int solve_device(bp_solver_s* S, double* x, double* r, double tol, int maxit, double* hist_rnorm,
                        double* hist_alpha, bp_solve_stats_t* stats, cudaStream_t s, bool record_events) {
  const int32_t N = S->N;
  BP_TRY(ensure_hist(S, maxit));
  BP_TRY(ensure_graph(S, x, r, s));
  if (record_events) BP_CUDA_TRY(cudaEventRecord(S->ev0, s));
  // r = b - A x
  BP_TRY(operator_apply(S, x, S->Ap.ptr, nullptr, s));
  cg_init_kernel<<<vec_grid(N), kThreads, 0, s>>>(N, S->Ap.ptr, r, S->invD.ptr, S->sc.ptr, tol, maxit, S->precon,
                                                  S->partials.ptr, S->counter.ptr);
  BP_CUDA_TRY(cudaGetLastError());
  const int nchunks = (maxit + kChunk - 1) / kChunk;
  CgScalars h{};
  for (int c = 0; c < nchunks; ++c) {
    BP_CUDA_TRY(cudaGraphLaunch(S->graph, s));
    if (tol > 0.0 && c + 1 < nchunks) {
      BP_CUDA_TRY(cudaMemcpyAsync(&h, S->sc.ptr, sizeof(CgScalars), cudaMemcpyDeviceToHost, s));
      BP_CUDA_TRY(cudaStreamSynchronize(s));
      if (h.done) break;
    }
  }
  cg_final_kernel<<<vec_grid(N), kThreads, 0, s>>>(N, x, S->p.ptr, S->sc.ptr);
  BP_CUDA_TRY(cudaGetLastError());
  if (record_events) BP_CUDA_TRY(cudaEventRecord(S->ev1, s));
  BP_CUDA_TRY(cudaMemcpyAsync(&h, S->sc.ptr, sizeof(CgScalars), cudaMemcpyDeviceToHost, s));
  BP_CUDA_TRY(cudaStreamSynchronize(s));
  const int it = h.iter;
  if (hist_alpha && it > 0)
    BP_CUDA_TRY(cudaMemcpy(hist_alpha, S->hist.ptr, sizeof(double) * it, cudaMemcpyDeviceToHost));
  if (hist_rnorm && it > 0)
    BP_CUDA_TRY(cudaMemcpy(hist_rnorm, S->hist.ptr + S->hist_len, sizeof(double) * it, cudaMemcpyDeviceToHost));
  if (stats) {
    stats->iterations = it;
    stats->rdotr0 = h.rdotr0;
    stats->rdotr = h.rdotr;
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

}  // namespace bp

extern "C" {

int bp_solver_create(bp_mesh_t mesh, const bp_solver_desc_t* d, bp_solver_t* out) {
  if (!mesh || !d || !out) return fail(BP_ERROR_ARG, "bp_solver_create: null pointer");
  *out = nullptr;
  if (d->bp != 5 && d->bp != 6) return fail(BP_ERROR_ARG, "bp_solver_create: only BP5 and BP6 are available");
  if ((d->bp == 6) != (mesh->Nfields == 3))
    return fail(BP_ERROR_ARG, "bp_solver_create: BP6 needs a 3-field mesh, BP5 a 1-field mesh");
  if (d->precon != BP_PRECON_NONE && d->precon != BP_PRECON_JACOBI)
    return fail(BP_ERROR_ARG, "bp_solver_create: unknown preconditioner");
  cudaStream_t s = default_stream();
  bp_solver_s* S = new bp_solver_s();
  S->mesh = mesh;
  S->bp = d->bp;
  S->lambda = d->lambda;
  S->precon = d->precon;
  S->N = mesh->Ngather;
  S->ax.bp = d->bp;
  S->ax.N = mesh->N;
  S->ax.affine = mesh->affine;
  S->ax.Nfields = mesh->Nfields;
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
    cudaError_t ce = cudaMemsetAsync(S->p.ptr, 0, sizeof(double) * S->N, s);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(S->counter.ptr, 0, sizeof(unsigned int) * 4, s);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(S->sc.ptr, 0, sizeof(CgScalars), s);
    if (ce == cudaSuccess) ce = cudaEventCreate(&S->ev0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&S->ev1);
    if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_solver_create", __FILE__, __LINE__); break; }
    if (S->precon == BP_PRECON_JACOBI) {
      if ((rc = S->invD.alloc(S->N))) break;
      if ((rc = bp_solver_diagonal(S, S->invD.ptr))) break;
      if ((rc = launch_reciprocal(S->N, S->invD.ptr, s))) break;
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
    BP_TRY(launch_rhs_analytic(m->N, m->affine, m->Nfields, m->E, m->EX.ptr, m->EY.ptr, m->EZ.ptr, m->gllz.ptr,
                               m->gllw.ptr, m->wJ.ptr, S->lambda, S->AqL.ptr, s));
  } else if (mode == BP_RHS_RANDOM) {
    DeviceArray<double> ftmp;
    double* f = f_out;
    if (!f) {
      BP_TRY(ftmp.alloc(S->N));
      f = ftmp.ptr;
    }
    BP_TRY(launch_rhs_random(S->N, seed, f, s));
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
  BP_TRY(launch_diag_local(m->N, m->affine, m->Nfields, m->E, m->ggeo.ptr, m->wJ.ptr, m->gllw.ptr, m->D.ptr,
                           S->lambda, S->AqL.ptr, s));
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
  BP_CUDA_TRY(cudaEventRecord(S->ev0, s));
  BP_CUDA_TRY(cudaMemcpyAsync(S->rw.ptr, b_host, bytes, cudaMemcpyHostToDevice, s));
  BP_CUDA_TRY(cudaMemsetAsync(S->xw.ptr, 0, bytes, s));
  cudaEvent_t e0 = S->ev0;
  // inner solve without its own events, then the copy back
  BP_TRY(solve_device(S, S->xw.ptr, S->rw.ptr, tol, maxit, nullptr, nullptr, stats, s, false));
  BP_CUDA_TRY(cudaMemcpyAsync(x_host, S->xw.ptr, bytes, cudaMemcpyDeviceToHost, s));
  BP_CUDA_TRY(cudaEventRecord(S->ev1, s));
  BP_CUDA_TRY(cudaEventSynchronize(S->ev1));
  if (stats) {
    float ms = 0.f;
    BP_CUDA_TRY(cudaEventElapsedTime(&ms, e0, S->ev1));
    stats->elapsed_ms = ms;
  }
  return BP_SUCCESS;
}

}  // extern "C"
