// FP64 instantiation of the over-integrated BP1-BP4 operators, and the
// element-local diagonal of those operators (the Jacobi preconditioner).
#define BP_CUB_REAL double
#include "bp_ax_cub.cuh"

namespace bp {

int launch_ax_cub(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const CubOperands<double>& ops, double lambda, const double* q, double* Aq, const int* skip,
                  cudaStream_t s, const CgFuse* fuse, int* nblocks) {
  return launch_ax_cub_impl(d, Nelements, elementList, G2L, ops, lambda, q, Aq, skip, s, fuse, nblocks);
}

// ---------------------------------------------------------------------------
// Diagonal of the curved-mesh BP1/BP3 element matrices.  The element matrix
// is B^T W B with B built from 1D columns, so entry (a,b,c) of the diagonal is
//   sum over grid points (i,j,k) of W(i,j,k) X(i,a) Y(j,b) Z(k,c)
// for each weighted term: the mass (lambda cubwJ, or cubwJ for BP1) with
// X=Y=Z=T^2, G00 with X=DV^2, the cross term 2 G01 with X=T DV, Y=T DV, ...
// (T the interpolation, DV = cubD T).  Each term is summed by
// sum-factorisation: i, then j, then k, one element per block.
// ---------------------------------------------------------------------------
template <int NQ>
__global__ void __launch_bounds__((NQ + 1) * (NQ + 1))
diag_cub_kernel(int Nfields, int stiff, const double* __restrict__ wJ, const double* __restrict__ ggeo,
                const double* __restrict__ Tg, const double* __restrict__ DVg, double lambda,
                double* __restrict__ dL) {
  constexpr int G = NQ + 1, G2 = G * G, GP = G * G * G, NQ2 = NQ * NQ, NP = NQ * NQ * NQ;
  extern __shared__ double smem[];
  double* s_W = smem;                   // [G][G][G]
  double* s_T1 = s_W + GP;              // [G k][G j][NQ a]
  double* s_T2 = s_T1 + G2 * NQ;        // [G k][NQ b][NQ a]
  double* s_A = s_T2 + G * NQ2;         // [3][G][NQ]: T^2, T DV, DV^2
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + G * ty;
  const int e = blockIdx.x;
  for (int t = tid; t < G * NQ; t += G2) {
    const double T = Tg[t], DV = DVg[t];
    s_A[t] = T * T;
    s_A[G * NQ + t] = T * DV;
    s_A[2 * G * NQ + t] = DV * DV;
  }
  // terms: mass, G00, G11, G22, G01, G02, G12 -> (table x, y, z, factor slot, coefficient)
  const int tabx[7] = {0, 2, 0, 0, 1, 1, 0}, taby[7] = {0, 0, 2, 0, 1, 0, 1}, tabz[7] = {0, 0, 0, 2, 0, 1, 1};
  const int slot[7] = {-1, 0, 3, 5, 1, 2, 4};
  const double coef[7] = {stiff ? lambda : 1.0, 1.0, 1.0, 1.0, 2.0, 2.0, 2.0};
  double d[NQ];
#pragma unroll
  for (int c = 0; c < NQ; ++c) d[c] = 0.0;
  const int nterms = stiff ? 7 : 1;
  for (int term = 0; term < nterms; ++term) {
    __syncthreads();   // previous term's reads of s_W / s_T2 done; s_A ready
    const size_t base = (size_t)e * GP;
    for (int n = tid; n < GP; n += G2)
      s_W[n] = coef[term] * (slot[term] < 0 ? wJ[base + n] : ggeo[6 * (base + n) + slot[term]]);
    __syncthreads();
    const double* X = s_A + tabx[term] * G * NQ;
    const double* Y = s_A + taby[term] * G * NQ;
    const double* Z = s_A + tabz[term] * G * NQ;
    {   // T1[k][j][a] = sum_i W[k][j][i] X[i][a]: thread (j, k)
      const int jj = tx, k = ty;
      for (int a = 0; a < NQ; ++a) {
        double acc = 0.0;
        for (int i = 0; i < G; ++i) acc += s_W[k * G2 + jj * G + i] * X[i * NQ + a];
        s_T1[(k * G + jj) * NQ + a] = acc;
      }
    }
    __syncthreads();
    if (tx < NQ) {   // T2[k][b][a] = sum_j T1[k][j][a] Y[j][b]: thread (a, k)
      const int a = tx, k = ty;
      for (int b = 0; b < NQ; ++b) {
        double acc = 0.0;
        for (int jj = 0; jj < G; ++jj) acc += s_T1[(k * G + jj) * NQ + a] * Y[jj * NQ + b];
        s_T2[(k * NQ + b) * NQ + a] = acc;
      }
    }
    __syncthreads();
    if (tx < NQ && ty < NQ) {   // d[c] += sum_k T2[k][b][a] Z[k][c]: thread (a, b)
      const int a = tx, b = ty;
#pragma unroll
      for (int c = 0; c < NQ; ++c) {
        double acc = 0.0;
        for (int k = 0; k < G; ++k) acc += s_T2[(k * NQ + b) * NQ + a] * Z[k * NQ + c];
        d[c] += acc;
      }
    }
  }
  if (tx < NQ && ty < NQ) {
    for (int f = 0; f < Nfields; ++f)
#pragma unroll
      for (int c = 0; c < NQ; ++c) dL[((size_t)e * Nfields + f) * NP + c * NQ2 + ty * NQ + tx] = d[c];
  }
}

// Affine BP1/BP3 diagonal: the factors are constant per element, so every
// term separates into products of 1D column sums.  BP1: wJ MM[a][a] MM[b][b]
// MM[c][c] (T = MM).  BP3 (T = invV, DV = cubD_modal invV): with
// S_p(a) = sum_i A_p(i,a) over the tables T^2, T DV, DV^2,
//   d = lambda wJ S0 S0 S0 + G00 S2 S0 S0 + G11 S0 S2 S0 + G22 S0 S0 S2
//     + 2 G01 S1 S1 S0 + 2 G02 S1 S0 S1 + 2 G12 S0 S1 S1.
__global__ void diag_cub_affine_kernel(int NQ, int E, int Nfields, int stiff, const double* __restrict__ wJ,
                                       const double* __restrict__ ggeo, const double* __restrict__ Tg,
                                       const double* __restrict__ DVg, double lambda, double* __restrict__ dL) {
  const int NP = NQ * NQ * NQ;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)E * NP) return;
  const int e = (int)(gid / NP), n = (int)(gid % NP);
  const int ab[3] = {n % NQ, (n / NQ) % NQ, n / (NQ * NQ)};
  double d;
  if (!stiff) {
    d = wJ[e] * Tg[ab[0] * NQ + ab[0]] * Tg[ab[1] * NQ + ab[1]] * Tg[ab[2] * NQ + ab[2]];
  } else {
    double S[3][3];   // S[dir][table]
    for (int r = 0; r < 3; ++r) {
      double s0 = 0, s1 = 0, s2 = 0;
      for (int i = 0; i < NQ; ++i) {
        const double T = Tg[i * NQ + ab[r]], DV = DVg[i * NQ + ab[r]];
        s0 += T * T; s1 += T * DV; s2 += DV * DV;
      }
      S[r][0] = s0; S[r][1] = s1; S[r][2] = s2;
    }
    const double* g = ggeo + 6 * (size_t)e;
    d = lambda * wJ[e] * S[0][0] * S[1][0] * S[2][0] + g[0] * S[0][2] * S[1][0] * S[2][0] +
        g[3] * S[0][0] * S[1][2] * S[2][0] + g[5] * S[0][0] * S[1][0] * S[2][2] +
        2 * g[1] * S[0][1] * S[1][1] * S[2][0] + 2 * g[2] * S[0][1] * S[1][0] * S[2][1] +
        2 * g[4] * S[0][0] * S[1][1] * S[2][1];
  }
  for (int f = 0; f < Nfields; ++f) dL[((size_t)e * Nfields + f) * NP + n] = d;
}

template <int NQ>
static int launch_diag_cub_nq(int32_t E, int Nfields, int stiff, const double* wJ, const double* ggeo,
                              const double* T, const double* DV, double lambda, double* dL, cudaStream_t s) {
  constexpr int G = NQ + 1;
  const size_t bytes = sizeof(double) * ((size_t)G * G * G + (size_t)G * G * NQ + (size_t)G * NQ * NQ + 3 * G * NQ);
  BP_CUDA_TRY(cudaFuncSetAttribute(diag_cub_kernel<NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  diag_cub_kernel<NQ><<<E, dim3(G, G), bytes, s>>>(Nfields, stiff, wJ, ggeo, T, DV, lambda, dL);
  BP_CUDA_TRY(cudaGetLastError());
  return BP_SUCCESS;
}

int launch_diag_cub(const bp_ax_desc_t& d, int32_t E, const double* wJ, const double* ggeo, const double* T,
                    const double* DV, double lambda, double* dL, cudaStream_t s) {
  if (d.bp < 1 || d.bp > 4) return fail(BP_ERROR_ARG, "over-integrated diagonal: bp must be 1..4");
  if (E == 0) return BP_SUCCESS;
  const int stiff = d.bp >= 3;
  if (d.affine) {
    const int NQ = d.N + 1;
    const long long tot = (long long)E * NQ * NQ * NQ;
    diag_cub_affine_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(NQ, E, d.Nfields, stiff, wJ, ggeo, T, DV,
                                                                         lambda, dL);
    BP_CUDA_TRY(cudaGetLastError());
    return BP_SUCCESS;
  }
  switch (d.N + 1) {
#define BP_DIAG_CASE(nq) \
  case nq:               \
    return launch_diag_cub_nq<nq>(E, d.Nfields, stiff, wJ, ggeo, T, DV, lambda, dL, s);
    BP_DIAG_CASE(2) BP_DIAG_CASE(3) BP_DIAG_CASE(4) BP_DIAG_CASE(5) BP_DIAG_CASE(6) BP_DIAG_CASE(7)
    BP_DIAG_CASE(8) BP_DIAG_CASE(9) BP_DIAG_CASE(10) BP_DIAG_CASE(11) BP_DIAG_CASE(12) BP_DIAG_CASE(13)
    BP_DIAG_CASE(14) BP_DIAG_CASE(15) BP_DIAG_CASE(16)
#undef BP_DIAG_CASE
    default:
      return fail(BP_ERROR_ARG, "over-integrated diagonal: degree N must be in 1..15");
  }
}

}  // namespace bp
