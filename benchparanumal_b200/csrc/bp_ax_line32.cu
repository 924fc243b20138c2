// FP32 instantiation of the line-per-thread BP5/BP6 element operator (mixed-precision CG).
#define BP_LINE_REAL float
#define BP_LINE_UNROLL_MAX 16
#include "bp_ax_line.cuh"
#include "bp_cg_persist.cuh"

namespace bp {

namespace {
// the line body as the operator phase of the persistent CG step
template <int NQ, bool AFFINE, class T>
struct LineStepOp {
  static constexpr int THREADS = LineShape<NQ, T>::THREADS;
  static constexpr int MINB = LineMinBlocks<NQ, T>::V;
  static __device__ __forceinline__ void run(int blk, const GrpStepArgs& a, unsigned char* smem) {
    ax_line_body<NQ, AFFINE, T>(blk, a.nblk_op, a.Nelements, 1, a.elementList, a.G2L, a.wJ, a.ggeo, a.gllw,
                                a.lambda, reinterpret_cast<const T*>(a.p), reinterpret_cast<T*>(a.AqL), a.parts,
                                smem);
  }
};

template <int NQ, int PK>
int launch_step_line_nq(const bp_ax_desc_t& d, GrpStepArgs a, int grid_cap, cudaStream_t s) {
  using T = Pack<float, PK>;
  using Sh = LineShape<NQ, T>;
  LineReal* tab = line_table_address();
  if (!tab) return fail(BP_ERROR_CUDA, "persistent CG step: constant table address lookup failed");
  BP_TRY(const_slot_copy(tab + Sh::SLOT, a.D, sizeof(float) * NQ * NQ, s));
  if (d.affine)
    BP_TRY(const_slot_copy(tab + Sh::SLOT + NQ * NQ, a.gllw, sizeof(float) * NQ, s));
  a.nblk_op = (a.Nelements + Sh::EPB - 1) / Sh::EPB;
  const dim3 block(NQ, NQ, Sh::EPB);
  if (d.affine) return launch_grp_step_kernel<PK, LineStepOp<NQ, true, T>>(a, block, Sh::smem(), grid_cap, s);
  return launch_grp_step_kernel<PK, LineStepOp<NQ, false, T>>(a, block, Sh::smem(), grid_cap, s);
}
}  // namespace

// One CG step of a packed group as one cooperative kernel with the line form
// of the operator (bp_cg_persist.cuh); pk = 4, Nq <= 12
int launch_grp_step_line(int pk, const bp_ax_desc_t& d, const GrpStepArgs& a, int grid_cap, cudaStream_t s) {
  if (pk != 4 || d.Nfields != 1 || d.dim == 2) return 1;
  switch (d.N + 1) {
#define BP_STEP_LINE(nq) \
  case nq:               \
    return launch_step_line_nq<nq, 4>(d, a, grid_cap, s);
    BP_STEP_LINE(2) BP_STEP_LINE(3) BP_STEP_LINE(4) BP_STEP_LINE(5) BP_STEP_LINE(6) BP_STEP_LINE(7)
    BP_STEP_LINE(8) BP_STEP_LINE(9) BP_STEP_LINE(10) BP_STEP_LINE(11) BP_STEP_LINE(12)
#undef BP_STEP_LINE
    default:
      return 1;
  }
}

int launch_ax_line(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                   const float* wJ, const float* ggeo, const float* gllw, const float* D, float lambda,
                   const float* q, float* Aq, const int* skip, cudaStream_t s, const CgFuse* fuse, int* nblocks) {
  return launch_ax_line_impl(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, s, fuse,
                             nblocks);
}

int launch_ax_line_packed(int pk, const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList,
                          const int32_t* G2L, const float* wJ, const float* ggeo, const float* gllw, const float* D,
                          float lambda, const float* q, float* Aq, const int* skip, const CgFuse* fuse,
                          cudaStream_t s, int* nblocks) {
  if (pk == 2)
    return launch_ax_line_pk<2>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, s, fuse,
                                nblocks);
  if (pk == 4)
    return launch_ax_line_pk<4>(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, s, fuse,
                                nblocks);
  return fail(BP_ERROR_ARG, "packed element operator: 2 or 4 lanes");
}

}  // namespace bp
