// FP32 instantiation of the line-per-thread BP5/BP6 element operator (mixed-precision CG).
#define BP_LINE_REAL float
#define BP_LINE_UNROLL_MAX 16
#include "bp_ax_line.cuh"

namespace bp {

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
