// FP32 instantiation of the over-integrated BP1-BP4 operators (mixed-precision CG).
#define BP_CUB_REAL float
#define BP_CUB_OUTER _Pragma("unroll")
#include "bp_ax_cub.cuh"

namespace bp {

int launch_ax_cub(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const CubOperands<float>& ops, float lambda, const float* q, float* Aq, const int* skip,
                  cudaStream_t s, const CgFuse* fuse, int* nblocks) {
  return launch_ax_cub_impl(d, Nelements, elementList, G2L, ops, lambda, q, Aq, skip, s, fuse, nblocks);
}

}  // namespace bp
