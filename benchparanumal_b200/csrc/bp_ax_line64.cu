// FP64 instantiation of the line-per-thread BP5/BP6 element operator.
#define BP_LINE_REAL double
#include "bp_ax_line.cuh"

namespace bp {

int launch_ax_line(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                   const double* wJ, const double* ggeo, const double* gllw, const double* D, double lambda,
                   const double* q, double* Aq, const int* skip, cudaStream_t s, const CgFuse* fuse, int* nblocks) {
  return launch_ax_line_impl(d, Nelements, elementList, G2L, wJ, ggeo, gllw, D, lambda, q, Aq, skip, s, fuse,
                             nblocks);
}

}  // namespace bp
