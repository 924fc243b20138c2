// bp_operator_hex3d_noalloc: the BP5/BP6 operator (element operator, then the
// ogs gather) for callers that may not allocate device memory.
//
// Some callers cannot call cudaMalloc: an application whose own pool allocator
// has taken the device memory budget and forbids allocations behind its back,
// or a pipeline that cannot accept the device-wide synchronisation that
// cudaMalloc/cudaFree imply while other streams are busy.  The allocating
// route (bp_solver_operator) keeps its element-local result in a buffer the
// solver allocates; this entry point keeps it in a fixed device array that
// is part of the library image instead, so a call allocates nothing.
#include <cuda_runtime.h>

#include <string>

#include "bp_internal.hpp"

namespace bp {
namespace {

constexpr int kMaxDevices = 64;

// Element-local results (E*Np*Nfields doubles) between the element operator
// and the gather.  BP_NOALLOC_MAX_LOCAL doubles = 8 MiB, resident on every GPU
// that loads the library until the process exits.  Every call writes all the
// entries it later reads, so nothing has to start at zero.
__device__ __align__(256) double g_noalloc_scratch[BP_NOALLOC_MAX_LOCAL];

// the scratch array's device address, per device (host code may not use the
// symbol itself as an address)
double* g_noalloc_addr[kMaxDevices] = {};

}  // namespace
}  // namespace bp

using namespace bp;

extern "C" int bp_operator_hex3d_noalloc(const bp_ax_desc_t* desc, int32_t Nelements, const int32_t* elementList,
                                         const int32_t* GlobalToLocal, const double* wJ, const double* ggeo,
                                         const double* gllw, const double* D, double lambda, int32_t Ngather,
                                         const int32_t* rowStarts, const int32_t* colIds, const double* q,
                                         double* Aq, bp_stream_t stream) {
  if (!desc) return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: null descriptor");
  if (desc->N < 1 || desc->N > 15) return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: degree N must be in 1..15");
  if (desc->Nfields != 1 && desc->Nfields != 3)
    return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: Nfields must be 1 or 3");
  if ((desc->bp == 6) != (desc->Nfields == 3) || (desc->bp != 5 && desc->bp != 6))
    return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: bp must be 5 (one field) or 6 (three fields)");
  if (Nelements < 0 || Ngather < 0) return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: negative size");
  const int64_t Nq = desc->N + 1;
  const int64_t NL = (int64_t)Nelements * Nq * Nq * Nq * desc->Nfields;
  if (NL > BP_NOALLOC_MAX_LOCAL)
    return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: Nelements*Np*Nfields = " + std::to_string(NL) +
                                  " exceeds the scratch maximum of " + std::to_string(BP_NOALLOC_MAX_LOCAL) +
                                  " local nodes; use bp_solver_operator for larger meshes");
  if (Nelements == 0 || Ngather == 0) return BP_SUCCESS;
  if (!elementList || !GlobalToLocal || !wJ || !ggeo || !D || !rowStarts || !colIds || !q || !Aq ||
      (desc->affine && !gllw))
    return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: null array");

  // set-up on the first call on each device, with that device current
  int dev = 0;
  BP_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: device ordinal too large");
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    BP_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev] = static_cast<double*>(p);
  }
  double* scratch = g_noalloc_addr[dev];
  const cudaStream_t s = to_stream(stream);
  BP_TRY(launch_ax(*desc, Nelements, elementList, GlobalToLocal, wJ, ggeo, gllw, D, lambda, q, scratch, s));
  return launch_gather(Ngather, rowStarts, colIds, scratch, Aq, s);
}
