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

#include <algorithm>
#include <atomic>
#include <string>

#include "bp_internal.hpp"

namespace bp {
namespace {

// Element-local results between the element operator and the gather:
// BP_NOALLOC_MAX_LOCAL doubles = 8 MiB, resident on every GPU that loads the
// library until the process exits.  Each call clears the first Nlocal entries
// before the element operator writes the listed elements, so a partial
// element list gathers zeros, not an earlier call's values, for the elements
// it leaves out.
__device__ __align__(256) double g_noalloc_scratch[BP_NOALLOC_MAX_LOCAL];

// Index check of one call: 0 when every index is in range, else the kind of
// the first violation recorded (1 element id, 2 row starts, 3 column index).
__device__ int g_noalloc_bad;

// The two arrays' device addresses, per device.  In host code the symbols
// name host-side stand-ins, not device addresses: a kernel given one would
// fault or, where the GPU can reach host memory, use the wrong memory.
std::atomic<double*> g_scratch_addr[kMaxDevices] = {};
std::atomic<int*> g_bad_addr[kMaxDevices] = {};

// Looks the addresses up on the first call on each device, with that device
// current (concurrent first calls store the same values).
int noalloc_addresses(double** scratch, int** bad) {
  int dev = 0;
  BP_TRY(current_device(&dev));
  double* s = g_scratch_addr[dev].load(std::memory_order_acquire);
  int* b = g_bad_addr[dev].load(std::memory_order_acquire);
  if (!s || !b) {
    BP_CUDA_TRY(cudaGetSymbolAddress((void**)&s, g_noalloc_scratch));
    BP_CUDA_TRY(cudaGetSymbolAddress((void**)&b, g_noalloc_bad));
    g_bad_addr[dev].store(b, std::memory_order_release);
    g_scratch_addr[dev].store(s, std::memory_order_release);
  }
  *scratch = s;
  *bad = b;
  return BP_SUCCESS;
}

// Every element id below Nelem_total, row starts that begin at 0 and never
// decrease, and every column index (the rowStarts[Ngather] entries of colIds)
// below Nlocal.  Grid-stride; records the kind of a violation in g_noalloc_bad.
__global__ void noalloc_check_kernel(int32_t Nelements, const int32_t* __restrict__ elementList, int32_t Nelem_total,
                                     int32_t Ngather, const int32_t* __restrict__ rowStarts,
                                     const int32_t* __restrict__ colIds, int32_t Nlocal) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t i = t0; i < Nelements; i += stride) {
    const int32_t e = elementList[i];
    if (e < 0 || e >= Nelem_total) atomicCAS(&g_noalloc_bad, 0, 1);
  }
  if (t0 == 0 && rowStarts[0] != 0) atomicCAS(&g_noalloc_bad, 0, 2);
  for (int64_t r = t0; r < Ngather; r += stride)
    if (rowStarts[r + 1] < rowStarts[r]) atomicCAS(&g_noalloc_bad, 0, 2);
  const int32_t nnz = rowStarts[Ngather];
  for (int64_t c = t0; c < nnz; c += stride) {
    const int32_t l = colIds[c];
    if (l < 0 || l >= Nlocal) atomicCAS(&g_noalloc_bad, 0, 3);
  }
}

}  // namespace
}  // namespace bp

using namespace bp;

extern "C" int bp_operator_hex3d_noalloc(const bp_ax_desc_t* desc, int32_t Nelements, const int32_t* elementList,
                                         const int32_t* GlobalToLocal, const double* wJ, const double* ggeo,
                                         const double* gllw, const double* D, double lambda, int32_t Nlocal,
                                         int32_t Ngather, const int32_t* rowStarts, const int32_t* colIds,
                                         const double* q, double* Aq, bp_stream_t stream) {
  if (!desc) return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: null descriptor");
  if (desc->N < 1 || desc->N > 15) return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: degree N must be in 1..15");
  if (desc->Nfields != 1 && desc->Nfields != 3)
    return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: Nfields must be 1 or 3");
  if ((desc->bp == 6) != (desc->Nfields == 3) || (desc->bp != 5 && desc->bp != 6))
    return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: bp must be 5 (one field) or 6 (three fields)");
  if (Nelements < 0 || Ngather < 0 || Nlocal < 0)
    return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: negative size");
  const int64_t Nq = desc->N + 1;
  const int64_t Nel = Nq * Nq * Nq * desc->Nfields;   // local nodes per element
  if (Nlocal > BP_NOALLOC_MAX_LOCAL)
    return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: Nlocal = " + std::to_string(Nlocal) +
                                  " exceeds the scratch maximum of " + std::to_string(BP_NOALLOC_MAX_LOCAL) +
                                  " local nodes; use bp_solver_operator for larger meshes");
  if (Nlocal % Nel != 0)
    return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: Nlocal = " + std::to_string(Nlocal) +
                                  " is not a whole number of elements of Np*Nfields = " + std::to_string(Nel) +
                                  " local nodes");
  if ((int64_t)Nelements * Nel > Nlocal)
    return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: Nelements*Np*Nfields exceeds Nlocal");
  if (Ngather == 0) return BP_SUCCESS;
  if (!rowStarts || !colIds || !Aq || (Nelements > 0 && (!elementList || !GlobalToLocal || !wJ || !ggeo || !D ||
                                                         !q || (desc->affine && !gllw))))
    return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: null array");

  double* scratch = nullptr;
  int* bad = nullptr;
  BP_TRY(noalloc_addresses(&scratch, &bad));
  const cudaStream_t s = to_stream(stream);

  // Check every index the launches below follow before they run, so an index
  // outside the scratch array is an error here and never a device access.
  // The check's result comes back through a 4-byte copy to this stack
  // variable, which waits for the stream.
  BP_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), s));
  const int64_t work = std::max<int64_t>(std::max<int64_t>(Nelements, Ngather), 1);
  const int grid = (int)std::min<int64_t>((work + 255) / 256, 4 * (int64_t)sm_count());
  noalloc_check_kernel<<<grid, 256, 0, s>>>(Nelements, elementList, (int32_t)(Nlocal / Nel), Ngather, rowStarts,
                                            colIds, Nlocal);
  BP_CUDA_TRY(cudaGetLastError());
  int h_bad = 0;
  BP_CUDA_TRY(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  BP_CUDA_TRY(cudaStreamSynchronize(s));
  if (h_bad == 1)
    return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: an elementList entry is outside [0, Nlocal/(Np*Nfields))");
  if (h_bad == 2) return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: rowStarts do not start at 0 and rise");
  if (h_bad == 3) return fail(BP_ERROR_ARG, "bp_operator_hex3d_noalloc: a colIds entry is outside [0, Nlocal)");

  if (Nlocal > 0) BP_CUDA_TRY(cudaMemsetAsync(scratch, 0, sizeof(double) * (size_t)Nlocal, s));
  if (Nelements > 0)
    BP_TRY(launch_ax(*desc, Nelements, elementList, GlobalToLocal, wJ, ggeo, gllw, D, lambda, q, scratch, s));
  return launch_gather(Ngather, rowStarts, colIds, scratch, Aq, s);
}
