// C ABI: platform (device, memory, streams, events), kernel entry points and
// mesh setup.  See include/bp_b200.h for the contract of each function.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "bp_cg_device.cuh"
#include "bp_internal.hpp"

namespace bp {

static thread_local std::string g_last_error;
static std::atomic<cudaStream_t> g_stream[kMaxDevices] = {};
static std::atomic<int> g_sm_count[kMaxDevices] = {};
static std::mutex g_device_state_lock;

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }
int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
int cuda_fail(cudaError_t err, const char* what, const char* file, int line) {
  char buf[512];
  std::snprintf(buf, sizeof(buf), "%s failed at %s:%d: %s", what, file, line, cudaGetErrorString(err));
  g_last_error = buf;
  return err == cudaErrorMemoryAllocation ? BP_ERROR_ALLOC : BP_ERROR_CUDA;
}

int current_device(int* dev) {
  BP_CUDA_TRY(cudaGetDevice(dev));
  if (*dev < 0 || *dev >= kMaxDevices)
    return fail(BP_ERROR_ARG, "device ordinal " + std::to_string(*dev) + " is beyond the library's " +
                                  std::to_string(kMaxDevices) + " per-device slots");
  return BP_SUCCESS;
}

void* DeviceSymbol::address() {
  int dev = 0;
  if (current_device(&dev) != BP_SUCCESS) return nullptr;
  void* p = addr_[dev].load(std::memory_order_acquire);
  if (p) return p;
  const cudaError_t e = cudaGetSymbolAddress(&p, symbol_);
  if (e != cudaSuccess) {
    cuda_fail(e, "cudaGetSymbolAddress", __FILE__, __LINE__);
    return nullptr;
  }
  addr_[dev].store(p, std::memory_order_release);   // concurrent first lookups store the same address
  return p;
}

cudaStream_t default_stream() {
  int dev = 0;
  if (current_device(&dev) != BP_SUCCESS) return nullptr;
  cudaStream_t s = g_stream[dev].load(std::memory_order_acquire);
  if (s) return s;
  std::lock_guard<std::mutex> lock(g_device_state_lock);
  s = g_stream[dev].load(std::memory_order_relaxed);
  if (!s && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess)
    g_stream[dev].store(s, std::memory_order_release);
  return s;
}

// The last copy captured into each constant-bank slot: (capture, stream,
// source, bytes).  Keyed by the slot's device address (unique across devices
// under unified addressing).
struct SlotCopy {
  unsigned long long capture = 0;
  cudaStream_t stream = nullptr;
  const void* src = nullptr;
  size_t bytes = 0;
};
static std::mutex g_slot_lock;
static std::map<void*, SlotCopy> g_slot_last;

int const_slot_copy(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  unsigned long long id = 0;
  BP_CUDA_TRY(cudaStreamGetCaptureInfo(s, &st, &id));
  if (st == cudaStreamCaptureStatusActive) {
    std::lock_guard<std::mutex> lock(g_slot_lock);
    SlotCopy& last = g_slot_last[dst];
    if (last.capture == id && last.stream == s && last.src == src && last.bytes == bytes) return BP_SUCCESS;
    BP_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
    last = SlotCopy{id, s, src, bytes};
    return BP_SUCCESS;
  }
  BP_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
  return BP_SUCCESS;
}

bool pdl_enabled() {
  static const bool on = [] {
    const char* e = getenv("BP_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}

int sm_count() {
  int dev = 0;
  if (current_device(&dev) != BP_SUCCESS) return 148;
  int n = g_sm_count[dev].load(std::memory_order_relaxed);
  if (n <= 0) {
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    g_sm_count[dev].store(n, std::memory_order_relaxed);
  }
  return n;
}

}  // namespace bp

using namespace bp;

extern "C" {

const char* bp_last_error(void) { return g_last_error.c_str(); }

const char* bp_version(void) { return "benchparanumal_b200 0.1 (sm_100a)"; }

int bp_test_wait_timeout(int withhold_slice) { return tma_wait_test(withhold_slice); }

int bp_tune_report(int32_t kind, int32_t N, int32_t Nfields, int32_t affine, int32_t precision_bytes, int32_t lanes,
                   int32_t fused, int32_t Nelements, int32_t* form, int32_t* nforms, int32_t* forms, float* ms,
                   int32_t cap) {
  if (!form || !nforms || (cap > 0 && (!forms || !ms))) return fail(BP_ERROR_ARG, "bp_tune_report: null pointer");
  const TuneConfig c{kind, N + 1, Nfields, affine ? 1 : 0, precision_bytes, lanes, fused ? 1 : 0,
                     element_class(Nelements)};
  int f = -1, n = 0;
  std::vector<int> fs(cap > 0 ? cap : 0);
  BP_TRY(tuned_report(c, &f, &n, fs.data(), ms, cap));
  *form = f;
  *nforms = n;
  for (int k = 0; k < n; ++k) forms[k] = fs[k];
  return BP_SUCCESS;
}

int bp_tune_reset(void) {
  tuned_clear();
  return BP_SUCCESS;
}

int bp_platform_init(int device_id) {
  int n = 0;
  BP_CUDA_TRY(cudaGetDeviceCount(&n));
  if (device_id < 0 || device_id >= n)
    return fail(BP_ERROR_ARG, "bp_platform_init: device " + std::to_string(device_id) + " not present (" +
                                  std::to_string(n) + " devices)");
  BP_CUDA_TRY(cudaSetDevice(device_id));
  BP_CUDA_TRY(cudaFree(0));
  int major = 0, minor = 0;
  BP_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device_id));
  BP_CUDA_TRY(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device_id));
  if (major != 10)
    return fail(BP_ERROR_ARG, "bp_platform_init: this build targets sm_100a (B200); device has sm_" +
                                  std::to_string(major) + std::to_string(minor));
  (void)default_stream();
  clear_error();
  return BP_SUCCESS;
}

int bp_device_count(int* count) {
  if (!count) return fail(BP_ERROR_ARG, "bp_device_count: null pointer");
  BP_CUDA_TRY(cudaGetDeviceCount(count));
  return BP_SUCCESS;
}

int bp_device_info(char* name, size_t name_len, int* sms) {
  int dev = 0;
  BP_CUDA_TRY(cudaGetDevice(&dev));
  cudaDeviceProp p;
  BP_CUDA_TRY(cudaGetDeviceProperties(&p, dev));
  if (name && name_len) {
    std::strncpy(name, p.name, name_len - 1);
    name[name_len - 1] = 0;
  }
  if (sms) *sms = p.multiProcessorCount;
  return BP_SUCCESS;
}

int bp_malloc(void** ptr, size_t bytes) {
  if (!ptr) return fail(BP_ERROR_ARG, "bp_malloc: null pointer");
  *ptr = nullptr;
  if (bytes == 0) return BP_SUCCESS;
  BP_CUDA_TRY(cudaMalloc(ptr, bytes));
  return BP_SUCCESS;
}

int bp_free(void* ptr) {
  if (ptr) BP_CUDA_TRY(cudaFree(ptr));
  return BP_SUCCESS;
}

int bp_host_malloc(void** ptr, size_t bytes) {
  if (!ptr) return fail(BP_ERROR_ARG, "bp_host_malloc: null pointer");
  *ptr = nullptr;
  if (bytes == 0) return BP_SUCCESS;
  BP_CUDA_TRY(cudaMallocHost(ptr, bytes));
  return BP_SUCCESS;
}

int bp_host_free(void* ptr) {
  if (ptr) BP_CUDA_TRY(cudaFreeHost(ptr));
  return BP_SUCCESS;
}

int bp_memcpy_htod(void* dst, const void* src, size_t bytes, bp_stream_t s) {
  if (bytes == 0) return BP_SUCCESS;
  BP_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, to_stream(s)));
  return BP_SUCCESS;
}

int bp_memcpy_dtoh(void* dst, const void* src, size_t bytes, bp_stream_t s) {
  if (bytes == 0) return BP_SUCCESS;
  BP_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, to_stream(s)));
  return BP_SUCCESS;
}

int bp_memcpy_dtod(void* dst, const void* src, size_t bytes, bp_stream_t s) {
  if (bytes == 0) return BP_SUCCESS;
  BP_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, to_stream(s)));
  return BP_SUCCESS;
}

int bp_memset(void* dst, int value, size_t bytes, bp_stream_t s) {
  if (bytes == 0) return BP_SUCCESS;
  BP_CUDA_TRY(cudaMemsetAsync(dst, value, bytes, to_stream(s)));
  return BP_SUCCESS;
}

int bp_stream_create(bp_stream_t* s) {
  if (!s) return fail(BP_ERROR_ARG, "bp_stream_create: null pointer");
  cudaStream_t cs;
  BP_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  *s = reinterpret_cast<bp_stream_t>(cs);
  return BP_SUCCESS;
}

int bp_stream_destroy(bp_stream_t s) {
  if (s) BP_CUDA_TRY(cudaStreamDestroy(reinterpret_cast<cudaStream_t>(s)));
  return BP_SUCCESS;
}

int bp_finish(bp_stream_t s) {
  BP_CUDA_TRY(cudaStreamSynchronize(to_stream(s)));
  return check_device_error();
}

int bp_event_create(bp_event_t* ev) {
  if (!ev) return fail(BP_ERROR_ARG, "bp_event_create: null pointer");
  cudaEvent_t e;
  BP_CUDA_TRY(cudaEventCreate(&e));
  *ev = reinterpret_cast<bp_event_t>(e);
  return BP_SUCCESS;
}

int bp_event_destroy(bp_event_t ev) {
  if (ev) BP_CUDA_TRY(cudaEventDestroy(reinterpret_cast<cudaEvent_t>(ev)));
  return BP_SUCCESS;
}

int bp_event_record(bp_event_t ev, bp_stream_t s) {
  BP_CUDA_TRY(cudaEventRecord(reinterpret_cast<cudaEvent_t>(ev), to_stream(s)));
  return BP_SUCCESS;
}

int bp_event_elapsed_ms(bp_event_t a, bp_event_t b, float* ms) {
  if (!ms) return fail(BP_ERROR_ARG, "bp_event_elapsed_ms: null pointer");
  BP_CUDA_TRY(cudaEventSynchronize(reinterpret_cast<cudaEvent_t>(b)));
  BP_CUDA_TRY(cudaEventElapsedTime(ms, reinterpret_cast<cudaEvent_t>(a), reinterpret_cast<cudaEvent_t>(b)));
  return BP_SUCCESS;
}

// ---------------------------------------------------------------------------
// kernel entry points
// ---------------------------------------------------------------------------
static int check_ax_desc(const bp_ax_desc_t* d) {
  if (!d) return fail(BP_ERROR_ARG, "bp_ax_hex3d: null descriptor");
  if (d->N < 1 || d->N > 15) return fail(BP_ERROR_ARG, "bp_ax_hex3d: degree N must be in 1..15");
  if (d->dim != 0 && d->dim != 2 && d->dim != 3) return fail(BP_ERROR_ARG, "bp_ax_hex3d: dim must be 2 or 3");
  const int nf6 = d->dim == 2 ? 2 : 3;   // BP6 has Nfields = dim
  if (d->Nfields != 1 && d->Nfields != nf6)
    return fail(BP_ERROR_ARG, d->dim == 2 ? "bp_ax_hex3d: Quad2D Nfields must be 1 or 2"
                                          : "bp_ax_hex3d: Nfields must be 1 or 3");
  if (d->bp != 5 && d->bp != 6) return fail(BP_ERROR_ARG, "bp_ax_hex3d: bp must be 5 or 6");
  if ((d->bp == 6) != (d->Nfields == nf6))
    return fail(BP_ERROR_ARG, "bp_ax_hex3d: BP6 has dim fields, BP5 one");
  return BP_SUCCESS;
}

int bp_ax_hex3d(const bp_ax_desc_t* desc, int32_t Nelements, const int32_t* elementList,
                const int32_t* GlobalToLocal, const double* wJ, const double* ggeo, const double* gllw,
                const double* D, double lambda, const double* q, double* Aq, bp_stream_t stream) {
  BP_TRY(check_ax_desc(desc));
  if (Nelements < 0) return fail(BP_ERROR_ARG, "bp_ax_hex3d: negative element count");
  if (Nelements == 0) return BP_SUCCESS;
  if (!elementList || !GlobalToLocal || !wJ || !ggeo || !D || !q || !Aq || (desc->affine && !gllw))
    return fail(BP_ERROR_ARG, "bp_ax_hex3d: null array");
  return launch_ax(*desc, Nelements, elementList, GlobalToLocal, wJ, ggeo, gllw, D, lambda, q, Aq,
                   to_stream(stream));
}

int bp_ax_tri2d(const bp_ax_desc_t* d, int32_t Nelements, const int32_t* elementList, const int32_t* GlobalToLocal,
                const double* wJ, const double* ggeo, const double* S, const double* MM, double lambda,
                const double* q, double* Aq, bp_stream_t stream) {
  if (!d) return fail(BP_ERROR_ARG, "bp_ax_tri2d: null descriptor");
  if (d->bp != 5 || d->Nfields != 1 || d->dim != 2 || !d->affine)
    return fail(BP_ERROR_ARG, "bp_ax_tri2d: the Tri2D operator is BP5, one field, dim 2, affine");
  if (d->N < 1 || d->N > 15) return fail(BP_ERROR_ARG, "bp_ax_tri2d: degree N must be in 1..15");
  if (Nelements < 0) return fail(BP_ERROR_ARG, "bp_ax_tri2d: negative element count");
  if (Nelements == 0) return BP_SUCCESS;
  if (!elementList || !GlobalToLocal || !wJ || !ggeo || !S || !MM || !q || !Aq)
    return fail(BP_ERROR_ARG, "bp_ax_tri2d: null array");
  return launch_ax_simplex(2, d->N, Nelements, elementList, GlobalToLocal, wJ, ggeo, S, MM, lambda, q, Aq, nullptr,
                           to_stream(stream));
}

int bp_ax_tet3d(const bp_ax_desc_t* d, int32_t Nelements, const int32_t* elementList, const int32_t* GlobalToLocal,
                const double* wJ, const double* ggeo, const double* S, const double* MM, double lambda,
                const double* q, double* Aq, bp_stream_t stream) {
  if (!d) return fail(BP_ERROR_ARG, "bp_ax_tet3d: null descriptor");
  if (d->bp != 5 || d->Nfields != 1 || (d->dim != 3 && d->dim != 0) || !d->affine)
    return fail(BP_ERROR_ARG, "bp_ax_tet3d: the Tet3D operator is BP5, one field, dim 3, affine");
  if (d->N < 1 || d->N > 15) return fail(BP_ERROR_ARG, "bp_ax_tet3d: degree N must be in 1..15");
  if (Nelements < 0) return fail(BP_ERROR_ARG, "bp_ax_tet3d: negative element count");
  if (Nelements == 0) return BP_SUCCESS;
  if (!elementList || !GlobalToLocal || !wJ || !ggeo || !S || !MM || !q || !Aq)
    return fail(BP_ERROR_ARG, "bp_ax_tet3d: null array");
  return launch_ax_simplex(3, d->N, Nelements, elementList, GlobalToLocal, wJ, ggeo, S, MM, lambda, q, Aq, nullptr,
                           to_stream(stream));
}

int bp_ax_hex3d_f32(const bp_ax_desc_t* desc, int32_t Nelements, const int32_t* elementList,
                    const int32_t* GlobalToLocal, const float* wJ, const float* ggeo, const float* gllw,
                    const float* D, float lambda, const float* q, float* Aq, bp_stream_t stream) {
  BP_TRY(check_ax_desc(desc));
  if (Nelements < 0) return fail(BP_ERROR_ARG, "bp_ax_hex3d_f32: negative element count");
  if (Nelements == 0) return BP_SUCCESS;
  if (!elementList || !GlobalToLocal || !wJ || !ggeo || !D || !q || !Aq || (desc->affine && !gllw))
    return fail(BP_ERROR_ARG, "bp_ax_hex3d_f32: null array");
  return launch_ax_skip(*desc, Nelements, elementList, GlobalToLocal, wJ, ggeo, gllw, D, lambda, q, Aq, nullptr,
                        to_stream(stream));
}

int bp_ax_hex3d_f32_multi(const bp_ax_desc_t* desc, int32_t nrhs, int32_t Nelements, const int32_t* elementList,
                          const int32_t* GlobalToLocal, const float* wJ, const float* ggeo, const float* gllw,
                          const float* D, float lambda, const float* q, float* Aq, bp_stream_t stream) {
  if (nrhs == 1)
    return bp_ax_hex3d_f32(desc, Nelements, elementList, GlobalToLocal, wJ, ggeo, gllw, D, lambda, q, Aq, stream);
  BP_TRY(check_ax_desc(desc));
  if (nrhs != 2 && nrhs != 4) return fail(BP_ERROR_ARG, "bp_ax_hex3d_f32_multi: nrhs must be 1, 2 or 4");
  if (desc->Nfields != 1 || desc->affine)
    return fail(BP_ERROR_ARG, "bp_ax_hex3d_f32_multi: one field, stored factors only");
  if (Nelements < 0) return fail(BP_ERROR_ARG, "bp_ax_hex3d_f32_multi: negative element count");
  if (Nelements == 0) return BP_SUCCESS;
  if (!elementList || !GlobalToLocal || !wJ || !ggeo || !D || !q || !Aq)
    return fail(BP_ERROR_ARG, "bp_ax_hex3d_f32_multi: null array");
  if ((reinterpret_cast<uintptr_t>(q) | reinterpret_cast<uintptr_t>(Aq)) % (sizeof(float) * nrhs))
    return fail(BP_ERROR_ARG, "bp_ax_hex3d_f32_multi: q and Aq must be aligned to nrhs floats");
  const cudaStream_t s = to_stream(stream);
  return launch_ax_packed(nrhs, *desc, Nelements, elementList, GlobalToLocal, wJ, ggeo, gllw, D, lambda, q, Aq,
                          nullptr, nullptr, s, nullptr);
}

int bp_ogs_owner_map(int32_t NL, const int32_t* GlobalToLocal, int32_t Ngather, const int32_t* rowStarts,
                     const int32_t* colIds, int32_t* ownerMap, bp_stream_t stream) {
  if (NL < 0 || Ngather < 0) return fail(BP_ERROR_ARG, "bp_ogs_owner_map: negative size");
  if (Ngather >= kOwnerBit) return fail(BP_ERROR_ARG, "bp_ogs_owner_map: Ngather must be below BP_OWNER_BIT");
  if ((NL && (!GlobalToLocal || !ownerMap)) || (Ngather && (!rowStarts || !colIds)))
    return fail(BP_ERROR_ARG, "bp_ogs_owner_map: null array");
  return launch_owner_map((size_t)NL, GlobalToLocal, Ngather, rowStarts, colIds, ownerMap, to_stream(stream));
}

// the fused step's common checks; lanes = values per node
static int check_dir_args(const char* who, const bp_ax_desc_t* desc, int lanes, int32_t Nelements,
                          const void* elementList, const void* ownerMap, const void* wJ, const void* ggeo,
                          const void* D, const void* r, const void* p_old, const void* p_new, const void* x,
                          const void* Aq, const void* partials) {
  BP_TRY(check_ax_desc(desc));
  if (Nelements < 0) return fail(BP_ERROR_ARG, std::string(who) + ": negative element count");
  if (desc->bp < 5 || !tma_covers(*desc, lanes))
    return fail(BP_ERROR_ARG, std::string(who) + ": the fused step covers stored factors at even Nq (packed: Nq 8..12, "
                                                 "one field; single: Nq <= 16, or <= 10 with three fields)");
  // the gathered vectors are only read at unmasked nodes: a mesh without any may pass NULL
  if (Nelements && (!elementList || !ownerMap || !wJ || !ggeo || !D || !Aq || !partials))
    return fail(BP_ERROR_ARG, std::string(who) + ": null array");
  if (p_old && p_old == p_new) return fail(BP_ERROR_ARG, std::string(who) + ": p_new must not alias p_old");
  return BP_SUCCESS;
}

int bp_cg_direction_ax_hex3d(const bp_ax_desc_t* desc, int32_t Nelements, const int32_t* elementList,
                             const int32_t* ownerMap, const double* wJ, const double* ggeo, const double* D,
                             double lambda, double alpha, double beta, const double* r, const double* invD,
                             const double* p_old, double* p_new, double* x, double* Aq, double* pAp_partials,
                             bp_stream_t stream) {
  BP_TRY(check_dir_args("bp_cg_direction_ax_hex3d", desc, 1, Nelements, elementList, ownerMap, wJ, ggeo, D, r,
                        p_old, p_new, x, Aq, pAp_partials));
  if (Nelements == 0) return BP_SUCCESS;
  CgFuse f;
  f.partials = pAp_partials;
  f.dir = 1;
  f.pbuf[0] = const_cast<double*>(p_old);
  f.pbuf[1] = p_new;
  f.r = r;
  f.invD = invD;
  f.x = x;
  f.alpha[0] = alpha;
  f.beta[0] = beta;
  const int rc = launch_ax_tma(*desc, Nelements, elementList, ownerMap, wJ, ggeo, D, lambda, nullptr, Aq, nullptr,
                               &f, to_stream(stream), nullptr);
  return rc == 1 ? fail(BP_ERROR_ARG, "bp_cg_direction_ax_hex3d: factor arrays must be 16-byte aligned") : rc;
}

int bp_cg_direction_ax_f32_multi(const bp_ax_desc_t* desc, int32_t nrhs, int32_t Nelements,
                                 const int32_t* elementList, const int32_t* ownerMap, const float* wJ,
                                 const float* ggeo, const float* D, float lambda, const double* alpha,
                                 const double* beta, const float* r, const float* invD, const float* p_old,
                                 float* p_new, float* x, float* Aq, double* pAp_partials, bp_stream_t stream) {
  if (nrhs != 1 && nrhs != 2 && nrhs != 4)
    return fail(BP_ERROR_ARG, "bp_cg_direction_ax_f32_multi: nrhs must be 1, 2 or 4");
  if (!alpha || !beta) return fail(BP_ERROR_ARG, "bp_cg_direction_ax_f32_multi: null coefficients");
  BP_TRY(check_dir_args("bp_cg_direction_ax_f32_multi", desc, nrhs, Nelements, elementList, ownerMap, wJ, ggeo, D, r,
                        p_old, p_new, x, Aq, pAp_partials));
  if (Nelements == 0) return BP_SUCCESS;
  if ((reinterpret_cast<uintptr_t>(r) | reinterpret_cast<uintptr_t>(p_old) | reinterpret_cast<uintptr_t>(p_new) |
       reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(Aq)) % (sizeof(float) * nrhs))
    return fail(BP_ERROR_ARG, "bp_cg_direction_ax_f32_multi: vectors must be aligned to nrhs floats");
  CgFuse f;
  f.partials = pAp_partials;
  f.dir = 1;
  f.pbuf[0] = const_cast<float*>(p_old);
  f.pbuf[1] = p_new;
  f.r = r;
  f.invD = invD;
  f.x = x;
  for (int k = 0; k < nrhs; ++k) {
    f.alpha[k] = alpha[k];
    f.beta[k] = beta[k];
  }
  const cudaStream_t s = to_stream(stream);
  const int rc = nrhs == 1 ? launch_ax_tma(*desc, Nelements, elementList, ownerMap, wJ, ggeo, D, lambda, nullptr, Aq,
                                           nullptr, &f, s, nullptr)
                           : launch_ax_tma_packed(nrhs, *desc, Nelements, elementList, ownerMap, wJ, ggeo, D, lambda,
                                                  nullptr, Aq, nullptr, &f, s, nullptr);
  return rc == 1 ? fail(BP_ERROR_ARG, "bp_cg_direction_ax_f32_multi: factor arrays must be 16-byte aligned") : rc;
}

int bp_convert_f64_f32(size_t n, const double* src, float* dst, bp_stream_t stream) {
  if (n > 0 && (!src || !dst)) return fail(BP_ERROR_ARG, "bp_convert_f64_f32: null array");
  return launch_d2f(n, src, dst, to_stream(stream));
}

int bp_ax_cub_hex3d(const bp_ax_desc_t* d, int32_t Nelements, const int32_t* elementList,
                    const int32_t* GlobalToLocal, const double* cubwJ, const double* cubggeo, const double* cubD,
                    const double* cubInterp, const double* invV, const double* MM, double lambda, const double* q,
                    double* Aq, bp_stream_t stream) {
  if (!d) return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d: null descriptor");
  if (d->N < 1 || d->N > 15) return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d: degree N must be in 1..15");
  if (d->bp < 1 || d->bp > 4) return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d: bp must be 1..4");
  if (d->dim == 2) return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d: the over-integrated forms are Hex3D only");
  if (d->Nfields != ((d->bp % 2) ? 1 : 3)) return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d: BP1/BP3 have 1 field, BP2/BP4 3");
  if (Nelements < 0) return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d: negative element count");
  if (Nelements == 0) return BP_SUCCESS;
  const bool stiff = d->bp >= 3;
  const double* T = !d->affine ? cubInterp : (stiff ? invV : MM);
  if (!elementList || !GlobalToLocal || !cubwJ || !T || !q || !Aq || (stiff && (!cubggeo || !cubD)))
    return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d: null array");
  const CubOperands<double> ops{cubwJ, cubggeo, cubD, T};
  return launch_ax_cub(*d, Nelements, elementList, GlobalToLocal, ops, lambda, q, Aq, nullptr, to_stream(stream));
}

int bp_ax_cub_hex3d_f32(const bp_ax_desc_t* d, int32_t Nelements, const int32_t* elementList,
                        const int32_t* GlobalToLocal, const float* cubwJ, const float* cubggeo, const float* cubD,
                        const float* cubInterp, const float* invV, const float* MM, float lambda, const float* q,
                        float* Aq, bp_stream_t stream) {
  if (!d) return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d_f32: null descriptor");
  if (d->N < 1 || d->N > 15) return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d_f32: degree N must be in 1..15");
  if (d->bp < 1 || d->bp > 4) return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d_f32: bp must be 1..4");
  if (d->dim == 2) return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d_f32: the over-integrated forms are Hex3D only");
  if (d->Nfields != ((d->bp % 2) ? 1 : 3))
    return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d_f32: BP1/BP3 have 1 field, BP2/BP4 3");
  if (Nelements < 0) return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d_f32: negative element count");
  if (Nelements == 0) return BP_SUCCESS;
  const bool stiff = d->bp >= 3;
  const float* T = !d->affine ? cubInterp : (stiff ? invV : MM);
  if (!elementList || !GlobalToLocal || !cubwJ || !T || !q || !Aq || (stiff && (!cubggeo || !cubD)))
    return fail(BP_ERROR_ARG, "bp_ax_cub_hex3d_f32: null array");
  const CubOperands<float> ops{cubwJ, cubggeo, cubD, T};
  return launch_ax_cub(*d, Nelements, elementList, GlobalToLocal, ops, lambda, q, Aq, nullptr, to_stream(stream));
}

int bp_ogs_gather(int32_t Nrows, const int32_t* rowStarts, const int32_t* colIds, const double* v, double* gv,
                  bp_stream_t stream) {
  if (Nrows < 0) return fail(BP_ERROR_ARG, "bp_ogs_gather: negative row count");
  if (Nrows == 0) return BP_SUCCESS;
  if (!rowStarts || !colIds || !v || !gv) return fail(BP_ERROR_ARG, "bp_ogs_gather: null array");
  return launch_gather(Nrows, rowStarts, colIds, v, gv, to_stream(stream));
}

int bp_ogs_scatter(int32_t Nrows, const int32_t* rowStarts, const int32_t* colIds, const double* gv, double* v,
                   bp_stream_t stream) {
  if (Nrows < 0) return fail(BP_ERROR_ARG, "bp_ogs_scatter: negative row count");
  if (Nrows == 0) return BP_SUCCESS;
  if (!rowStarts || !colIds || !v || !gv) return fail(BP_ERROR_ARG, "bp_ogs_scatter: null array");
  return launch_scatter(Nrows, rowStarts, colIds, gv, v, to_stream(stream));
}

int bp_linalg_set(int32_t N, double alpha, double* x, bp_stream_t s) {
  if (N < 0 || (N > 0 && !x)) return fail(BP_ERROR_ARG, "bp_linalg_set: bad arguments");
  return launch_set(N, alpha, x, to_stream(s));
}

int bp_linalg_axpy(int32_t N, double alpha, const double* x, double beta, double* y, bp_stream_t s) {
  if (N < 0 || (N > 0 && (!x || !y))) return fail(BP_ERROR_ARG, "bp_linalg_axpy: bad arguments");
  return launch_axpy(N, alpha, x, beta, y, to_stream(s));
}

// scratch for the standalone reductions, per device: partial sums and the
// arrival counter (allocated on the first reduction on each device)
struct RedScratch {
  double* partials = nullptr;
  unsigned int* counter = nullptr;
};
static RedScratch g_red[kMaxDevices];
static DeviceOnce g_red_once;
static int red_scratch(RedScratch** out) {
  int dev = 0;
  BP_TRY(current_device(&dev));
  BP_TRY(once_per_device(g_red_once, [dev]() -> int {
    RedScratch& r = g_red[dev];
    BP_CUDA_TRY(cudaMalloc(&r.partials, sizeof(double) * 4 * reduction_blocks()));
    BP_CUDA_TRY(cudaMalloc(&r.counter, sizeof(unsigned int) * 4));
    BP_CUDA_TRY(cudaMemset(r.counter, 0, sizeof(unsigned int) * 4));
    return BP_SUCCESS;
  }));
  *out = &g_red[dev];
  return BP_SUCCESS;
}

int bp_linalg_inner_prod(int32_t N, const double* x, const double* y, double* result, bp_stream_t s) {
  if (N < 0 || !result || (N > 0 && (!x || !y))) return fail(BP_ERROR_ARG, "bp_linalg_inner_prod: bad arguments");
  RedScratch* r = nullptr;
  BP_TRY(red_scratch(&r));
  return launch_dot(N, x, y, result, r->partials, r->counter, to_stream(s));
}

int bp_linalg_norm2(int32_t N, const double* x, double* result, bp_stream_t s) {
  if (N < 0 || !result || (N > 0 && !x)) return fail(BP_ERROR_ARG, "bp_linalg_norm2: bad arguments");
  RedScratch* r = nullptr;
  BP_TRY(red_scratch(&r));
  BP_TRY(launch_dot(N, x, x, result, r->partials, r->counter, to_stream(s)));
  return launch_sqrt1(result, to_stream(s));
}

int bp_update_cg(int32_t N, const double* Ap, double alpha, double* r, double* rdotr, bp_stream_t s) {
  if (N < 0 || !rdotr || (N > 0 && (!Ap || !r))) return fail(BP_ERROR_ARG, "bp_update_cg: bad arguments");
  RedScratch* rs = nullptr;
  BP_TRY(red_scratch(&rs));
  return launch_update_cg(N, Ap, alpha, r, rdotr, rs->partials, rs->counter, to_stream(s));
}

// ---------------------------------------------------------------------------
// mesh
// ---------------------------------------------------------------------------
// The Quad2D box: vertices, numbering and factors on the host (a 2D box is
// small next to a 3D one of the same degree), then uploaded.
static int mesh_create_quad(const bp_box_desc_t* d, bp_mesh_t* out) {
  if (d->nx < 1 || d->ny < 1) return fail(BP_ERROR_ARG, "bp_mesh_create: element counts must be >= 1");
  if (d->N < 1 || d->N > 15) return fail(BP_ERROR_ARG, "bp_mesh_create: degree must be in 1..15");
  if (d->Nfields != 1 && d->Nfields != 2) return fail(BP_ERROR_ARG, "bp_mesh_create: Quad2D Nfields must be 1 or 2");
  if (!(d->pert >= 0.0 && d->pert < 0.5)) return fail(BP_ERROR_ARG, "bp_mesh_create: perturbation must be in [0, 0.5)");
  const int Nq = d->N + 1, Np = Nq * Nq;
  const int64_t E64 = (int64_t)d->nx * d->ny;
  if (E64 * Np * d->Nfields >= (int64_t)INT32_MAX)
    return fail(BP_ERROR_ARG, "bp_mesh_create: local node count exceeds int32 (dlong) range");
  cudaStream_t s = default_stream();
  HostMesh hm;
  hm.dim = 2;
  hm.N = d->N; hm.Nq = Nq; hm.Np = Np;
  hm.nx = d->nx; hm.ny = d->ny; hm.nz = 1;
  hm.E = (int)E64; hm.affine = d->affine ? 1 : 0; hm.Nfields = d->Nfields;
  gll_nodes_weights(hm.N, hm.gllz, hm.gllw);
  diff_matrix(hm.gllz, hm.D);
  box_vertices_2d(hm, d->pert, d->pert_seed);
  box_numbering_2d(hm);
  std::vector<double> wJ, ggeo;
  if (!quad_geometry(hm, wJ, ggeo))
    return fail(BP_ERROR_NUMERIC, "bp_mesh_create: non-positive Jacobian found (perturbation too large?)");
  bp_mesh_s* m = new bp_mesh_s();
  m->dim = 2;
  m->N = hm.N; m->Nq = Nq; m->Np = Np; m->E = hm.E; m->Nfields = hm.Nfields; m->affine = hm.affine;
  m->Ngather = hm.Ngather; m->nnz = hm.nnz;
  std::vector<int32_t> elist(hm.E);
  for (int e = 0; e < hm.E; ++e) elist[e] = e;
  int rc = BP_SUCCESS;
  do {
    if ((rc = m->elementList.upload(elist, s))) break;
    if ((rc = m->G2L.upload(hm.G2L, s))) break;
    if ((rc = m->rowStarts.upload(hm.rowStarts, s))) break;
    if ((rc = m->colIds.upload(hm.colIds, s))) break;
    if ((rc = m->D.upload(hm.D, s))) break;
    if ((rc = m->gllz.upload(hm.gllz, s))) break;
    if ((rc = m->gllw.upload(hm.gllw, s))) break;
    if ((rc = m->EX.upload(hm.EX, s))) break;
    if ((rc = m->EY.upload(hm.EY, s))) break;
    if ((rc = m->wJ.upload(wJ, s))) break;
    if ((rc = m->ggeo.upload(ggeo, s))) break;
    cudaError_t ce = cudaStreamSynchronize(s);   // the host vectors are released on return
    if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_mesh_create", __FILE__, __LINE__); break; }
  } while (0);
  if (rc != BP_SUCCESS) {
    delete m;
    return rc;
  }
  *out = m;
  return BP_SUCCESS;
}

// the node-fastest device layout of row-major Np x Np blocks: out[k*Np + n] = in[n*Np + k]
static std::vector<double> node_fastest(const std::vector<double>& rm, int Np) {
  std::vector<double> t(rm.size());
  const size_t NP2 = (size_t)Np * Np;
  for (size_t b = 0; b < rm.size() / NP2; ++b)
    for (int n = 0; n < Np; ++n)
      for (int k = 0; k < Np; ++k) t[b * NP2 + (size_t)k * Np + n] = rm[b * NP2 + (size_t)n * Np + k];
  return t;
}

static int mesh_create_tri(const bp_box_desc_t* d, bp_mesh_t* out) {
  if (d->nx < 1 || d->ny < 1) return fail(BP_ERROR_ARG, "bp_mesh_create: element counts must be >= 1");
  if (d->N < 1 || d->N > 15) return fail(BP_ERROR_ARG, "bp_mesh_create: degree must be in 1..15");
  if (d->Nfields != 1) return fail(BP_ERROR_ARG, "bp_mesh_create: Tri2D meshes take one field (BP5)");
  if (!d->affine) return fail(BP_ERROR_ARG, "bp_mesh_create: Tri2D meshes are affine here (-a)");
  if (d->pert != 0.0) return fail(BP_ERROR_ARG, "bp_mesh_create: the Tri2D box has no vertex perturbation");
  TriBasis tb;
  if (!tri_basis(d->N, tb)) return fail(BP_ERROR_NUMERIC, "bp_mesh_create: singular Tri2D Vandermonde matrix");
  const int Np = tb.Np;
  const int64_t E64 = 2 * (int64_t)d->nx * d->ny;
  if (E64 * Np >= (int64_t)INT32_MAX)
    return fail(BP_ERROR_ARG, "bp_mesh_create: local node count exceeds int32 (dlong) range");
  cudaStream_t s = default_stream();
  HostMesh hm;
  hm.dim = 2;
  hm.N = d->N; hm.Nq = d->N + 1; hm.Np = Np;
  hm.nx = d->nx; hm.ny = d->ny; hm.nz = 1;
  hm.E = (int)E64; hm.affine = 1; hm.Nfields = 1;
  std::vector<double> wJ, ggeo;
  if (!box_tri(hm, tb, wJ, ggeo))
    return fail(BP_ERROR_NUMERIC, "bp_mesh_create: non-positive Jacobian found");
  std::vector<double> D(tb.Dr);
  D.insert(D.end(), tb.Ds.begin(), tb.Ds.end());
  std::vector<double> xn, yn;
  tri_nodes_xy(hm, tb, xn, yn);
  bp_mesh_s* m = new bp_mesh_s();
  m->dim = 2;
  m->simplex = 1;
  m->N = hm.N; m->Nq = hm.Nq; m->Np = Np; m->E = hm.E; m->Nfields = 1; m->affine = 1;
  m->Ngather = hm.Ngather; m->nnz = hm.nnz;
  std::vector<int32_t> elist(hm.E);
  for (int e = 0; e < hm.E; ++e) elist[e] = e;
  int rc = BP_SUCCESS;
  do {
    if ((rc = m->elementList.upload(elist, s))) break;
    if ((rc = m->G2L.upload(hm.G2L, s))) break;
    if ((rc = m->rowStarts.upload(hm.rowStarts, s))) break;
    if ((rc = m->colIds.upload(hm.colIds, s))) break;
    if ((rc = m->D.upload(node_fastest(D, Np), s))) break;
    if ((rc = m->S.upload(node_fastest(tb.S, Np), s))) break;
    if ((rc = m->MM.upload(tb.MM, s))) break;   // symmetric
    if ((rc = m->x.upload(xn, s))) break;
    if ((rc = m->y.upload(yn, s))) break;
    if ((rc = m->EX.upload(hm.EX, s))) break;
    if ((rc = m->EY.upload(hm.EY, s))) break;
    if ((rc = m->wJ.upload(wJ, s))) break;
    if ((rc = m->ggeo.upload(ggeo, s))) break;
    cudaError_t ce = cudaStreamSynchronize(s);   // the host vectors are released on return
    if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_mesh_create", __FILE__, __LINE__); break; }
  } while (0);
  if (rc != BP_SUCCESS) {
    delete m;
    return rc;
  }
  *out = m;
  return BP_SUCCESS;
}

static int mesh_create_tet(const bp_box_desc_t* d, bp_mesh_t* out) {
  if (d->nx < 1 || d->ny < 1 || d->nz < 1) return fail(BP_ERROR_ARG, "bp_mesh_create: element counts must be >= 1");
  if (d->N < 1 || d->N > 15) return fail(BP_ERROR_ARG, "bp_mesh_create: degree must be in 1..15");
  if (d->Nfields != 1) return fail(BP_ERROR_ARG, "bp_mesh_create: Tet3D meshes take one field (BP5)");
  if (!d->affine) return fail(BP_ERROR_ARG, "bp_mesh_create: Tet3D meshes are affine here (-a)");
  if (d->pert != 0.0) return fail(BP_ERROR_ARG, "bp_mesh_create: the Tet3D box has no vertex perturbation");
  TetBasis tb;
  if (!tet_basis(d->N, tb)) return fail(BP_ERROR_NUMERIC, "bp_mesh_create: singular Tet3D Vandermonde matrix");
  const int Np = tb.Np;
  const int64_t E64 = 6 * (int64_t)d->nx * d->ny * d->nz;
  if (E64 * Np >= (int64_t)INT32_MAX)
    return fail(BP_ERROR_ARG, "bp_mesh_create: local node count exceeds int32 (dlong) range");
  cudaStream_t s = default_stream();
  HostMesh hm;
  hm.dim = 3;
  hm.N = d->N; hm.Nq = d->N + 1; hm.Np = Np;
  hm.nx = d->nx; hm.ny = d->ny; hm.nz = d->nz;
  hm.E = (int)E64; hm.affine = 1; hm.Nfields = 1;
  std::vector<double> wJ, ggeo, xn, yn, zn;
  if (!box_tet(hm, tb, wJ, ggeo, xn, yn, zn))
    return fail(BP_ERROR_NUMERIC, "bp_mesh_create: non-positive Jacobian found");
  std::vector<double> D(tb.Dr);
  D.insert(D.end(), tb.Ds.begin(), tb.Ds.end());
  D.insert(D.end(), tb.Dt.begin(), tb.Dt.end());
  bp_mesh_s* m = new bp_mesh_s();
  m->dim = 3;
  m->simplex = 1;
  m->N = hm.N; m->Nq = hm.Nq; m->Np = Np; m->E = hm.E; m->Nfields = 1; m->affine = 1;
  m->Ngather = hm.Ngather; m->nnz = hm.nnz;
  std::vector<int32_t> elist(hm.E);
  for (int e = 0; e < hm.E; ++e) elist[e] = e;
  int rc = BP_SUCCESS;
  do {
    if ((rc = m->elementList.upload(elist, s))) break;
    if ((rc = m->G2L.upload(hm.G2L, s))) break;
    if ((rc = m->rowStarts.upload(hm.rowStarts, s))) break;
    if ((rc = m->colIds.upload(hm.colIds, s))) break;
    if ((rc = m->D.upload(node_fastest(D, Np), s))) break;
    if ((rc = m->S.upload(node_fastest(tb.S, Np), s))) break;
    if ((rc = m->MM.upload(tb.MM, s))) break;   // symmetric
    if ((rc = m->x.upload(xn, s))) break;
    if ((rc = m->y.upload(yn, s))) break;
    if ((rc = m->z.upload(zn, s))) break;
    if ((rc = m->EX.upload(hm.EX, s))) break;
    if ((rc = m->EY.upload(hm.EY, s))) break;
    if ((rc = m->EZ.upload(hm.EZ, s))) break;
    if ((rc = m->wJ.upload(wJ, s))) break;
    if ((rc = m->ggeo.upload(ggeo, s))) break;
    cudaError_t ce = cudaStreamSynchronize(s);   // the host vectors are released on return
    if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_mesh_create", __FILE__, __LINE__); break; }
  } while (0);
  if (rc != BP_SUCCESS) {
    delete m;
    return rc;
  }
  *out = m;
  return BP_SUCCESS;
}

int bp_mesh_create(const bp_box_desc_t* d, bp_mesh_t* out) {
  if (!d || !out) return fail(BP_ERROR_ARG, "bp_mesh_create: null pointer");
  *out = nullptr;
  if (d->dim != 0 && d->dim != 2 && d->dim != 3) return fail(BP_ERROR_ARG, "bp_mesh_create: dim must be 2 or 3");
  if (d->dim == 2 && d->simplex) return mesh_create_tri(d, out);
  if (d->simplex) return mesh_create_tet(d, out);
  if (d->dim == 2) return mesh_create_quad(d, out);
  if (d->nx < 1 || d->ny < 1 || d->nz < 1) return fail(BP_ERROR_ARG, "bp_mesh_create: element counts must be >= 1");
  if (d->N < 1 || d->N > 15) return fail(BP_ERROR_ARG, "bp_mesh_create: degree must be in 1..15");
  if (d->Nfields != 1 && d->Nfields != 3) return fail(BP_ERROR_ARG, "bp_mesh_create: Nfields must be 1 or 3");
  if (!(d->pert >= 0.0 && d->pert < 0.5)) return fail(BP_ERROR_ARG, "bp_mesh_create: perturbation must be in [0, 0.5)");
  const int64_t E64 = (int64_t)d->nx * d->ny * d->nz;
  const int Nq = d->N + 1, Np = Nq * Nq * Nq;
  if (E64 * Np * d->Nfields >= (int64_t)INT32_MAX)
    return fail(BP_ERROR_ARG, "bp_mesh_create: local node count exceeds int32 (dlong) range");
  cudaStream_t s = default_stream();

  HostMesh hm;
  hm.N = d->N; hm.Nq = Nq; hm.Np = Np;
  hm.nx = d->nx; hm.ny = d->ny; hm.nz = d->nz;
  hm.E = (int)E64; hm.affine = d->affine ? 1 : 0; hm.Nfields = d->Nfields;
  gll_nodes_weights(hm.N, hm.gllz, hm.gllw);
  diff_matrix(hm.gllz, hm.D);
  box_vertices(hm, d->pert, d->pert_seed);
  int64_t ngather = 0, nnz = 0;
  box_numbering_counts(hm.nx, hm.ny, hm.nz, hm.N, hm.Nfields, &ngather, &nnz);

  bp_mesh_s* m = new bp_mesh_s();
  m->N = hm.N; m->Nq = Nq; m->Np = Np; m->E = hm.E; m->Nfields = hm.Nfields; m->affine = hm.affine;
  m->Ngather = (int32_t)ngather; m->nnz = (int32_t)nnz;
  std::vector<int32_t> elist(hm.E);
  for (int e = 0; e < hm.E; ++e) elist[e] = e;
  int rc = BP_SUCCESS;
  int* d_bad = nullptr;
  do {
    if ((rc = m->elementList.upload(elist, s))) break;
    // the numbering is computed on the device (closed form, bit-identical to
    // the host box_numbering): no O(E*Np) host pass, no 0.35 GB upload at 40^3 p=7
    if ((rc = m->G2L.alloc((size_t)hm.E * Np * hm.Nfields))) break;
    if ((rc = m->rowStarts.alloc((size_t)ngather + 1))) break;
    if ((rc = m->colIds.alloc((size_t)nnz))) break;
    if ((rc = launch_box_numbering(hm.nx, hm.ny, hm.nz, hm.N, hm.Nfields, m->G2L.ptr, m->rowStarts.ptr,
                                   m->colIds.ptr, s)))
      break;
    if ((rc = m->D.upload(hm.D, s))) break;
    if ((rc = m->gllz.upload(hm.gllz, s))) break;
    if ((rc = m->gllw.upload(hm.gllw, s))) break;
    if ((rc = m->EX.upload(hm.EX, s))) break;
    if ((rc = m->EY.upload(hm.EY, s))) break;
    if ((rc = m->EZ.upload(hm.EZ, s))) break;
    const size_t ng = hm.affine ? (size_t)hm.E : (size_t)hm.E * Np;
    if ((rc = m->wJ.alloc(ng))) break;
    if ((rc = m->ggeo.alloc(6 * ng))) break;
    cudaError_t ce = cudaMalloc(&d_bad, sizeof(int));
    if (ce != cudaSuccess) { rc = cuda_fail(ce, "cudaMalloc", __FILE__, __LINE__); break; }
    cudaMemsetAsync(d_bad, 0, sizeof(int), s);
    if ((rc = launch_geometry(hm.N, hm.affine, hm.E, m->EX.ptr, m->EY.ptr, m->EZ.ptr, m->gllz.ptr, m->gllw.ptr,
                              m->wJ.ptr, m->ggeo.ptr, d_bad, s)))
      break;
    int bad = 0;
    ce = cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) { rc = cuda_fail(ce, "geometry setup", __FILE__, __LINE__); break; }
    if (bad) { rc = fail(BP_ERROR_NUMERIC, "bp_mesh_create: non-positive Jacobian found (perturbation too large?)"); break; }
  } while (0);
  if (d_bad) cudaFree(d_bad);
  if (rc != BP_SUCCESS) {
    delete m;
    return rc;
  }
  *out = m;
  return BP_SUCCESS;
}

int bp_mesh_view(bp_mesh_t m, bp_mesh_view_t* v) {
  if (!m || !v) return fail(BP_ERROR_ARG, "bp_mesh_view: null pointer");
  v->N = m->N; v->Nq = m->Nq; v->Np = m->Np; v->Nelements = m->E; v->Nfields = m->Nfields;
  v->affine = m->affine; v->Ngather = m->Ngather; v->nnz = m->nnz;
  v->Nlocal = (int64_t)m->E * m->Np * m->Nfields;
  v->elementList = m->elementList.ptr; v->GlobalToLocal = m->G2L.ptr;
  v->rowStarts = m->rowStarts.ptr; v->colIds = m->colIds.ptr;
  v->wJ = m->wJ.ptr; v->ggeo = m->ggeo.ptr; v->D = m->D.ptr; v->gllz = m->gllz.ptr; v->gllw = m->gllw.ptr;
  v->EX = m->EX.ptr; v->EY = m->EY.ptr; v->EZ = m->EZ.ptr;
  v->dim = m->dim;
  v->simplex = m->simplex;
  v->S = m->simplex ? m->S.ptr : nullptr;
  v->MM = m->simplex ? m->MM.ptr : nullptr;
  return BP_SUCCESS;
}

int bp_mesh_cubature(bp_mesh_t m) {
  if (!m) return fail(BP_ERROR_ARG, "bp_mesh_cubature: null mesh");
  if (m->dim == 2 || m->simplex)
    return fail(BP_ERROR_ARG, "bp_mesh_cubature: the over-integrated BP1-BP4 forms are Hex3D only");
  if (m->cubNq) return BP_SUCCESS;
  cudaStream_t s = default_stream();
  std::vector<double> z(m->Nq);
  BP_CUDA_TRY(cudaMemcpy(z.data(), m->gllz.ptr, sizeof(double) * m->Nq, cudaMemcpyDeviceToHost));
  CubBasis cb;
  cubature_basis(m->N, z, cb);
  const int Nq = m->Nq, G = cb.cNq;
  std::vector<double> DV;
  if (m->affine) {
    DV.assign((size_t)Nq * Nq, 0.0);
    for (int i = 0; i < Nq; ++i)
      for (int a = 0; a < Nq; ++a) {
        double acc = 0;
        for (int l = 0; l < Nq; ++l) acc += cb.Dmodal[(size_t)i * Nq + l] * cb.invV[(size_t)l * Nq + a];
        DV[(size_t)i * Nq + a] = acc;
      }
  } else {
    DV.assign((size_t)G * Nq, 0.0);
    for (int i = 0; i < G; ++i)
      for (int a = 0; a < Nq; ++a) {
        double acc = 0;
        for (int l = 0; l < G; ++l) acc += cb.D[(size_t)i * G + l] * cb.I[(size_t)l * Nq + a];
        DV[(size_t)i * Nq + a] = acc;
      }
  }
  int rc = BP_SUCCESS;
  int* d_bad = nullptr;
  do {
    if ((rc = m->cubr.upload(cb.r, s))) break;
    if ((rc = m->cubw.upload(cb.w, s))) break;
    if ((rc = m->cubInterp.upload(cb.I, s))) break;
    if ((rc = m->cubD.upload(cb.D, s))) break;
    if ((rc = m->invV.upload(cb.invV, s))) break;
    if ((rc = m->cubDmodal.upload(cb.Dmodal, s))) break;
    if ((rc = m->MM.upload(cb.MM, s))) break;
    if ((rc = m->cubDV.upload(DV, s))) break;
    if (!m->affine) {
      const size_t n = (size_t)m->E * G * G * G;
      if ((rc = m->cubwJ_c.alloc(n))) break;
      if ((rc = m->cubggeo_c.alloc(6 * n))) break;
      cudaError_t ce = cudaMalloc(&d_bad, sizeof(int));
      if (ce == cudaSuccess) ce = cudaMemsetAsync(d_bad, 0, sizeof(int), s);
      if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_mesh_cubature", __FILE__, __LINE__); break; }
      if ((rc = launch_geometry_at(G, m->E, m->EX.ptr, m->EY.ptr, m->EZ.ptr, m->cubr.ptr, m->cubw.ptr,
                                   m->cubwJ_c.ptr, m->cubggeo_c.ptr, d_bad, s)))
        break;
      int bad = 0;
      ce = cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s);
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
      if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_mesh_cubature", __FILE__, __LINE__); break; }
      if (bad) { rc = fail(BP_ERROR_NUMERIC, "bp_mesh_cubature: non-positive Jacobian at a Gauss point"); break; }
    } else {
      cudaError_t ce = cudaStreamSynchronize(s);
      if (ce != cudaSuccess) { rc = cuda_fail(ce, "bp_mesh_cubature", __FILE__, __LINE__); break; }
    }
  } while (0);
  if (d_bad) cudaFree(d_bad);
  if (rc != BP_SUCCESS) {
    m->cubwJ_c.release();
    m->cubggeo_c.release();
    return rc;
  }
  m->cubNq = G;
  return BP_SUCCESS;
}

int bp_mesh_cubature_view(bp_mesh_t m, bp_cubature_view_t* v) {
  if (!m || !v) return fail(BP_ERROR_ARG, "bp_mesh_cubature_view: null pointer");
  if (!m->cubNq) return fail(BP_ERROR_ARG, "bp_mesh_cubature_view: call bp_mesh_cubature first");
  v->cubNq = m->cubNq;
  v->cubNp = m->cubNq * m->cubNq * m->cubNq;
  v->cubr = m->cubr.ptr; v->cubw = m->cubw.ptr; v->cubInterp = m->cubInterp.ptr;
  v->cubD = m->affine ? m->cubDmodal.ptr : m->cubD.ptr;
  v->invV = m->invV.ptr; v->MM = m->MM.ptr;
  v->cubwJ = m->cubwJ(); v->cubggeo = m->cubggeo();
  return BP_SUCCESS;
}

int bp_mesh_write_vtu(bp_mesh_t m, const double* xL, const char* filename) {
  if (!m || !xL || !filename) return fail(BP_ERROR_ARG, "bp_mesh_write_vtu: null pointer");
  if (m->dim == 2 || m->simplex) return fail(BP_ERROR_ARG, "bp_mesh_write_vtu: Hex3D meshes only");
  const int Nq = m->Nq, Np = m->Np, E = m->E, Nf = m->Nfields, N = m->N;
  std::vector<double> EX((size_t)8 * E), EY((size_t)8 * E), EZ((size_t)8 * E), z(Nq);
  BP_CUDA_TRY(cudaMemcpy(EX.data(), m->EX.ptr, sizeof(double) * EX.size(), cudaMemcpyDeviceToHost));
  BP_CUDA_TRY(cudaMemcpy(EY.data(), m->EY.ptr, sizeof(double) * EY.size(), cudaMemcpyDeviceToHost));
  BP_CUDA_TRY(cudaMemcpy(EZ.data(), m->EZ.ptr, sizeof(double) * EZ.size(), cudaMemcpyDeviceToHost));
  BP_CUDA_TRY(cudaMemcpy(z.data(), m->gllz.ptr, sizeof(double) * Nq, cudaMemcpyDeviceToHost));
  FILE* fp = std::fopen(filename, "w");
  if (!fp) return fail(BP_ERROR, std::string("bp_mesh_write_vtu: cannot open ") + filename);
  // VTK XML unstructured grid (the reference's mesh_t::PlotFields3D,
  // libs/mesh/meshPlotFields3D.cpp:31-113): every element's GLL nodes are
  // points, each sub-cube of the node lattice is cut into six tetrahedra along
  // its main diagonal
  const int ncell = 6 * N * N * N;
  std::fprintf(fp, "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"BigEndian\">\n");
  std::fprintf(fp, "  <UnstructuredGrid>\n");
  std::fprintf(fp, "    <Piece NumberOfPoints=\"%d\" NumberOfCells=\"%d\">\n", E * Np, E * ncell);
  std::fprintf(fp, "      <Points>\n");
  std::fprintf(fp, "        <DataArray type=\"Float32\" NumberOfComponents=\"3\" Format=\"ascii\">\n");
  for (int e = 0; e < E; ++e)
    for (int k = 0; k < Nq; ++k)
      for (int j = 0; j < Nq; ++j)
        for (int i = 0; i < Nq; ++i)
          std::fprintf(fp, "       %g %g %g\n", trilinear(&EX[8 * (size_t)e], z[i], z[j], z[k]),
                       trilinear(&EY[8 * (size_t)e], z[i], z[j], z[k]), trilinear(&EZ[8 * (size_t)e], z[i], z[j], z[k]));
  std::fprintf(fp, "        </DataArray>\n");
  std::fprintf(fp, "      </Points>\n");
  std::fprintf(fp, "      <PointData Scalars=\"scalars\">\n");
  std::fprintf(fp, "        <DataArray type=\"Float32\" Name=\"Fields\" NumberOfComponents=\"%d\" Format=\"ascii\">\n",
               Nf);
  for (int e = 0; e < E; ++e)
    for (int n = 0; n < Np; ++n) {
      std::fprintf(fp, "       ");
      for (int f = 0; f < Nf; ++f) std::fprintf(fp, "%g ", xL[((size_t)e * Nf + f) * Np + n]);
      std::fprintf(fp, "\n");
    }
  std::fprintf(fp, "       </DataArray>\n");
  std::fprintf(fp, "     </PointData>\n");
  std::fprintf(fp, "    <Cells>\n");
  std::fprintf(fp, "      <DataArray type=\"Int32\" Name=\"connectivity\" Format=\"ascii\">\n");
  // the six tetrahedra of a sub-cube: the lattice paths from its low corner to
  // its high corner, one per order of the three axes; for an odd order the
  // second and third vertices are swapped so every tetrahedron has positive
  // orientation in reference coordinates
  static const int kAxisOrder[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {0, 2, 1}, {1, 0, 2}, {2, 1, 0}};
  for (int e = 0; e < E; ++e)
    for (int c = 0; c < N; ++c)
      for (int b = 0; b < N; ++b)
        for (int a = 0; a < N; ++a)
          for (int o = 0; o < 6; ++o) {
            int off[3] = {a, b, c}, id[4];
            for (int v = 0; v < 4; ++v) {
              if (v > 0) off[kAxisOrder[o][v - 1]] += 1;
              id[v] = e * Np + off[0] + off[1] * Nq + off[2] * Nq * Nq;
            }
            if (o >= 3) std::swap(id[1], id[2]);
            std::fprintf(fp, "       %d %d %d %d \n", id[0], id[1], id[2], id[3]);
          }
  std::fprintf(fp, "        </DataArray>\n");
  std::fprintf(fp, "        <DataArray type=\"Int32\" Name=\"offsets\" Format=\"ascii\">\n");
  for (int c = 1; c <= E * ncell; ++c) std::fprintf(fp, "       %d\n", 4 * c);
  std::fprintf(fp, "       </DataArray>\n");
  std::fprintf(fp, "       <DataArray type=\"Int32\" Name=\"types\" Format=\"ascii\">\n");
  for (int c = 0; c < E * ncell; ++c) std::fprintf(fp, "10\n");
  std::fprintf(fp, "        </DataArray>\n");
  std::fprintf(fp, "      </Cells>\n");
  std::fprintf(fp, "    </Piece>\n");
  std::fprintf(fp, "  </UnstructuredGrid>\n");
  std::fprintf(fp, "</VTKFile>\n");
  const bool ok = std::ferror(fp) == 0;
  std::fclose(fp);
  if (!ok) return fail(BP_ERROR, std::string("bp_mesh_write_vtu: write error on ") + filename);
  return BP_SUCCESS;
}

int bp_mesh_destroy(bp_mesh_t m) {
  delete m;
  return BP_SUCCESS;
}

}  // extern "C"
