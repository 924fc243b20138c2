// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bp_b200.h"

namespace bp {

// ---- error state (libp::exception / LIBP_ABORT replacement) ----
void set_error(const std::string& msg);
void clear_error();
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t err, const char* what, const char* file, int line);

#define BP_CUDA_TRY(call)                                                   \
  do {                                                                      \
    cudaError_t bp_err_ = (call);                                           \
    if (bp_err_ != cudaSuccess) return bp::cuda_fail(bp_err_, #call, __FILE__, __LINE__); \
  } while (0)

#define BP_TRY(call)                    \
  do {                                  \
    int bp_rc_ = (call);                \
    if (bp_rc_ != BP_SUCCESS) return bp_rc_; \
  } while (0)

// ---- per-device state ----
// Every cache of device-side state (symbol addresses, function attributes,
// scratch buffers, the default stream) is kept per device: a process may
// switch devices with bp_platform_init, and each device has its own copy of
// the library image.
constexpr int kMaxDevices = 64;
int current_device(int* dev);   // BP_SUCCESS, or an error for an ordinal >= kMaxDevices

// Runs `init` once per device (the current one), serialised by a lock; a
// failed `init` is not recorded, so the next call retries it.
struct DeviceOnce {
  std::atomic<uint64_t> done{0};
  std::mutex m;
};
template <class Fn>
int once_per_device(DeviceOnce& o, Fn&& init) {
  int dev = 0;
  BP_TRY(current_device(&dev));
  const uint64_t bit = uint64_t(1) << dev;
  if (o.done.load(std::memory_order_acquire) & bit) return BP_SUCCESS;
  std::lock_guard<std::mutex> lock(o.m);
  if (o.done.load(std::memory_order_relaxed) & bit) return BP_SUCCESS;
  BP_TRY(init());
  o.done.fetch_or(bit, std::memory_order_release);
  return BP_SUCCESS;
}

// The device address of a __device__ or __constant__ symbol on the current
// device, looked up on first use per device.  Host code may not use the
// symbol itself as a device address: it names a host-side shadow.
class DeviceSymbol {
 public:
  explicit DeviceSymbol(const void* symbol) : symbol_(symbol) {}
  void* address();   // nullptr (error text set) when the lookup fails
 private:
  const void* symbol_;
  std::atomic<void*> addr_[kMaxDevices] = {};
};

// the library's default stream on the current device (created on first use)
cudaStream_t default_stream();
inline cudaStream_t to_stream(bp_stream_t s) {
  return s ? reinterpret_cast<cudaStream_t>(s) : default_stream();
}
int sm_count();   // multiprocessors of the current device

// Copies `bytes` of device memory `src` into the constant-bank slot `dst` on
// stream s.  Inside a stream capture, a copy of the same source into the same
// slot already captured on the same stream in the same capture is still in
// effect (stream order), so it is not captured again: a CUDA graph of many CG
// iterations holds one copy per slot rather than one per operator launch (and
// its kernels stay adjacent for programmatic dependent launch).  Outside
// captures every call copies.
int const_slot_copy(void* dst, const void* src, size_t bytes, cudaStream_t s);

// Programmatic dependent launch for the kernels of a CG iteration: launched
// with launch_pdl, a kernel may be scheduled while its predecessor on the
// stream finishes.  Every such kernel calls pdl_wait() before it reads
// anything (it returns once the predecessor has completed and its memory is
// visible; at once for a kernel launched without the attribute) and
// pdl_release() to let its own successor be scheduled.  BP_PDL=0, read once,
// launches without the attribute.
bool pdl_enabled();
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}
#endif

// ---- device buffer owned by the library ----
template <class T>
struct DeviceArray {
  T* ptr = nullptr;
  size_t n = 0;
  DeviceArray() = default;
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  ~DeviceArray() { release(); }
  int alloc(size_t count) {
    release();
    n = count;
    if (count == 0) return BP_SUCCESS;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&ptr), count * sizeof(T));
    if (e != cudaSuccess) {
      ptr = nullptr;
      n = 0;
      return fail(BP_ERROR_ALLOC, std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) +
                                      " bytes failed: " + cudaGetErrorString(e));
    }
    return BP_SUCCESS;
  }
  int upload(const std::vector<T>& h, cudaStream_t s) {
    BP_TRY(alloc(h.size()));
    if (!h.empty()) BP_CUDA_TRY(cudaMemcpyAsync(ptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    return BP_SUCCESS;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    n = 0;
  }
};

// ---- host-side mesh description produced by the setup code ----
struct HostMesh {
  int N = 0, Nq = 0, Np = 0, nx = 0, ny = 0, nz = 0, E = 0, affine = 0, Nfields = 1;
  int dim = 3;                           // 2: Quad2D (Np = Nq^2, 4 vertices, 3 factors)
  std::vector<double> gllz, gllw, D;
  std::vector<double> EX, EY, EZ;        // E*8 (perturbed vertices)
  int32_t Ngather = 0, nnz = 0;
  std::vector<int32_t> G2L;              // E*Np*Nf
  std::vector<int32_t> rowStarts;        // Ngather+1
  std::vector<int32_t> colIds;           // nnz
};

// basis (GLL nodes by Newton iteration, lumped weights, differentiation matrix)
void gll_nodes_weights(int N, std::vector<double>& z, std::vector<double>& w);
void diff_matrix(const std::vector<double>& z, std::vector<double>& D);
// Gauss-Legendre points and weights (n points)
void gauss_nodes_weights(int n, std::vector<double>& r, std::vector<double>& w);
// 1D data of the over-integrated (BP1-BP4) operators
struct CubBasis {
  int cNq = 0;                        // N+2 Gauss points
  std::vector<double> r, w;           // Gauss points and weights [cNq]
  std::vector<double> I;              // GLL -> Gauss interpolation [cNq*Nq]
  std::vector<double> D;              // differentiation on the Gauss points [cNq*cNq]
  std::vector<double> invV;           // inverse orthonormal Legendre Vandermonde on GLL [Nq*Nq]
  std::vector<double> Dmodal;         // invV * Vr [Nq*Nq]
  std::vector<double> MM;             // exact GLL mass matrix [Nq*Nq]
};
void cubature_basis(int N, const std::vector<double>& gllz, CubBasis& cb);
// box vertices with optional seeded interior perturbation
void box_vertices(HostMesh& m, double pert, uint64_t seed);
// masked gathered numbering, CSR and GlobalToLocal for the box
void box_numbering(HostMesh& m);
// the same for the Quad2D box (dim 2): vertices [E*4], numbering, and the
// geometric factors at the GLL nodes (wJ, ggeo = G00, G01, G11 with the weights
// folded in; affine: per element, without weights).  quad_geometry returns
// false on a Jacobian below 1e-8 (the reference's check).
void box_vertices_2d(HostMesh& m, double pert, uint64_t seed);
void box_numbering_2d(HostMesh& m);
bool quad_geometry(const HostMesh& m, std::vector<double>& wJ, std::vector<double>& ggeo);
// Tri2D (dim 2, simplex): reference-element nodes and matrices (row-major),
// and the box with its affine factors and masked numbering (HostMesh EX/EY
// hold 3 vertices per element)
struct TriBasis {
  int N = 0, Np = 0;
  std::vector<double> r, s;           // nodes [Np]
  std::vector<double> Dr, Ds, MM;     // [Np*Np]
  std::vector<double> S;              // Srr, Srs, Sss [3*Np*Np]
};
bool tri_basis(int N, TriBasis& b);
bool box_tri(HostMesh& m, const TriBasis& b, std::vector<double>& wJ, std::vector<double>& ggeo);
// physical node coordinates of the Tri2D box [E*Np] each (meshPhysicalNodesTri2D.cpp)
void tri_nodes_xy(const HostMesh& m, const TriBasis& b, std::vector<double>& x, std::vector<double>& y);
// Tet3D (dim 3, simplex): reference element (r, s, t; Dr, Ds, Dt, MM; S = Srr,
// Srs, Srt, Sss, Sst, Stt, row-major) and the box of six tetrahedra per cell
// with its affine factors (wJ [E], ggeo [6E]), numbering (HostMesh EX/EY/EZ hold
// 4 vertices per element) and physical node coordinates
struct TetBasis {
  int N = 0, Np = 0;
  std::vector<double> r, s, t;
  std::vector<int> bary;              // [Np*4] lattice weights of the nodes on the vertices
  std::vector<double> Dr, Ds, Dt, MM;
  std::vector<double> S;              // [6*Np*Np]
};
bool tet_basis(int N, TetBasis& b);
bool box_tet(HostMesh& m, const TetBasis& b, std::vector<double>& wJ, std::vector<double>& ggeo,
             std::vector<double>& x, std::vector<double>& y, std::vector<double>& z);

// trilinear map of the eight hex vertices v (mesh_t vertex order) at (r,s,t)
__host__ __device__ inline double trilinear(const double* v, double r, double s, double t) {
  return 0.125 * ((1 - r) * (1 - s) * (1 - t) * v[0] + (1 + r) * (1 - s) * (1 - t) * v[1] +
                  (1 + r) * (1 + s) * (1 - t) * v[2] + (1 - r) * (1 + s) * (1 - t) * v[3] +
                  (1 - r) * (1 - s) * (1 + t) * v[4] + (1 + r) * (1 - s) * (1 + t) * v[5] +
                  (1 + r) * (1 + s) * (1 + t) * v[6] + (1 - r) * (1 + s) * (1 + t) * v[7]);
}

}  // namespace bp

// ---- the opaque objects of the C ABI ----
struct bp_mesh_s {
  int N, Nq, Np, E, Nfields, affine;
  int dim = 3;                                  // 2: Quad2D, or Tri2D when simplex
  int simplex = 0;                              // 1: Tri2D (dim 2) or Tet3D (dim 3), affine
  int32_t Ngather, nnz;
  bp::DeviceArray<int32_t> elementList, G2L, rowStarts, colIds;
  // GlobalToLocal with the owner bit (kOwnerBit) of each gathered node's first
  // local node, for operators with the fused CG direction update; built on first use
  bp::DeviceArray<int32_t> G2Lo;
  bp::DeviceArray<double> wJ, ggeo, D, gllz, gllw, EX, EY, EZ;
  // cubature of the BP1-BP4 operators (bp_mesh_cubature); cubNq = 0 until set up
  int cubNq = 0;
  bp::DeviceArray<double> cubr, cubw, cubInterp, cubD, invV, cubDmodal, MM;
  bp::DeviceArray<double> cubDV;                // derivative columns for the diagonal: cubD*cubInterp
                                                // (curved) or cubDmodal*invV (affine)
  bp::DeviceArray<double> cubwJ_c, cubggeo_c;   // curved mesh only
  // simplex: the stiffness matrices S_ab [3 or 6 Np*Np] node-fastest (X[k*Np + n]
  // weighs node k in output n); MM above holds the element mass matrix and D
  // the derivative matrices
  bp::DeviceArray<double> S;
  bp::DeviceArray<double> x, y, z;              // simplex: physical node coordinates [E*Np]
  // factors at the quadrature points: curved [E*cubNp], [6*E*cubNp]; affine the
  // per-element wJ and ggeo
  const double* cubwJ() const { return affine ? wJ.ptr : cubwJ_c.ptr; }
  const double* cubggeo() const { return affine ? ggeo.ptr : cubggeo_c.ptr; }
  // FP32 copies of the operator data for mixed-precision solvers, one set per
  // operator family (0: GLL collocation, 1: BP3/BP4 cubature, 2: BP1/BP2
  // cubature), built on first use and shared by the solvers on this mesh
  struct Fp32Ops {
    bp::DeviceArray<float> wJ, ggeo, gllw, D, T;
    bool ready = false;
  } f32[3];
};

struct bp_solver_s;

// ---- simplex elements: Tri2D (dim 2), Tet3D (dim 3) (bp_ax_simplex.cu) ----
namespace bp {
int launch_ax_simplex(int dim, int N, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                      const double* wJ, const double* ggeo, const double* S, const double* MM, double lambda,
                      const double* q, double* Aq, const int* skip, cudaStream_t s, double* partials = nullptr,
                      int* nblocks = nullptr);
int launch_ax_simplex(int dim, int N, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                      const float* wJ, const float* ggeo, const float* S, const float* MM, float lambda,
                      const float* q, float* Aq, const int* skip, cudaStream_t s, double* partials = nullptr,
                      int* nblocks = nullptr);
int launch_mass_local_simplex(int dim, int N, int32_t Nelements, const int32_t* G2L, const double* wJ,
                              const double* MM, const double* f, double* bL, cudaStream_t s);
int launch_diag_local_simplex(int dim, int N, int32_t Nelements, const double* wJ, const double* ggeo,
                              const double* S, const double* MM, double lambda, double* dL, cudaStream_t s);
int launch_rhs_analytic_simplex(int dim, int N, int32_t Nelements, const double* wJ, const double* MM,
                                const double* x, const double* y, const double* z, double lambda, double* bL,
                                cudaStream_t s);
}  // namespace bp

// ---- kernel launchers (bp_kernels.cu) ----
namespace bp {
struct CgFuse;
// element operator; with `fuse` it also produces p.Ap and alpha for CG (bp_cg_device.cuh)
int launch_ax_skip(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                   const double* wJ, const double* ggeo, const double* gllw, const double* D, double lambda,
                   const double* q, double* Aq, const int* skip, cudaStream_t s, const CgFuse* fuse = nullptr,
                   int* nblocks = nullptr);
int launch_ax_skip(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                   const float* wJ, const float* ggeo, const float* gllw, const float* D, float lambda,
                   const float* q, float* Aq, const int* skip, cudaStream_t s, const CgFuse* fuse = nullptr,
                   int* nblocks = nullptr);
int launch_ax(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
              const double* wJ, const double* ggeo, const double* gllw, const double* D, double lambda,
              const double* q, double* Aq, cudaStream_t s);
int launch_gather(int32_t Nrows, const int32_t* rowStarts, const int32_t* colIds, const double* v, double* gv,
                  cudaStream_t s);
int launch_scatter(int32_t Nrows, const int32_t* rowStarts, const int32_t* colIds, const double* gv, double* v,
                   cudaStream_t s);
// masked gathered numbering of the box on the device: GlobalToLocal, CSR row
// starts (Ngather + 1) and columns, as box_numbering computes them on the host
void box_numbering_counts(int nx, int ny, int nz, int N, int Nf, int64_t* Ngather, int64_t* nnz);
int launch_box_numbering(int nx, int ny, int nz, int N, int Nf, int32_t* G2L, int32_t* rowStarts, int32_t* colIds,
                         cudaStream_t s);
int launch_geometry(int N, int affine, int E, const double* EX, const double* EY, const double* EZ,
                    const double* gllz, const double* gllw, double* wJ, double* ggeo, int* bad, cudaStream_t s);
int launch_rhs_analytic(int N, int affine, int Nfields, int E, const double* EX, const double* EY,
                        const double* EZ, const double* gllz, const double* gllw, const double* wJ, double lambda,
                        double* rL, cudaStream_t s);
int launch_rhs_random(int32_t Ngather, uint64_t seed, double* f, cudaStream_t s);
int launch_mass_local(int N, int affine, int Nfields, int E, const int32_t* G2L, const double* gllw,
                      const double* wJ, const double* f, double* rL, cudaStream_t s);
int launch_diag_local(int N, int affine, int Nfields, int E, const double* ggeo, const double* wJ,
                      const double* gllw, const double* D, double lambda, double* dL, cudaStream_t s);
int launch_set(int32_t N, double alpha, double* x, cudaStream_t s);
int launch_d2f(size_t n, const double* a, float* b, cudaStream_t s);   // b = (float) a
int launch_axpy(int32_t N, double alpha, const double* x, double beta, double* y, cudaStream_t s);
int launch_reciprocal(int32_t N, double* x, cudaStream_t s);
int launch_sqrt1(double* v, cudaStream_t s);   // v[0] = sqrt(v[0]) on the device

// deterministic fused reductions: result[0] = sum over i of term(i)
int launch_dot(int32_t N, const double* x, const double* y, double* result, double* partials,
               unsigned int* counter, cudaStream_t s);
int launch_update_cg(int32_t N, const double* Ap, double alpha, double* r, double* result, double* partials,
                     unsigned int* counter, cudaStream_t s);

int reduction_blocks();

// TMA-staged stored-factor operator (bp_ax_tma.cu); returns 1 when the
// configuration is not covered and nothing was launched
int launch_ax_tma(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const double* wJ, const double* ggeo, const double* D, double lambda, const double* q, double* Aq,
                  const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks);
int launch_ax_tma(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const float* wJ, const float* ggeo, const float* D, float lambda, const float* q, float* Aq,
                  const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks);
// line-per-thread BP5/BP6 element operator (bp_ax_line*.cu), same arguments
// as launch_ax_skip
int launch_ax_line(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                   const double* wJ, const double* ggeo, const double* gllw, const double* D, double lambda,
                   const double* q, double* Aq, const int* skip, cudaStream_t s, const CgFuse* fuse, int* nblocks);
int launch_ax_line(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                   const float* wJ, const float* ggeo, const float* gllw, const float* D, float lambda,
                   const float* q, float* Aq, const int* skip, cudaStream_t s, const CgFuse* fuse, int* nblocks);
// over-integrated BP1-BP4 operator (bp_ax_cub*.cu).  T is the 1D transform:
// curved cubInterp [cubNq*Nq]; affine BP3/BP4 invV [Nq*Nq]; affine BP1/BP2 MM
// [Nq*Nq].  D is cubD (curved) or the modal cubD (affine BP3/BP4); unused for
// BP1/BP2.  With fuse, the block partials of q.Aq go to fuse->partials.
template <class F>
struct CubOperands {
  const F* wJ;
  const F* ggeo;
  const F* D;
  const F* T;
};
int launch_ax_cub(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const CubOperands<double>& ops, double lambda, const double* q, double* Aq, const int* skip,
                  cudaStream_t s, const CgFuse* fuse = nullptr, int* nblocks = nullptr);
int launch_ax_cub(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const CubOperands<float>& ops, float lambda, const float* q, float* Aq, const int* skip,
                  cudaStream_t s, const CgFuse* fuse = nullptr, int* nblocks = nullptr);
// element-local diagonal of the BP1-BP4 operators (DV = D*T, the derivative columns)
int launch_diag_cub(const bp_ax_desc_t& d, int32_t Nelements, const double* wJ, const double* ggeo,
                    const double* T, const double* DV, double lambda, double* dL, cudaStream_t s);
// cubature geometric factors of a curved mesh at the Gauss points
int launch_geometry_at(int Nq, int E, const double* EX, const double* EY, const double* EZ, const double* r,
                       const double* w, double* wJ, double* ggeo, int* bad, cudaStream_t s);
// the same FP32 operator on pk (2 or 4) right-hand sides packed per node; 1 when not covered
int launch_ax_tma_packed(int pk, const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList,
                         const int32_t* G2L, const float* wJ, const float* ggeo, const float* D, float lambda,
                         const float* q, float* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s,
                         int* nblocks);
// the line-per-thread FP32 operator on pk (2 or 4) packed right-hand sides (any Nq up to 12)
int launch_ax_line_packed(int pk, const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList,
                          const int32_t* G2L, const float* wJ, const float* ggeo, const float* gllw, const float* D,
                          float lambda, const float* q, float* Aq, const int* skip, const CgFuse* fuse,
                          cudaStream_t s, int* nblocks);
// affine operator on the tensor cores (bp_ax_mma.cu: DMMA in FP64, split TF32
// in FP32); returns 1 when the configuration is not covered (stored factors,
// or Nq other than 16) and nothing was launched
int launch_ax_mma(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const double* wJ, const double* ggeo, const double* gllw, const double* D, double lambda,
                  const double* q, double* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks);
int launch_ax_mma(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                  const float* wJ, const float* ggeo, const float* gllw, const float* D, float lambda,
                  const float* q, float* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks);
// ---- kernel-form autotuner (bp_tune.cu) ----
// Forms of the element operator; kind 0 = one value per node, 1 = packed lanes.
enum { FORM_MMA = 0, FORM_TMA = 1, FORM_LINE = 2, FORM_PENCIL = 3, FORM_RB = 4 };
struct TuneConfig {
  int kind, nq, nf, affine, bytes, lanes, fused;
  int ecls;   // size class: floor(log2(elements))
};
inline int element_class(int32_t E) {
  int c = 0;
  while (E > 1) {
    E >>= 1;
    ++c;
  }
  return c;
}
// The form to launch for configuration c: the tuned one once measured, else
// (while s is capturing) forms[0].  run(f) launches form f on s and returns 1
// when f does not apply.
int tuned_form(const TuneConfig& c, const std::vector<int>& forms, const std::function<int(int)>& run,
               cudaStream_t s, int* form);
// the chosen form (-1: not tuned yet) and the measured times of configuration c
int tuned_report(const TuneConfig& c, int* form, int* nforms, int* forms, float* ms, int cap);
void tuned_clear();

// Element-operator variant forced by BP_AX_VARIANT (pencil, line, tma, mma),
// else AX_AUTO: the tuned choice per configuration.
enum { AX_AUTO = 0, AX_PENCIL = 1, AX_LINE = 2, AX_MMA = 3, AX_TMA = 4, AX_RB = 5 };
int ax_variant();
// the packed FP32 operator (2 or 4 rhs per node) in its tuned form (bp_kernels.cu)
int launch_ax_packed(int pk, const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList,
                     const int32_t* G2L, const float* wJ, const float* ggeo, const float* gllw, const float* D,
                     float lambda, const float* q, float* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s,
                     int* nblocks);
// the register-blocked packed FP32 stored-factor operator (4 rhs, Nq = 8; one
// lane of four pencils per thread, bp_ax_tma.cu); 1 when not covered
int launch_ax_rb_packed(int pk, const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList,
                        const int32_t* G2L, const float* wJ, const float* ggeo, const float* D, float lambda,
                        const float* q, float* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s,
                        int* nblocks);
// the packed FP32 stored-factor operator (4 rhs) at Nq = 8 on the tensor cores;
// 1 when not covered
int launch_ax_mma_packed(int pk, const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList,
                         const int32_t* G2L, const float* wJ, const float* ggeo, const float* D, float lambda,
                         const float* q, float* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s,
                         int* nblocks);
// Quad2D forms (bp_ax_quad.cu): the BP5/BP6 element operator (FP64 and FP32;
// 1 with a fused direction update, which it does not take), the forcing, the
// lumped mass and the element diagonal
int launch_ax_quad(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                   const double* wJ, const double* ggeo, const double* gllw, const double* D, double lambda,
                   const double* q, double* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks);
int launch_ax_quad(const bp_ax_desc_t& d, int32_t Nelements, const int32_t* elementList, const int32_t* G2L,
                   const float* wJ, const float* ggeo, const float* gllw, const float* D, float lambda,
                   const float* q, float* Aq, const int* skip, const CgFuse* fuse, cudaStream_t s, int* nblocks);
int launch_rhs_analytic_quad(int N, int affine, int Nfields, int E, const double* EX, const double* EY,
                             const double* gllz, const double* gllw, const double* wJ, double lambda, double* rL,
                             cudaStream_t s);
int launch_mass_local_quad(int N, int affine, int Nfields, int E, const int32_t* G2L, const double* gllw,
                           const double* wJ, const double* f, double* rL, cudaStream_t s);
int launch_diag_local_quad(int N, int affine, int Nfields, int E, const double* ggeo, const double* wJ,
                           const double* gllw, const double* D, double lambda, double* dL, cudaStream_t s);
// whether the TMA form covers d with `lanes` values per node (1, or 2 or 4
// packed FP32 lanes); with factor arrays 16-byte aligned
bool tma_covers(const bp_ax_desc_t& d, int lanes);
// the form a CG launch of the element operator (p.Ap fused) of d takes now:
// forced by BP_AX_VARIANT, tuned, or the static choice while untuned
int ax_current_form(const bp_ax_desc_t& d, int bytes, int lanes, int32_t Nelements);
// G2Lo = G2L (NL entries) with kOwnerBit on the first column of every CSR row
int launch_owner_map(size_t NL, const int32_t* G2L, int32_t Ngather, const int32_t* rowStarts, const int32_t* colIds,
                     int32_t* G2Lo, cudaStream_t s);
// One CG step of a packed group (4 lanes) as one cooperative kernel
// (bp_cg_persist.cuh), with the TMA or the line form of the operator; 1 when
// the form does not cover d.  grid_cap limits the resident blocks.
struct GrpStepArgs;
int launch_grp_step_tma(int pk, const bp_ax_desc_t& d, const GrpStepArgs& a, int grid_cap, cudaStream_t s);
int launch_grp_step_line(int pk, const bp_ax_desc_t& d, const GrpStepArgs& a, int grid_cap, cudaStream_t s);
// the device error word set by kernels whose bounded waits gave up
int* device_error_word();
int check_device_error();
// test hook: a stored-factor launch whose slice `withhold` never arrives (bp_ax_tma.cu)
int tma_wait_test(int withhold);
}  // namespace bp
