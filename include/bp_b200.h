/*
 * bp_b200.h -- C ABI of the B200-native BK/BP Hex3D hot path.
 *
 * The library replaces the OCCA platform layer and the OKL kernels of
 * benchParanumal for the Hex3D BK/BP path (one rank, one GPU, CUDA only).
 * Every entry point returns BP_SUCCESS (0) or a negative error code; the text
 * of the last error is available from bp_last_error().  Pointers named
 * "device" must come from bp_malloc (or any CUDA device allocation); all other
 * arrays are host memory.  The library is not thread-safe: drive it from one
 * host thread, like the reference drives OCCA.
 *
 * Reference interfaces replaced are cited as path:line relative to the
 * reference project root.
 */
#ifndef BP_B200_H
#define BP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: LIBP_SUCCESS / LIBP_ERROR (include/utils.hpp:47-48) plus detail. */
#define BP_SUCCESS 0
#define BP_ERROR -1            /* generic failure (LIBP_ABORT)                      */
#define BP_ERROR_ARG -2        /* invalid argument or unsupported configuration    */
#define BP_ERROR_CUDA -3       /* a CUDA runtime call failed                        */
#define BP_ERROR_ALLOC -4      /* device or pinned-host allocation failed           */
#define BP_ERROR_NUMERIC -5    /* non-positive Jacobian, CG breakdown, NaN          */
#define BP_ERROR_TIMEOUT -6    /* a bounded device-side wait gave up                */

typedef void* bp_stream_t;     /* cudaStream_t; NULL = the library's default stream */
typedef void* bp_event_t;      /* cudaEvent_t                                       */

/* Text of the most recent error (empty string when none).
   Replaces the message carried by libp::exception (libs/core/exception.cpp:78-90). */
const char* bp_last_error(void);

/* Library version string. */
const char* bp_version(void);

/* ---------------------------------------------------------------------------
 * Platform: device, memory, streams, timing.
 * Replaces platform_t (include/platform.hpp:61-185), platform_t::malloc /
 * hostMalloc (platform.hpp:99-144), deviceMemory<T>::copyFrom/copyTo
 * (include/memory.hpp:288-464), platform.finish() (platform.hpp:161-163).
 * ------------------------------------------------------------------------- */

/* "-m CUDA -d id" device selection (libs/core/platformDeviceConfig.cpp:63-101). */
int bp_platform_init(int device_id);
int bp_device_count(int* count);
/* Name and SM count of the current device. */
int bp_device_info(char* name, size_t name_len, int* sm_count);

int bp_malloc(void** device_ptr, size_t bytes);
int bp_free(void* device_ptr);
int bp_host_malloc(void** host_ptr, size_t bytes);       /* pinned host memory */
int bp_host_free(void* host_ptr);
int bp_memcpy_htod(void* device_dst, const void* host_src, size_t bytes, bp_stream_t stream);
int bp_memcpy_dtoh(void* host_dst, const void* device_src, size_t bytes, bp_stream_t stream);
int bp_memcpy_dtod(void* device_dst, const void* device_src, size_t bytes, bp_stream_t stream);
int bp_memset(void* device_ptr, int value, size_t bytes, bp_stream_t stream);

int bp_stream_create(bp_stream_t* stream);
int bp_stream_destroy(bp_stream_t stream);
/* platform.finish(): wait for all work on the stream. */
int bp_finish(bp_stream_t stream);
int bp_event_create(bp_event_t* event);
int bp_event_destroy(bp_event_t event);
int bp_event_record(bp_event_t event, bp_stream_t stream);
int bp_event_elapsed_ms(bp_event_t start, bp_event_t end, float* ms);

/* ---------------------------------------------------------------------------
 * Device kernels.  Each replaces one OKL kernel with the same argument
 * meaning; compile-time OKL defines (p_N, p_Nfields, affine) become fields of
 * bp_ax_desc_t.  Index arrays are int32 (dlong, include/types.h:59-63).
 * ------------------------------------------------------------------------- */

typedef struct bp_ax_desc {
  int32_t bp;        /* benchmark problem 1..6; odd: Nfields 1, even: Nfields 3;
                        bp_ax_hex3d takes 5/6, bp_ax_cub_hex3d 1..4               */
  int32_t N;         /* polynomial degree 1..15 (p_N)                             */
  int32_t affine;    /* 1: per-element factors (bp5AxAffineHex3D)                 */
  int32_t Nfields;   /* 1 or 3 (p_Nfields); Quad2D BP6: 2 (Nfields = dim)          */
  int32_t dim;       /* 0 or 3: Hex3D; 2: Quad2D (bp 5/6 only: bp5AxQuad2D,
                        bp5AxAffineQuad2D, bp6AxQuad2D of okl/; ggeo holds
                        G00, G01, G11 per node, or per element when affine)     */
} bp_ax_desc_t;

/* Element-local stiffness + lambda*mass operator, Aq[e] = A_e q[GlobalToLocal].
   Replaces bp5AxHex3D (okl/bp5AxHex3D.okl:415-569, :50-185),
   bp5AxAffineHex3D (okl/bp5AxAffineHex3D.okl:419-579) and the BP6 variants
   (okl/bp6AxHex3D.okl:50-255).  Argument order follows the OKL signature
   (okl/bp5AxHex3D.okl:415-427) minus the unused vgeo, S and MM.
   ggeo: non-affine [E*Np*6] node-major G00,G01,G02,G11,G12,G22 with the GLL
   weights folded in, wJ [E*Np]; affine ggeo [E*6], wJ [E] (weights applied in
   the kernel from gllw).  D: [Nq*Nq] row-major, D[i*Nq+m] = l_m'(r_i).
   q: gathered vector; Aq: E-vector [E*Np*Nfields], layout e*Np*Nf + f*Np + n. */
int bp_ax_hex3d(const bp_ax_desc_t* desc, int32_t Nelements, const int32_t* elementList,
                const int32_t* GlobalToLocal, const double* wJ, const double* ggeo,
                const double* gllw, const double* D, double lambda, const double* q,
                double* Aq, bp_stream_t stream);

/* Tri2D affine stiffness + lambda*mass operator, Aq[e] = A_e q[GlobalToLocal]
   with A_e = G00 Srr + G01 Srs + G11 Sss + lambda J MM.  Replaces
   bp5AxAffineTri2D (okl/bp5AxAffineTri2D.okl:27-89); argument order follows its
   signature minus the unused vgeo, gllw and D.  desc: bp 5, N 1..15, affine 1,
   Nfields 1, dim 2.  wJ [E] (J), ggeo [E*3] (G00, G01, G11), S [3*Np*Np] and
   MM [Np*Np] as in bp_mesh_view_t (node-fastest); Aq [E*Np]. */
int bp_ax_tri2d(const bp_ax_desc_t* desc, int32_t Nelements, const int32_t* elementList,
                const int32_t* GlobalToLocal, const double* wJ, const double* ggeo, const double* S,
                const double* MM, double lambda, const double* q, double* Aq, bp_stream_t stream);

/* Tet3D affine stiffness + lambda*mass operator, A_e = sum_ab G_ab S_ab +
   lambda J MM over ab = rr, rs, rt, ss, st, tt.  Replaces bp5AxAffineTet3D
   (okl/bp5AxAffineTet3D.okl); desc: bp 5, N 1..15, affine 1, Nfields 1, dim 3.
   wJ [E], ggeo [E*6], S [6*Np*Np] and MM [Np*Np] as in bp_mesh_view_t. */
int bp_ax_tet3d(const bp_ax_desc_t* desc, int32_t Nelements, const int32_t* elementList,
                const int32_t* GlobalToLocal, const double* wJ, const double* ggeo, const double* S,
                const double* MM, double lambda, const double* q, double* Aq, bp_stream_t stream);

/* The same operator in FP32 (the inner operator of the mixed-precision CG):
   all arrays FP32, dot products of the CG stay FP64.  No counterpart in the
   reference (dfloat is FP64 there, include/types.h:31-39). */
int bp_ax_hex3d_f32(const bp_ax_desc_t* desc, int32_t Nelements, const int32_t* elementList,
                    const int32_t* GlobalToLocal, const float* wJ, const float* ggeo, const float* gllw,
                    const float* D, float lambda, const float* q, float* Aq, bp_stream_t stream);
/* The FP32 operator on nrhs (1, 2 or 4) right-hand sides at once: q and Aq hold
   nrhs consecutive floats per gathered row / local node (system k at offset k),
   so the index and factor traffic is shared by the systems.  One field, stored
   factors.  No counterpart in the reference (one vector per Operator call). */
int bp_ax_hex3d_f32_multi(const bp_ax_desc_t* desc, int32_t nrhs, int32_t Nelements, const int32_t* elementList,
                          const int32_t* GlobalToLocal, const float* wJ, const float* ggeo, const float* gllw,
                          const float* D, float lambda, const float* q, float* Aq, bp_stream_t stream);
/* GlobalToLocal with owner marks for the fused CG step below: ownerMap[n] =
   GlobalToLocal[n], with BP_OWNER_BIT added on the first local node (the first
   column of its CSR row) of every gathered row; masked entries stay -1.
   Needs Ngather < BP_OWNER_BIT.  ownerMap may equal GlobalToLocal (in place).
   No counterpart in the reference. */
#define BP_OWNER_BIT (1 << 30)
int bp_ogs_owner_map(int32_t NL, const int32_t* GlobalToLocal, int32_t Ngather, const int32_t* rowStarts,
                     const int32_t* colIds, int32_t* ownerMap, bp_stream_t stream);

/* One CG step's direction update fused into the stored-factor element operator
   (the TMA-staged form: even Nq, stored factors).  For every system k of nrhs
   (FP64: 1; FP32: 1, 2 or 4 packed as in bp_ax_hex3d_f32_multi), at every
   gathered node g:
     p_new[g] = z[g] + beta[k] p_old[g],  z = invD .* r (r if invD is NULL),
                or p_new = z where beta[k] == 0 (the first step);
     x[g]    += alpha[k] p_old[g]          (skipped where alpha[k] == 0);
   and Aq = A_e p_new[GlobalToLocal] element by element, with the block sums of
   p_new.Aq per system in pAp_partials[k * nblocks + b] (nblocks <= Nelements).
   It replaces the pair linAlg axpy (p = r + beta p, libs/core/linearSolverCG.cpp:
   105-107) + Operator(p, Ap) (:109-110, BP/BP5/src/bp5Operator.cpp:29-85) of the
   reference's iteration, and takes over the x update of its UpdateCG
   (:131-156), one step later, so p, r, invD and x are read in the pass over the
   factors that the operator makes anyway;
   ownerMap comes from bp_ogs_owner_map.  p_new must not alias p_old; the
   gathered vectors (r, invD, p_old, p_new, x) are read and written at unmasked
   nodes only, so a mesh whose nodes are all masked may pass NULL.  Returns
   BP_ERROR_ARG where the TMA form does not cover desc. */
int bp_cg_direction_ax_hex3d(const bp_ax_desc_t* desc, int32_t Nelements, const int32_t* elementList,
                             const int32_t* ownerMap, const double* wJ, const double* ggeo, const double* D,
                             double lambda, double alpha, double beta, const double* r, const double* invD,
                             const double* p_old, double* p_new, double* x, double* Aq, double* pAp_partials,
                             bp_stream_t stream);
int bp_cg_direction_ax_f32_multi(const bp_ax_desc_t* desc, int32_t nrhs, int32_t Nelements,
                                 const int32_t* elementList, const int32_t* ownerMap, const float* wJ,
                                 const float* ggeo, const float* D, float lambda, const double* alpha,
                                 const double* beta, const float* r, const float* invD, const float* p_old,
                                 float* p_new, float* x, float* Aq, double* pAp_partials, bp_stream_t stream);

/* dst[i] = (float) src[i], i < n, device arrays (to build FP32 operands). */
int bp_convert_f64_f32(size_t n, const double* src, float* dst, bp_stream_t stream);

/* Element-local over-integrated operators of BP1-BP4 on N+2 Gauss points per
   direction, Aq[e] = A_e q[GlobalToLocal].  Replaces bp1AxHex3D / bp2AxHex3D
   (mass, okl/bp1AxHex3D.okl, okl/bp2AxHex3D.okl), bp3AxHex3D / bp4AxHex3D
   (stiffness + lambda mass, okl/bp3AxHex3D.okl:29-340, okl/bp4AxHex3D.okl) and
   their Affine variants (okl/bp1AxAffineHex3D.okl:29-135,
   okl/bp3AxAffineHex3D.okl:29-258).  Argument order follows the OKL signature
   (okl/bp3AxHex3D.okl:29-41) minus the unused S; the arrays are those of
   bp_cubature_view_t.  Curved mesh: cubwJ [E*cubNp], cubggeo [E*cubNp*6],
   cubD [cubNq^2], cubInterp [cubNq*Nq]; affine mesh: cubwJ [E], cubggeo [E*6]
   (the GLL wJ/ggeo), cubD the modal [Nq^2], invV [Nq^2] (BP3/BP4) or MM
   [Nq^2] (BP1/BP2).  Arrays a form does not use may be NULL; BP1/BP2 ignore
   lambda. */
int bp_ax_cub_hex3d(const bp_ax_desc_t* desc, int32_t Nelements, const int32_t* elementList,
                    const int32_t* GlobalToLocal, const double* cubwJ, const double* cubggeo, const double* cubD,
                    const double* cubInterp, const double* invV, const double* MM, double lambda, const double* q,
                    double* Aq, bp_stream_t stream);

/* The same over-integrated operators in FP32 (the inner operator of the
   mixed-precision CG for BP1-BP4), every array FP32. */
int bp_ax_cub_hex3d_f32(const bp_ax_desc_t* desc, int32_t Nelements, const int32_t* elementList,
                        const int32_t* GlobalToLocal, const float* cubwJ, const float* cubggeo, const float* cubD,
                        const float* cubInterp, const float* invV, const float* MM, float lambda, const float* q,
                        float* Aq, bp_stream_t stream);

/* ogs Gather(Add, Trans): gv[r] = sum over c in row r of v[colIds[c]] in column
   order.  Replaces ogsOperator_t::Gather (libs/ogs/ogsOperator.cpp:160-188) and
   the OKL gather kernel (libs/ogs/okl/ogsKernels.okl:86-122), K=1, T=double. */
int bp_ogs_gather(int32_t Nrows, const int32_t* rowStarts, const int32_t* colIds,
                  const double* v, double* gv, bp_stream_t stream);

/* ogs Scatter(NoTrans): v[colIds[c]] = gv[r] for every c in row r.
   Replaces the OKL scatter kernel (libs/ogs/okl/ogsKernels.okl:127-164). */
int bp_ogs_scatter(int32_t Nrows, const int32_t* rowStarts, const int32_t* colIds,
                   const double* gv, double* v, bp_stream_t stream);

/* linAlg_t vector kernels (libs/core/linAlg.cpp:38-89, libs/core/okl/linAlg*.okl).
   Reductions write their result to a device scalar instead of a pinned host
   buffer, so no host synchronisation is implied. */
int bp_linalg_set(int32_t N, double alpha, double* x, bp_stream_t stream);
int bp_linalg_axpy(int32_t N, double alpha, const double* x, double beta, double* y,
                   bp_stream_t stream);
int bp_linalg_inner_prod(int32_t N, const double* x, const double* y, double* result,
                         bp_stream_t stream);
int bp_linalg_norm2(int32_t N, const double* x, double* result, bp_stream_t stream);

/* cg::UpdateCG first half (libs/core/linearSolverCG.cpp:131-156,
   libs/core/okl/linearSolverUpdateCG.okl:29-103): r <- r - alpha Ap and
   rdotr <- r.r, written to a device scalar. */
int bp_update_cg(int32_t N, const double* Ap, double alpha, double* r, double* rdotr,
                 bp_stream_t stream);

/* The BP5/BP6 operator, Aq = Gather(A_e q[GlobalToLocal]), without any device
   allocation.  No counterpart in the reference: it exists for callers that
   cannot call cudaMalloc -- an application whose own pool allocator owns the
   device memory budget, or a pipeline that cannot accept the device-wide
   synchronisation that cudaMalloc/cudaFree imply.  The element-local results
   live in a fixed 8 MiB array inside the library image (every GPU that loads
   the library holds it until the process exits).
   Nlocal is the length of the element-local vector that elementList and the
   CSR index: the mesh's total element count times Np*Nfields.  It may not
   exceed BP_NOALLOC_MAX_LOCAL; larger meshes are rejected with BP_ERROR_ARG
   (use bp_solver_operator for them).  elementList may name any subset of the
   mesh's elements (entries below Nlocal/(Np*Nfields)); every colIds entry must
   be below Nlocal.  Before launching the operator the call checks every
   element id, row start and column index on the device and waits for that
   check (a synchronisation of `stream`, no allocation): an index out of range
   returns BP_ERROR_ARG and touches nothing.  Elements left out of a partial
   list contribute zero: the call clears the first Nlocal entries of the
   array before the element operator writes.
   The first call on a device looks up the array's device address with that
   device current; make that first call before any stream capture.  All calls
   share the one array, so calls that overlap on the GPU -- on different
   streams, or from several host threads -- race with each other.  Arguments
   are those of bp_ax_hex3d plus Nlocal and the gather's CSR (Ngather,
   rowStarts [Ngather+1], colIds); q [Ngather] in, Aq [Ngather] out, both
   device memory. */
#define BP_NOALLOC_MAX_LOCAL (1 << 20)
int bp_operator_hex3d_noalloc(const bp_ax_desc_t* desc, int32_t Nelements, const int32_t* elementList,
                              const int32_t* GlobalToLocal, const double* wJ, const double* ggeo,
                              const double* gllw, const double* D, double lambda, int32_t Nlocal,
                              int32_t Ngather, const int32_t* rowStarts, const int32_t* colIds,
                              const double* q, double* Aq, bp_stream_t stream);

/* ---------------------------------------------------------------------------
 * Mesh and masked gather-scatter setup.  Replaces mesh_t::Setup for the Hex3D
 * box (libs/mesh/meshSetup.cpp:31-85, meshSetupBoxHex3D.cpp:31-131,
 * meshGeometricFactorsHex3D.cpp:31-153), mesh_t::MaskedGatherScatterSetup
 * (libs/mesh/meshMaskedGatherScatterSetup.cpp:31-77), ogs_t::Setup
 * (libs/ogs/ogsSetup.cpp:87-290) and ogs_t::SetupGlobalToLocalMapping
 * (libs/ogs/ogsSetup.cpp:833-849).  All arrays live on the device.
 * ------------------------------------------------------------------------- */

typedef struct bp_mesh_s* bp_mesh_t;

typedef struct bp_box_desc {
  int32_t nx, ny, nz;   /* -nx -ny -nz: elements per direction                    */
  int32_t N;            /* -p: degree 1..15                                        */
  int32_t affine;       /* -a                                                      */
  int32_t Nfields;      /* 1 (BP1/3/5) or 3 (BP2/4/6)                              */
  double pert;          /* interior vertex perturbation, fraction of h (0 = none)  */
  uint64_t pert_seed;   /* LCG seed of the perturbation                            */
  int32_t dim;          /* 0 or 3: Hex3D box nx x ny x nz (-e Hex); 2: Quad2D box
                           nx x ny (-e Quad, meshSetupBoxQuad2D.cpp:30-100; nz
                           ignored; Nfields 1 or 2)                                */
  int32_t simplex;      /* 1 with dim 2: Tri2D box (-e Tri, meshSetupBoxTri2D.cpp:
                           30-107), two triangles per cell; 1 with dim 3: Tet3D
                           box (-e Tet, meshSetupBoxTet3D.cpp), six tetrahedra
                           per cell; affine, one field, no perturbation; 0
                           otherwise                                               */
} bp_box_desc_t;

typedef struct bp_mesh_view {
  int32_t N, Nq, Np, Nelements, Nfields, affine;
  int32_t Ngather;           /* CG unknowns (masked, gathered rows)              */
  int32_t nnz;               /* unmasked local nodes (= colIds length)            */
  int64_t Nlocal;            /* E * Np * Nfields                                  */
  /* device arrays */
  const int32_t* elementList;     /* [E]                                          */
  const int32_t* GlobalToLocal;   /* [Nlocal], -1 = masked                        */
  const int32_t* rowStarts;       /* [Ngather+1]                                  */
  const int32_t* colIds;          /* [nnz]                                        */
  const double* wJ;               /* [E*Np] (affine: [E])                         */
  const double* ggeo;             /* [E*Np*6] (affine: [E*6])                     */
  const double* D;                /* [Nq*Nq]                                      */
  const double* gllz;             /* [Nq]                                         */
  const double* gllw;             /* [Nq]                                         */
  const double* EX;               /* [E*8] vertex coordinates (Quad2D: [E*4])    */
  const double* EY;
  const double* EZ;               /* NULL for Quad2D                              */
  int32_t dim;                    /* 3, or 2 for Quad2D: Np = Nq^2, ggeo [E*Np*3]
                                     (affine [E*3]), G00, G01, G11               */
  int32_t simplex;                /* 1: Tri2D (dim 2): Np = (N+1)(N+2)/2, affine:
                                     wJ [E], ggeo [E*3] G00, G01, G11; EX, EY
                                     [E*3]; D [2*Np*Np] Dr, Ds.  Tet3D (dim 3):
                                     Np = (N+1)(N+2)(N+3)/6, ggeo [E*6] G00, G01,
                                     G02, G11, G12, G22; EX, EY, EZ [E*4]; D
                                     [3*Np*Np].  gllz, gllw NULL               */
  const double* S;                /* simplex: Srr, Srs, Sss [3*Np*Np] (Tri2D) or
                                     Srr, Srs, Srt, Sss, Sst, Stt [6*Np*Np]
                                     (Tet3D); X[k*Np + n] is the weight of node k
                                     in output n (the layout of the reference's
                                     o_S, o_D); else NULL                       */
  const double* MM;               /* simplex: mass matrix [Np*Np] (symmetric)     */
} bp_mesh_view_t;

int bp_mesh_create(const bp_box_desc_t* desc, bp_mesh_t* mesh);

/* Host-only pieces of the same setup (no device needed).
   bp_box_numbering: the masked gathered numbering of the box
   (ogsSetup.cpp:492-579 EnumerateGatherGroups + :833-849
   SetupGlobalToLocalMapping).  Call with NULL arrays to get Ngather and nnz,
   then with GlobalToLocal [E*Np*Nfields], rowStarts [Ngather+1], colIds [nnz].
   bp_basis_gll: GLL nodes z, weights w [N+1] and D [(N+1)^2]
   (meshBasis1D.cpp:218-264 JacobiGLL, :114-136 Dmatrix1D).
   bp_box_vertices: vertex coordinates EX/EY/EZ [E*8] with the seeded
   perturbation (meshSetupBoxHex3D.cpp:31-131). */
/* Cubature data of the BP1-BP4 operators (device arrays), filled by
   bp_mesh_cubature.  Replaces mesh_t::CubatureSetupHex3D
   (libs/mesh/meshCubatureSetupHex3D.cpp:31-258). */
typedef struct bp_cubature_view {
  int32_t cubNq, cubNp;     /* N+2 Gauss points per direction, cubNq^3          */
  const double* cubr;       /* [cubNq] Gauss points                              */
  const double* cubw;       /* [cubNq] Gauss weights                             */
  const double* cubInterp;  /* [cubNq*Nq] GLL -> Gauss interpolation             */
  const double* cubD;       /* curved [cubNq^2] on the Gauss points; affine the
                               modal invV*Vr [Nq^2]                              */
  const double* invV;       /* [Nq^2] inverse orthonormal-Legendre Vandermonde   */
  const double* MM;         /* [Nq^2] exact GLL mass matrix                      */
  const double* cubwJ;      /* curved [E*cubNp] J*w_i*w_j*w_k; affine = wJ [E]   */
  const double* cubggeo;    /* curved [E*cubNp*6]; affine = ggeo [E*6]           */
} bp_cubature_view_t;

/* Set up (once; later calls return at once) the cubature of a mesh: the 1D
   data and, for a curved mesh, the factors at the Gauss points
   (7*8*E*cubNp bytes of device memory). */
int bp_mesh_cubature(bp_mesh_t mesh);
int bp_mesh_cubature_view(bp_mesh_t mesh, bp_cubature_view_t* view);

/* Host-only Tri2D reference element of degree N (meshReferenceNodesTri2D.cpp:
   31-52, meshBasisTri2D.cpp): warp & blend nodes r, s [Np]; D [2*Np*Np] (Dr, Ds),
   MM [Np*Np], S [3*Np*Np] (Srr, Srs, Sss), node-fastest as in bp_mesh_view_t.
   Np = (N+1)(N+2)/2; any pointer may be NULL. */
int bp_basis_tri2d(int32_t N, double* r, double* s, double* D, double* MM, double* S);
/* Host-only Tet3D reference element of degree N (meshReferenceNodesTet3D.cpp,
   meshBasisTet3D.cpp): warp & blend nodes r, s, t [Np]; D [3*Np*Np] (Dr, Ds,
   Dt), MM [Np*Np], S [6*Np*Np] (Srr, Srs, Srt, Sss, Sst, Stt), node-fastest.
   Np = (N+1)(N+2)(N+3)/6; any pointer may be NULL. */
int bp_basis_tet3d(int32_t N, double* r, double* s, double* t, double* D, double* MM, double* S);

/* Host-only 1D cubature data for degree N (meshCubatureSetupHex3D.cpp:31-51,
   meshBasis1D.cpp JacobiGQ / InterpolationMatrix1D / Dmatrix1D / MassMatrix1D):
   r, w [N+2], I [(N+2)*(N+1)], D [(N+2)^2], invV, Dmodal, MM [(N+1)^2]. */
int bp_basis_cubature(int32_t N, double* r, double* w, double* I, double* D, double* invV, double* Dmodal,
                      double* MM);

int bp_box_numbering(const bp_box_desc_t* desc, int32_t* Ngather, int32_t* nnz, int32_t* GlobalToLocal,
                     int32_t* rowStarts, int32_t* colIds);
int bp_basis_gll(int32_t N, double* z, double* w, double* D);
int bp_box_vertices(const bp_box_desc_t* desc, double* EX, double* EY, double* EZ);
int bp_mesh_view(bp_mesh_t mesh, bp_mesh_view_t* view);
/* Write a host E-vector xL [E*Np*Nfields] (e.g. the solution scattered to the
   local nodes) as a VTK XML unstructured grid (ASCII) of the element nodes and
   six tetrahedra per node sub-cube: mesh_t::PlotFields3D
   (libs/mesh/meshPlotFields3D.cpp:31-113), used by the "-o" output of the BP
   drivers (BP/BP5/src/bp5Run.cpp:220-238). */
int bp_mesh_write_vtu(bp_mesh_t mesh, const double* xL, const char* filename);
int bp_mesh_destroy(bp_mesh_t mesh);

/* ---------------------------------------------------------------------------
 * Benchmark problem: operator, forcing and CG.  Replaces bp5_t::Setup /
 * Operator / Run (BP/BP5/src/bp5Setup.cpp:29-95, bp5Operator.cpp:29-85,
 * bp5Run.cpp:30-239) and cg::Solve (libs/core/linearSolverCG.cpp:62-129).
 * ------------------------------------------------------------------------- */

typedef struct bp_solver_s* bp_solver_t;

#define BP_PRECON_NONE 0
#define BP_PRECON_JACOBI 1

#define BP_PRECISION_FP64 0    /* every operation in FP64 (the reference's dfloat)       */
#define BP_PRECISION_MIXED 1   /* FP32 CG with FP64 reliable updates (extension)          */

typedef struct bp_solver_desc {
  int32_t bp;          /* 1..6; BP2/BP4/BP6 need a 3-field mesh, BP1/3/5 one field  */
  double lambda;       /* 1.0 for BP3-BP6 (BP/BP5/bp5Main.cpp:47)                   */
  int32_t precon;      /* BP_PRECON_NONE (reference) or BP_PRECON_JACOBI             */
  int32_t precision;   /* BP_PRECISION_FP64 or BP_PRECISION_MIXED                    */
} bp_solver_desc_t;

#define BP_RHS_ANALYTIC 0   /* rhsHex3D forcing (okl/rhsHex3D.okl:29-128)         */
#define BP_RHS_RANDOM 1     /* f = 2u-1 per gathered row (seeded LCG), b = M f     */

typedef struct bp_solve_stats {
  int32_t iterations;      /* cg::Solve return value (mixed: FP32 iterations)      */
  double rdotr0;           /* initial r.r                                          */
  double rdotr;            /* final r.r (mixed: of the FP64 residual b - A x)      */
  double elapsed_ms;       /* device time of the solve (CUDA events)               */
  int32_t updates;         /* mixed: FP64 residual replacements; FP64: 0           */
  int64_t kernel_launches; /* kernels launched by the solve, CUDA-graph nodes included */
} bp_solve_stats_t;

int bp_solver_create(bp_mesh_t mesh, const bp_solver_desc_t* desc, bp_solver_t* solver);
int bp_solver_destroy(bp_solver_t solver);
/* Number of CG unknowns (ogs.Ngather). */
int bp_solver_size(bp_solver_t solver, int32_t* Ngather);
/* solver_t::Operator (include/solver.hpp:47-49): Aq = Gather(A_e q[G2L]). */
int bp_solver_operator(bp_solver_t solver, const double* q, double* Aq, bp_stream_t stream);
/* Forcing then Trans-gather into the device vector b [Ngather]
   (bp5Run.cpp:53-64).  For BP_RHS_RANDOM, f_out (device, may be NULL) receives f. */
int bp_solver_rhs(bp_solver_t solver, int32_t mode, uint64_t seed, double* b, double* f_out);
/* Assembled operator diagonal (device [Ngather]), the Jacobi preconditioner's inverse. */
int bp_solver_diagonal(bp_solver_t solver, double* diag);
/* cg::Solve on device vectors: x (initial guess in, solution out) and r
   (b in, final residual out).  tol and maxit as in the reference; with the
   Jacobi preconditioner the stop rule is ||r|| <= tol ||b||.  A solver made
   with BP_PRECISION_MIXED runs the CG recursion, the operator and the stored
   factors in FP32 and replaces the FP32 residual by the FP64 residual b - A x
   (x accumulated in FP64) whenever the FP32 residual has dropped by 1e-2 since
   the last replacement; it stops on the FP64 residual, ||b - A x|| <= tol ||b||
   (tol > 0 required), and r returns that FP64 residual.  hist_rnorm and
   hist_alpha (host, length maxit, may be NULL) receive sqrt(r.r) and alpha of
   every iteration (the "-v" output).  No host synchronisation happens inside
   the iteration loop except one flag read every 20 iterations when tol > 0. */
int bp_solver_solve(bp_solver_t solver, double* x, double* r, double tol, int32_t maxit,
                    double* hist_rnorm, double* hist_alpha, bp_solve_stats_t* stats);
/* The same solve from HOST buffers: copies b (host, pinned or pageable) to the
   device, solves from x=0, copies x back to x_host.  The device time reported
   in stats covers the copies and the solve. */
int bp_solver_solve_host(bp_solver_t solver, const double* b_host, double* x_host, double tol,
                         int32_t maxit, bp_solve_stats_t* stats);

/* ---------------------------------------------------------------------------
 * Batched solves (extension; the reference solves one problem per run).
 * Many independent problems -- each its own perturbed box, degree and element
 * count -- with several right-hand sides each, solved together: every
 * (problem, rhs) pair is one CG system, and one CUDA graph launch advances
 * all systems by 20 iterations, small and large problems side by side on the
 * GPU.  Each system behaves exactly as bp_solver_solve on its own problem
 * (same kernels, same stop rules, same mixed-precision reliable updates).
 * ------------------------------------------------------------------------- */

typedef struct bp_batch_s* bp_batch_t;

typedef struct bp_batch_problem {
  int32_t nx, ny, nz;   /* elements per direction                                  */
  int32_t N;            /* degree 1..15                                             */
  double pert;          /* interior vertex perturbation, fraction of h              */
  uint64_t pert_seed;   /* LCG seed of the perturbation                             */
  int32_t nrhs;         /* right-hand sides: BP_RHS_RANDOM forcing ...              */
  uint64_t rhs_seed;    /* ... with seeds rhs_seed, rhs_seed+1, ..., +nrhs-1        */
  int32_t affine;       /* nonzero: per-element (affine) factors, as bp_box_desc_t  */
} bp_batch_problem_t;

/* Meshes, solvers (desc: bp 1, 3 or 5; preconditioner; precision) and
   right-hand sides for every system, in problem order, rhs order within a
   problem.  Each problem's mesh has stored per-node factors unless its
   affine flag is set. */
int bp_batch_create(const bp_batch_problem_t* problems, int32_t nproblems, const bp_solver_desc_t* desc,
                    bp_batch_t* batch);
int bp_batch_destroy(bp_batch_t batch);
int bp_batch_systems(bp_batch_t batch, int32_t* nsystems);
/* problem index and number of unknowns of a system (either may be NULL) */
int bp_batch_system_info(bp_batch_t batch, int32_t system, int32_t* problem, int32_t* Ngather);
/* Solve every system from x = 0 to its own stop rule (see bp_solver_solve).
   stats (host, one entry per system, may be NULL) and elapsed_ms (device
   time of the whole batch, may be NULL). */
int bp_batch_solve(bp_batch_t batch, double tol, int32_t maxit, bp_solve_stats_t* stats, double* elapsed_ms);
/* Device pointers of a system's solution x and right-hand side b [Ngather]. */
int bp_batch_vectors(bp_batch_t batch, int32_t system, double** x, double** b);
/* The solver object of a system (owned by the batch), e.g. for bp_solver_operator. */
int bp_batch_solver(bp_batch_t batch, int32_t system, bp_solver_t* solver);

/* ---------------------------------------------------------------------------
 * Drivers: the BK/BP executables' main() with the reference's command-line
 * keys (libs/core/platformSettings.cpp:31-50, libs/mesh/meshSettings.cpp:31-62,
 * BP/BP5/src/bp5Settings.cpp:30-46) and result line (bp5Run.cpp:208-217,
 * BK/BK5/src/bk5Run.cpp:186-194).  name is "BP5" or "BK5".
 * ------------------------------------------------------------------------- */
int bp_driver_main(const char* name, int argc, char** argv);

/* ---------------------------------------------------------------------------
 * Kernel-form autotuner (extension: the reference picks its OKL variant by a
 * compile-time rule on the degree, okl/bp5AxHex3D.okl:27-41).  The element
 * operator has several forms; the first launch of a configuration outside a
 * stream capture times every applicable form on the caller's operands (one
 * untimed and three timed launches each) and keeps the fastest for that
 * configuration and element-count class (floor(log2(Nelements))) on the
 * device.  Solvers launch their operator once before capturing their graphs.
 * While a stream captures, an untuned configuration takes the measured static
 * choice.  BP_AUTOTUNE=0 in the environment keeps the static choice.
 * ------------------------------------------------------------------------- */
#define BP_FORM_MMA 0     /* tensor-core MMA (affine Nq = 16; packed Nq = 8) */
#define BP_FORM_TMA 1     /* TMA-staged register pencils (stored factors, even Nq) */
#define BP_FORM_LINE 2    /* line-per-thread */
#define BP_FORM_PENCIL 3  /* register pencil */

/* The form chosen for a configuration (-1 when not tuned yet) and the forms
   measured with their times in ms (up to cap entries).  kind 0: one value per
   node (precision_bytes 8 or 4); kind 1: `lanes` packed FP32 right-hand sides.
   fused: 1 for the CG launches that also form p.Ap. */
int bp_tune_report(int32_t kind, int32_t N, int32_t Nfields, int32_t affine, int32_t precision_bytes, int32_t lanes,
                   int32_t fused, int32_t Nelements, int32_t* form, int32_t* nforms, int32_t* forms, float* ms,
                   int32_t cap);
/* Forget every tuned choice (the next launches measure again). */
int bp_tune_reset(void);

/* ---------------------------------------------------------------------------
 * Validation and failure detection.
 * ------------------------------------------------------------------------- */

/* Host-side check of a masked numbering handed in from outside (for example
   the reference's own mesh_t / ogs_t set-up, libs/ogs/ogsSetup.cpp:492-579,
   833-849): every GlobalToLocal entry in [-1, Ngather); rowStarts starting at
   0, non-decreasing, ending at the number of unmasked local nodes; every row
   non-empty; and row r's colIds exactly the local indices l with
   GlobalToLocal[l] == r, ascending.  All arrays are HOST memory.  Returns
   BP_ERROR_ARG naming the first index that breaks a rule, without touching a
   device.  No counterpart in the reference, which trusts its own set-up. */
int bp_ogs_check(int64_t Nlocal, const int32_t* GlobalToLocal, int32_t Ngather, const int32_t* rowStarts,
                 const int32_t* colIds);

/* Test hook for the bounded device-side waits: one element of the FP64
   stored-factor operator at degree 7 through a kernel instantiation whose
   producer arms the mbarrier of slice `withhold_slice` (0, 3, 5 or 7) but
   issues none of its bulk copies, so the consumers' wait runs out after a
   short limit (about a millisecond) with nothing in flight; -1 runs the
   product kernel.  Returns the library's device error status: BP_ERROR_TIMEOUT
   when a wait gave up (the status is then cleared and the context stays
   usable), BP_SUCCESS otherwise.  Allocates its own small buffers. */
int bp_test_wait_timeout(int withhold_slice);

#ifdef __cplusplus
}
#endif

#endif /* BP_B200_H */
