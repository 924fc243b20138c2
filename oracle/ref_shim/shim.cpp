// Implementations behind the host-only shims (TEST INFRASTRUCTURE):
//
//  * MPI for one rank (ref_shim/mpi.h): collectives copy this rank's
//    contribution; point-to-point messages to this rank are matched by tag.
//  * Stand-ins for the LAPACK routines the reference's Hex3D basis setup calls
//    (libs/core/linAlgMatrixInverse.cpp, linAlgMatrixRightSolve.cpp,
//    linAlgMatrixEig.cpp): LU with partial pivoting for dgesv/dgetrf/dgetri
//    and cyclic Jacobi rotations for dgeev on the symmetric Golub-Welsch
//    matrix of JacobiGQ (libs/mesh/meshBasis1D.cpp:266-338).  The system
//    LAPACK the reference links (OpenBLAS, unpinned) is absent here.
//  * The three platform_t members that wrap OCCA's device setup
//    (libs/core/platformDeviceConfig.cpp, platformProperties.cpp,
//    platformBuildKernel.cpp): a host "device" and named kernels that are
//    never run.
//
// Nothing here is product code; it exists so the reference's own mesh, ogs and
// primitives sources run on the CPU and produce golden data.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "mpi.h"
#include "platform.hpp"

// ---------------------------------------------------------------------------
// MPI, one rank
// ---------------------------------------------------------------------------
namespace {

inline size_t type_bytes(MPI_Datatype t) { return (size_t)(t >> 4); }

struct Message {
  const void* sbuf = nullptr;        // Isend: the sender's buffer (valid until its wait)
  std::vector<char> copy;            // Send: a buffered copy
  void* rbuf = nullptr;              // Irecv: the receiver's buffer
  size_t bytes = 0;
  int tag = 0;
  bool is_send = false;
  bool done = false;
};
std::vector<Message> g_msgs;   // request handle = index + 1

void fail(const char* what) {
  std::fprintf(stderr, "mpi shim: %s\n", what);
  throw std::runtime_error(std::string("mpi shim: ") + what);
}

// deliver a send to a posted receive (or the reverse) when both are present
void match() {
  for (auto& s : g_msgs) {
    if (!s.is_send || s.done) continue;
    for (auto& r : g_msgs) {
      if (r.is_send || r.done || r.tag != s.tag) continue;
      if (r.bytes < s.bytes) fail("receive buffer smaller than the message");
      std::memcpy(r.rbuf, s.sbuf ? s.sbuf : s.copy.data(), s.bytes);
      s.done = r.done = true;
      break;
    }
  }
}

int post(Message m) {
  g_msgs.push_back(std::move(m));
  match();
  return (int)g_msgs.size();
}

void copy_in_place(const void* snd, void* rcv, size_t bytes) {
  if (snd != MPI_IN_PLACE && bytes && snd != rcv) std::memmove(rcv, snd, bytes);
}

}  // namespace

extern "C" {

int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out) { *out = comm; return MPI_SUCCESS; }
int MPI_Comm_split(MPI_Comm comm, int, int, MPI_Comm* out) { *out = comm; return MPI_SUCCESS; }
int MPI_Comm_free(MPI_Comm* comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }
int MPI_Get_processor_name(char* name, int* len) {
  std::snprintf(name, MPI_MAX_PROCESSOR_NAME, "localhost");
  *len = (int)std::strlen(name);
  return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype* out) {
  *out = (int)((count * type_bytes(old)) << 4);
  return MPI_SUCCESS;
}
int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype*) { return MPI_SUCCESS; }

int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm) {
  if (dest != 0) fail("send to a rank other than 0");
  Message m;
  m.bytes = count * type_bytes(type);
  m.copy.assign(static_cast<const char*>(buf), static_cast<const char*>(buf) + m.bytes);
  m.tag = tag;
  m.is_send = true;
  post(std::move(m));
  return MPI_SUCCESS;
}
int MPI_Recv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm, MPI_Status*) {
  if (source != 0) fail("receive from a rank other than 0");
  Message m;
  m.rbuf = buf;
  m.bytes = count * type_bytes(type);
  m.tag = tag;
  const int h = post(std::move(m));
  if (!g_msgs[h - 1].done) fail("blocking receive with no matching send (would deadlock)");
  return MPI_SUCCESS;
}
int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm, MPI_Request* req) {
  if (dest != 0) fail("send to a rank other than 0");
  Message m;
  m.sbuf = buf;
  m.bytes = count * type_bytes(type);
  m.tag = tag;
  m.is_send = true;
  *req = post(std::move(m));
  return MPI_SUCCESS;
}
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm, MPI_Request* req) {
  if (source != 0) fail("receive from a rank other than 0");
  Message m;
  m.rbuf = buf;
  m.bytes = count * type_bytes(type);
  m.tag = tag;
  *req = post(std::move(m));
  return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request* req, MPI_Status*) {
  if (*req > 0) {
    match();
    if (!g_msgs[*req - 1].done) fail("wait on a message that was never matched (would deadlock)");
  }
  *req = MPI_REQUEST_NULL;
  bool all = true;
  for (auto& m : g_msgs) all = all && m.done;
  if (all) g_msgs.clear();
  return MPI_SUCCESS;
}
int MPI_Waitall(int count, MPI_Request* reqs, MPI_Status*) {
  for (int i = 0; i < count; ++i) MPI_Wait(&reqs[i], MPI_STATUS_IGNORE);
  return MPI_SUCCESS;
}

int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Reduce(const void* snd, void* rcv, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm) {
  if (rcv) copy_in_place(snd, rcv, count * type_bytes(type));
  return MPI_SUCCESS;
}
int MPI_Allreduce(const void* snd, void* rcv, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
  copy_in_place(snd, rcv, count * type_bytes(type));
  return MPI_SUCCESS;
}
int MPI_Iallreduce(const void* snd, void* rcv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm,
                   MPI_Request* req) {
  *req = MPI_REQUEST_NULL;
  return MPI_Allreduce(snd, rcv, count, type, op, comm);
}
int MPI_Scan(const void* snd, void* rcv, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
  copy_in_place(snd, rcv, count * type_bytes(type));
  return MPI_SUCCESS;
}
int MPI_Gather(const void* snd, int scount, MPI_Datatype stype, void* rcv, int, MPI_Datatype, int, MPI_Comm) {
  copy_in_place(snd, rcv, scount * type_bytes(stype));
  return MPI_SUCCESS;
}
int MPI_Gatherv(const void* snd, int scount, MPI_Datatype stype, void* rcv, const int*, const int* displs,
                MPI_Datatype rtype, int, MPI_Comm) {
  copy_in_place(snd, static_cast<char*>(rcv) + displs[0] * type_bytes(rtype), scount * type_bytes(stype));
  return MPI_SUCCESS;
}
int MPI_Scatter(const void* snd, int, MPI_Datatype, void* rcv, int rcount, MPI_Datatype rtype, int, MPI_Comm) {
  if (rcv != MPI_IN_PLACE) copy_in_place(snd, rcv, rcount * type_bytes(rtype));
  return MPI_SUCCESS;
}
int MPI_Scatterv(const void* snd, const int*, const int* displs, MPI_Datatype stype, void* rcv, int rcount,
                 MPI_Datatype rtype, int, MPI_Comm) {
  if (rcv != MPI_IN_PLACE)
    copy_in_place(static_cast<const char*>(snd) + displs[0] * type_bytes(stype), rcv, rcount * type_bytes(rtype));
  return MPI_SUCCESS;
}
int MPI_Allgather(const void* snd, int scount, MPI_Datatype stype, void* rcv, int, MPI_Datatype, MPI_Comm) {
  copy_in_place(snd, rcv, scount * type_bytes(stype));
  return MPI_SUCCESS;
}
int MPI_Allgatherv(const void* snd, int scount, MPI_Datatype stype, void* rcv, const int*, const int* displs,
                   MPI_Datatype rtype, MPI_Comm) {
  copy_in_place(snd, static_cast<char*>(rcv) + displs[0] * type_bytes(rtype), scount * type_bytes(stype));
  return MPI_SUCCESS;
}
int MPI_Alltoall(const void* snd, int scount, MPI_Datatype stype, void* rcv, int, MPI_Datatype, MPI_Comm) {
  copy_in_place(snd, rcv, scount * type_bytes(stype));
  return MPI_SUCCESS;
}
int MPI_Alltoallv(const void* snd, const int* scounts, const int* sdispls, MPI_Datatype stype, void* rcv,
                  const int*, const int* rdispls, MPI_Datatype rtype, MPI_Comm) {
  copy_in_place(static_cast<const char*>(snd) + sdispls[0] * type_bytes(stype),
                static_cast<char*>(rcv) + rdispls[0] * type_bytes(rtype), scounts[0] * type_bytes(stype));
  return MPI_SUCCESS;
}
int MPI_Ialltoallv(const void* snd, const int* scounts, const int* sdispls, MPI_Datatype stype, void* rcv,
                   const int* rcounts, const int* rdispls, MPI_Datatype rtype, MPI_Comm comm, MPI_Request* req) {
  *req = MPI_REQUEST_NULL;
  return MPI_Alltoallv(snd, scounts, sdispls, stype, rcv, rcounts, rdispls, rtype, comm);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// LAPACK stand-ins (column-major, Fortran calling convention)
// ---------------------------------------------------------------------------
namespace {

// LU factorisation with partial pivoting, A (n x n, leading dimension lda)
// overwritten by L\U, ipiv 1-based as LAPACK returns it; info > 0 on a zero pivot
template <class T>
void lu(int n, T* A, int lda, int* ipiv, int* info) {
  *info = 0;
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(A[i + k * lda]) > std::fabs(A[p + k * lda])) p = i;
    ipiv[k] = p + 1;
    if (A[p + k * lda] == T(0)) {
      if (!*info) *info = k + 1;
      continue;
    }
    if (p != k)
      for (int j = 0; j < n; ++j) std::swap(A[k + j * lda], A[p + j * lda]);
    for (int i = k + 1; i < n; ++i) {
      A[i + k * lda] /= A[k + k * lda];
      const T l = A[i + k * lda];
      for (int j = k + 1; j < n; ++j) A[i + j * lda] -= l * A[k + j * lda];
    }
  }
}

template <class T>
void lu_solve(int n, const T* A, int lda, const int* ipiv, T* b) {
  for (int k = 0; k < n; ++k) std::swap(b[k], b[ipiv[k] - 1]);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < i; ++k) b[i] -= A[i + k * lda] * b[k];
  for (int i = n - 1; i >= 0; --i) {
    for (int k = i + 1; k < n; ++k) b[i] -= A[i + k * lda] * b[k];
    b[i] /= A[i + i * lda];
  }
}

template <class T>
void gesv(int n, int nrhs, T* A, int lda, int* ipiv, T* B, int ldb, int* info) {
  lu(n, A, lda, ipiv, info);
  if (*info) return;
  for (int c = 0; c < nrhs; ++c) lu_solve(n, A, lda, ipiv, B + (size_t)c * ldb);
}

template <class T>
void getri(int n, T* A, int lda, const int* ipiv, int* info) {
  *info = 0;
  std::vector<T> LU((size_t)n * n), col(n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) LU[i + (size_t)j * n] = A[i + (size_t)j * lda];
  for (int j = 0; j < n; ++j) {
    std::fill(col.begin(), col.end(), T(0));
    col[j] = T(1);
    lu_solve(n, LU.data(), n, ipiv, col.data());
    for (int i = 0; i < n; ++i) A[i + (size_t)j * lda] = col[i];
  }
}

// Eigen-decomposition of a symmetric matrix by cyclic Jacobi rotations; the
// eigenvectors (columns of V) have unit 2-norm, as dgeev returns them.
template <class T>
void geev_symmetric(int n, T* A, int lda, T* wr, T* wi, T* vr, int ldvr, int* info) {
  *info = 0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < i; ++j)
      if (std::fabs(A[i + j * lda] - A[j + i * lda]) > 1e-12 * (std::fabs(A[i + j * lda]) + 1.0)) {
        *info = -1;   // only the symmetric (Golub-Welsch) matrices of the Hex3D setup are supported
        return;
      }
  std::vector<double> a((size_t)n * n), v((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) a[i + (size_t)j * n] = A[i + (size_t)j * lda];
  for (int i = 0; i < n; ++i) v[i + (size_t)i * n] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += a[p + (size_t)q * n] * a[p + (size_t)q * n];
    if (off == 0.0) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a[p + (size_t)q * n];
        if (apq == 0.0) continue;
        const double app = a[p + (size_t)p * n], aqq = a[q + (size_t)q * n];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {   // columns p, q
          const double akp = a[k + (size_t)p * n], akq = a[k + (size_t)q * n];
          a[k + (size_t)p * n] = c * akp - s * akq;
          a[k + (size_t)q * n] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {   // rows p, q
          const double apk = a[p + (size_t)k * n], aqk = a[q + (size_t)k * n];
          a[p + (size_t)k * n] = c * apk - s * aqk;
          a[q + (size_t)k * n] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = v[k + (size_t)p * n], vkq = v[k + (size_t)q * n];
          v[k + (size_t)p * n] = c * vkp - s * vkq;
          v[k + (size_t)q * n] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < n; ++i) {
    wr[i] = (T)a[i + (size_t)i * n];
    wi[i] = T(0);
  }
  if (vr)
    for (int j = 0; j < n; ++j) {
      double nrm = 0.0;
      for (int i = 0; i < n; ++i) nrm += v[i + (size_t)j * n] * v[i + (size_t)j * n];
      nrm = std::sqrt(nrm);
      for (int i = 0; i < n; ++i) vr[i + (size_t)j * ldvr] = (T)(v[i + (size_t)j * n] / nrm);
    }
}

}  // namespace

extern "C" {

void dgesv_(int* N, int* NRHS, double* A, int* LDA, int* IPIV, double* B, int* LDB, int* INFO) {
  gesv(*N, *NRHS, A, *LDA, IPIV, B, *LDB, INFO);
}
void sgesv_(int* N, int* NRHS, float* A, int* LDA, int* IPIV, float* B, int* LDB, int* INFO) {
  gesv(*N, *NRHS, A, *LDA, IPIV, B, *LDB, INFO);
}
void dgetrf_(int* M, int* N, double* A, int* LDA, int* IPIV, int* INFO) {
  if (*M != *N) { *INFO = -1; return; }
  lu(*N, A, *LDA, IPIV, INFO);
}
void sgetrf_(int* M, int* N, float* A, int* LDA, int* IPIV, int* INFO) {
  if (*M != *N) { *INFO = -1; return; }
  lu(*N, A, *LDA, IPIV, INFO);
}
void dgetri_(int* N, double* A, int* LDA, int* IPIV, double*, int*, int* INFO) { getri(*N, A, *LDA, IPIV, INFO); }
void sgetri_(int* N, float* A, int* LDA, int* IPIV, float*, int*, int* INFO) { getri(*N, A, *LDA, IPIV, INFO); }
void dgeev_(char*, char* JOBVR, int* N, double* A, int* LDA, double* WR, double* WI, double*, int*, double* VR,
            int* LDVR, double*, int*, int* INFO) {
  geev_symmetric(*N, A, *LDA, WR, WI, *JOBVR == 'V' ? VR : nullptr, *LDVR, INFO);
}
void sgeev_(char*, char* JOBVR, int* N, float* A, int* LDA, float* WR, float* WI, float*, int*, float* VR,
            int* LDVR, float*, int*, int* INFO) {
  geev_symmetric(*N, A, *LDA, WR, WI, *JOBVR == 'V' ? VR : nullptr, *LDVR, INFO);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// platform_t's OCCA device layer
// ---------------------------------------------------------------------------
namespace libp {

void platform_t::DeviceConfig() {
  properties_t mode;
  mode["mode"] = "Serial";
  device = occa::device(mode);
}

void platform_t::DeviceProperties() {}

kernel_t platform_t::buildKernel(std::string fileName, std::string kernelName, properties_t&) {
  (void)fileName;
  return occa::kernel(kernelName);
}

}  // namespace libp
