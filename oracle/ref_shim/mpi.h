/* Single-rank stand-in for the MPI surface the reference's host code uses
   (include/comm.hpp, libs/core/comm.cpp, libs/ogs/*.cpp).  TEST
   INFRASTRUCTURE: with one rank every collective is a copy of this rank's
   contribution, and point-to-point messages can only go to this rank, where
   they are matched by tag.  Implemented in ref_shim/shim.cpp.

   A datatype handle encodes its size in bytes (handle >> 4) and a kind
   (handle & 15), so the predefined types stay distinct. */
#ifndef BP_REF_SHIM_MPI_H
#define BP_REF_SHIM_MPI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_IN_PLACE ((void*)1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_REQUEST_NULL 0
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_SUCCESS 0

#define MPI_CHAR ((1 << 4) | 1)
#define MPI_INT ((4 << 4) | 2)
#define MPI_LONG_LONG_INT ((8 << 4) | 3)
#define MPI_FLOAT ((4 << 4) | 4)
#define MPI_DOUBLE ((8 << 4) | 5)

#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUM 3
#define MPI_PROD 4
#define MPI_LAND 5
#define MPI_LOR 6
#define MPI_LXOR 7

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* out);
int MPI_Comm_free(MPI_Comm* comm);
int MPI_Get_processor_name(char* name, int* len);
int MPI_Barrier(MPI_Comm comm);

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype* out);
int MPI_Type_commit(MPI_Datatype* type);
int MPI_Type_free(MPI_Datatype* type);

int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Status* status);
int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Wait(MPI_Request* req, MPI_Status* status);
int MPI_Waitall(int count, MPI_Request* reqs, MPI_Status* statuses);

int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void* snd, void* rcv, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void* snd, void* rcv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Iallreduce(const void* snd, void* rcv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm,
                   MPI_Request* req);
int MPI_Scan(const void* snd, void* rcv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Gather(const void* snd, int scount, MPI_Datatype stype, void* rcv, int rcount, MPI_Datatype rtype, int root,
               MPI_Comm comm);
int MPI_Gatherv(const void* snd, int scount, MPI_Datatype stype, void* rcv, const int* rcounts, const int* displs,
                MPI_Datatype rtype, int root, MPI_Comm comm);
int MPI_Scatter(const void* snd, int scount, MPI_Datatype stype, void* rcv, int rcount, MPI_Datatype rtype, int root,
                MPI_Comm comm);
int MPI_Scatterv(const void* snd, const int* scounts, const int* displs, MPI_Datatype stype, void* rcv, int rcount,
                 MPI_Datatype rtype, int root, MPI_Comm comm);
int MPI_Allgather(const void* snd, int scount, MPI_Datatype stype, void* rcv, int rcount, MPI_Datatype rtype,
                  MPI_Comm comm);
int MPI_Allgatherv(const void* snd, int scount, MPI_Datatype stype, void* rcv, const int* rcounts, const int* displs,
                   MPI_Datatype rtype, MPI_Comm comm);
int MPI_Alltoall(const void* snd, int scount, MPI_Datatype stype, void* rcv, int rcount, MPI_Datatype rtype,
                 MPI_Comm comm);
int MPI_Alltoallv(const void* snd, const int* scounts, const int* sdispls, MPI_Datatype stype, void* rcv,
                  const int* rcounts, const int* rdispls, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Ialltoallv(const void* snd, const int* scounts, const int* sdispls, MPI_Datatype stype, void* rcv,
                   const int* rcounts, const int* rdispls, MPI_Datatype rtype, MPI_Comm comm, MPI_Request* req);

#ifdef __cplusplus
}
#endif

#endif
