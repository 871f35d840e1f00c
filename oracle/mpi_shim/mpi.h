/*
 * In-process, thread-per-rank stand-in for the subset of MPI that the
 * dsDecompX Host path calls.  TEST INFRASTRUCTURE ONLY: it exists so that the
 * reference's own Host-mode sources (src/{runtime,decomp,topology,grid,halo,
 * migration,buffer,backend_selection}.cpp and src/backends/mpi_backend.cpp)
 * can be compiled unmodified and run as the correctness oracle and as the
 * timed CPU baseline, with P virtual ranks = P threads of one process.
 *
 * Model:
 *   - a "world" of P ranks is created by shim_world_create(P); each rank is a
 *     thread that calls shim_bind_rank(world, rank) before any MPI call;
 *   - every communicator spans all ranks of its world in the same order (the
 *     Host path only ever duplicates the world, makes a Cartesian grid without
 *     reorder, or splits by shared memory, which keeps everyone);
 *   - point-to-point sends are eager (copied into a FIFO mailbox keyed by
 *     communicator, source, destination and tag), so Isend completes at once
 *     and Waitall only blocks for receives;
 *   - collectives exchange pointers through per-communicator slots between
 *     two barriers and reduce in rank order (deterministic).
 */
#ifndef DSX_ORACLE_MPI_SHIM_H
#define DSX_ORACLE_MPI_SHIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef ptrdiff_t MPI_Aint;
typedef struct shim_request_t* MPI_Request;

typedef struct MPI_Status {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    size_t bytes;
} MPI_Status;

#define MPI_COMM_NULL ((MPI_Comm)0)
#define MPI_COMM_WORLD ((MPI_Comm)1)
#define MPI_COMM_SELF ((MPI_Comm)2)

#define MPI_DATATYPE_NULL ((MPI_Datatype)0)
#define MPI_BYTE ((MPI_Datatype)1)
#define MPI_CHAR ((MPI_Datatype)2)
#define MPI_INT ((MPI_Datatype)3)
#define MPI_UNSIGNED ((MPI_Datatype)4)
#define MPI_LONG_LONG ((MPI_Datatype)5)
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype)6)
#define MPI_DOUBLE ((MPI_Datatype)7)
#define MPI_UINT64_T ((MPI_Datatype)8)
#define MPI_INT64_T ((MPI_Datatype)9)
#define MPI_FLOAT ((MPI_Datatype)10)

#define MPI_OP_NULL ((MPI_Op)0)
#define MPI_SUM ((MPI_Op)1)
#define MPI_MIN ((MPI_Op)2)
#define MPI_MAX ((MPI_Op)3)

#define MPI_INFO_NULL ((MPI_Info)0)
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_PROC_NULL (-2)
#define MPI_ANY_SOURCE (-1)
#define MPI_UNDEFINED (-32766)
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_MAX_ERROR_STRING 256
#define MPI_COMM_TYPE_SHARED 1

#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

/* ---- stand-in control (not part of MPI) ---- */
typedef struct shim_world_t shim_world;
shim_world* shim_world_create(int size);
void shim_world_destroy(shim_world* world);
void shim_bind_rank(shim_world* world, int rank);
void shim_unbind_rank(void);

/* ---- the MPI subset ---- */
int MPI_Init(int* argc, char*** argv);
int MPI_Init_thread(int* argc, char*** argv, int required, int* provided);
int MPI_Initialized(int* flag);
int MPI_Finalized(int* flag);
int MPI_Finalize(void);
int MPI_Query_thread(int* provided);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);
int MPI_Get_processor_name(char* name, int* length);
int MPI_Error_string(int code, char* text, int* length);

int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out);
int MPI_Comm_free(MPI_Comm* comm);
int MPI_Comm_split_type(MPI_Comm comm, int split_type, int key, MPI_Info info,
                        MPI_Comm* out);

int MPI_Dims_create(int nnodes, int ndims, int* dims);
int MPI_Cart_create(MPI_Comm comm, int ndims, const int* dims,
                    const int* periods, int reorder, MPI_Comm* out);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int* coords);
int MPI_Cart_rank(MPI_Comm comm, const int* coords, int* rank);

int MPI_Get_address(const void* location, MPI_Aint* address);
int MPI_Type_create_struct(int count, const int* block_lengths,
                           const MPI_Aint* displacements,
                           const MPI_Datatype* types, MPI_Datatype* out);
int MPI_Type_commit(MPI_Datatype* type);
int MPI_Type_free(MPI_Datatype* type);
int MPI_Type_size(MPI_Datatype type, int* size);

int MPI_Isend(const void* buffer, int count, MPI_Datatype type, int dest,
              int tag, MPI_Comm comm, MPI_Request* request);
int MPI_Irecv(void* buffer, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request* request);
int MPI_Wait(MPI_Request* request, MPI_Status* status);
int MPI_Waitall(int count, MPI_Request* requests, MPI_Status* statuses);

int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void* buffer, int count, MPI_Datatype type, int root,
              MPI_Comm comm);
int MPI_Allreduce(const void* send, void* receive, int count,
                  MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void* send, void* receive, int count, MPI_Datatype type,
               MPI_Op op, int root, MPI_Comm comm);
int MPI_Allgather(const void* send, int send_count, MPI_Datatype send_type,
                  void* receive, int receive_count, MPI_Datatype receive_type,
                  MPI_Comm comm);
int MPI_Allgatherv(const void* send, int send_count, MPI_Datatype send_type,
                   void* receive, const int* receive_counts,
                   const int* displacements, MPI_Datatype receive_type,
                   MPI_Comm comm);
int MPI_Alltoall(const void* send, int send_count, MPI_Datatype send_type,
                 void* receive, int receive_count, MPI_Datatype receive_type,
                 MPI_Comm comm);
int MPI_Alltoallv(const void* send, const int* send_counts,
                  const int* send_displacements, MPI_Datatype send_type,
                  void* receive, const int* receive_counts,
                  const int* receive_displacements, MPI_Datatype receive_type,
                  MPI_Comm comm);

#ifdef __cplusplus
}
#endif

#endif
