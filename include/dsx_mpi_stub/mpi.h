/*
 * Single-process stand-in for <mpi.h>, header only, for building and running
 * the dsDecompX drop-in where no MPI is installed.  The drop-in handles one
 * rank per process, so every communicator here has size 1.  Programs that do
 * have an MPI should compile against that MPI instead (the library's
 * dsx_dropin.cpp must then be compiled against the same <mpi.h>, since
 * MPI_Comm is part of Decomp's signature).
 */
#ifndef DSX_MPI_STUB_H
#define DSX_MPI_STUB_H

#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_NULL ((MPI_Comm)0)
#define MPI_COMM_WORLD ((MPI_Comm)1)
#define MPI_COMM_SELF ((MPI_Comm)2)
#define MPI_SUCCESS 0
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_IN_PLACE ((void*)1)

#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_BYTE ((MPI_Datatype)1)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_UNSIGNED ((MPI_Datatype)4)
#define MPI_FLOAT ((MPI_Datatype)4)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_LONG_LONG ((MPI_Datatype)8)
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype)8)
#define MPI_UINT64_T ((MPI_Datatype)8)
#define MPI_INT64_T ((MPI_Datatype)8)

#define MPI_SUM ((MPI_Op)1)
#define MPI_MIN ((MPI_Op)2)
#define MPI_MAX ((MPI_Op)3)

static inline int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Init_thread(int* argc, char*** argv, int required, int* provided) {
    (void)argc; (void)argv; (void)required;
    if (provided) *provided = MPI_THREAD_MULTIPLE;
    return MPI_SUCCESS;
}
static inline int MPI_Initialized(int* flag) { *flag = 1; return MPI_SUCCESS; }
static inline int MPI_Finalized(int* flag) { *flag = 0; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm comm, int* size) { (void)comm; *size = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm comm, int* rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out) { *out = comm; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm* comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }
/* one rank: a reduction or gather is a copy (MPI_Datatype is the element size) */
static inline int MPI_Allreduce(const void* send, void* receive, int count, MPI_Datatype type,
                                MPI_Op op, MPI_Comm comm) {
    (void)op; (void)comm;
    if (send != MPI_IN_PLACE && count > 0) memcpy(receive, send, (size_t)count * (size_t)type);
    return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void* send, void* receive, int count, MPI_Datatype type, MPI_Op op,
                             int root, MPI_Comm comm) {
    (void)root;
    return MPI_Allreduce(send, receive, count, type, op, comm);
}
/* wall-clock seconds, as MPI_Wtime is defined (timespec_get: ISO C11 and
 * C++17, no POSIX feature macro needed) */
static inline double MPI_Wtime(void) {
    struct timespec t;
    timespec_get(&t, TIME_UTC);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

#endif
