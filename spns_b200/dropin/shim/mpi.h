/* mpi.h -- single-rank stand-ins for the MPI calls made by the reference
 * driver (src/MAIN.cpp, src/util.cpp of adalbal/SpNS) when it runs on one GPU
 * through libspns: one process, rank 0 of 1, so every collective is a copy and
 * every barrier returns at once.  Only the names those two files use exist. */
#ifndef SPNS_SHIM_MPI_H
#define SPNS_SHIM_MPI_H

#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_INFO_NULL 0

#define MPI_BYTE 1
#define MPI_INT 2
#define MPI_FLOAT 3
#define MPI_DOUBLE 4

#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUM 3

static inline size_t spns_mpi_type_size(MPI_Datatype t) {
    return t == MPI_DOUBLE ? sizeof(double) : t == MPI_FLOAT ? sizeof(float) : t == MPI_INT ? sizeof(int) : 1;
}
static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Init_thread(int *argc, char ***argv, int required, int *provided) {
    (void)argc; (void)argv; *provided = required; return MPI_SUCCESS;
}
static inline int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int *size) { (void)c; *size = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
/* The reference aborts the job after printing its crash message: exit non-zero. */
static inline int MPI_Abort(MPI_Comm c, int code) { (void)c; exit(code != 0 ? code : 1); return code; }
static inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
    (void)op; (void)c;
    if (send != recv) memcpy(recv, send, (size_t)count * spns_mpi_type_size(t));
    return MPI_SUCCESS;
}
static inline int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm c) {
    (void)buf; (void)count; (void)t; (void)root; (void)c; return MPI_SUCCESS;
}

#endif
