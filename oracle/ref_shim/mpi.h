/* mpi.h -- single-process stand-in for the MPI calls of the reference solver
 * (adalbal/SpNS src/*.cpp), so that its sources compile unchanged into a CPU
 * executable under oracle/_ref/.  TEST INFRASTRUCTURE ONLY: the build of the
 * reference that checks the oracle and serves as the timed CPU baseline.
 *
 * One rank of one: collectives copy the send buffer into the receive buffer
 * (a reduction over one rank is that rank's value), broadcasts and barriers
 * return at once, and MPI-IO maps onto stdio with the reference's open modes
 * (src/HIT_LES.cpp:622-686 reads, src/HIT_LES_output.cpp:22-114 writes). */
#ifndef SPNS_REF_SHIM_MPI_H
#define SPNS_REF_SHIM_MPI_H

#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef struct { int count; } MPI_Status;
typedef struct spns_ref_mpi_file {
    FILE *f;
    int delete_on_close;
    char path[4096];
} *MPI_File;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_ERR_FILE 27
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

#define MPI_MODE_CREATE 1
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_MODE_DELETE_ON_CLOSE 16
#define MPI_MODE_EXCL 64
#define MPI_SEEK_SET 600

static inline size_t spns_ref_type_size(MPI_Datatype t) {
    return t == MPI_DOUBLE ? sizeof(double) : (t == MPI_FLOAT ? sizeof(float) : (t == MPI_INT ? sizeof(int) : 1));
}

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Init_thread(int *argc, char ***argv, int required, int *provided) {
    (void)argc; (void)argv; *provided = required; return MPI_SUCCESS;
}
static inline int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int *size) { (void)c; *size = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm c, int code) { (void)c; exit(code != 0 ? code : 1); return code; }
static inline int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm c) {
    (void)buf; (void)count; (void)t; (void)root; (void)c; return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
    (void)op; (void)c;
    if (send != recv) memmove(recv, send, (size_t)count * spns_ref_type_size(t));
    return MPI_SUCCESS;
}
static inline int MPI_Gather(const void *send, int scount, MPI_Datatype st, void *recv, int rcount, MPI_Datatype rt, int root,
                             MPI_Comm c) {
    (void)rcount; (void)rt; (void)root; (void)c;
    if (send != recv) memmove(recv, send, (size_t)scount * spns_ref_type_size(st));
    return MPI_SUCCESS;
}
static inline int MPI_Gatherv(const void *send, int scount, MPI_Datatype st, void *recv, const int *rcounts, const int *displs,
                              MPI_Datatype rt, int root, MPI_Comm c) {
    (void)rcounts; (void)root; (void)c;
    char *dst = (char *)recv + (size_t)displs[0] * spns_ref_type_size(rt);
    if ((const void *)dst != send) memmove(dst, send, (size_t)scount * spns_ref_type_size(st));
    return MPI_SUCCESS;
}
static inline int MPI_Allgatherv(const void *send, int scount, MPI_Datatype st, void *recv, const int *rcounts, const int *displs,
                                 MPI_Datatype rt, MPI_Comm c) {
    return MPI_Gatherv(send, scount, st, recv, rcounts, displs, rt, 0, c);
}

/* MPI-IO on one process.  An exclusive create of an existing file fails, as the
 * reference expects before it deletes and recreates an output file; opening for
 * writing does not truncate (MPI semantics). */
static inline int MPI_File_open(MPI_Comm c, const char *name, int amode, MPI_Info info, MPI_File *fh) {
    (void)c; (void)info;
    *fh = NULL;
    int flags = (amode & MPI_MODE_RDONLY) ? O_RDONLY : O_WRONLY;
    if (amode & MPI_MODE_CREATE) flags |= O_CREAT;
    if (amode & MPI_MODE_EXCL) flags |= O_EXCL;
    const int fd = open(name, flags, 0644);
    if (fd < 0) return MPI_ERR_FILE;
    FILE *f = fdopen(fd, (amode & MPI_MODE_RDONLY) ? "rb" : "wb");
    if (!f) { close(fd); return MPI_ERR_FILE; }
    MPI_File h = (MPI_File)calloc(1, sizeof(*h));
    h->f = f;
    h->delete_on_close = (amode & MPI_MODE_DELETE_ON_CLOSE) != 0;
    strncpy(h->path, name, sizeof(h->path) - 1);
    *fh = h;
    return MPI_SUCCESS;
}
static inline int MPI_File_close(MPI_File *fh) {
    if (!fh || !*fh) return MPI_SUCCESS;
    fclose((*fh)->f);
    if ((*fh)->delete_on_close) remove((*fh)->path);
    free(*fh);
    *fh = NULL;
    return MPI_SUCCESS;
}
static inline int MPI_File_get_size(MPI_File fh, MPI_Offset *size) {
    struct stat st;
    if (fstat(fileno(fh->f), &st) != 0) return MPI_ERR_FILE;
    *size = (MPI_Offset)st.st_size;
    return MPI_SUCCESS;
}
static inline int MPI_File_seek(MPI_File fh, MPI_Offset off, int whence) {
    (void)whence;
    return fseeko(fh->f, (off_t)off, SEEK_SET) == 0 ? MPI_SUCCESS : MPI_ERR_FILE;
}
static inline int MPI_File_read_all(MPI_File fh, void *buf, int count, MPI_Datatype t, MPI_Status *status) {
    const size_t n = fread(buf, spns_ref_type_size(t), (size_t)count, fh->f);
    if (status) status->count = (int)n;
    return n == (size_t)count ? MPI_SUCCESS : MPI_ERR_FILE;
}
static inline int MPI_File_write(MPI_File fh, const void *buf, int count, MPI_Datatype t, MPI_Status *status) {
    const size_t n = fwrite(buf, spns_ref_type_size(t), (size_t)count, fh->f);
    if (status) status->count = (int)n;
    return n == (size_t)count ? MPI_SUCCESS : MPI_ERR_FILE;
}

#endif
