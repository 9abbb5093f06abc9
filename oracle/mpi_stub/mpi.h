/*
 * Single-rank MPI stand-in used ONLY to build the reference programs as the
 * parity oracle (test infrastructure; never linked into the product library).
 *
 * It provides exactly the MPI surface that the reference drivers and its CPU
 * baseline call (tc.cu, sg.cu, wcc.cu, single_join.cu, tc_nl.cu, sg_nl.cu,
 * common/comm.cu, common/parallel_io.cu, common/utils.cu, rough/tc_mpi.cpp):
 * with one rank every collective is a local copy and MPI-IO is pread/pwrite.
 * Like MPI_File_open with MPI_MODE_CREATE, files are opened without truncation
 * (common/parallel_io.cu:117 relies on that), so callers delete stale outputs.
 */
#ifndef ORACLE_MPI_STUB_H
#define ORACLE_MPI_STUB_H

#include <fcntl.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef struct { int fd; } MPI_File_s;
typedef MPI_File_s *MPI_File;
typedef int MPI_Status;
typedef int64_t MPI_Offset;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *) 0)
#define MPI_MAX_ERROR_STRING 256
#define MPI_ERR_COUNT 2

#define MPI_INT 1
#define MPI_LONG 2
#define MPI_LONG_LONG_INT 3
#define MPI_LONG_LONG 3
#define MPI_DOUBLE 4
#define MPI_UINT64_T 5
#define MPI_FLOAT 6
#define MPI_CHAR 7

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

#define MPI_MODE_RDONLY 1
#define MPI_MODE_WRONLY 2
#define MPI_MODE_RDWR 4
#define MPI_MODE_CREATE 8

static inline size_t mpi_stub_type_size(MPI_Datatype t) {
    switch (t) {
        case MPI_INT: return sizeof(int);
        case MPI_LONG: return sizeof(long);
        case MPI_LONG_LONG_INT: return sizeof(long long);
        case MPI_DOUBLE: return sizeof(double);
        case MPI_UINT64_T: return sizeof(uint64_t);
        case MPI_FLOAT: return sizeof(float);
        case MPI_CHAR: return 1;
        default: fprintf(stderr, "mpi stub: unknown datatype %d\n", t); exit(2);
    }
}

static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
static inline double MPI_Wtime(void) {
    struct timeval tv;
    gettimeofday(&tv, 0);
    return (double) tv.tv_sec + 1e-6 * (double) tv.tv_usec;
}
static inline int MPI_Abort(MPI_Comm, int code) { exit(code); return code; }
static inline int MPI_Error_string(int code, char *s, int *len) {
    *len = snprintf(s, MPI_MAX_ERROR_STRING, "mpi stub error %d", code);
    return MPI_SUCCESS;
}

static inline void mpi_stub_copy(const void *src, void *dst, int count, MPI_Datatype t) {
    if (src != dst && count > 0) memmove(dst, src, (size_t) count * mpi_stub_type_size(t));
}
static inline int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
    mpi_stub_copy(s, r, count, t);
    return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    mpi_stub_copy(s, r, count, t);
    return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
    mpi_stub_copy(s, r, sc, st);
    return MPI_SUCCESS;
}
static inline int MPI_Alltoall(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
    mpi_stub_copy(s, r, sc, st);
    return MPI_SUCCESS;
}
/* Buffers may live in device memory when the caller is CUDA-aware; the
 * reference programs only pass host buffers in their default (non CUDA-aware)
 * mode, which is the only mode the oracle runs. */
static inline int MPI_Alltoallv(const void *s, const int *sc, const int *sd, MPI_Datatype st,
                                void *r, const int *, const int *rd, MPI_Datatype, MPI_Comm) {
    size_t es = mpi_stub_type_size(st);
    mpi_stub_copy((const char *) s + (size_t) sd[0] * es, (char *) r + (size_t) rd[0] * es, sc[0], st);
    return MPI_SUCCESS;
}

static inline int MPI_File_open(MPI_Comm, const char *name, int mode, MPI_Info, MPI_File *fh) {
    int flags = 0;
    if (mode & MPI_MODE_RDWR) flags = O_RDWR;
    else if (mode & MPI_MODE_WRONLY) flags = O_WRONLY;
    else flags = O_RDONLY;
    if (mode & MPI_MODE_CREATE) flags |= O_CREAT;
    int fd = open(name, flags, 0644);
    if (fd < 0) return 1;
    *fh = (MPI_File) malloc(sizeof(MPI_File_s));
    (*fh)->fd = fd;
    return MPI_SUCCESS;
}
static inline int MPI_File_close(MPI_File *fh) {
    if (*fh) { close((*fh)->fd); free(*fh); *fh = 0; }
    return MPI_SUCCESS;
}
static inline int MPI_File_read_at(MPI_File fh, MPI_Offset off, void *buf, int count, MPI_Datatype t, MPI_Status *) {
    if (count < 0) return MPI_ERR_COUNT; /* as MPI does; nothing is read */
    size_t want = (size_t) count * mpi_stub_type_size(t), got = 0;
    while (got < want) {
        ssize_t k = pread(fh->fd, (char *) buf + got, want - got, (off_t) off + (off_t) got);
        if (k <= 0) break;
        got += (size_t) k;
    }
    return MPI_SUCCESS;
}
static inline int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int count, MPI_Datatype t, MPI_Status *) {
    /* A count that overflowed int (the reference passes rows * 2 as an int)
     * is rejected as MPI rejects it: nothing is written. */
    if (count < 0) return MPI_ERR_COUNT;
    size_t want = (size_t) count * mpi_stub_type_size(t), put = 0;
    while (put < want) {
        ssize_t k = pwrite(fh->fd, (const char *) buf + put, want - put, (off_t) off + (off_t) put);
        if (k <= 0) break;
        put += (size_t) k;
    }
    return MPI_SUCCESS;
}

#endif
