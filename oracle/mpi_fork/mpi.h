/*
 * Multi-process MPI stand-in on one host: fork + shared memory. Test and
 * baseline infrastructure only (never linked into the product library).
 *
 * It lets the reference's CPU program (rough/tc_mpi.cpp) run as several MPI
 * ranks on the host's cores without an MPI installation: MPI_Init forks
 * MPI_FORK_RANKS - 1 children (default 1 rank), every rank gets a slice of
 * one shared anonymous mapping, and each collective is "write my part into
 * my slice, barrier, read the others' parts, barrier" with a process-shared
 * pthread barrier. It covers exactly the MPI surface tc_mpi.cpp calls:
 * Init/Finalize/Abort, Barrier, Comm_size/rank, Wtime, Alltoall, Alltoallv,
 * Allreduce (SUM/MAX/MIN), Allgather, Reduce and MPI-IO read/write_at
 * (pread/pwrite). A rank's send data must fit its slice (MPI_FORK_SLICE_MB,
 * default 1024 MiB; the mapping reserves no memory up front); larger data
 * aborts with a message.
 */
#ifndef ORACLE_MPI_FORK_H
#define ORACLE_MPI_FORK_H

#include <fcntl.h>
#include <pthread.h>
#include <signal.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/time.h>
#include <sys/wait.h>
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
#define MPI_ERR_COUNT 2
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *) 0)
#define MPI_MAX_ERROR_STRING 256

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

#define MPI_FORK_MAX_RANKS 512

typedef struct {
    pthread_barrier_t barrier;
    int64_t counts[MPI_FORK_MAX_RANKS][MPI_FORK_MAX_RANKS];  /* Alltoallv: [src][dst] count */
    int64_t displs[MPI_FORK_MAX_RANKS][MPI_FORK_MAX_RANKS];  /* and displacement (elements) */
} mpi_fork_control;

static mpi_fork_control *mpi_fork_ctl = 0;
static char *mpi_fork_arena = 0;
static size_t mpi_fork_slice = 0;
static int mpi_fork_rank = 0, mpi_fork_size = 1;
static pid_t mpi_fork_children[MPI_FORK_MAX_RANKS];

static inline size_t mpi_stub_type_size(MPI_Datatype t) {
    switch (t) {
        case MPI_INT: return sizeof(int);
        case MPI_LONG: return sizeof(long);
        case MPI_LONG_LONG_INT: return sizeof(long long);
        case MPI_DOUBLE: return sizeof(double);
        case MPI_UINT64_T: return sizeof(uint64_t);
        case MPI_FLOAT: return sizeof(float);
        case MPI_CHAR: return 1;
        default: return 1;
    }
}

static inline char *mpi_fork_slice_of(int r) { return mpi_fork_arena + (size_t) r * mpi_fork_slice; }

static inline void mpi_fork_die(const char *msg) {
    fprintf(stderr, "mpi_fork rank %d: %s\n", mpi_fork_rank, msg);
    fflush(stderr);
    if (mpi_fork_rank == 0)
        for (int i = 1; i < mpi_fork_size; ++i) kill(mpi_fork_children[i], SIGKILL);
    _exit(3);
}

static inline void mpi_fork_put(const void *src, size_t bytes, size_t at) {
    if (at + bytes > mpi_fork_slice) mpi_fork_die("send data larger than the slice (raise MPI_FORK_SLICE_MB)");
    if (bytes) memcpy(mpi_fork_slice_of(mpi_fork_rank) + at, src, bytes);
}

static inline int MPI_Barrier(MPI_Comm) {
    if (mpi_fork_size > 1) pthread_barrier_wait(&mpi_fork_ctl->barrier);
    return MPI_SUCCESS;
}

static inline int MPI_Init(int *, char ***) {
    const char *e = getenv("MPI_FORK_RANKS");
    mpi_fork_size = e ? atoi(e) : 1;
    if (mpi_fork_size < 1) mpi_fork_size = 1;
    if (mpi_fork_size > MPI_FORK_MAX_RANKS) mpi_fork_size = MPI_FORK_MAX_RANKS;
    const char *sl = getenv("MPI_FORK_SLICE_MB");
    mpi_fork_slice = (size_t) (sl ? atoll(sl) : 1024) << 20;
    const size_t bytes = sizeof(mpi_fork_control) + (size_t) mpi_fork_size * mpi_fork_slice;
    void *p = mmap(0, bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    if (p == MAP_FAILED) mpi_fork_die("mmap of the shared arena failed");
    mpi_fork_ctl = (mpi_fork_control *) p;
    mpi_fork_arena = (char *) p + sizeof(mpi_fork_control);
    pthread_barrierattr_t a;
    pthread_barrierattr_init(&a);
    pthread_barrierattr_setpshared(&a, PTHREAD_PROCESS_SHARED);
    pthread_barrier_init(&mpi_fork_ctl->barrier, &a, (unsigned) mpi_fork_size);
    fflush(stdout);
    fflush(stderr);
    for (int i = 1; i < mpi_fork_size; ++i) {
        pid_t c = fork();
        if (c < 0) mpi_fork_die("fork failed");
        if (c == 0) {
            mpi_fork_rank = i;
            return MPI_SUCCESS;
        }
        mpi_fork_children[i] = c;
    }
    return MPI_SUCCESS;
}

static inline int MPI_Finalize(void) {
    MPI_Barrier(MPI_COMM_WORLD);
    if (mpi_fork_rank != 0) {
        fflush(stdout);
        fflush(stderr);
        _exit(0);
    }
    int bad = 0;
    for (int i = 1; i < mpi_fork_size; ++i) {
        int st = 0;
        if (waitpid(mpi_fork_children[i], &st, 0) < 0 || !WIFEXITED(st) || WEXITSTATUS(st) != 0) bad = 1;
    }
    if (bad) mpi_fork_die("a rank did not exit cleanly");
    return MPI_SUCCESS;
}

static inline int MPI_Abort(MPI_Comm, int code) {
    if (mpi_fork_rank == 0)
        for (int i = 1; i < mpi_fork_size; ++i) kill(mpi_fork_children[i], SIGKILL);
    exit(code);
}

static inline int MPI_Comm_size(MPI_Comm, int *s) {
    *s = mpi_fork_size;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_rank(MPI_Comm, int *r) {
    *r = mpi_fork_rank;
    return MPI_SUCCESS;
}
static inline double MPI_Wtime(void) {
    struct timeval tv;
    gettimeofday(&tv, 0);
    return (double) tv.tv_sec + 1e-6 * (double) tv.tv_usec;
}
static inline int MPI_Error_string(int, char *s, int *len) {
    strcpy(s, "mpi_fork error");
    *len = (int) strlen(s);
    return MPI_SUCCESS;
}

/* Every rank sends sc elements to every rank. */
static inline int MPI_Alltoall(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
    const size_t blk = (size_t) sc * mpi_stub_type_size(st);
    mpi_fork_put(s, blk * (size_t) mpi_fork_size, 0);
    MPI_Barrier(MPI_COMM_WORLD);
    for (int src = 0; src < mpi_fork_size; ++src)
        memcpy((char *) r + (size_t) src * blk, mpi_fork_slice_of(src) + (size_t) mpi_fork_rank * blk, blk);
    MPI_Barrier(MPI_COMM_WORLD);
    return MPI_SUCCESS;
}

static inline int MPI_Alltoallv(const void *s, const int *sc, const int *sd, MPI_Datatype st, void *r,
                                const int *rc, const int *rd, MPI_Datatype, MPI_Comm) {
    const size_t es = mpi_stub_type_size(st);
    size_t end = 0;
    for (int d = 0; d < mpi_fork_size; ++d) {
        mpi_fork_ctl->counts[mpi_fork_rank][d] = sc[d];
        mpi_fork_ctl->displs[mpi_fork_rank][d] = sd[d];
        const size_t e = (size_t) sd[d] + (size_t) sc[d];
        if (sc[d] && e > end) end = e;
    }
    mpi_fork_put(s, end * es, 0);
    MPI_Barrier(MPI_COMM_WORLD);
    for (int src = 0; src < mpi_fork_size; ++src) {
        const int64_t n = mpi_fork_ctl->counts[src][mpi_fork_rank];
        if (n != rc[src]) mpi_fork_die("Alltoallv: receive count differs from the sender's count");
        memcpy((char *) r + (size_t) rd[src] * es,
               mpi_fork_slice_of(src) + (size_t) mpi_fork_ctl->displs[src][mpi_fork_rank] * es, (size_t) n * es);
    }
    MPI_Barrier(MPI_COMM_WORLD);
    return MPI_SUCCESS;
}

#define MPI_FORK_REDUCE(T)                                                  \
    for (int i = 0; i < count; ++i) {                                       \
        T acc = ((const T *) mpi_fork_slice_of(0))[i];                      \
        for (int src = 1; src < mpi_fork_size; ++src) {                     \
            const T v = ((const T *) mpi_fork_slice_of(src))[i];            \
            acc = op == MPI_SUM ? acc + v : op == MPI_MAX ? (v > acc ? v : acc) : (v < acc ? v : acc); \
        }                                                                   \
        ((T *) r)[i] = acc;                                                 \
    }

static inline int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm) {
    const size_t bytes = (size_t) count * mpi_stub_type_size(t);
    mpi_fork_put(s, bytes, 0);
    MPI_Barrier(MPI_COMM_WORLD);
    switch (t) {
        case MPI_INT: MPI_FORK_REDUCE(int) break;
        case MPI_LONG: MPI_FORK_REDUCE(long) break;
        case MPI_LONG_LONG_INT: MPI_FORK_REDUCE(long long) break;
        case MPI_DOUBLE: MPI_FORK_REDUCE(double) break;
        case MPI_UINT64_T: MPI_FORK_REDUCE(uint64_t) break;
        case MPI_FLOAT: MPI_FORK_REDUCE(float) break;
        default: mpi_fork_die("Allreduce: unsupported type");
    }
    MPI_Barrier(MPI_COMM_WORLD);
    return MPI_SUCCESS;
}

static inline int MPI_Reduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, int, MPI_Comm c) {
    return MPI_Allreduce(s, r, count, t, op, c);
}

static inline int MPI_Allgather(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
    const size_t blk = (size_t) sc * mpi_stub_type_size(st);
    mpi_fork_put(s, blk, 0);
    MPI_Barrier(MPI_COMM_WORLD);
    for (int src = 0; src < mpi_fork_size; ++src) memcpy((char *) r + (size_t) src * blk, mpi_fork_slice_of(src), blk);
    MPI_Barrier(MPI_COMM_WORLD);
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
    if (count < 0) return MPI_ERR_COUNT;
    size_t want = (size_t) count * mpi_stub_type_size(t), got = 0;
    while (got < want) {
        ssize_t k = pread(fh->fd, (char *) buf + got, want - got, (off_t) off + (off_t) got);
        if (k <= 0) break;
        got += (size_t) k;
    }
    return MPI_SUCCESS;
}
static inline int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int count, MPI_Datatype t, MPI_Status *) {
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
