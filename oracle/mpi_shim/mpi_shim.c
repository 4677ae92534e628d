/*
 * Single-rank MPI shim implementation (oracle test infrastructure only; see
 * mpi.h for the contract). Every collective over one rank is a copy of the
 * caller's own contribution; MPI-IO is pread/pwrite.
 */
#define _GNU_SOURCE
#include "mpi.h"

#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include <time.h>
#include <unistd.h>

#define SHIM_MAX_DERIVED 64
static long long g_derived_size[SHIM_MAX_DERIVED];
static int g_derived_count = 0;

static long long type_size(MPI_Datatype t)
{
    if (t >= 0x10000) {
        int idx = t - 0x10000;
        if (idx < 0 || idx >= g_derived_count) {
            fprintf(stderr, "mpi shim: unknown datatype %d\n", t);
            abort();
        }
        return g_derived_size[idx];
    }
    return (long long)(t & 0xff);
}

static void shim_fail(const char *what)
{
    fprintf(stderr, "mpi shim: %s is not possible in a single-rank job\n", what);
    abort();
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm comm, int code) { (void)comm; fflush(stdout); exit(code & 0xff ? code & 0xff : 1); }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }

double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int MPI_Get_address(const void *loc, MPI_Aint *addr)
{
    *addr = (MPI_Aint)(uintptr_t)loc;
    return MPI_SUCCESS;
}

int MPI_Type_create_struct(int count, const int blens[], const MPI_Aint displs[],
                           const MPI_Datatype types[], MPI_Datatype *newtype)
{
    long long extent = 0;
    for (int i = 0; i < count; i++) {
        long long end = displs[i] + (long long)blens[i] * type_size(types[i]);
        if (end > extent) extent = end;
    }
    /* round the extent up to the largest member alignment (8 for Vite's structs) */
    extent = (extent + 7) & ~7LL;
    if (g_derived_count >= SHIM_MAX_DERIVED) shim_fail("registering more derived types");
    g_derived_size[g_derived_count] = extent;
    *newtype = 0x10000 + g_derived_count;
    g_derived_count++;
    return MPI_SUCCESS;
}
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }

static void copy_elems(void *dst, const void *src, int n, MPI_Datatype t)
{
    if (src == MPI_IN_PLACE || n <= 0 || dst == src) return;
    memmove(dst, src, (size_t)n * (size_t)type_size(t));
}

int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    (void)op; (void)c;
    copy_elems(r, s, n, t);
    return MPI_SUCCESS;
}

int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{
    (void)op; (void)c; (void)root;
    copy_elems(r, s, n, t);
    return MPI_SUCCESS;
}

int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{
    (void)b; (void)n; (void)t; (void)root; (void)c;
    return MPI_SUCCESS;
}

int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt,
                  MPI_Comm c)
{
    (void)rn; (void)rt; (void)c;
    copy_elems(r, s, sn, st);
    return MPI_SUCCESS;
}

int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt,
               int root, MPI_Comm c)
{
    (void)rn; (void)rt; (void)root; (void)c;
    copy_elems(r, s, sn, st);
    return MPI_SUCCESS;
}

int MPI_Gatherv(const void *s, int sn, MPI_Datatype st, void *r, const int rcounts[],
                const int displs[], MPI_Datatype rt, int root, MPI_Comm c)
{
    (void)rcounts; (void)root; (void)c;
    if (s == MPI_IN_PLACE) return MPI_SUCCESS;
    copy_elems((char *)r + (size_t)displs[0] * (size_t)type_size(rt), s, sn, st);
    return MPI_SUCCESS;
}

int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt,
                 MPI_Comm c)
{
    (void)rn; (void)rt; (void)c;
    copy_elems(r, s, sn, st);
    return MPI_SUCCESS;
}

int MPI_Ialltoall(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt,
                  MPI_Comm c, MPI_Request *req)
{
    MPI_Alltoall(s, sn, st, r, rn, rt, c);
    *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}

int MPI_Alltoallv(const void *s, const int scounts[], const int sdispls[], MPI_Datatype st,
                  void *r, const int rcounts[], const int rdispls[], MPI_Datatype rt,
                  MPI_Comm c)
{
    (void)rcounts; (void)c;
    if (scounts[0] > 0)
        memmove((char *)r + (size_t)rdispls[0] * (size_t)type_size(rt),
                (const char *)s + (size_t)sdispls[0] * (size_t)type_size(st),
                (size_t)scounts[0] * (size_t)type_size(st));
    return MPI_SUCCESS;
}

int MPI_Isend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c,
              MPI_Request *req)
{
    (void)b; (void)t; (void)tag; (void)c;
    if (dest != MPI_PROC_NULL && n > 0) shim_fail("MPI_Isend to a rank");
    *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}

int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *req)
{
    (void)b; (void)t; (void)tag; (void)c;
    if (src != MPI_PROC_NULL && n > 0) shim_fail("MPI_Irecv from a rank");
    *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}

int MPI_Sendrecv(const void *sb, int sn, MPI_Datatype st, int dest, int stag, void *rb, int rn,
                 MPI_Datatype rt, int src, int rtag, MPI_Comm c, MPI_Status *status)
{
    (void)sb; (void)sn; (void)st; (void)stag; (void)rb; (void)rt; (void)rtag; (void)c;
    (void)status;
    if (dest != MPI_PROC_NULL && sn > 0) shim_fail("MPI_Sendrecv to a rank");
    if (src != MPI_PROC_NULL && rn > 0) shim_fail("MPI_Sendrecv from a rank");
    return MPI_SUCCESS;
}

int MPI_Wait(MPI_Request *req, MPI_Status *status) { (void)req; (void)status; return MPI_SUCCESS; }
int MPI_Waitall(int n, MPI_Request reqs[], MPI_Status statuses[])
{
    (void)n; (void)reqs; (void)statuses;
    return MPI_SUCCESS;
}
int MPI_Test(MPI_Request *req, int *flag, MPI_Status *status)
{
    (void)req; (void)status;
    *flag = 1;
    return MPI_SUCCESS;
}
int MPI_Testany(int n, MPI_Request reqs[], int *idx, int *flag, MPI_Status *status)
{
    (void)n; (void)reqs; (void)status;
    *idx = -32766; /* MPI_UNDEFINED */
    *flag = 1;
    return MPI_SUCCESS;
}

int MPI_Info_create(MPI_Info *info) { *info = 1; return MPI_SUCCESS; }
int MPI_Info_set(MPI_Info info, const char *key, const char *value)
{
    (void)info; (void)key; (void)value;
    return MPI_SUCCESS;
}
int MPI_Info_free(MPI_Info *info) { *info = MPI_INFO_NULL; return MPI_SUCCESS; }

int MPI_File_open(MPI_Comm c, const char *name, int amode, MPI_Info info, MPI_File *fh)
{
    (void)c; (void)info;
    int flags = (amode & MPI_MODE_WRONLY) ? O_WRONLY : O_RDONLY;
    if (amode & MPI_MODE_CREATE) flags |= O_CREAT;
    int fd = open(name, flags, 0644);
    if (fd < 0) return MPI_ERR_OTHER;
    *fh = (MPI_File)malloc(sizeof(**fh));
    (*fh)->fd = fd;
    (*fh)->pos = 0;
    return MPI_SUCCESS;
}

int MPI_File_close(MPI_File *fh)
{
    if (*fh) {
        close((*fh)->fd);
        free(*fh);
        *fh = NULL;
    }
    return MPI_SUCCESS;
}

static int full_pread(int fd, void *buf, size_t len, long long off)
{
    char *p = (char *)buf;
    while (len > 0) {
        ssize_t got = pread(fd, p, len, (off_t)off);
        if (got <= 0) return MPI_ERR_OTHER;
        p += got; len -= (size_t)got; off += got;
    }
    return MPI_SUCCESS;
}

int MPI_File_read_at(MPI_File fh, MPI_Offset off, void *buf, int n, MPI_Datatype t,
                     MPI_Status *status)
{
    (void)status;
    return full_pread(fh->fd, buf, (size_t)n * (size_t)type_size(t), off);
}

int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int n, MPI_Datatype t,
                      MPI_Status *status)
{
    (void)status;
    const char *p = (const char *)buf;
    size_t len = (size_t)n * (size_t)type_size(t);
    while (len > 0) {
        ssize_t put = pwrite(fh->fd, p, len, (off_t)off);
        if (put <= 0) return MPI_ERR_OTHER;
        p += put; len -= (size_t)put; off += put;
    }
    return MPI_SUCCESS;
}

int MPI_File_read_all(MPI_File fh, void *buf, int n, MPI_Datatype t, MPI_Status *status)
{
    (void)status;
    size_t len = (size_t)n * (size_t)type_size(t);
    int rc = full_pread(fh->fd, buf, len, fh->pos);
    fh->pos += (long long)len;
    return rc;
}
