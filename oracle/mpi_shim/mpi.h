/*
 * Single-rank MPI shim (test infrastructure for the oracle build only).
 *
 * The reference (Vite) is an MPI+OpenMP C++ code. No MPI is installed here, so
 * the unmodified reference sources are compiled against this header, which
 * implements the subset of MPI-3 that Vite calls, with the semantics of a job
 * that has exactly one rank (`mpirun -n 1`):
 *   - collectives copy the send buffer to the receive buffer (or do nothing
 *     for MPI_IN_PLACE), since a reduction over one rank is the identity;
 *   - point-to-point calls only ever target MPI_PROC_NULL or are skipped by
 *     Vite's own `i != me` guards for one rank; any real self-message aborts;
 *   - MPI-IO maps to pread/pwrite on a POSIX file descriptor.
 * Nothing here is used by the GPU product path.
 */
#ifndef VITE_ORACLE_MPI_SHIM_H
#define VITE_ORACLE_MPI_SHIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef long long MPI_Aint;
typedef struct { int fd; long long pos; } *MPI_File;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; long long count; } MPI_Status;

#define MPI_COMM_WORLD     ((MPI_Comm)1)
#define MPI_SUCCESS        0
#define MPI_ERR_OTHER      15
#define MPI_PROC_NULL      (-2)
#define MPI_REQUEST_NULL   ((MPI_Request)0)
#define MPI_INFO_NULL      ((MPI_Info)0)
#define MPI_STATUS_IGNORE   ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE       ((void *)-1)

#define MPI_MODE_RDONLY    2
#define MPI_MODE_WRONLY    4
#define MPI_MODE_CREATE    1

/* Datatype handles: the low 8 bits hold the element size in bytes;
 * handles >= 0x10000 are derived types registered at run time. */
#define MPI_BYTE      ((MPI_Datatype)(0x0100 | 1))
#define MPI_INT       ((MPI_Datatype)(0x0200 | 4))
#define MPI_INT32_T   ((MPI_Datatype)(0x0300 | 4))
#define MPI_INT64_T   ((MPI_Datatype)(0x0400 | 8))
#define MPI_LONG      ((MPI_Datatype)(0x0500 | 8))
#define MPI_FLOAT     ((MPI_Datatype)(0x0600 | 4))
#define MPI_DOUBLE    ((MPI_Datatype)(0x0700 | 8))

#define MPI_SUM ((MPI_Op)1)
#define MPI_MIN ((MPI_Op)2)
#define MPI_MAX ((MPI_Op)3)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
double MPI_Wtime(void);
int MPI_Barrier(MPI_Comm comm);

int MPI_Get_address(const void *loc, MPI_Aint *addr);
int MPI_Type_create_struct(int count, const int blens[], const MPI_Aint displs[],
                           const MPI_Datatype types[], MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Type_free(MPI_Datatype *t);

int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c);
int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c);
int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt,
                  MPI_Comm c);
int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt,
               int root, MPI_Comm c);
int MPI_Gatherv(const void *s, int sn, MPI_Datatype st, void *r, const int rcounts[],
                const int displs[], MPI_Datatype rt, int root, MPI_Comm c);
int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt,
                 MPI_Comm c);
int MPI_Ialltoall(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt,
                  MPI_Comm c, MPI_Request *req);
int MPI_Alltoallv(const void *s, const int scounts[], const int sdispls[], MPI_Datatype st,
                  void *r, const int rcounts[], const int rdispls[], MPI_Datatype rt,
                  MPI_Comm c);

int MPI_Isend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c,
              MPI_Request *req);
int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *req);
int MPI_Sendrecv(const void *sb, int sn, MPI_Datatype st, int dest, int stag, void *rb, int rn,
                 MPI_Datatype rt, int src, int rtag, MPI_Comm c, MPI_Status *status);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Waitall(int n, MPI_Request reqs[], MPI_Status statuses[]);
int MPI_Test(MPI_Request *req, int *flag, MPI_Status *status);
int MPI_Testany(int n, MPI_Request reqs[], int *idx, int *flag, MPI_Status *status);

int MPI_Info_create(MPI_Info *info);
int MPI_Info_set(MPI_Info info, const char *key, const char *value);
int MPI_Info_free(MPI_Info *info);
int MPI_File_open(MPI_Comm c, const char *name, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_close(MPI_File *fh);
int MPI_File_read_at(MPI_File fh, MPI_Offset off, void *buf, int n, MPI_Datatype t,
                     MPI_Status *status);
int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int n, MPI_Datatype t,
                      MPI_Status *status);
int MPI_File_read_all(MPI_File fh, void *buf, int n, MPI_Datatype t, MPI_Status *status);

#ifdef __cplusplus
}
#endif

#endif
