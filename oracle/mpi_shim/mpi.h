/*
 * ORACLE (test infrastructure only).  The MPI names the reference's host code uses
 * (hpc-engine/tdwslda_checkpoint.c, and the TD drivers pca.c / cpca.c / ccpca.c with their
 * pca_utils.c, wslda_writevars.c and lib/wdata) for one process: either a one-rank run (the
 * drivers; collectives copy or do nothing) or one process that plays the ranks of a run one
 * after another (oracle/ck_ref.c sets which rank it is, how many there are and the IO group
 * size).  File calls are POSIX pread/pwrite; MPI_Comm_split groups ranks by color as the
 * reference's rank / HowMany does.
 */
#ifndef ORACLE_MPI_SHIM_H
#define ORACLE_MPI_SHIM_H
#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Info;
typedef struct { int fd; } *MPI_File;
typedef struct { int count; } MPI_Status;
typedef long long MPI_Offset;

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
/* a datatype is its size in bytes */
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_BYTE 1
#define MPI_CHAR 1
#define MPI_LONG 8
#define MPI_UNSIGNED_LONG 8
typedef int MPI_Op;
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_IN_PLACE ((void *)1)
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_SUCCESS 0
#define MPI_MODE_RDONLY 1
#define MPI_MODE_WRONLY 2
#define MPI_MODE_CREATE 4

extern int shim_rank, shim_size, shim_howmany;

int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm);
int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_close(MPI_File *fh);
int MPI_File_read_at(MPI_File fh, MPI_Offset offset, void *buf, int count, MPI_Datatype type, MPI_Status *st);
int MPI_File_write_at(MPI_File fh, MPI_Offset offset, const void *buf, int count, MPI_Datatype type, MPI_Status *st);
int MPI_Abort(MPI_Comm comm, int code);
/* one rank: initialisation, barriers and broadcasts do nothing, reductions and gathers copy */
int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Gather(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, int rcount, MPI_Datatype rtype,
               int root, MPI_Comm comm);
int MPI_Gatherv(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, const int *rcounts,
                const int *displs, MPI_Datatype rtype, int root, MPI_Comm comm);
int MPI_Get_processor_name(char *name, int *len);
double MPI_Wtime(void);
#endif
