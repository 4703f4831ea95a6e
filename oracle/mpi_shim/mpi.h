/*
 * ORACLE (test infrastructure only).  The few MPI names hpc-engine/tdwslda_checkpoint.c uses,
 * for one process that plays the ranks of a run one after another (oracle/ck_ref.c sets which
 * rank it is, how many there are and the IO group size).  File calls are POSIX pread/pwrite;
 * MPI_Comm_split groups ranks by color as the reference's rank / HowMany does.
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
#define MPI_DOUBLE 8
#define MPI_INT 4
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
#endif
