/*
 * ORACLE (test infrastructure only).  The MPI calls of mpi.h for one process that plays the
 * ranks of a run one after another: shim_rank / shim_size / shim_howmany say which rank it is,
 * how many ranks the run has and the IO group size (the reference's rank / HowMany colouring).
 */
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <fcntl.h>
#include <unistd.h>
#include "mpi.h"

int shim_rank = 0, shim_size = 1, shim_howmany = 1;

int MPI_Comm_size(MPI_Comm comm, int *size)
{
    if (comm == MPI_COMM_WORLD) { *size = shim_size; return 0; }
    int g = comm - 1, first = g * shim_howmany;
    *size = (shim_size - first < shim_howmany) ? shim_size - first : shim_howmany;
    return 0;
}
int MPI_Comm_rank(MPI_Comm comm, int *rank)
{
    *rank = (comm == MPI_COMM_WORLD) ? shim_rank : shim_rank - (comm - 1) * shim_howmany;
    return 0;
}
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm)
{
    (void)comm; (void)key;
    *newcomm = color + 1;
    return 0;
}
int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh)
{
    (void)comm; (void)info;
    int fl = (amode & MPI_MODE_WRONLY) ? O_WRONLY : O_RDONLY;
    if (amode & MPI_MODE_CREATE) fl |= O_CREAT;
    int fd = open(name, fl, 0644);
    if (fd < 0) { *fh = NULL; return 1; }
    *fh = (MPI_File)malloc(sizeof(**fh));
    (*fh)->fd = fd;
    return 0;
}
int MPI_File_close(MPI_File *fh)
{
    if (*fh) { close((*fh)->fd); free(*fh); *fh = NULL; }
    return 0;
}
int MPI_File_read_at(MPI_File fh, MPI_Offset off, void *buf, int count, MPI_Datatype type, MPI_Status *st)
{
    ssize_t r = pread(fh->fd, buf, (size_t)count * type, (off_t)off);
    if (st) st->count = (int)(r / type);
    return r == (ssize_t)((size_t)count * type) ? 0 : 1;
}
int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int count, MPI_Datatype type, MPI_Status *st)
{
    ssize_t r = pwrite(fh->fd, buf, (size_t)count * type, (off_t)off);
    if (st) st->count = (int)(r / type);
    return r == (ssize_t)((size_t)count * type) ? 0 : 1;
}
int MPI_Abort(MPI_Comm comm, int code) { (void)comm; exit(code); }

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return 0; }
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm)
{
    (void)buf; (void)count; (void)type; (void)root; (void)comm;
    return 0;
}
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm)
{
    (void)op; (void)root; (void)comm;
    if (sendbuf != MPI_IN_PLACE && sendbuf != recvbuf) memmove(recvbuf, sendbuf, (size_t)count * (size_t)type);
    return 0;
}
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm)
{
    return MPI_Reduce(sendbuf, recvbuf, count, type, op, 0, comm);
}
int MPI_Gather(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, int rcount, MPI_Datatype rtype,
               int root, MPI_Comm comm)
{
    (void)rcount; (void)rtype; (void)root; (void)comm;
    if (sendbuf != MPI_IN_PLACE && sendbuf != recvbuf) memmove(recvbuf, sendbuf, (size_t)scount * (size_t)stype);
    return 0;
}
int MPI_Gatherv(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, const int *rcounts,
                const int *displs, MPI_Datatype rtype, int root, MPI_Comm comm)
{
    (void)rcounts; (void)root; (void)comm;
    char *dst = (char *)recvbuf + (size_t)displs[0] * (size_t)rtype;
    if (sendbuf != MPI_IN_PLACE && sendbuf != dst) memmove(dst, sendbuf, (size_t)scount * (size_t)stype);
    return 0;
}
int MPI_Get_processor_name(char *name, int *len)
{
    strcpy(name, "localhost");
    *len = (int)strlen(name);
    return 0;
}
double MPI_Wtime(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}
