/*
 * ORACLE (test infrastructure only).  The reference's checkpoint writer and reader
 * (hpc-engine/tdwslda_checkpoint.c, compiled where it lies by the `ckref` target of
 * oracle/Makefile against oracle/mpi_shim) driven for one rank of an emulated run at a time.
 * The reference's device copies (memcopy_gpu2host / memcopy_host2gpu) become host copies, so
 * every "device" array here is host memory.
 *
 *   ckref_save(dir, rank, nranks, howmany, scheme, nwf, y, f1..f5, pots, meta[8], En, kperp)
 *   ckref_load(dir, rank, nranks, howmany, scheme, y, f1..f5, pots, meta[8], &nwf, En, kperp)
 *
 * meta = [t0, mu_a, mu_b, ec, kF, eF, Effg, beta]; y and f_k hold the rank's 2 nwfip N complex
 * values; f4, f5 may be NULL below AB4AM5 / AB5AM5.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <fcntl.h>
#include <unistd.h>
#include <complex.h>
#include "mpi.h"
#include "predefines.h"
#include "pca_settings.h"
#include "tdwslda_checkpoint.h"

#if CODEDIM == 1
#define CK_N NX
#elif CODEDIM == 2
#define CK_N NXY
#else
#define CK_N NXYZ
#endif

/* the process id that the reference's drivers keep globally (pca.c:39) */
int wsldapid = 0;

/* the reference's host/device copies, on host memory */
int memcopy_host2gpu(void *host, void *gpu, size_t size) { memcpy(gpu, host, size); return 0; }
int memcopy_gpu2host(void *gpu, void *host, size_t size) { memcpy(host, gpu, size); return 0; }

static void set_rank(int rank, int nranks, int howmany)
{
    shim_rank = rank; shim_size = nranks; shim_howmany = howmany;
}

int ckref_save(const char *dir, int rank, int nranks, int howmany, int scheme, int nwf, double complex *y,
               double complex *f1, double complex *f2, double complex *f3, double complex *f4, double complex *f5,
               double *pots, const double *meta, double *En, double *kperp)
{
    set_rank(rank, nranks, howmany);
    int nwfip;
    getnwfip(rank, nranks, nwf, &nwfip);
    double complex *scratch = (double complex *)malloc((size_t)2 * nwfip * CK_N * sizeof(double complex));
    double m[8];
    memcpy(m, meta, sizeof(m));
    int rc = save_checkpoint(scratch, MPI_COMM_WORLD, (char *)dir, y, f1, f2, f3, f4, f5, pots, &m[0], nwf, nwfip,
                             En, kperp, &m[1], &m[3], &m[4], &m[5], &m[6], &m[7], howmany, scheme);
    free(scratch);
    return rc;
}

int ckref_load(const char *dir, int rank, int nranks, int howmany, int scheme, double complex *y,
               double complex *f1, double complex *f2, double complex *f3, double complex *f4, double complex *f5,
               double *pots, double *meta, int *nwf, double *En, double *kperp)
{
    set_rank(rank, nranks, howmany);
    int nwfip = 0;
    int rc = load_nwf(MPI_COMM_WORLD, (char *)dir, nwf, &nwfip, howmany);
    if (rc != 0) return rc;
    double complex *scratch = (double complex *)malloc((size_t)2 * nwfip * CK_N * sizeof(double complex));
    rc = load_checkpoint(scratch, MPI_COMM_WORLD, (char *)dir, y, f1, f2, f3, f4, f5, pots, &meta[0], nwf, &nwfip,
                         En, kperp, &meta[1], &meta[3], &meta[4], &meta[5], &meta[6], &meta[7], howmany, scheme);
    free(scratch);
    return rc;
}
