/*
 * ORACLE (test infrastructure only).  The reference's W-data output of the TD codes
 * (hpc-engine/wslda_writevars.c over lib/wdata/c/wdata.c, compiled where they lie by the
 * `wdref` target of oracle/Makefile against oracle/mpi_shim on one process).
 *
 *   wdref_begin(prefix, vars, t0, dt, spinsymmetry, kF, eF, mu_a, mu_b, float_prec)
 *       create_wdata_metadata + the constants of pca.c:1026-1030 + clear_files
 *   wdref_write(it, dens, pots, vext_a, vext_b, velext_a, velext_b, dext)
 *       write_measurments for one cycle; the external fields the reference evaluates on the
 *       GPU (get_v_ext, get_delta_ext, get_velocity_ext) come in as host arrays
 *   wdref_meta(path)
 *       wdata_print_metadata of the set into path
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>
#include "mpi.h"
#include "wdata.h"
#include "predefines.h"
#include "pca_settings.h"
#include "pca_utils.h"
#include "wslda_writevars.h"

#if CODEDIM == 1
#define WD_N NX
#elif CODEDIM == 2
#define WD_N NXY
#else
#define WD_N NXYZ
#endif

/* the process id that the reference's drivers keep globally (pca.c:39) */
int wsldapid = 0;

/* file helpers of pca_io.h (which needs MPI) */
#include <unistd.h>
int exists(const char *filename) { return access(filename, F_OK) == 0; }
int urm(const char *fn) { return unlink(fn); }

static wdata_metadata g_set;
static const double *g_vext[2], *g_velext[2], *g_dext;

/* the external fields of this cycle, as the reference's CUDA helpers would return them */
int get_v_ext(int datadim, int spin, int it, double *data)
{
    (void)datadim; (void)it;
    memcpy(data, g_vext[spin], sizeof(double) * WD_N);
    return 0;
}
int get_delta_ext(int datadim, int it, void *deltain, void *data)
{
    (void)datadim; (void)it; (void)deltain;
    memcpy(data, g_dext, sizeof(double) * 2 * WD_N);
    return 0;
}
int get_velocity_ext(int datadim, int spin, int it, double *data)
{
    (void)datadim; (void)it;
    memcpy(data, g_velext[spin], sizeof(double) * 3 * WD_N);
    return 0;
}

int wdref_begin(const char *prefix, const char *vars, double t0, double dt, int spinsymmetry, double kF, double eF,
                double mu_a, double mu_b, int float_prec)
{
    char list[1024];
    snprintf(list, sizeof(list), "%s", vars);
    md.nwritevar = 0;
    for (char *tok = strtok(list, " ,"); tok; tok = strtok(NULL, " ,")) strcpy(md.writevar[md.nwritevar++], tok);
    snprintf(md.outprefix, sizeof(md.outprefix), "%s", prefix);
    md.writeprec = float_prec ? 'f' : 'd';
    md.overwrite = 1;
    int r = create_wdata_metadata(&md, CODEDIM, t0, dt, spinsymmetry, &g_set);
    if (r) return r;
    wdata_setconst(&g_set, "kF", kF);
    wdata_setconst(&g_set, "eF", eF);
    wdata_setconst(&g_set, "mu_a", mu_a);
    wdata_setconst(&g_set, "mu_b", mu_b);
    return clear_files(&md, &g_set);
}

int wdref_write(int it, double *dens, double *pots, const double *vext_a, const double *vext_b,
                const double *velext_a, const double *velext_b, const double *dext)
{
    g_vext[0] = vext_a; g_vext[1] = vext_b;
    g_velext[0] = velext_a; g_velext[1] = velext_b;
    g_dext = dext;
    double mu[2] = {0.0, 0.0};
    wslda_density D = convert_into_wslda_density(dens, WD_N);
    wslda_potential P = convert_into_wslda_potential(pots, WD_N, mu);
    return write_measurments(&g_set, MPI_COMM_WORLD, "td", it, D, P);
}

int wdref_meta(const char *path)
{
    FILE *f = fopen(path, "w");
    if (!f) return 1;
    wdata_print_metadata(&g_set, f);
    fclose(f);
    return 0;
}
