/*
 * ORACLE (test infrastructure only).  Runs the reference's uniform-solution generator for one
 * td-gauss replay case and writes the initial state the reference's TD driver starts from
 * (inittype 0, pca.c:257-330; cpca.c:258-325; ccpca.c).  It is compiled, by the `uniform`
 * target of oracle/Makefile, from hpc-engine/pca_uniform.h, pca_utils.c and
 * wslda_wavevectors.h where they lie, against a gauss_* project's predefines.h.
 *
 *   uniform_init <input.txt> <out.bin>
 *
 * Steps, as the reference's driver takes them: parse the input file (pca_utils.c:162), fix the
 * particle numbers of UNIFORM_TEST_MODE (pca.c:195-203), solve the uniform problem for the
 * functional (pca.c:263-270), count the states the 1D/2D engines evolve (cpca.c:268), create
 * the states of all ranks at once (pca.c:312).
 *
 * out.bin: int32 [codedim, N, nwf, spinsymmetry], then float64 [n0_a, n0_b, mu_a, mu_b, V_a,
 * V_b, alph_a, alph_b, ec, delta, beta, sclgth], float64 E_n[nwf], float64 k_perp (nwf in 2D: k_z;
 * 2 nwf in 1D: k_y then k_z; none in 3D), int32 cnt[nwf] (1D degeneracy, else 1), complex128
 * states [u_0..u_{nwf-1}, v_0..v_{nwf-1}] of N points each.
 */
#include <stdlib.h>
#include <stddef.h>
#include <stdio.h>
#include <string.h>
#include <math.h>
#include <complex.h>
#define TDWSLDA_MAIN /* as pca.c:1: the host prototypes of pca_kernels.h take double complex */
#include "predefines.h"
#include "pca_settings.h"
#include "pca_macro.h"
#include "pca_utils.h"
#include "pca_kernels.h" /* prototypes of the host EDF functions (*_h) */
#include "wslda_wavevectors.h"
#include "pca_uniform.h"

/* the process id that the reference's drivers keep globally (pca.c:39); one process here */
int wsldapid = 0;

/* file helpers of pca_io.h, referenced only by save_uniform/read_uniform (pca_uniform.h:504-635),
 * which this driver never calls; pca_io.h itself needs MPI */
int exists(const char *filename) { (void)filename; return 0; }
int urm(const char *fn) { (void)fn; return 0; }

#if CODEDIM == 3
#define UI_N NXYZ
#elif CODEDIM == 2
#define UI_N NXY
#else
#define UI_N NX
#endif

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s <input.txt> <out.bin>\n", argv[0]);
        return 1;
    }
    if (parse_input_file(argv[1]) != 1) return 2; /* 1 = parsed (pca_utils.c:618) */
#ifdef SPINSYMMETRY_MODE
    md.spinsymmetry = 1;
#else
    md.spinsymmetry = 0;
#endif
#ifdef UNIFORM_TEST_MODE
    md.Na = ceil(1.0 / (6.0 * M_PI * M_PI) * LXYZ);
    md.Nb = (md.spinsymmetry == 1) ? md.Na : md.Na + 1;
    md.init0Na = md.Na;
    md.init0Nb = md.Nb;
#endif
    int nwf = 0, rc;
#if FUNCTIONAL == BDG
    rc = solve_uniform_problem_bdg(md.init0Na / LXYZ, md.init0Nb / LXYZ, &nwf, 1);
#elif FUNCTIONAL == SLDAE
    rc = solve_uniform_problem_sldae(md.init0Na / LXYZ, md.init0Nb / LXYZ, &nwf, 1);
#else
    rc = solve_uniform_problem(md.init0Na / LXYZ, md.init0Nb / LXYZ, &nwf, 1);
#endif
    if (rc != 0) return 3;
#if CODEDIM == 2
    if (get_nwf_to_evolve_2d(&nwf) != 0) return 4;
#elif CODEDIM == 1
    if (get_nwf_to_evolve_1d(&nwf) != 0) return 4;
#endif
    double complex *wf = (double complex *)calloc((size_t)2 * nwf * UI_N, sizeof(double complex));
    double *fEn = (double *)calloc(nwf, sizeof(double)), *En = (double *)calloc(nwf, sizeof(double));
    double *kk = (double *)calloc(2 * (size_t)nwf, sizeof(double));
    int *cnt = (int *)calloc(nwf, sizeof(int));
    double mu_a, mu_b, ec;
    for (int i = 0; i < nwf; i++) cnt[i] = 1;
#if CODEDIM == 3
    rc = create_uniform_wf(0, nwf, wf, &mu_a, &mu_b, &ec, fEn, En, 1);
    int nk = 0;
#elif CODEDIM == 2
    rc = create_uniform_wf_2d(0, nwf, wf, &mu_a, &mu_b, &ec, fEn, kk, En, 1);
    int nk = nwf;
#else
    rc = create_uniform_wf_1d(0, nwf, wf, &mu_a, &mu_b, &ec, fEn, kk, cnt, En, 1);
    int nk = 2 * nwf;
#endif
    if (rc != 0) return 5;
    FILE *f = fopen(argv[2], "wb");
    if (!f) return 6;
    int hdr[4] = {CODEDIM, UI_N, nwf, md.spinsymmetry};
    double m[12] = {__md_pca_uniform.n0_a, __md_pca_uniform.n0_b, mu_a, mu_b, __md_pca_uniform.V_a,
                    __md_pca_uniform.V_b, __md_pca_uniform.alph_a, __md_pca_uniform.alph_b, ec,
                    __md_pca_uniform.delta, __md_pca_uniform.beta, md.sclgth};
    fwrite(hdr, sizeof(int), 4, f);
    fwrite(m, sizeof(double), 12, f);
    fwrite(fEn, sizeof(double), nwf, f);
    fwrite(kk, sizeof(double), nk, f);
    fwrite(cnt, sizeof(int), nwf, f);
    fwrite(wf, sizeof(double complex), (size_t)2 * nwf * UI_N, f);
    fclose(f);
    free(wf); free(fEn); free(En); free(kk); free(cnt);
    return 0;
}
