/*
 * Names a W-SLDA project's problem-definition.h expects to exist when it is compiled into the
 * kernel translation unit (td-project-template/problem-definition.h; the reference provides
 * them through hpc-engine/wslda_cuda_utils.h:21-34, pca_macro.h:134-160, wslda_potdens.h:53-98
 * and pca_utils.h:16-172).  Kept name-for-name so an unmodified user file compiles:
 *   - Complex == thrust::complex<double>
 *   - __constant__ dc_mu_a, dc_mu_b, dc_ec, dc_t0, dc_dt, dc_kF, dc_eF, dc_nF, dc_sclgth,
 *     dc_params[MAX_USER_PARAMS], dc_extra_data, dc_extra_data_size
 *   - wslda_density / wslda_potential pointer bundles (same field order and meaning)
 *   - metadata_t with the run-time fields hooks read (input->akF, input->sclgth, md.params ...)
 *   - index decoding macros ixyz2ixiyiz / ixy2ixiy2d
 * Include after predefines.h and wtd_settings.h, before problem-definition.h.
 */
#ifndef WTD_SURFACE_H
#define WTD_SURFACE_H

#include <cuda_runtime.h>
#include <thrust/complex.h>
#include <stdio.h>
#include <math.h>
typedef thrust::complex<double> Complex;

__constant__ double dc_mu_a;
__constant__ double dc_mu_b;
__constant__ double dc_ec;
__constant__ double dc_t0;
__constant__ double dc_dt;
__constant__ double dc_kF;
__constant__ double dc_eF;
__constant__ double dc_nF;
__constant__ double dc_sclgth;
__constant__ void *dc_extra_data;
__constant__ size_t dc_extra_data_size;
__constant__ double dc_params[MAX_USER_PARAMS];

/* host mirrors of the constants (wslda_cuda_utils.h:36-45) */
static double hc_mu_a = 0.0, hc_mu_b = 0.0, hc_ec = 0.0, hc_t0 = 0.0, hc_dt = 0.0;
static double hc_kF = 0.0, hc_eF = 0.0, hc_nF = 0.0, hc_sclgth = 0.0;

#define ixyz2ixiyiz(ixyz,_ix,_iy,_iz,i) \
    i=(int)(ixyz);                      \
    _ix=i/(NY*NZ);                      \
    i=i-_ix*NY*NZ;                      \
    _iy=i/NZ;                           \
    _iz=i-_iy*NZ;

#define ixy2ixiy2d(ixy,_ix,_iy) \
    _ix=(int)(ixy)/NY;          \
    _iy=(int)(ixy)-_ix*NY;

typedef struct {
    int nx, ny, nz, datadim, blocklength;
    Complex *nu;
    double *rho_a, *rho_b, *tau_a, *tau_b;
    double *j_a_x, *j_a_y, *j_a_z, *j_b_x, *j_b_y, *j_b_z;
} wslda_density;

typedef struct {
    int nx, ny, nz, datadim, blocklength;
    Complex *delta;
    double *alpha_a, *alpha_b, *V_a, *V_b;
    double *A_a_x, *A_a_y, *A_a_z, *A_b_x, *A_b_y, *A_b_z;
    double *mu;
} wslda_potential;

/* density array layout [nu(c), rho_a, tau_a, j_a_xyz, rho_b, tau_b, j_b_xyz]
 * (pca_dens.cu:233-243, wslda_potdens.c:14-38): 12 blocks of doubles */
static inline wslda_density convert_into_wslda_density(double *d, int bl)
{
    wslda_density r;
    r.nx = NX; r.ny = (CODEDIM >= 2) ? NY : 1; r.nz = (CODEDIM >= 3) ? NZ : 1;
    r.datadim = CODEDIM; r.blocklength = bl;
    r.nu = (Complex *)(d + 0 * (size_t)bl);
    r.rho_a = d + 2 * (size_t)bl; r.tau_a = d + 3 * (size_t)bl;
    r.j_a_x = d + 4 * (size_t)bl; r.j_a_y = d + 5 * (size_t)bl; r.j_a_z = d + 6 * (size_t)bl;
    r.rho_b = d + 7 * (size_t)bl; r.tau_b = d + 8 * (size_t)bl;
    r.j_b_x = d + 9 * (size_t)bl; r.j_b_y = d + 10 * (size_t)bl; r.j_b_z = d + 11 * (size_t)bl;
    return r;
}

/* potential array layout [V_a, V_b, delta(c), alpha_a, alpha_b, A_a_xyz, A_b_xyz]
 * (wslda_potdens.c:44-70): 12 blocks of doubles */
static inline wslda_potential convert_into_wslda_potential(double *d, int bl, double *mu)
{
    wslda_potential r;
    r.nx = NX; r.ny = (CODEDIM >= 2) ? NY : 1; r.nz = (CODEDIM >= 3) ? NZ : 1;
    r.datadim = CODEDIM; r.blocklength = bl;
    r.V_a = d + 0 * (size_t)bl; r.V_b = d + 1 * (size_t)bl;
    r.delta = (Complex *)(d + 2 * (size_t)bl);
    r.alpha_a = d + 4 * (size_t)bl; r.alpha_b = d + 5 * (size_t)bl;
    r.A_a_x = d + 6 * (size_t)bl; r.A_a_y = d + 7 * (size_t)bl; r.A_a_z = d + 8 * (size_t)bl;
    r.A_b_x = d + 9 * (size_t)bl; r.A_b_y = d + 10 * (size_t)bl; r.A_b_z = d + 11 * (size_t)bl;
    r.mu = mu;
    return r;
}

/* Run-time inputs of a TD run that hook code may read (subset of pca_utils.h:16-172). */
#define MD_CHAR_LGTH 128
typedef struct {
    int inittype, measurements, timesteps;
    double dt, kc, ec;
    char inprefix[MD_CHAR_LGTH], outprefix[MD_CHAR_LGTH];
    int nthreads, batch, selfstart;
    double qfalpha, qfbeta, qfgamma, qfNreq, qfstart, qfstop, qfswitch;
    double Na, Nb, npart;
    double alpha, beta, temperature, referencekF;
    int spinsymmetry;
    double ccstart, ccstop, ccswitch;
    int hkf_mode;
    double hkf_mu, hkf_T;
    double sclgth, akF;
    double params[MAX_USER_PARAMS];
} metadata_t;

metadata_t md;
metadata_t *input = &md;

#endif
