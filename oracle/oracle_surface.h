/*
 * ORACLE (test infrastructure only; never linked into the product library).
 *
 * Host emulation of the names a W-SLDA problem-definition.h uses, so the same unmodified user
 * file compiles as plain C++ into the CPU oracle: Complex and the thrust:: calls map onto
 * std::complex<double>, CUDA qualifiers vanish, the __constant__ dc_* values become host
 * globals, and per-point __global__ kernels (CUSTOMEDF functional, modify_potentials) are run
 * by a host loop that sets threadIdx.x.  Mirrors hpc-engine/wslda_cuda_utils.h:21-34 and
 * pca_macro.h:134-160 name-for-name.
 */
#ifndef ORACLE_SURFACE_H
#define ORACLE_SURFACE_H
#include <complex>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef std::complex<double> Complex;
namespace thrust {
template <class T> using complex = std::complex<T>;
using std::conj; using std::norm; using std::abs; using std::arg;
using std::sqrt; using std::log; using std::exp; using std::polar; using std::pow;
}
#define __device__
#define __host__
#define __global__
#define __constant__
#define __forceinline__ inline

struct orc_dim3 { unsigned int x, y, z; };
static orc_dim3 threadIdx = {0, 0, 0}, blockIdx = {0, 0, 0}, blockDim = {1, 1, 1};

static double dc_mu_a, dc_mu_b, dc_ec, dc_t0, dc_dt, dc_kF, dc_eF, dc_nF, dc_sclgth;
static void *dc_extra_data = nullptr;
static size_t dc_extra_data_size = 0;

#define ixyz2ixiyiz(ixyz,_ix,_iy,_iz,i) \
    i=(int)(ixyz); _ix=i/(NY*NZ); i=i-_ix*NY*NZ; _iy=i/NZ; _iz=i-_iy*NZ;
#define ixy2ixiy2d(ixy,_ix,_iy) _ix=(int)(ixy)/NY; _iy=(int)(ixy)-_ix*NY;

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
    double params[64];
} metadata_t;
static metadata_t md;
static metadata_t *input = &md;
#endif
