/*
 * wslda_td_compat.h — the reference's per-kernel C ABI, provided by this library with the
 * same names, argument meaning and error behaviour (0 = success, nonzero = error code), so
 * the reference's host drivers hpc-engine/pca.c, cpca.c, ccpca.c can link against libwtd.so
 * in place of the objects of hpc-engine/mk.td:44-51 (NVCCSRCS1D/2D/3D + reduce_many.o +
 * tdwslda_memory_management.o).
 *
 * Every array is a caller-owned device buffer, as in the reference.  Complex arrays are
 * cufftDoubleComplex (two doubles, re/im) — declared here as wtd_z so the header needs no CUDA
 * include; the ABI is identical.  Work is issued on the legacy default stream and every call
 * returns after the work is complete, the reference's synchronous contract
 * (hpc-engine/pca_macro.h:63-74: callers read results right after return).
 *
 * Dimension-specific signatures follow the reference: 3D (pca_*), 2D (cpca_*: d_kkz replaces
 * the z derivative, calculate_densities takes kkz), 1D (ccpca_*: kkyz = [ky(n), kz(n)],
 * calculate_densities takes kkyz and cnt).  Compile-time WTD_CODEDIM selects them for C
 * callers (1, 2 or 3; default 3).
 */
#ifndef WSLDA_TD_COMPAT_H
#define WSLDA_TD_COMPAT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double x, y; } wtd_z; /* layout of cufftDoubleComplex / double complex */

#ifndef WTD_CODEDIM
#define WTD_CODEDIM 3
#endif

/* constants and memory (hpc-engine/wslda_cuda_utils.h:44-330) */
int memcopy_const(double mu_a, double mu_b, double ec, double t0, double dt, double kF);
int memcopy_const_params(double *params);
int memcopy_const_sclgth(double a);
int memcopy_extra_data(size_t extra_data_size, void *extra_data);
int set_gpu(int device);
int gpu_malloc(size_t size, void **pointer);
int gpu_free(void *pointer);
int host_malloc_pl(size_t size, void **pointer);
int host_free_pl(void *pointer);
int memcopy_host2gpu(void *host, void *gpu, size_t size);
int memcopy_gpu2host(void *gpu, void *host, size_t size);
int memcopy_gpu2gpu(void *gpusrc, void *gpudst, size_t size);

/* workspace (hpc-engine/pca_derivative.cu:41-133, tdwslda_memory_management.cu:31-94):
 * create_cufftPlans reports the bytes of the work area the library needs for nwfip states;
 * the caller allocates it and hands it over with set_workspace_for_cufftPlan.  No cuFFT is
 * used: the transforms are this library's own.  qp energies are left in work[0..nwfip). */
int create_cufftPlans(int batch_size, int nwfip, size_t *workSize);
int set_workspace_for_cufftPlan(void *workArea);
size_t mm_get_size_of_kernels_workspace(size_t n);
size_t mm_get_size_of_derivatives_workspace(size_t n);
size_t mm_get_size_of_total_workspace(size_t n);
void *mm_get_pointer_to_kernels_workspace(size_t n);
void *mm_get_pointer_to_derivatives_workspace(size_t n);
void *mm_get_pointer_to_total_workspace(size_t n);

/* host forms of the energy-density-functional pieces (hpc-engine/pca_kernels.h:11-30,
 * cpca_kernels.h, ccpca_kernels.h; pca_edf.h:46-350), called by the drivers' uniform-solution
 * start (pca_uniform.h) */
double polarization_h(double n_a, double n_b);
double der_polarization__der_na_h(double n_a, double n_b);
double der_polarization__der_nb_h(double n_a, double n_b);
double alpha_h(double p);
double alpha_a_h(double p);
double alpha_b_h(double p);
double alpha_plus_h(double p);
double alpha_minus_h(double p);
double der_alpha_plus__der_na_h(double n_a, double n_b);
double der_alpha_plus__der_nb_h(double n_a, double n_b);
double der_alpha_minus__der_na_h(double n_a, double n_b);
double der_alpha_minus__der_nb_h(double n_a, double n_b);
double funG_h(double p);
double funD_h(double n_a, double n_b);
double der_funD__der_na_h(double n_a, double n_b);
double der_funD__der_nb_h(double n_a, double n_b);
double tildeC_h(double n_a, double n_b);
double der_tildeC__der_na_h(double n_a, double n_b);
double der_tildeC__der_nb_h(double n_a, double n_b);

/* ABM predictor / corrector (hpc-engine/tdwslda_ode_integrator.h:106, :195) */
int abm_step1(int n, wtd_z *ykm1, wtd_z *fkm1, wtd_z *fkm2, wtd_z *fkm3, wtd_z *fkm4, wtd_z *fkm5,
              int abm_scheme, int nthreads);
int abm_step4(int n, wtd_z *ykm1_in, wtd_z *ykm1_out, wtd_z *fkm_last, int abm_scheme, int nthreads);
/* normalisation (hpc-engine/pca_kernels.cu:955) */
int normalize_wf(int n, wtd_z *wf, int nthreads);
/* spectral derivatives of n fields (hpc-engine/pca_derivative.cu:217, :332) */
int compute_derivatives(int n, wtd_z *wf, wtd_z *wf_d_dx, wtd_z *wf_d_dy, wtd_z *wf_d_dz, wtd_z *wf_laplace, int nthreads);
int compute_laplace(int n, wtd_z *wf, wtd_z *wf_laplace, int nthreads);
/* real-field derivatives (hpc-engine/pca_derivative.cu:444, 548, 630, 710) */
int compute_gradient_real_f(double *f, double *df_dx, double *df_dy, double *df_dz, int nthreads);
int compute_derivative_real_vector_f(double *fx, double *fy, double *fz, double *dfx_dx, double *dfy_dy, double *dfz_dz, int nthreads);
int compute_laplace_real_f(double *f, double *laplace_f, int nthreads);
int compute_divergence_real_vector_f(double *fx, double *fy, double *fz, double *divf, int nthreads);
/* Fermi-Dirac high-k filters, FD(k^2/2; mu, T) in k-space (hpc-engine/pca_derivative.cu:829,
 * 906, 950); out may alias in */
int high_frequency_filter_d(double *in, double *out, double fd_mu, double fd_T, int nthreads);
int high_frequency_filter_c(wtd_z *in, wtd_z *out, double fd_mu, double fd_T, int nthreads);
int high_frequency_filter_massive_d(int n, double *in, double *out, double fd_mu, double fd_T, int nthreads);

/* densities (hpc-engine/pca_dens.cu:220, cpca_dens.cu:239, ccpca_dens.cu:239) */
#if WTD_CODEDIM == 3
int calculate_densities(int n, wtd_z *wf, wtd_z *wf_d_dx, wtd_z *wf_d_dy, wtd_z *wf_d_dz, wtd_z *d_wf_laplace,
                        double *d_fbetaEn, double *weights, double *d_densities, int gradients_computed, int nthreads);
#elif WTD_CODEDIM == 2
int calculate_densities(int n, wtd_z *wf, wtd_z *wf_d_dx, wtd_z *wf_d_dy, wtd_z *d_wf_laplace, double *kkz,
                        double *d_fbetaEn, double *weights, double *d_densities, int gradients_computed, int nthreads);
#else
int calculate_densities(int n, wtd_z *wf, wtd_z *wf_d_dx, wtd_z *d_wf_laplace, double *kkyz,
                        double *d_fbetaEn, double *weights, int *cnt, double *d_densities, int gradients_computed, int nthreads);
#endif
/* quantum-friction densities [U_a, U_b, D (complex)] (4 N doubles; the reference keeps them at
 * d_densities + 12 N) from the states and their laplacians (hpc-engine/pca_dens.cu:431,
 * cpca_dens.cu:471, ccpca_dens.cu:470); apply_hamiltonian reads them there when qfswitch > 0 */
#if WTD_CODEDIM == 3
int calculate_quantum_friction_densities(int n, wtd_z *wf, wtd_z *d_wf_laplace, double *d_fbetaEn, double *weights,
                                         double *d_qf_densities, int nthreads);
#elif WTD_CODEDIM == 2
int calculate_quantum_friction_densities(int n, wtd_z *wf, wtd_z *d_wf_laplace, double *kkz, double *d_fbetaEn,
                                         double *weights, double *d_qf_densities, int nthreads);
#else
int calculate_quantum_friction_densities(int n, wtd_z *wf, wtd_z *d_wf_laplace, double *kkyz, double *d_fbetaEn,
                                         double *weights, int *cnt, double *d_qf_densities, int nthreads);
#endif
#define WTD_ERR_NOALLOC_SIZE -6
/* calculate_densities_noalloc: no counterpart in the reference.  Same arguments, result and
 * error behaviour as calculate_densities above, for callers that cannot call cudaMalloc (a
 * host whose device memory is owned by a pool reserved at start-up, an embedding runtime that
 * forbids the library from allocating): it needs no work area and allocates nothing.  Its
 * scratch is a fixed 8 MiB device array inside the library, so it accepts lattices with
 * 12*N doubles <= 1 Mi words (N <= 87381 points) and returns WTD_ERR_NOALLOC_SIZE (-6)
 * otherwise.  The array is shared by all calls: calls that overlap on the GPU race on it.
 * The first call on a device resolves the array's device address with that device current;
 * make that first call before any stream capture on the device. */
#if WTD_CODEDIM == 3
int calculate_densities_noalloc(int n, wtd_z *wf, wtd_z *wf_d_dx, wtd_z *wf_d_dy, wtd_z *wf_d_dz, wtd_z *d_wf_laplace,
                                double *d_fbetaEn, double *weights, double *d_densities, int gradients_computed, int nthreads);
#elif WTD_CODEDIM == 2
int calculate_densities_noalloc(int n, wtd_z *wf, wtd_z *wf_d_dx, wtd_z *wf_d_dy, wtd_z *d_wf_laplace, double *kkz,
                                double *d_fbetaEn, double *weights, double *d_densities, int gradients_computed, int nthreads);
#else
int calculate_densities_noalloc(int n, wtd_z *wf, wtd_z *wf_d_dx, wtd_z *d_wf_laplace, double *kkyz,
                                double *d_fbetaEn, double *weights, int *cnt, double *d_densities, int gradients_computed, int nthreads);
#endif
int density_caculate_tau(double *d_densities, int nthreads);
int symmetrize_densities_device(double *d_densities);

/* functional and H psi (hpc-engine/pca_kernels.cu:81, 674, 1020; cpca_kernels.cu:676;
 * ccpca_kernels.cu:625).  qfswitch > 0 adds the quantum-friction terms built from the friction
 * densities after the 12 N density words (pca_kernels.cu:497-539) to H, with pccoeff the
 * particle-control coefficient. */
int compute_potentials(int it, double *d_densities, double *d_potentials, double cccoeff, int nthreads);
int multiply_wf_by_alpha(int n, wtd_z *wf_in, wtd_z *wf_out, double *d_potentials, int nthreads);
#if WTD_CODEDIM == 3
int apply_hamiltonian(int it, int n, wtd_z *wf_in, wtd_z *wf_out, wtd_z *wf_d_dx, wtd_z *wf_d_dy, wtd_z *wf_d_dz,
                      wtd_z *wf_laplace, wtd_z *alphawf_laplace, double *d_densities, double *d_potentials,
                      double qfswitch, double *useqpe, double pccoeff, int nthreads);
#elif WTD_CODEDIM == 2
int apply_hamiltonian(int it, int n, wtd_z *wf_in, wtd_z *wf_out, wtd_z *wf_d_dx, wtd_z *wf_d_dy, double *d_kkz,
                      wtd_z *wf_laplace, wtd_z *alphawf_laplace, double *d_densities, double *d_potentials,
                      double qfswitch, double *useqpe, double pccoeff, int nthreads);
#else
int apply_hamiltonian(int it, int n, wtd_z *wf_in, wtd_z *wf_out, wtd_z *wf_d_dx, double *d_kkyz,
                      wtd_z *wf_laplace, wtd_z *alphawf_laplace, double *d_densities, double *d_potentials,
                      double qfswitch, double *useqpe, double pccoeff, int nthreads);
#endif
/* energies: 11 doubles left at d_workarea[0..10] (hpc-engine/tdwslda_energy_generic.h:21) */
int compute_energy(int it, double *d_densities, double *d_potentials, double *d_workarea, int nthreads);
/* n sums of length m: out[k] = sum_i in[k*m + i] (hpc-engine/reduce_many.cu:155) */
int local_reductions_many(int n, int m, double *d_in, double *d_out);
/* overlaps <wf1_n|wf2_n> dV (hpc-engine/pca_kernels.cu:871) */
int compute_ovelap(int n, wtd_z *wf1, wtd_z *wf2, double *overlap_re, double *overlap_im, double *workarea, int nthreads);
/* Taylor self-start term (hpc-engine/pca_kernels.cu:1075) */
int taylor_expansion_contribution(int it, double dt, int n, wtd_z *wf_hpsi, wtd_z *wf_update, wtd_z *wf_contr, int nthreads);
/* external fields to host arrays (hpc-engine/pca_kernels.cu:1110-1181) */
int get_v_ext(int datadim, int spin, int it, double *data);
int get_delta_ext(int datadim, int it, void *deltain, void *data);
int get_velocity_ext(int datadim, int spin, int it, double *data);

#ifdef __cplusplus
}
#endif
#endif
