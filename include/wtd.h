/*
 * wtd.h — C ABI of the B200 TD-(A)SLDA/BdG step library (one library per W-SLDA project,
 * built from the project's predefines.h and problem-definition.h).
 *
 * This is the fused entry surface.  It replaces, as one stream-ordered unit, the sequence the
 * reference's host driver issues per time step through its C ABI
 *   hpc-engine/pca.c:1401-1571 (cpca.c:1262-, ccpca.c:1137-) calling
 *   abm_step1 / abm_step4          hpc-engine/tdwslda_ode_integrator.h:106, :195
 *   normalize_wf                   hpc-engine/pca_kernels.cu:955
 *   compute_derivatives / _laplace hpc-engine/pca_derivative.cu:217, :332
 *   calculate_densities            hpc-engine/pca_dens.cu:220
 *   density_caculate_tau           hpc-engine/pca_dens.cu:300
 *   compute_potentials             hpc-engine/pca_kernels.cu:81
 *   apply_hamiltonian              hpc-engine/pca_kernels.cu:674
 *   compute_energy                 hpc-engine/pca_kernels.cu:211
 * and the constant setters memcopy_const / memcopy_const_params / memcopy_const_sclgth /
 * memcopy_extra_data (hpc-engine/wslda_cuda_utils.h:47-105).
 *
 * Conventions (kept from the reference):
 *  - N = NX (1D), NX*NY (2D), NX*NY*NZ (3D); x is the slowest index.
 *  - states: 2*nwf*N complex numbers [u_0..u_{nwf-1}, v_0..v_{nwf-1}], interleaved (re, im)
 *    doubles on the host, as cufftDoubleComplex / double complex in the reference.
 *  - densities: 12*N doubles [nu (complex), rho_a, tau_a, j_a_x, j_a_y, j_a_z,
 *    rho_b, tau_b, j_b_x, j_b_y, j_b_z] (hpc-engine/pca_dens.cu:233-243).
 *  - potentials: 12*N doubles [V_a, V_b, Delta (complex), alpha_a, alpha_b, A_a_xyz, A_b_xyz]
 *    (hpc-engine/wslda_potdens.c:44-70).
 *  - energy: TDWSLDAITEMS = 11 doubles [E_kin, E_pot, E_pair, E_curr, E_ext_V, E_ext_Delta,
 *    E_ext_v, N_a, N_b, L_za, L_zb] (hpc-engine/pca_settings.h:143-158).
 *  - return value 0 = success; nonzero = error (see wtd_error_string).  No call exits the
 *    process.
 *  - every call is ordered on the context's CUDA stream; calls that return host data
 *    synchronise before returning.
 */
#ifndef WTD_H
#define WTD_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct wtd_ctx wtd_ctx;

/* precision forms */
#define WTD_FP64 0        /* states, history, FFT and H psi in FP64 (drop-in form) */
#define WTD_MIXED_H64 1   /* states, FFT and H psi in FP32; ABM history/P stored in FP64 */
#define WTD_MIXED_H32 2   /* states, history, FFT and H psi in FP32; ABM sums, norms, densities FP64 */

/* error codes */
#define WTD_OK 0
#define WTD_ERR_ARG -1
#define WTD_ERR_CUDA -2
#define WTD_ERR_UNSUPPORTED -3
#define WTD_ERR_STATE -4
#define WTD_ERR_NOMEM -5
#define WTD_ERR_COMM -7   /* density exchange failed (NCCL missing or a collective error) */
#define WTD_ERR_IO -8     /* checkpoint file missing, short or not writable */

/* lattice and build facts of this library: dims[3], numel, codedim, scheme history length,
 * functional id (111 SLDA, 112 ASLDA, 113 BDG, 114 CUSTOMEDF), const-mass flag */
int wtd_info(int *dims, int *numel, int *codedim, int *nhist, int *functional, int *const_mass);
/* device bytes a context of nwf states in the given precision needs */
size_t wtd_device_bytes(int nwf, int precision);

int wtd_create(wtd_ctx **ctx, int nwf, int precision, int device);
int wtd_destroy(wtd_ctx *ctx);
const char *wtd_error_string(int code);

/* constants: replaces memcopy_const (wslda_cuda_utils.h:50), memcopy_const_params (:80),
 * memcopy_const_sclgth (:90), memcopy_extra_data (:44) */
int wtd_set_constants(wtd_ctx *ctx, double mu_a, double mu_b, double ec, double t0, double dt, double kF);
int wtd_set_params(wtd_ctx *ctx, const double *params /* MAX_USER_PARAMS */);
int wtd_set_sclgth(wtd_ctx *ctx, double a);
int wtd_set_extra_data(wtd_ctx *ctx, const void *host, size_t bytes);
/* user host hook process_params from problem-definition.h (pca.c:903) */
int wtd_process_params(wtd_ctx *ctx, double *params, double *kF, double *mu);

/* data in: occupations f_n (pca.c:837) and, for 1D/2D, per-state plane-wave ky, kz and
 * degeneracy cnt (NULL = 0, 0, 1) */
int wtd_upload_states(wtd_ctx *ctx, const double *host_states);
int wtd_upload_potentials(wtd_ctx *ctx, const double *host_pots);
int wtd_upload_occupations(wtd_ctx *ctx, const double *fbeta, const double *kky, const double *kkz, const int *cnt);
/* reference ABM history f1..fq (hpc-engine/tdwslda_checkpoint.c:223-364 layout, f1 newest);
 * slot in [0, q) */
int wtd_upload_history(wtd_ctx *ctx, int slot, const double *host);
int wtd_download_history(wtd_ctx *ctx, int slot, double *host);

/* initial measurement (pca.c:939-958): normalise, all densities, tau; zero ABM history */
int wtd_initial_measurement(wtd_ctx *ctx, int it0);
/* Taylor self-start (pca.c:1086-1330, input "selfstart 1"), after wtd_initial_measurement:
 * the first q steps (q = history length) are taken with a Taylor expansion of exp(-i H dt)
 * (midpoint potentials from a half step), recording (H - <H>) psi of each start state as the
 * ABM history; as in the reference, potentials and H use time index 0 during these steps and
 * the time index does not advance.  FP64 only. */
int wtd_selfstart(wtd_ctx *ctx);
/* nsteps ABM steps forming one measurement block (pca.c:1401-1571): tau and j are formed on
 * the block's last step (constant mass) or on every step (variable mass) */
int wtd_steps(wtd_ctx *ctx, int nsteps);
/* compute_energy (hpc-engine/tdwslda_energy_generic.h:21-111) into host[11] */
int wtd_energy(wtd_ctx *ctx, double *host11);
int wtd_sync(wtd_ctx *ctx);
int wtd_time_index(wtd_ctx *ctx);

int wtd_download_states(wtd_ctx *ctx, double *host_states);
int wtd_download_densities(wtd_ctx *ctx, double *host_dens);
int wtd_download_potentials(wtd_ctx *ctx, double *host_pots);
/* <psi_n|H|psi_n> dV of the last H application (left in d_workarea by the reference) */
int wtd_download_qpe(wtd_ctx *ctx, double *host_qpe);
/* densities (12 N, with tau and j) of a weighted subset of the current states: the reference's
 * subset tracking (pca.c:842-870, 1056-1066) with weights[n] = 1 for the tracked states, 0
 * otherwise (any real weights are accepted).  FP64. */
int wtd_subset_densities(wtd_ctx *ctx, const double *weights, double *host_dens);

/* Checkpoints in the reference's file layout (hpc-engine/tdwslda_checkpoint.c; restart with
 * inittype 5, pca.c:781-830): <dir>/checkpoint_<rank / howmany>, one file per IO group of
 * `howmany` ranks (MPI_NP_PER_IO_GROUP).  Every rank of a run calls save / load with its own
 * context, whose state count must be the rank's share of info.nwf (getnwfip,
 * pca_utils.c:660). */
typedef struct {
    double t0;                        /* time of the state */
    double mu_a, mu_b, ec, kF, eF, Effg, beta;
    int nwf;                          /* states of all ranks */
} wtd_checkpoint_info;
/* the file header (load_nwf, tdwslda_checkpoint.c:26-66) */
int wtd_checkpoint_info_read(const char *dir, int rank, int howmany, wtd_checkpoint_info *info);
/* write this rank's part (save_checkpoint, :215-364): E_n (ctx S values), k_perp (2D: k_z;
 * 1D: S k_y then S k_z; NULL in 3D), the states, the ABM history and, from the first rank of
 * a group, the header and the potentials */
int wtd_checkpoint_save(wtd_ctx *ctx, const char *dir, int rank, int nranks, int howmany,
                        const wtd_checkpoint_info *info, const double *En, const double *kperp);
/* read this rank's part back (load_checkpoint, :69-212): states, history, potentials, the
 * occupations fbeta(E_n, beta) and k_perp (1D: cnt = the degeneracy counts the run started
 * with, which the file does not hold); then the restart's measurement (densities, history
 * kept).  Set the constants first (t0 = info.t0 from wtd_checkpoint_info_read).  The outputs
 * may be NULL. */
int wtd_checkpoint_load(wtd_ctx *ctx, const char *dir, int rank, int nranks, int howmany, const int *cnt,
                        wtd_checkpoint_info *info, double *En, double *kperp);

/* Measurements in the W-data format of the reference's TD codes (wslda_writevars.c, lib/wdata):
 * <prefix>.wtxt plus <prefix>_<var>.wdat per variable.  vars: the input file's writevar tags
 * (rho, j, tau, V, V_ext, velocity_ext, delta, delta_ext, nu, alpha, A), separated by spaces or
 * commas; NULL or "" gives the reference's default "rho delta j".  dt_cycle: the time between
 * cycles (timesteps * dt); float_prec: 1 writes f32 (writeprec f).  begin removes the set's
 * old .wdat files; each write appends one cycle of the current densities and potentials at the
 * context's time index and rewrites the metadata. */
int wtd_wdata_begin(wtd_ctx *ctx, const char *prefix, const char *vars, double t0, double dt_cycle, int float_prec);
int wtd_wdata_write(wtd_ctx *ctx);

/* device pointers (for callers that keep data on the GPU): states, densities, potentials */
int wtd_device_pointers(wtd_ctx *ctx, void **states, double **dens, double **pots);
/* CUDA stream the context orders its work on (cudaStream_t) */
void *wtd_stream(wtd_ctx *ctx);
/* kernels launched by this context since creation (the fused passes and O(N) kernels) */
long long wtd_launch_count(wtd_ctx *ctx);
/* device timing of the two fused stream passes (CUDA events on the context stream around each
 * launch): enable, then read the summed milliseconds and launch counts since the last read */
int wtd_set_timing(wtd_ctx *ctx, int on);
int wtd_pass_times(wtd_ctx *ctx, double *ms_pass_a, double *ms_pass_b, int *count_a, int *count_b);

/* Optimal-control gradient (no counterpart in the reference, which has no adjoint).
 * From the states currently uploaded, runs wtd_initial_measurement(it0) and nsteps steps and
 * returns L = sum_r |Delta(r, T)|^2 mask(r) dV of the final pairing field (mask NULL = 1).
 * With grad non-NULL it also returns dL/dparams[j], j < nparam, through a hand-written
 * adjoint of the step: the forward keeps a checkpoint every checkpoint_every steps (0: the
 * largest interval whose step records fit in free device memory, all nsteps when they do),
 * records the last segment as it runs, and the reverse sweep recomputes each earlier segment
 * once.  Requires a contact-BdG project (Delta = -g nu, V = v_ext; WTD_ADJOINT_CONTACT_BDG
 * names the params index of g), constant mass, FP64 and a lattice on the fused path;
 * otherwise WTD_ERR_UNSUPPORTED.  The context is left as after the forward; its device
 * workspace is kept for the next call until wtd_adjoint_release or wtd_destroy. */
int wtd_adjoint(wtd_ctx *ctx, int it0, int nsteps, int checkpoint_every, const double *mask, int nparam,
                double *loss, double *grad);
int wtd_adjoint_release(wtd_ctx *ctx);
/* The same in two calls, for callers with a separate backward (an autograd function):
 * wtd_adjoint_forward runs the forward of wtd_adjoint with its checkpoints and records and
 * returns L; wtd_adjoint_backward then runs the reverse sweep and returns dL/dparams[0..nparam).
 * Between the two the context must not change: any launch, upload or setter on it makes the
 * backward return WTD_ERR_STATE (so does a backward without a forward, or a second backward:
 * the reverse sweep reuses the forward's records).  After the backward the context is again
 * where the forward left it. */
int wtd_adjoint_forward(wtd_ctx *ctx, int it0, int nsteps, int checkpoint_every, const double *mask, double *loss);
int wtd_adjoint_backward(wtd_ctx *ctx, int nparam, double *grad);
/* device time of the last adjoint forward (initial measurement, nsteps steps with checkpoints
 * and records, the loss) and of the last reverse sweep after it (recomputed segments and the
 * adjoint steps; 0 if none); WTD_ERR_STATE before any adjoint call */
int wtd_adjoint_times(wtd_ctx *ctx, double *ms_forward, double *ms_reverse);

/* high-k filters of the fields H is built from, f -> IFFT[FD(k^2/2; mu, T) FFT f], in place
 * after every functional evaluation, as the reference's driver and apply_hamiltonian do
 * (hkf_mode, pca_utils.h:131-133): mode >= 1 filters V_a, V_b (pca_kernels.cu:700-704), the
 * effective masses in variable-mass builds (pca.c:1448-1453) and the A components with
 * current corrections outside BdG (pca_kernels.cu:791-795); mode >= 2 also the pairing field
 * (pca_kernels.cu:758-762).  mu and T are energies (the reference's input gives them in units
 * of E_max = pi^2 / (2 dx^2), pca.c:183-185); mode 0 turns filtering off. */
int wtd_set_high_k_filter(wtd_ctx *ctx, int mode, double mu, double T);

/* quantum friction (cooling), as the reference's input qfalpha, qfbeta, qfgamma, qfNreq,
 * qfstart, qfstop, qfswitch (the times in units of 1/eF): in every step whose switch
 * (pca_utils.c:779-790, 1055-1060) is on, the friction densities are accumulated with the
 * gradient densities and H is built from V_s - U_s alpha/nF and the phase and particle-control
 * corrections of delta (pca_kernels.cu:497-539); the potentials themselves are not changed.
 * All coefficients 0 turns it off.  Fused-path lattices only (WTD_ERR_UNSUPPORTED otherwise). */
int wtd_set_quantum_friction(wtd_ctx *ctx, double qfalpha, double qfbeta, double qfgamma, double qfNreq,
                             double qfstart, double qfstop, double qfswitch);

/* ---- state-sharded runs (one process per GPU, each context holding a block of the states) ----
 * Densities are sums over states, so every density reduction of a sharded run is followed by a
 * sum over ranks: the reference's MPI_Allreduce of d_densities (hpc-engine/pca.c:948, 1433,
 * 1505).  Each context then holds the full densities and computes the same potentials.
 * Either attach an NCCL communicator (the sum runs on the context stream, no host sync), or
 * register a host hook (e.g. MPI after a stream sync).  Without either, the context's own
 * states are the whole system. */

/* NCCL: a 128-byte ncclUniqueId made on one rank and sent to all (any channel), then
 * wtd_nccl_attach on every rank.  libnccl.so.2 is loaded at run time (the process's copy if
 * one is already loaded). */
int wtd_nccl_unique_id(void *id128);
int wtd_nccl_attach(wtd_ctx *ctx, const void *id128, int nranks, int rank);

/* host hook: called after each density reduction with the device array of count doubles
 * (partial sums of this rank's states) and the context's cudaStream_t; it must leave the sum
 * over ranks in place, ordered on that stream, and return 0.  fn NULL removes the hook. */
typedef int (*wtd_exchange_fn)(void *user, double *dens, size_t count, void *stream);
int wtd_set_density_exchange(wtd_ctx *ctx, wtd_exchange_fn fn, void *user);

#ifdef __cplusplus
}
#endif
#endif
