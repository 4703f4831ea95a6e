/*
 * Host side of the fused C ABI (include/wtd.h): a context owns the device state of one run —
 * states, the ABM history ring, densities, potentials, per-point H coefficients and the
 * density partial slots — and orders all work on one CUDA stream.
 *
 * One step (wtd_steps) issues, on the context stream:
 *   pass A  -> reduce density slots -> [tau] -> potentials(it+1) -> coefficients(it+1)
 *   pass B  -> reduce density slots -> [tau] -> potentials(it+1) -> coefficients(it+1)
 * which is the reference's per-step sequence (hpc-engine/pca.c:1401-1571) with its ~30
 * whole-array kernels per half step folded into one stream pass.
 */
#ifndef WTD_API_CUH
#define WTD_API_CUH

#include <dlfcn.h>
#include <nccl.h>
#include "wtd_lattice.cuh"

struct wtd_ctx {
    int dev, S, prec;
    size_t ysz, hsz;            /* bytes per state array (y) and per history slot */
    void *y;
    void *hist[WTD_NHIST];      /* physical slots */
    int head;                   /* ring position 0 = physical slot head */
    double *cf, *occ, *kp2, *wcnt, *dslot, *qpe, *dens, *pots, *ework, *eout;
    double2 *tw;
    double *ktab;
    double2 *stage;             /* FP64 staging for conversions (mixed precision) */
    void *extra;
    size_t extra_bytes;
    int grid;
    int block;                  /* threads per CTA of the fused passes on large lattices */
    int prefetch;               /* L2 prefetch set of the fused passes (StepArgs::prefetch) */
    int it;
    int fk_given;
    int have_coef;
    double dt;
    cudaStream_t st;
    long long launches;
    long long mut;              /* uploads and setters so far (a recorded adjoint forward checks it) */
    /* optional device timing of the fused passes: events around each pass, summed on demand */
    int timing;
    cudaEvent_t ev[2][2][4096];
    int nev[2];
    /* large 3D lattices (state larger than one CTA's shared memory): the line path
     * (wtd_path3d.cuh), or the staged path where the line path does not apply (quantum
     * friction, large 2D lattices) */
    int staged;
    double2 *ddx, *ddy, *ddz, *dlap, *dalap, *stage3d;
    int line;                   /* line path in use */
    void *kbuf;                 /* K_yz of every state, compute precision */
    int ncl;                    /* clusters of the x-line kernel */
    int g2;                     /* state chunks of the plane density kernel */
    int p1grid;                 /* CTAs of the plane H kernel */
    void *xfer;                 /* bounded staging buffer of the mixed-precision uploads/downloads */
    /* state-sharded runs: sum of the density partials over ranks (NCCL or a host hook) */
    void *nccl;
    wtd_exchange_fn xfn;
    void *xuser;
    /* adjoint workspace kept between gradient calls (AdjWork, released with the context) */
    void *adj;
    /* W-data output set (wtd_wdata.cuh) and its destructor */
    void *wdata;
    void (*wdata_free)(void *);
    /* high-k filter of the effective masses after every functional evaluation (variable mass) */
    int hkf_mode;
    double hkf_mu, hkf_T;
    /* quantum friction: alpha, beta, gamma, N_req, start, stop, ramp (times in 1/eF); the switch
     * value of the current step; particle-control coefficient (device); the fields H uses */
    double qf[7];
    double qfsw;
    double *dqf, *qfld;
    int sstride;                /* density-slot words per CTA: 12 N, 16 N with quantum friction */
    int sdg;                    /* state chunks of the staged density kernel (staged_dens_chunks) */
};

static void adj_release(wtd_ctx *c);

#define WTD_LAUNCHED(ctx) do { (ctx)->launches++; cudaError_t _e = cudaGetLastError(); if (_e != cudaSuccess) return WTD_ERR_CUDA; } while (0)

/* ---------------------------------------------------------------------------------------
 * density exchange of state-sharded runs.  NCCL is loaded at run time so that the library has
 * no link-time dependency and shares the process's NCCL when one is already loaded.
 * -------------------------------------------------------------------------------------*/
struct NcclApi {
    ncclResult_t (*get_unique_id)(ncclUniqueId *);
    ncclResult_t (*comm_init_rank)(ncclComm_t *, int, ncclUniqueId, int);
    ncclResult_t (*all_reduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t);
    ncclResult_t (*comm_destroy)(ncclComm_t);
};

static const NcclApi *nccl_api()
{
    static NcclApi api;
    static int state = 0; /* 0 untried, 1 loaded, -1 unavailable */
    if (state == 0) {
        state = -1;
        void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
        if (h) {
            api.get_unique_id = (decltype(api.get_unique_id))dlsym(h, "ncclGetUniqueId");
            api.comm_init_rank = (decltype(api.comm_init_rank))dlsym(h, "ncclCommInitRank");
            api.all_reduce = (decltype(api.all_reduce))dlsym(h, "ncclAllReduce");
            api.comm_destroy = (decltype(api.comm_destroy))dlsym(h, "ncclCommDestroy");
            if (api.get_unique_id && api.comm_init_rank && api.all_reduce && api.comm_destroy) state = 1;
        }
    }
    return state == 1 ? &api : NULL;
}

/* in-place sum over ranks of count doubles on the context stream (no-op for a lone context) */
static int exchange(wtd_ctx *c, double *buf, size_t count)
{
    if (c->nccl) {
        const NcclApi *a = nccl_api();
        if (!a || a->all_reduce(buf, buf, count, ncclFloat64, ncclSum, (ncclComm_t)c->nccl, c->st) != ncclSuccess)
            return WTD_ERR_COMM;
    } else if (c->xfn) {
        if (c->xfn(c->xuser, buf, count, (void *)c->st) != 0) return WTD_ERR_COMM;
    }
    return WTD_OK;
}

/* complex numbers per chunk of the mixed-precision uploads and downloads (64 MiB of FP64) */
#define WTD_XFER ((size_t)1 << 22)

static size_t elem_bytes_y(int prec) { return prec == WTD_FP64 ? sizeof(double2) : sizeof(float2); }
static size_t elem_bytes_h(int prec) { return prec == WTD_MIXED_H32 ? sizeof(float2) : sizeof(double2); }

/* ---------------------------------------------------------------------------------------
 * fused pass dispatch
 * -------------------------------------------------------------------------------------*/
template <typename TC, int NBUF> static constexpr size_t fused_smem() { return FusedSmem<WG, TC, NBUF>::bytes; }

template <typename TY, typename TH, typename TC, int PASS, bool GRAD>
static int launch_pass_t(wtd_ctx *c, StepArgs &a)
{
    constexpr int NBUF = WTD_VAR ? 4 : (GRAD ? 3 : 2);
    constexpr size_t sm = fused_smem<TC, NBUF>();
    if (sm > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
    else {
        if (c->block == 1024 && WG::ntot >= 2048) {
            auto k = wtd_fused_pass<WG, TY, TH, TC, WTD_NHIST, PASS, WTD_VAR, GRAD, 1024>;
            WTD_ONCE_PER_DEVICE(
                WTD_CU(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)));
            k<<<c->grid, 1024, sm, c->st>>>(a, c->tw, c->ktab);
        } else {
            auto k = wtd_fused_pass<WG, TY, TH, TC, WTD_NHIST, PASS, WTD_VAR, GRAD, 512>;
            WTD_ONCE_PER_DEVICE(
                WTD_CU(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)));
            int threads = WG::ntot >= 512 ? 512 : ((WG::ntot + 31) / 32) * 32;
            k<<<c->grid, threads, sm, c->st>>>(a, c->tw, c->ktab);
        }
        WTD_LAUNCHED(c);
    }
    return WTD_OK;
}

template <int PASS, bool GRAD>
static int launch_pass(wtd_ctx *c, StepArgs &a)
{
    if (c->prec == WTD_FP64) return launch_pass_t<double2, double2, double, PASS, GRAD>(c, a);
    if (c->prec == WTD_MIXED_H64) return launch_pass_t<float2, double2, float, PASS, GRAD>(c, a);
    return launch_pass_t<float2, float2, float, PASS, GRAD>(c, a);
}

static void ring_slots(wtd_ctx *c, void **slot)
{
    for (int r = 0; r < WTD_NHIST; r++) slot[r] = c->hist[(c->head + r) % WTD_NHIST];
}

static StepArgs make_args(wtd_ctx *c)
{
    StepArgs a;
    memset(&a, 0, sizeof(a));
    a.y = c->y;
    ring_slots(c, a.slot);
    a.cf = c->cf; a.occ = c->occ; a.kp2 = c->kp2; a.wcnt = c->wcnt;
    a.dslot = c->dslot; a.qpe = c->qpe; a.dt = c->dt; a.S = c->S;
    a.fk_given = c->fk_given;
    a.prefetch = c->prefetch;
    a.accumulate = 0;
    a.sstride = c->sstride;
    a.qf = c->qfsw > 0.0 ? 1 : 0;
    return a;
}

static int run_pass(wtd_ctx *c, int pass, bool grad)
{
    StepArgs a = make_args(c);
    if (c->timing && pass < 2 && c->nev[pass] < 4096) {
        cudaEventRecord(c->ev[pass][0][c->nev[pass]], c->st);
        int r = (pass == 0) ? (grad ? launch_pass<0, true>(c, a) : launch_pass<0, false>(c, a))
                            : (grad ? launch_pass<1, true>(c, a) : launch_pass<1, false>(c, a));
        cudaEventRecord(c->ev[pass][1][c->nev[pass]], c->st);
        c->nev[pass]++;
        return r;
    }
    if (pass == 0) return grad ? launch_pass<0, true>(c, a) : launch_pass<0, false>(c, a);
    if (pass == 1) return grad ? launch_pass<1, true>(c, a) : launch_pass<1, false>(c, a);
    if (pass == 3) return launch_pass<3, false>(c, a);
    return grad ? launch_pass<2, true>(c, a) : launch_pass<2, false>(c, a);
}

static int line_pass(wtd_ctx *c, int pass, bool grad, const StepArgs *given = NULL);

/* f1 = (H - <H>) psi of the current state and its quasiparticle energies, as the reference
 * leaves them after a step (pca.c:1565, d_workarea[0..n)); later steps reuse f1 */
static int ensure_fk(wtd_ctx *c)
{
    if (c->fk_given) return WTD_OK;
    if (!c->have_coef) return WTD_ERR_STATE;
    if (c->line) WTD_TRY(line_pass(c, 3, false));
    else WTD_TRY(run_pass(c, 3, false));
    c->fk_given = 1;
    return WTD_OK;
}

/* high-k filters (hkf_mode) of the fields H is built from, in place, f -> IFFT[FD FFT f]:
 *   filter_alpha: alpha_a, alpha_b in variable-mass runs, after each functional evaluation
 *                 (the driver, pca.c:1448-1453; hkf_mode >= 1);
 *   filter_h:     V_a, V_b (hkf_mode >= 1, pca_kernels.cu:700-704), the pairing field (>= 2,
 *                 :758-762) and, with current corrections outside BdG, the six A components
 *                 (>= 1, :791-795) — the reference filters these at the top of every
 *                 apply_hamiltonian, which a step calls once after each functional evaluation */
static int filter_real(wtd_ctx *c, double *f, int nf)
{
    constexpr size_t sm = (size_t)WG::padded * sizeof(double2) + WG::twtotal * sizeof(double2) + sizeof(KTab<WG>);
    if (WTD_BIG) return big_filter_real(f, nf, c->hkf_mu, c->hkf_T, c->stage3d, c->tw, c->ktab, c->st);
    if (sm > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
    WTD_ONCE_PER_DEVICE(WTD_CU(cudaFuncSetAttribute(wtd_hkf_kernel<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)));
    wtd_hkf_kernel<WG><<<nf, 512, sm, c->st>>>(f, c->hkf_mu, c->hkf_T, c->tw, c->ktab);
    WTD_LAUNCHED(c);
    return WTD_OK;
}

static int filter_alpha(wtd_ctx *c)
{
    if (c->hkf_mode < 1 || !WTD_VAR) return WTD_OK;
    return filter_real(c, c->pots + 4 * (size_t)WTD_NUMEL, 2);
}

/* fld: [V_a, V_b, delta] to filter (the potentials, or the friction-modified copy) */
static int filter_h(wtd_ctx *c, double *fld = NULL)
{
    if (c->hkf_mode < 1) return WTD_OK;
    constexpr size_t N = WTD_NUMEL;
    if (!fld) fld = c->pots;
    WTD_TRY(filter_real(c, fld, 2));
#if defined(CURRENT_CORRECTIONS) && !defined(BDG_MODE)
    WTD_TRY(filter_real(c, c->pots + 6 * N, 6));
#endif
    if (c->hkf_mode >= 2) {
        double2 *delta = (double2 *)(fld + 2 * N);
        if (WTD_BIG) return big_derivs(delta, 1, delta, NULL, NULL, NULL, c->tw, c->ktab, c->st, 1, c->hkf_mu, c->hkf_T);
        constexpr size_t sm = (size_t)WG::padded * sizeof(double2) + WG::twtotal * sizeof(double2) + sizeof(KTab<WG>);
        if (sm > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
        WTD_ONCE_PER_DEVICE(WTD_CU(cudaFuncSetAttribute(wtd_hkf_c_kernel<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)));
        wtd_hkf_c_kernel<WG><<<1, 512, sm, c->st>>>(delta, delta, c->hkf_mu, c->hkf_T, c->tw, c->ktab);
        WTD_LAUNCHED(c);
    }
    return WTD_OK;
}

static int filter_fields(wtd_ctx *c)
{
    WTD_TRY(filter_alpha(c));
    return filter_h(c);
}

/* per-point H coefficients from the potentials at time index it (variable mass: lap alpha /4
 * and -div A /2 by spectral derivatives) */
static int coef_from_pots(wtd_ctx *c, int it, const double *fld = NULL)
{
    constexpr int N = WTD_NUMEL;
    wslda_potential P = convert_into_wslda_potential(c->pots, N, NULL);
    if (fld) { /* V_a, V_b, delta from the friction-modified fields */
        P.V_a = (double *)fld;
        P.V_b = (double *)fld + N;
        P.delta = (Complex *)(fld + 2 * (size_t)N);
    }
    wtd_prep_coef<<<(N + 127) / 128, 128, 0, c->st>>>(it, P, c->cf);
    WTD_LAUNCHED(c);
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
    if (WTD_BIG) {
        WTD_TRY(big_prep_var(c->cf, c->stage3d, c->tw, c->ktab, c->st));
    } else {
        constexpr size_t sm = (size_t)WG::padded * sizeof(double2) + WG::twtotal * sizeof(double2) + sizeof(KTab<WG>);
        if (sm > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
        WTD_ONCE_PER_DEVICE(WTD_CU(cudaFuncSetAttribute(wtd_prep_var<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)));
        wtd_prep_var<WG><<<2, 256, sm, c->st>>>(c->cf, c->tw, c->ktab);
        WTD_LAUNCHED(c);
    }
#endif
    c->have_coef = 1;
    return WTD_OK;
}

/* the functional at time index it (potentials kernel and the user's modify_potentials) */
static int functional(wtd_ctx *c, int it)
{
    constexpr int N = WTD_NUMEL;
    wslda_density D = convert_into_wslda_density(c->dens, N);
    wslda_potential P = convert_into_wslda_potential(c->pots, N, NULL);
    wtd_potentials_kernel<<<(N + WTD_POT_THREADS - 1) / WTD_POT_THREADS, WTD_POT_THREADS, 0, c->st>>>(it, D, P, 1.0);
    WTD_LAUNCHED(c);
#ifdef ENABLE_MODIFY_POTENTIALS
    modify_potentials<<<(N + 127) / 128, 128, 0, c->st>>>(it, D, P);
    WTD_LAUNCHED(c);
#endif
    return WTD_OK;
}

/* the effective-mass filter, then the H coefficients from the potentials at time index it:
 * filtered in place, or, while quantum friction acts, from the friction-modified fields */
static int coef_with_friction(wtd_ctx *c, int it)
{
    constexpr int N = WTD_NUMEL;
    WTD_TRY(filter_alpha(c));
    if (!(c->qfsw > 0.0)) {
        WTD_TRY(filter_h(c));
        return coef_from_pots(c, it);
    }
    /* quantum friction: H is built from V, delta plus the friction terms, filtered, while the
     * potentials keep their values (the reference adds and removes the terms around H,
     * pca_kernels.cu:497-539) */
    wtd_qf_pccoeff<<<1, 512, 0, c->st>>>(c->dens, N, WTD_VOLEL, c->qf[3], c->dqf);
    WTD_LAUNCHED(c);
    wtd_qf_fields<<<(N + 255) / 256, 256, 0, c->st>>>(c->pots, c->dens + 12 * (size_t)N, c->dqf, c->qf[0] * c->qfsw,
                                                      c->qf[1] * c->qfsw, c->qf[2] * c->qfsw, hc_nF, c->qfld, N);
    WTD_LAUNCHED(c);
    WTD_TRY(filter_h(c, c->qfld));
    WTD_TRY(coef_from_pots(c, it, c->qfld));
#if CODEDIM == 2
    /* the 2D engine leaves the friction terms in (cpca_kernels.cu:846 commented out): the
     * potentials take the modified, filtered fields and the friction-density words the
     * originals (kernel_add_quantum_friction, cpca_kernels.cu:521-525) */
    WTD_CU(cudaMemcpyAsync(c->dens + 12 * (size_t)N, c->pots, 4 * (size_t)N * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
    WTD_CU(cudaMemcpyAsync(c->pots, c->qfld, 4 * (size_t)N * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
#endif
    return WTD_OK;
}

/* densities from the slots, tau, potentials and H coefficients at time index it */
static int after_pass(wtd_ctx *c, bool full, int it)
{
    constexpr int N = WTD_NUMEL;
    const bool qf = c->qfsw > 0.0;
    const int words = (qf ? 16 : 12) * N;
    wtd_dens_reduce<<<(words + 255) / 256, 256, 0, c->st>>>(c->dslot, c->grid, c->dens, N, full ? 1 : 0, 1.0 / WTD_LPERP,
                                                            (size_t)c->sstride, words);
    WTD_LAUNCHED(c);
    WTD_TRY(exchange(c, c->dens, (size_t)words));
    if (full) {
        constexpr size_t sm = (size_t)WG::padded * sizeof(double2) + WG::twtotal * sizeof(double2) + sizeof(KTab<WG>);
        if (sm > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
        WTD_ONCE_PER_DEVICE(WTD_CU(cudaFuncSetAttribute(wtd_tau_kernel<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)));
        wtd_tau_kernel<WG><<<2, 512, sm, c->st>>>(c->dens, c->tw, c->ktab);
        WTD_LAUNCHED(c);
    }
    if (it < 0) return WTD_OK;
    WTD_TRY(functional(c, it));
    return coef_with_friction(c, it);
}

/* the friction switch at time t (pca_utils.c:779-790, 1055-1060): 0 when every coefficient is
 * 0, else the smooth step of the qfstart/qfstop/qfswitch times (1/eF) */
static double qf_switch(const wtd_ctx *c, double t)
{
    if (c->qf[0] == 0.0 && c->qf[1] == 0.0 && c->qf[2] == 0.0) return 0.0;
    const double a = c->qf[4] / hc_eF, b = c->qf[5] / hc_eF, r = c->qf[6] / hc_eF;
    auto ramp = [](double x, double T) { return 0.5 * (1.0 + tanh(tan(M_PI_2 * (2.0 * x / T - 1.0)))); };
    if (t <= a || t >= b) return 0.0;
    if (t >= a + r && t <= b - r) return 1.0;
    if (t > a && t < a + r) return ramp(t - a, r);
    return 1.0 - ramp(t - b + r, r);
}

/* ---------------------------------------------------------------------------------------
 * staged step for lattices whose state does not fit one CTA (32^3, 48^3): the reference's
 * per-step sequence (pca.c:1401-1571) on this library's kernels — plane/pencil spectral
 * derivatives (wtd_fft3d.cuh), CTA-per-state renormalisation and H psi with <H> subtraction,
 * slot-accumulated densities, the ABM update as one elementwise kernel per half step.
 * -------------------------------------------------------------------------------------*/
/* the plane/pencil path computes in FP64.  In the mixed form (WTD_MIXED_H64) the states
 * stay complex64 between calls and the step works on an FP64 copy in c->stage, rounded to
 * complex64 where the fused form stores the states: after each renormalisation */
static double2 *st_y(wtd_ctx *c) { return c->prec == WTD_FP64 ? (double2 *)c->y : c->stage; }
static int st_load(wtd_ctx *c)
{
    if (c->prec == WTD_FP64) return WTD_OK;
    const size_t n2 = (size_t)2 * c->S * WTD_NUMEL;
    wtd_convert_out<float2><<<(unsigned)((n2 + 255) / 256), 256, 0, c->st>>>((const float2 *)c->y, c->stage, n2);
    WTD_LAUNCHED(c);
    return WTD_OK;
}
/* store the FP64 copy as the complex64 states and continue from the stored values */
static int st_round(wtd_ctx *c)
{
    if (c->prec == WTD_FP64) return WTD_OK;
    const size_t n2 = (size_t)2 * c->S * WTD_NUMEL;
    wtd_convert_in<float2><<<(unsigned)((n2 + 255) / 256), 256, 0, c->st>>>(c->stage, (float2 *)c->y, n2);
    WTD_LAUNCHED(c);
    return st_load(c);
}

/* state chunks of the staged density kernel: WTD_DP_T-point tiles times chunks make one full
 * wave of resident CTAs, at most one chunk per slot of the context.  Computed once per context
 * (wtd_create); the densities' summation order follows the chunks, so it is fixed for a given
 * GPU model and build (bitwise reproducible run to run), not across GPU models. */
static int staged_dens_chunks(wtd_ctx *c, int *G)
{
    constexpr int N = WTD_NUMEL;
    const int tiles = (N + WTD_DP_T - 1) / WTD_DP_T;
    int nsm = 0, per_sm = 0;
    WTD_CU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->dev));
    WTD_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dens_points, WTD_DP_T, 0));
    int g = nsm * (per_sm > 0 ? per_sm : 1) / tiles;
    if (g > c->grid) g = c->grid;
    if (g > c->S) g = c->S;
    *G = g < 1 ? 1 : g;
    return WTD_OK;
}

static int staged_densities(wtd_ctx *c, bool grads)
{
    constexpr int N = WTD_NUMEL;
    const int S = c->S;
    const int tiles = (N + WTD_DP_T - 1) / WTD_DP_T;
    const int G = c->sdg > 0 ? c->sdg : 1;
    k_dens_points<<<dim3(tiles, G), WTD_DP_T, 0, c->st>>>(S, G, st_y(c), c->ddx, c->ddy, c->ddz, c->dlap, c->occ,
                                                          c->kp2, c->wcnt, c->dslot, grads ? 1 : 0);
    WTD_LAUNCHED(c);
    wtd_dens_reduce<<<(12 * N + 255) / 256, 256, 0, c->st>>>(c->dslot, G, c->dens, N, grads ? 1 : 0, 1.0 / WTD_LPERP);
    WTD_LAUNCHED(c);
    const bool qf = c->qfsw > 0.0;
    if (qf) {
        /* the friction densities U_a, U_b, D after the 12 N words (pca.c:1426-1429) */
        k_qf_dens_compat<<<(N + 255) / 256, 256, 0, c->st>>>(S, st_y(c), c->dlap, c->occ, NULL, c->kp2,
                                                            c->wcnt, c->dens + 12 * (size_t)N, 1.0 / WTD_LPERP);
        WTD_LAUNCHED(c);
    }
    WTD_TRY(exchange(c, c->dens, (qf ? 16 : 12) * (size_t)N));
    if (grads) WTD_TRY(big_tau(c->dens, c->stage3d, c->tw, c->ktab, c->st));
    return WTD_OK;
}

static int staged_derivs(wtd_ctx *c, bool grads)
{
    const int nf = 2 * c->S;
    c->launches += 2;
    if (grads)
        return big_derivs_sep(st_y(c), nf, c->dlap, c->ddx, c->ddy, CODEDIM >= 3 ? c->ddz : NULL, NULL, NULL, c->tw,
                              c->ktab, c->st);
    return big_derivs_sep(st_y(c), nf, c->dlap, NULL, NULL, NULL, NULL, NULL, c->tw, c->ktab, c->st);
}

static int staged_potentials(wtd_ctx *c, int it)
{
    constexpr int N = WTD_NUMEL;
    wslda_density D = convert_into_wslda_density(c->dens, N);
    wslda_potential P = convert_into_wslda_potential(c->pots, N, NULL);
    int pb = (N + 127) / 128;
    (void)D; (void)pb;
    WTD_TRY(functional(c, it));
    WTD_TRY(coef_with_friction(c, it));
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
    /* lap(alpha psi) for the variable-mass kinetic term (pca.c:1455-1456), the product with
     * alpha taken as the fields are loaded */
    WTD_TRY(big_derivs_sep(st_y(c), 2 * c->S, c->dalap, NULL, NULL, NULL, P.alpha_a, P.alpha_b, c->tw, c->ktab, c->st));
    c->launches += 2;
#endif
    c->have_coef = 1;
    return WTD_OK;
}

static int staged_hamiltonian(wtd_ctx *c, double2 *out)
{
    k_hamiltonian_compat<<<c->S, 256, 0, c->st>>>(c->S, st_y(c), out, c->ddx, c->ddy, c->ddz, c->dlap,
                                                  c->dalap, c->cf, c->kp2, c->qpe, NULL);
    WTD_LAUNCHED(c);
    return WTD_OK;
}

static int staged_initial(wtd_ctx *c)
{
    WTD_TRY(st_load(c));
    k_normalize<<<c->S, 256, 0, c->st>>>(c->S, st_y(c));
    WTD_LAUNCHED(c);
    WTD_TRY(st_round(c));
    WTD_TRY(staged_derivs(c, true));
    return staged_densities(c, true);
}

static int staged_step(wtd_ctx *c, bool last)
{
    constexpr int N = WTD_NUMEL;
    const int NH = WTD_NHIST;
    const size_t M = (size_t)2 * c->S * N;
    const unsigned nb = (unsigned)((M + 255) / 256);
    /* the reference's f1..fq from the ring (f1 newest at ring position NH-1) */
    double2 *f[5] = {NULL, NULL, NULL, NULL, NULL};
    for (int sl = 0; sl < NH; sl++) f[sl] = (double2 *)c->hist[(c->head + (sl == 0 ? NH - 1 : sl - 1)) % NH];
    const bool var = WTD_VAR;
    /* the friction switch of this step (pca.c:1405); while it acts every half step takes the
     * gradient path (pca.c:1412-1414, 1483-1485) */
    c->qfsw = qf_switch(c, hc_t0 + (c->it + 1) * c->dt);
    const bool qf = c->qfsw > 0.0;
    /* predictor (pca.c:1407-1465) */
    WTD_TRY(st_load(c));
    double2 *Y = st_y(c);
    if (NH == 3) k_abm_step1<3><<<nb, 256, 0, c->st>>>(M, Y, f[0], f[1], f[2], NULL, NULL, c->dt);
    else if (NH == 4) k_abm_step1<4><<<nb, 256, 0, c->st>>>(M, Y, f[0], f[1], f[2], f[3], NULL, c->dt);
    else k_abm_step1<5><<<nb, 256, 0, c->st>>>(M, Y, f[0], f[1], f[2], f[3], f[4], c->dt);
    WTD_LAUNCHED(c);
    k_normalize<<<c->S, 256, 0, c->st>>>(c->S, Y);
    WTD_LAUNCHED(c);
    WTD_TRY(st_round(c));
    WTD_TRY(staged_derivs(c, var || qf));
    WTD_TRY(staged_densities(c, var || qf));
    WTD_TRY(staged_potentials(c, c->it + 1));
    WTD_TRY(staged_hamiltonian(c, c->dlap));
    /* corrector (pca.c:1469-1566) */
    const double cc = (NH == 3) ? 9. / 24. : 251. / 720.;
    k_abm_step4<<<nb, 256, 0, c->st>>>(M, c->dlap, Y, f[NH - 1], c->dt, cc);
    WTD_LAUNCHED(c);
    k_normalize<<<c->S, 256, 0, c->st>>>(c->S, Y);
    WTD_LAUNCHED(c);
    WTD_TRY(st_round(c));
    const bool g = var || last || qf;
    WTD_TRY(staged_derivs(c, g));
    WTD_TRY(staged_densities(c, g));
    WTD_TRY(staged_potentials(c, c->it + 1));
    /* pointer rotation (pca.c:1543-1562): the old f_q slot (P, consumed) becomes f1 */
    WTD_TRY(staged_hamiltonian(c, f[NH - 1]));
    c->head = (c->head + NH - 1) % NH;
    c->fk_given = 1;
    c->it++;
    return WTD_OK;
}

/* ---------------------------------------------------------------------------------------
 * line path (3D lattices beyond one CTA, wtd_path3d.cuh): per half step k3_plane_h (when H is
 * formed), k3_xline, and k3_plane_dens on gradient half steps; then the slot reduction, tau,
 * the functional and the coefficients as the fused path does them.
 * -------------------------------------------------------------------------------------*/
#if CODEDIM == 3
/* compile-time choice of the x-line kernel's cluster size CL, threads per x-line TX, pad of its
 * H lines and whether it keeps the state's lines in shared memory (YS): the first candidate
 * that fits one CTA (<= 1024 threads, shared memory) in the order: clusters of 16 CTAs before
 * 8, teams of line_team(NX) threads before 2 and 1, a pad of 4 before 1, the state's lines in
 * shared memory before not */
template <typename TC, int CL, int TX, int HPAD, bool YS> struct LineFit {
    static constexpr bool ok = TX >= 1 && XSmem<TC, CL, TX, HPAD, YS>::ok &&
                               XSmem<TC, CL, TX, HPAD, YS>::bytes + 64 <= WTD_SMEM_MAX;
};
template <typename TC> struct LineCfg {
    static constexpr int T0 = line_team(NX), T1 = T0 > 2 ? 2 : 1;
    /* candidate i: YS = !(i & 1); j = i / 2 gives HPAD (4, 1), CL (16, 16, 8, 8) and TX (T0 for
     * j < 4, T1 for j < 8, else 1) */
    static constexpr int cl(int i) { return ((i / 2) % 4 < 2) ? 16 : 8; }
    static constexpr int tx(int i) { return (i / 2) < 4 ? T0 : (i / 2) < 8 ? T1 : 1; }
    static constexpr int hp(int i) { return ((i / 2) % 2 == 0) ? 4 : 1; }
    static constexpr bool ys(int i) { return (i & 1) == 0; }
    template <int I, bool = (I < 24)> struct Find {
        static constexpr int value = LineFit<TC, cl(I), tx(I), hp(I), ys(I)>::ok ? I : Find<I + 1>::value;
    };
    template <int I> struct Find<I, false> { static constexpr int value = 24; };
    static constexpr int k = Find<0>::value;
    static constexpr int CL = cl(k < 24 ? k : 0), TX = tx(k < 24 ? k : 0), HPAD = hp(k < 24 ? k : 0);
    static constexpr bool YS = ys(k < 24 ? k : 0);
    static constexpr bool ok = k < 24 && PlaneGeo::ok && PlaneSmem<TC>::h_bytes <= WTD_SMEM_MAX &&
                               PlaneSmem<TC>::d_bytes <= WTD_SMEM_MAX;
};

static bool line_fits(int prec)
{
    if (!WTD_BIG) return false;
    return prec == WTD_FP64 ? LineCfg<double>::ok : LineCfg<float>::ok;
}

/* the x-line kernel's attributes (shared memory beyond 48 KB; clusters of 16 CTAs) */
template <typename TY, typename TH, typename TC, int PASS, bool GRAD>
static cudaError_t line_x_attrs()
{
    typedef LineCfg<TC> L;
    typedef XSmem<TC, L::CL, L::TX, L::HPAD, L::YS> SM;
    auto k = k3_xline<TY, TH, TC, WTD_NHIST, PASS, WTD_VAR, GRAD, L::CL, L::TX, L::HPAD, L::YS>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM::bytes);
    if (e == cudaSuccess && L::CL > 8) e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    return e;
}

/* launch configuration of ncl clusters on the context stream */
template <typename TC>
static void line_x_config(wtd_ctx *c, cudaLaunchConfig_t &cfg, cudaLaunchAttribute *at, int ncl)
{
    typedef LineCfg<TC> L;
    typedef XSmem<TC, L::CL, L::TX, L::HPAD, L::YS> SM;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3((unsigned)(ncl * L::CL));
    cfg.blockDim = dim3(SM::XT);
    cfg.dynamicSmemBytes = SM::bytes;
    cfg.stream = c->st;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = L::CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
}

template <typename TY, typename TH, typename TC, int PASS, bool GRAD>
static int line_launch_x(wtd_ctx *c, const StepArgs &a)
{
    typedef LineCfg<TC> L;
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute at[1];
    WTD_ONCE_PER_DEVICE(WTD_CU((line_x_attrs<TY, TH, TC, PASS, GRAD>())));
    line_x_config<TC>(c, cfg, at, c->ncl);
    X3Args xa;
    xa.s = a;
    xa.K = c->kbuf;
    WTD_CU(cudaLaunchKernelEx(&cfg, k3_xline<TY, TH, TC, WTD_NHIST, PASS, WTD_VAR, GRAD, L::CL, L::TX, L::HPAD, L::YS>, xa,
                              (const double2 *)c->tw, (const double *)c->ktab));
    WTD_LAUNCHED(c);
    return WTD_OK;
}

template <typename TY, typename TC>
static int line_launch_h(wtd_ctx *c, const void *y)
{
    typedef PlaneSmem<TC> SM;
    auto k = k3_plane_h<TY, TC, WTD_VAR>;
    WTD_ONCE_PER_DEVICE(WTD_CU(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM::h_bytes)));
    k<<<c->p1grid, PlaneGeo::PT * SM::HS, SM::h_bytes, c->st>>>((const TY *)y, (typename cplx<TC>::t *)c->kbuf, c->cf, c->S, c->tw,
                                                        c->ktab);
    WTD_LAUNCHED(c);
    return WTD_OK;
}

template <typename TY, typename TC>
static int line_launch_dens(wtd_ctx *c, const void *y)
{
    typedef PlaneSmem<TC> SM;
    constexpr size_t N = WTD_NUMEL;
    auto k = k3_plane_dens<TY, TC>;
    WTD_ONCE_PER_DEVICE(WTD_CU(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM::d_bytes)));
    k<<<2 * NX * c->g2, PlaneGeo::PT, SM::d_bytes, c->st>>>((const TY *)y, c->occ, c->wcnt, c->S, c->g2,
                                                             c->dslot + (size_t)c->ncl * 12 * N, 12 * N, c->tw, c->ktab);
    WTD_LAUNCHED(c);
    return WTD_OK;
}

template <typename TY, typename TH, typename TC, int PASS, bool GRAD>
static int line_pass_t(wtd_ctx *c, const StepArgs &a)
{
    const bool haveH = PASS == 1 || PASS == 3 || (PASS == 0 && !a.fk_given);
    if (haveH) WTD_TRY((line_launch_h<TY, TC>(c, a.y)));
    WTD_TRY((line_launch_x<TY, TH, TC, PASS, GRAD>(c, a)));
    if (GRAD && PASS != 3) WTD_TRY((line_launch_dens<TY, TC>(c, a.yout ? a.yout : a.y)));
    return WTD_OK;
}

template <int PASS, bool GRAD>
static int line_pass_p(wtd_ctx *c, const StepArgs &a)
{
    if (c->prec == WTD_FP64) return line_pass_t<double2, double2, double, PASS, GRAD>(c, a);
    if (c->prec == WTD_MIXED_H64) return line_pass_t<float2, double2, float, PASS, GRAD>(c, a);
    return line_pass_t<float2, float2, float, PASS, GRAD>(c, a);
}

/* one half step's kernels (pass 0: H y_k + predictor, 1: H y_pred + corrector, 2: initial
 * measurement, 3: f_k only), timed like the fused passes when timing is on */
static int line_pass(wtd_ctx *c, int pass, bool grad, const StepArgs *given)
{
    StepArgs a = given ? *given : make_args(c);
    a.sstride = 12 * WTD_NUMEL;
    const bool timed = c->timing && pass < 2 && c->nev[pass] < 4096;
    if (timed) cudaEventRecord(c->ev[pass][0][c->nev[pass]], c->st);
    int r;
    if (pass == 0) r = grad ? line_pass_p<0, true>(c, a) : line_pass_p<0, false>(c, a);
    else if (pass == 1) r = grad ? line_pass_p<1, true>(c, a) : line_pass_p<1, false>(c, a);
    else if (pass == 2) r = line_pass_p<2, true>(c, a);
    else r = line_pass_p<3, false>(c, a);
    if (timed) {
        cudaEventRecord(c->ev[pass][1][c->nev[pass]], c->st);
        c->nev[pass]++;
    }
    return r;
}

/* slots -> densities (x-line slots, plus the plane slots on gradient passes), exchange, tau,
 * potentials and coefficients at time index it (it < 0: none) */
static int line_after(wtd_ctx *c, bool full, int it)
{
    constexpr int N = WTD_NUMEL;
    const int nslots = c->ncl + (full ? c->g2 : 0);
    wtd_dens_reduce<<<(12 * N + 255) / 256, 256, 0, c->st>>>(c->dslot, nslots, c->dens, N, full ? 1 : 0, 1.0 / WTD_LPERP,
                                                             12 * (size_t)N, 12 * N);
    WTD_LAUNCHED(c);
    WTD_TRY(exchange(c, c->dens, 12 * (size_t)N));
    if (full) WTD_TRY(big_tau(c->dens, c->stage3d, c->tw, c->ktab, c->st));
    if (it < 0) return WTD_OK;
    WTD_TRY(functional(c, it));
    return coef_with_friction(c, it);
}

static int line_step(wtd_ctx *c, bool last)
{
    const bool var = WTD_VAR;
    if (!c->fk_given && !c->have_coef) return WTD_ERR_STATE;
    c->qfsw = 0.0;
    WTD_TRY(line_pass(c, 0, var));
    WTD_TRY(line_after(c, var, c->it + 1));
    const bool g = var || last;
    WTD_TRY(line_pass(c, 1, g));
    WTD_TRY(line_after(c, g, c->it + 1));
    c->head = (c->head + WTD_NHIST - 1) % WTD_NHIST;
    c->fk_given = 0;
    c->it++;
    return WTD_OK;
}

static int line_initial(wtd_ctx *c)
{
    WTD_TRY(line_pass(c, 2, true));
    return line_after(c, true, -1);
}

/* grid sizes of the line kernels on this device */
template <typename TY, typename TH, typename TC>
static int line_setup_t(wtd_ctx *c, int nsm)
{
    typedef LineCfg<TC> L;
    int per = 0;
    {
        typedef PlaneSmem<TC> SM;
        auto k = k3_plane_h<TY, TC, WTD_VAR>;
        WTD_CU(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM::h_bytes));
        WTD_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, PlaneGeo::PT * SM::HS, SM::h_bytes));
        /* a whole number of CTAs per (component, x-plane) pair */
        const int pairs = 2 * NX, nch = nsm * (per > 0 ? per : 1) / pairs;
        c->p1grid = pairs * (nch > 0 ? nch : 1);
        auto kd = k3_plane_dens<TY, TC>;
        WTD_CU(cudaFuncSetAttribute(kd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM::d_bytes));
        WTD_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kd, PlaneGeo::PT, SM::d_bytes));
        int g = nsm * (per > 0 ? per : 1) / (2 * NX);
        c->g2 = g < 1 ? 1 : (g > c->S ? c->S : g);
    }
    {
        cudaLaunchConfig_t cfg;
        cudaLaunchAttribute at[1];
        WTD_CU((line_x_attrs<TY, TH, TC, 0, false>()));
        line_x_config<TC>(c, cfg, at, 1);
        int ncl = 0;
        if (cudaOccupancyMaxActiveClusters(&ncl, k3_xline<TY, TH, TC, WTD_NHIST, 0, WTD_VAR, false, L::CL, L::TX, L::HPAD, L::YS>,
                                           &cfg) != cudaSuccess || ncl < 1) {
            cudaGetLastError();
            ncl = nsm / L::CL;
        }
        if (ncl < 1) ncl = 1;
        if (ncl > c->S) ncl = c->S;
        c->ncl = ncl;
    }
    return WTD_OK;
}

static int line_setup(wtd_ctx *c, int nsm)
{
    if (c->prec == WTD_FP64) return line_setup_t<double2, double2, double>(c, nsm);
    if (c->prec == WTD_MIXED_H64) return line_setup_t<float2, double2, float>(c, nsm);
    return line_setup_t<float2, float2, float>(c, nsm);
}
#else
static bool line_fits(int) { return false; }
static int line_pass(wtd_ctx *, int, bool, const StepArgs *) { return WTD_ERR_UNSUPPORTED; }
static int line_step(wtd_ctx *, bool) { return WTD_ERR_UNSUPPORTED; }
static int line_initial(wtd_ctx *) { return WTD_ERR_UNSUPPORTED; }
static int line_setup(wtd_ctx *, int) { return WTD_ERR_UNSUPPORTED; }
#endif

/* what the adjoint's reverse sweep needs of one fused step */
struct StepRecord {
    double2 *yk, *yp;           /* state before the step, normalised predictor state */
    double *cfA, *cfB;          /* H coefficients of pass A and pass B */
    double *EA, *EB, *nA, *nB;  /* <H> and update norms of both half steps */
    int hasH;                   /* pass A formed f_k with H (0 on the first step) */
};

/* one fused step: pass A, functional, pass B, functional.
 * rec != NULL records the step without copying states: pass A reads y_k from rec->yk and
 * writes y_pred into rec->yp, pass B writes y_{k+1} into yk_next (the next record's yk) or,
 * when yk_next is NULL, into the context's states. */
static int fused_step(wtd_ctx *c, bool last, StepRecord *rec, double2 *yk_next = NULL)
{
    const bool var = WTD_VAR;
    constexpr int N = WTD_NUMEL;
    if (!c->fk_given && !c->have_coef) return WTD_ERR_STATE;
    /* quantum friction of this step (pca.c:1405, 1467): gradients and friction densities */
    c->qfsw = qf_switch(c, hc_t0 + (c->it + 1) * c->dt);
    const bool qf = c->qfsw > 0.0;
    if (rec) {
        WTD_CU(cudaMemcpyAsync(rec->cfA, c->cf, CF_COUNT * (size_t)N * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
        rec->hasH = c->fk_given ? 0 : 1;
    }
    /* predictor: f_k, y_pred, P; densities of y_pred */
    if (!rec) {
        WTD_TRY(run_pass(c, 0, var || qf));
    } else {
        StepArgs a = make_args(c);
        a.y = rec->yk;
        a.yout = rec->yp;
        a.nrm_out = rec->nA;
        a.qpe = rec->EA;
        WTD_TRY((var ? launch_pass<0, true>(c, a) : launch_pass<0, false>(c, a)));
    }
    WTD_TRY(after_pass(c, var || qf, c->it + 1));
    if (rec) WTD_CU(cudaMemcpyAsync(rec->cfB, c->cf, CF_COUNT * (size_t)N * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
    /* corrector */
    const bool g = var || last || qf;
    if (!rec) {
        WTD_TRY(run_pass(c, 1, g));
    } else {
        StepArgs a = make_args(c);
        a.y = rec->yp;
        a.yout = yk_next ? (void *)yk_next : c->y;
        a.nrm_out = rec->nB;
        a.qpe = rec->EB;
        WTD_TRY((g ? launch_pass<1, true>(c, a) : launch_pass<1, false>(c, a)));
    }
    WTD_TRY(after_pass(c, g, c->it + 1));
    /* ring: f_k becomes the newest history entry, P's slot becomes free */
    c->head = (c->head + WTD_NHIST - 1) % WTD_NHIST;
    c->fk_given = 0;
    c->it++;
    return WTD_OK;
}

template <typename TY, typename TH, typename TC>
static int occupancy_t(int block)
{
    /* resident CTAs of the step's ordinary passes (PASS 0 without gradients); the gradient
     * passes (one more buffer) may then run the same grid in more than one wave */
    constexpr int NBUF = WTD_VAR ? 4 : 2;
    constexpr size_t sm = fused_smem<TC, NBUF>();
    if (sm > WTD_SMEM_MAX) return 1;
    int nb = 1;
    if (block == 1024 && WG::ntot >= 2048) {
        auto k = wtd_fused_pass<WG, TY, TH, TC, WTD_NHIST, 0, WTD_VAR, false, 1024>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, 1024, sm);
    } else {
        auto k = wtd_fused_pass<WG, TY, TH, TC, WTD_NHIST, 0, WTD_VAR, false, 512>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        int threads = WG::ntot >= 512 ? 512 : ((WG::ntot + 31) / 32) * 32;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, threads, sm);
    }
    cudaGetLastError();
    return nb < 1 ? 1 : (nb > 16 ? 16 : nb);
}

static int occupancy_per_sm(wtd_ctx *c)
{
    if (c->prec == WTD_FP64) return occupancy_t<double2, double2, double>(c->block);
    if (c->prec == WTD_MIXED_H64) return occupancy_t<float2, double2, float>(c->block);
    return occupancy_t<float2, float2, float>(c->block);
}

/* ---------------------------------------------------------------------------------------
 * C ABI
 * -------------------------------------------------------------------------------------*/
extern "C" {

int wtd_info(int *dims, int *numel, int *codedim, int *nhist, int *functional, int *const_mass)
{
    if (dims) { dims[0] = WG::N0; dims[1] = WG::N1; dims[2] = WG::N2; }
    if (numel) *numel = WTD_NUMEL;
    if (codedim) *codedim = CODEDIM;
    if (nhist) *nhist = WTD_NHIST;
    if (functional) *functional = FUNCTIONAL;
    if (const_mass) *const_mass = WTD_VAR ? 0 : 1;
    return WTD_OK;
}

size_t wtd_device_bytes(int nwf, int precision)
{
    size_t n2 = (size_t)2 * nwf * WTD_NUMEL;
    size_t b = n2 * (elem_bytes_y(precision) + WTD_NHIST * elem_bytes_h(precision)) +
               (size_t)300 * 16 * WTD_NUMEL * sizeof(double);
    if (WTD_BIG) b += n2 * sizeof(double2) * ((CODEDIM >= 3 ? 4 : 3) + (WTD_VAR ? 1 : 0));
    return b;
}

const char *wtd_error_string(int code)
{
    switch (code) {
    case WTD_OK: return "ok";
    case WTD_ERR_ARG: return "invalid argument";
    case WTD_ERR_CUDA: return "CUDA error";
    case WTD_ERR_UNSUPPORTED: return "lattice/mode not supported by this build";
    case WTD_ERR_STATE: return "call out of order";
    case WTD_ERR_NOMEM: return "out of device memory";
    case WTD_ERR_COMM: return "density exchange failed (NCCL not loadable, or a collective or hook error)";
    case -6: return "lattice too large for the fixed scratch of calculate_densities_noalloc (12*N doubles > 1 Mi words)";
    case WTD_ERR_IO: return "checkpoint file missing, short or not writable";
    default: return "unknown error";
    }
}

int wtd_create(wtd_ctx **out, int nwf, int precision, int device)
{
    if (!out || nwf <= 0 || precision < 0 || precision > 2) return WTD_ERR_ARG;
    *out = NULL;
    WTD_CU(cudaSetDevice(device));
    wtd_ctx *c = (wtd_ctx *)calloc(1, sizeof(wtd_ctx));
    if (!c) return WTD_ERR_NOMEM;
    c->dev = device; c->S = nwf; c->prec = precision;
    const size_t N = WTD_NUMEL, n2 = (size_t)2 * nwf * N;
    c->ysz = n2 * elem_bytes_y(precision);
    c->hsz = n2 * elem_bytes_h(precision);
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    c->block = 512;
    {
        const char *b = getenv("WTD_BLOCK");
        if (b && atoi(b) == 1024) c->block = 1024;
    }
    /* persistent grid: as many CTAs as fit on every SM for the step's ordinary passes (two per
     * SM for the FP32 compute forms), one slot layout for all pass variants of a run */
    /* L2 prefetch of the next state's y only: prefetching the history as well overflows L2
     * with one FP64 or two FP32 CTAs per SM in flight and is re-read from HBM */
    c->prefetch = 1;
    {
        const char *pf = getenv("WTD_PREFETCH");
        if (pf) c->prefetch = atoi(pf) & 15;
    }
    /* lattices beyond one CTA.  The FP32-mixed forms take the 3D line path (FP32 arithmetic,
     * complex64 history possible); FP64 takes the staged path, which measures faster in FP64
     * on 32^3.  WTD_3D_PATH=line or =staged selects either for every form. */
    {
        const char *pp = getenv("WTD_3D_PATH");
        bool want_line = precision != WTD_FP64;
        if (pp && strcmp(pp, "line") == 0) want_line = true;
        if (pp && strcmp(pp, "staged") == 0) want_line = false;
        c->line = (WTD_BIG && line_fits(precision) && want_line) ? 1 : 0;
    }
    c->staged = (WTD_BIG && !c->line) ? 1 : 0;
    if (c->staged && precision == WTD_MIXED_H32) { free(c); return WTD_ERR_UNSUPPORTED; }
    if (c->line && line_setup(c, nsm) != WTD_OK) { free(c); return WTD_ERR_CUDA; }
    int per_sm = WTD_BIG ? 2 : occupancy_per_sm(c);
    c->grid = nsm * per_sm;
    if (c->grid > nwf) c->grid = nwf;
    if (c->staged && staged_dens_chunks(c, &c->sdg) != WTD_OK) { cudaGetLastError(); free(c); return WTD_ERR_CUDA; }
    cudaError_t e = cudaSuccess;
#define ALLOC(p, bytes) if (e == cudaSuccess) e = cudaMalloc((void **)&(p), (bytes))
    ALLOC(c->y, c->ysz);
    for (int h = 0; h < WTD_NHIST; h++) ALLOC(c->hist[h], c->hsz);
    ALLOC(c->cf, (size_t)CF_COUNT * N * sizeof(double));
    ALLOC(c->occ, nwf * sizeof(double));
    ALLOC(c->kp2, nwf * sizeof(double));
    ALLOC(c->wcnt, nwf * sizeof(double));
    {
        /* density slots: per CTA of the fused passes (12 N words, 16 N with quantum friction);
         * on the line path per cluster and per plane chunk (12 N words) */
        size_t slots = (size_t)c->grid * 16 * N;
        if (c->line && (size_t)(c->ncl + c->g2) * 12 * N > slots) slots = (size_t)(c->ncl + c->g2) * 12 * N;
        ALLOC(c->dslot, slots * sizeof(double));
    }
    ALLOC(c->qpe, nwf * sizeof(double));
    ALLOC(c->dens, 16 * N * sizeof(double));
    ALLOC(c->qfld, 4 * N * sizeof(double));
    ALLOC(c->dqf, 4 * sizeof(double));
    ALLOC(c->pots, 12 * N * sizeof(double));
    ALLOC(c->ework, (size_t)TDWSLDAITEMS * N * sizeof(double));
    ALLOC(c->eout, 16 * sizeof(double));
    ALLOC(c->tw, WG::twtotal * sizeof(double2));
    ALLOC(c->ktab, 6 * WTD_KT * sizeof(double));
    if (precision != WTD_FP64) {
        ALLOC(c->xfer, WTD_XFER * sizeof(double2));
        if (c->staged) ALLOC(c->stage, n2 * sizeof(double2));
    }
    if (c->line) {
        ALLOC(c->kbuf, n2 * (precision == WTD_FP64 ? sizeof(double2) : sizeof(float2)));
        ALLOC(c->stage3d, 2 * N * sizeof(double2));
    }
    if (c->staged) {
        ALLOC(c->ddx, n2 * sizeof(double2));
        ALLOC(c->ddy, n2 * sizeof(double2));
        if (CODEDIM >= 3) ALLOC(c->ddz, n2 * sizeof(double2));
        ALLOC(c->dlap, n2 * sizeof(double2));
        if (WTD_VAR) ALLOC(c->dalap, n2 * sizeof(double2));
        ALLOC(c->stage3d, 2 * N * sizeof(double2));
    }
#undef ALLOC
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) { wtd_destroy(c); return e == cudaErrorMemoryAllocation ? WTD_ERR_NOMEM : WTD_ERR_CUDA; }
    cudaMemsetAsync(c->cf, 0, (size_t)CF_COUNT * N * sizeof(double), c->st);
    cudaMemsetAsync(c->qpe, 0, nwf * sizeof(double), c->st);
    cudaMemsetAsync(c->dens, 0, 16 * N * sizeof(double), c->st);
    cudaMemsetAsync(c->dqf, 0, 4 * sizeof(double), c->st);
    c->sstride = 12 * (int)N;
    {
        double2 tw[WG::twtotal];
        double kt[6 * WTD_KT];
        wtd_make_tables(tw, kt);
        cudaMemcpyAsync(c->tw, tw, sizeof(tw), cudaMemcpyHostToDevice, c->st);
        cudaMemcpyAsync(c->ktab, kt, sizeof(kt), cudaMemcpyHostToDevice, c->st);
        cudaStreamSynchronize(c->st);
    }
    /* defaults: f_n = 0, no plane-wave momentum, unit degeneracy */
    {
        double *h = (double *)calloc(nwf, sizeof(double));
        cudaMemcpy(c->occ, h, nwf * sizeof(double), cudaMemcpyHostToDevice);
        cudaMemcpy(c->kp2, h, nwf * sizeof(double), cudaMemcpyHostToDevice);
        for (int i = 0; i < nwf; i++) h[i] = 1.0;
        cudaMemcpy(c->wcnt, h, nwf * sizeof(double), cudaMemcpyHostToDevice);
        free(h);
    }
    for (int h = 0; h < WTD_NHIST; h++) cudaMemsetAsync(c->hist[h], 0, c->hsz, c->st);
    c->fk_given = 1;
    e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) { wtd_destroy(c); return WTD_ERR_CUDA; }
    *out = c;
    return WTD_OK;
}

int wtd_destroy(wtd_ctx *c)
{
    if (!c) return WTD_OK;
    cudaSetDevice(c->dev);
    if (c->st) cudaStreamSynchronize(c->st);
    adj_release(c);
    if (c->wdata && c->wdata_free) c->wdata_free(c->wdata);
    if (c->nccl && nccl_api()) nccl_api()->comm_destroy((ncclComm_t)c->nccl);
    if (c->timing)
        for (int p = 0; p < 2; p++)
            for (int k = 0; k < 2; k++)
                for (int i = 0; i < 4096; i++) cudaEventDestroy(c->ev[p][k][i]);
    void *ptrs[] = {c->y, c->cf, c->occ, c->kp2, c->wcnt, c->dslot, c->qpe, c->dens, c->pots, c->qfld, c->dqf, c->ework,
                    c->eout, c->tw, c->ktab, c->stage, c->extra, c->ddx, c->ddy, c->ddz, c->dlap, c->dalap, c->stage3d,
                    c->kbuf, c->xfer};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) if (ptrs[i]) cudaFree(ptrs[i]);
    for (int h = 0; h < WTD_NHIST; h++) if (c->hist[h]) cudaFree(c->hist[h]);
    if (c->st) cudaStreamDestroy(c->st);
    free(c);
    return WTD_OK;
}

int wtd_set_constants(wtd_ctx *c, double mu_a, double mu_b, double ec, double t0, double dt, double kF)
{
    if (!c) return WTD_ERR_ARG;
    c->mut++;
    WTD_CU(cudaSetDevice(c->dev));
    double eF = kF * kF / 2., nF = kF * kF * kF / (3. * M_PI * M_PI);
    WTD_CU(cudaMemcpyToSymbol(dc_mu_a, &mu_a, sizeof(double)));
    WTD_CU(cudaMemcpyToSymbol(dc_mu_b, &mu_b, sizeof(double)));
    WTD_CU(cudaMemcpyToSymbol(dc_ec, &ec, sizeof(double)));
    WTD_CU(cudaMemcpyToSymbol(dc_t0, &t0, sizeof(double)));
    WTD_CU(cudaMemcpyToSymbol(dc_dt, &dt, sizeof(double)));
    WTD_CU(cudaMemcpyToSymbol(dc_kF, &kF, sizeof(double)));
    WTD_CU(cudaMemcpyToSymbol(dc_eF, &eF, sizeof(double)));
    WTD_CU(cudaMemcpyToSymbol(dc_nF, &nF, sizeof(double)));
    hc_mu_a = mu_a; hc_mu_b = mu_b; hc_ec = ec; hc_t0 = t0; hc_dt = dt; hc_kF = kF; hc_eF = eF; hc_nF = nF;
    md.dt = dt; md.ec = ec;
    c->dt = dt;
    return WTD_OK;
}

int wtd_set_params(wtd_ctx *c, const double *params)
{
    if (!c || !params) return WTD_ERR_ARG;
    c->mut++;
    WTD_CU(cudaSetDevice(c->dev));
    WTD_CU(cudaMemcpyToSymbol(dc_params, params, MAX_USER_PARAMS * sizeof(double)));
    memcpy(md.params, params, MAX_USER_PARAMS * sizeof(double));
    return WTD_OK;
}

int wtd_set_sclgth(wtd_ctx *c, double a)
{
    if (!c) return WTD_ERR_ARG;
    c->mut++;
    WTD_CU(cudaSetDevice(c->dev));
    WTD_CU(cudaMemcpyToSymbol(dc_sclgth, &a, sizeof(double)));
    hc_sclgth = a;
    md.sclgth = a;
    return WTD_OK;
}

int wtd_set_extra_data(wtd_ctx *c, const void *host, size_t bytes)
{
    if (!c || (bytes && !host)) return WTD_ERR_ARG;
    c->mut++;
    WTD_CU(cudaSetDevice(c->dev));
    if (c->extra) { cudaFree(c->extra); c->extra = NULL; }
    if (bytes) {
        WTD_CU(cudaMalloc(&c->extra, bytes));
        WTD_CU(cudaMemcpy(c->extra, host, bytes, cudaMemcpyHostToDevice));
    }
    c->extra_bytes = bytes;
    WTD_CU(cudaMemcpyToSymbol(dc_extra_data, &c->extra, sizeof(void *)));
    WTD_CU(cudaMemcpyToSymbol(dc_extra_data_size, &bytes, sizeof(size_t)));
    return WTD_OK;
}

int wtd_process_params(wtd_ctx *c, double *params, double *kF, double *mu)
{
    if (!params || !kF || !mu) return WTD_ERR_ARG;
    process_params(params, kF, mu, c ? c->extra_bytes : 0, NULL);
    return WTD_OK;
}

/* complex64 arrays go through the bounded staging buffer in chunks of WTD_XFER complex
 * numbers (host FP64 <-> device complex64), in stream order */
static int upload_array(wtd_ctx *c, void *dst, int prec_elem64, const double *host)
{
    const size_t n2 = (size_t)2 * c->S * WTD_NUMEL;
    if (prec_elem64) {
        WTD_CU(cudaMemcpyAsync(dst, host, n2 * sizeof(double2), cudaMemcpyHostToDevice, c->st));
    } else {
        for (size_t o = 0; o < n2; o += WTD_XFER) {
            const size_t m = n2 - o < WTD_XFER ? n2 - o : WTD_XFER;
            WTD_CU(cudaMemcpyAsync(c->xfer, host + 2 * o, m * sizeof(double2), cudaMemcpyHostToDevice, c->st));
            wtd_convert_in<float2><<<(unsigned)((m + 255) / 256), 256, 0, c->st>>>((const double2 *)c->xfer, (float2 *)dst + o, m);
            WTD_LAUNCHED(c);
        }
    }
    return WTD_OK;
}
static int download_array(wtd_ctx *c, const void *src, int prec_elem64, double *host)
{
    const size_t n2 = (size_t)2 * c->S * WTD_NUMEL;
    if (prec_elem64) {
        WTD_CU(cudaMemcpyAsync(host, src, n2 * sizeof(double2), cudaMemcpyDeviceToHost, c->st));
    } else {
        for (size_t o = 0; o < n2; o += WTD_XFER) {
            const size_t m = n2 - o < WTD_XFER ? n2 - o : WTD_XFER;
            wtd_convert_out<float2><<<(unsigned)((m + 255) / 256), 256, 0, c->st>>>((const float2 *)src + o, (double2 *)c->xfer, m);
            WTD_LAUNCHED(c);
            WTD_CU(cudaMemcpyAsync(host + 2 * o, c->xfer, m * sizeof(double2), cudaMemcpyDeviceToHost, c->st));
        }
    }
    WTD_CU(cudaStreamSynchronize(c->st));
    return WTD_OK;
}

int wtd_upload_states(wtd_ctx *c, const double *host)
{
    if (!c || !host) return WTD_ERR_ARG;
    c->mut++;
    WTD_CU(cudaSetDevice(c->dev));
    return upload_array(c, c->y, c->prec == WTD_FP64, host);
}

int wtd_download_states(wtd_ctx *c, double *host)
{
    if (!c || !host) return WTD_ERR_ARG;
    WTD_CU(cudaSetDevice(c->dev));
    return download_array(c, c->y, c->prec == WTD_FP64, host);
}

/* reference slot s (f_{s+1}, f1 newest) lives at ring position NH-1 for s = 0 (the "given"
 * f_k) and at ring position s-1 for s >= 1 */
static int ring_of_ref_slot(int s) { return s == 0 ? WTD_NHIST - 1 : s - 1; }

int wtd_upload_history(wtd_ctx *c, int slot, const double *host)
{
    if (!c || !host || slot < 0 || slot >= WTD_NHIST) return WTD_ERR_ARG;
    c->mut++;
    WTD_CU(cudaSetDevice(c->dev));
    void *s[5];
    ring_slots(c, s);
    WTD_TRY(upload_array(c, s[ring_of_ref_slot(slot)], c->prec != WTD_MIXED_H32, host));
    c->fk_given = 1;
    return WTD_OK;
}

int wtd_download_history(wtd_ctx *c, int slot, double *host)
{
    if (!c || !host || slot < 0 || slot >= WTD_NHIST) return WTD_ERR_ARG;
    WTD_CU(cudaSetDevice(c->dev));
    if (slot == 0) WTD_TRY(ensure_fk(c));
    void *s[5];
    ring_slots(c, s);
    return download_array(c, s[ring_of_ref_slot(slot)], c->prec != WTD_MIXED_H32, host);
}

int wtd_upload_potentials(wtd_ctx *c, const double *host)
{
    if (!c || !host) return WTD_ERR_ARG;
    c->mut++;
    WTD_CU(cudaSetDevice(c->dev));
    WTD_CU(cudaMemcpyAsync(c->pots, host, 12 * (size_t)WTD_NUMEL * sizeof(double), cudaMemcpyHostToDevice, c->st));
    return WTD_OK;
}

int wtd_upload_occupations(wtd_ctx *c, const double *fbeta, const double *kky, const double *kkz, const int *cnt)
{
    if (!c || !fbeta) return WTD_ERR_ARG;
    c->mut++;
    WTD_CU(cudaSetDevice(c->dev));
    const int S = c->S;
    double *kp2 = (double *)malloc(S * sizeof(double)), *w = (double *)malloc(S * sizeof(double));
    for (int n = 0; n < S; n++) {
        double ky = kky ? kky[n] : 0.0, kz = kkz ? kkz[n] : 0.0;
#if CODEDIM == 2
        kp2[n] = kz * kz;
        w[n] = (fabs(kz) < 1.0e-12) ? 1.0 : 2.0;  /* +kz and -kz (cpca_dens.cu:52-58) */
#ifdef USE_CUBIC_CUTOFF
        if (fabs(kz + M_PI / DZ) < 1.0e-12) w[n] = 1.0;
#endif
#elif CODEDIM == 1
        kp2[n] = ky * ky + kz * kz;
        w[n] = cnt ? (double)cnt[n] : 1.0;       /* ccpca_dens.cu:47 */
#else
        (void)ky; (void)kz;
        kp2[n] = 0.0;
        w[n] = 1.0;
#endif
    }
    cudaError_t e = cudaMemcpy(c->occ, fbeta, S * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->kp2, kp2, S * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->wcnt, w, S * sizeof(double), cudaMemcpyHostToDevice);
    free(kp2); free(w);
    return wtd_cuerr(e);
}

int wtd_initial_measurement(wtd_ctx *c, int it0)
{
    if (!c) return WTD_ERR_ARG;
    WTD_CU(cudaSetDevice(c->dev));
    c->it = it0;
    c->head = 0;
    c->qfsw = 0.0;
    for (int h = 0; h < WTD_NHIST; h++) WTD_CU(cudaMemsetAsync(c->hist[h], 0, c->hsz, c->st));
    c->fk_given = 1;
    if (c->staged) {
        WTD_TRY(staged_initial(c));
        return wtd_cuerr(cudaGetLastError());
    }
    if (c->line) {
        WTD_TRY(line_initial(c));
        return wtd_cuerr(cudaGetLastError());
    }
    WTD_TRY(run_pass(c, 2, true));
    WTD_TRY(after_pass(c, true, -1));
    return wtd_cuerr(cudaGetLastError());
}

int wtd_steps(wtd_ctx *c, int nsteps)
{
    if (!c || nsteps < 0) return WTD_ERR_ARG;
    WTD_CU(cudaSetDevice(c->dev));
    const bool var = WTD_VAR;
    if (c->staged) {
        for (int s = 0; s < nsteps; s++) WTD_TRY(staged_step(c, s == nsteps - 1));
        return WTD_OK;
    }
    if (c->line) {
        for (int s = 0; s < nsteps; s++) WTD_TRY(line_step(c, s == nsteps - 1));
        return WTD_OK;
    }
    (void)var;
    for (int s = 0; s < nsteps; s++) WTD_TRY(fused_step(c, s == nsteps - 1, NULL));
    return WTD_OK;
}

int wtd_energy(wtd_ctx *c, double *host11)
{
    if (!c || !host11) return WTD_ERR_ARG;
    WTD_CU(cudaSetDevice(c->dev));
    constexpr int N = WTD_NUMEL;
    wslda_density D = convert_into_wslda_density(c->dens, N);
    wslda_potential P = convert_into_wslda_potential(c->pots, N, NULL);
    int pb = (N + 127) / 128;
    double *e = c->ework;
    wtd_energy_kernel<<<pb, 128, 0, c->st>>>(c->it, D, P, e + EKIN * (size_t)N, e + EPOT * (size_t)N,
                                             e + EPAIR * (size_t)N, e + ECURRENT * (size_t)N);
    WTD_LAUNCHED(c);
    wtd_energy_ext_kernel<<<pb, 128, 0, c->st>>>(c->it, D, P, e);
    WTD_LAUNCHED(c);
#ifdef ENABLE_MODIFY_ENERGIES
    modify_energies<<<pb, 128, 0, c->st>>>(c->it, D, P, e);
    WTD_LAUNCHED(c);
#endif
    wtd_sum_items<<<TDWSLDAITEMS, 256, 0, c->st>>>(e, N, c->eout, WTD_VOLEL);
    WTD_LAUNCHED(c);
    WTD_CU(cudaMemcpyAsync(host11, c->eout, TDWSLDAITEMS * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    WTD_CU(cudaStreamSynchronize(c->st));
    return WTD_OK;
}

int wtd_sync(wtd_ctx *c)
{
    if (!c) return WTD_ERR_ARG;
    return wtd_cuerr(cudaStreamSynchronize(c->st));
}

int wtd_time_index(wtd_ctx *c) { return c ? c->it : 0; }

int wtd_download_densities(wtd_ctx *c, double *host)
{
    if (!c || !host) return WTD_ERR_ARG;
    WTD_CU(cudaMemcpyAsync(host, c->dens, 12 * (size_t)WTD_NUMEL * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    return wtd_cuerr(cudaStreamSynchronize(c->st));
}

int wtd_download_potentials(wtd_ctx *c, double *host)
{
    if (!c || !host) return WTD_ERR_ARG;
    WTD_CU(cudaMemcpyAsync(host, c->pots, 12 * (size_t)WTD_NUMEL * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    return wtd_cuerr(cudaStreamSynchronize(c->st));
}

int wtd_download_qpe(wtd_ctx *c, double *host)
{
    if (!c || !host) return WTD_ERR_ARG;
    WTD_CU(cudaSetDevice(c->dev));
    WTD_TRY(ensure_fk(c));
    WTD_CU(cudaMemcpyAsync(host, c->qpe, c->S * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    return wtd_cuerr(cudaStreamSynchronize(c->st));
}

int wtd_device_pointers(wtd_ctx *c, void **states, double **dens, double **pots)
{
    if (!c) return WTD_ERR_ARG;
    if (states) *states = c->y;
    if (dens) *dens = c->dens;
    if (pots) *pots = c->pots;
    return WTD_OK;
}

void *wtd_stream(wtd_ctx *c) { return c ? (void *)c->st : NULL; }

int wtd_set_timing(wtd_ctx *c, int on)
{
    if (!c) return WTD_ERR_ARG;
    WTD_CU(cudaSetDevice(c->dev));
    if (on && !c->timing) {
        for (int p = 0; p < 2; p++)
            for (int k = 0; k < 2; k++)
                for (int i = 0; i < 4096; i++) WTD_CU(cudaEventCreate(&c->ev[p][k][i]));
    }
    c->timing = on;
    c->nev[0] = c->nev[1] = 0;
    return WTD_OK;
}

int wtd_pass_times(wtd_ctx *c, double *ms_a, double *ms_b, int *count_a, int *count_b)
{
    if (!c || !c->timing) return WTD_ERR_STATE;
    WTD_CU(cudaStreamSynchronize(c->st));
    double t[2] = {0.0, 0.0};
    for (int p = 0; p < 2; p++)
        for (int i = 0; i < c->nev[p]; i++) {
            float ms = 0.f;
            WTD_CU(cudaEventElapsedTime(&ms, c->ev[p][0][i], c->ev[p][1][i]));
            t[p] += ms;
        }
    if (ms_a) *ms_a = t[0];
    if (ms_b) *ms_b = t[1];
    if (count_a) *count_a = c->nev[0];
    if (count_b) *count_b = c->nev[1];
    c->nev[0] = c->nev[1] = 0;
    return WTD_OK;
}
long long wtd_launch_count(wtd_ctx *c) { return c ? c->launches : 0; }

int wtd_nccl_unique_id(void *id128)
{
    if (!id128) return WTD_ERR_ARG;
    const NcclApi *a = nccl_api();
    ncclUniqueId id;
    if (!a || a->get_unique_id(&id) != ncclSuccess) return WTD_ERR_COMM;
    memcpy(id128, &id, sizeof(id));
    return WTD_OK;
}

int wtd_nccl_attach(wtd_ctx *c, const void *id128, int nranks, int rank)
{
    if (!c || !id128 || nranks < 1 || rank < 0 || rank >= nranks) return WTD_ERR_ARG;
    const NcclApi *a = nccl_api();
    if (!a) return WTD_ERR_COMM;
    WTD_CU(cudaSetDevice(c->dev));
    if (c->nccl) { a->comm_destroy((ncclComm_t)c->nccl); c->nccl = NULL; }
    ncclUniqueId id;
    memcpy(&id, id128, sizeof(id));
    ncclComm_t comm = NULL;
    if (a->comm_init_rank(&comm, nranks, id, rank) != ncclSuccess) return WTD_ERR_COMM;
    c->nccl = comm;
    return WTD_OK;
}

int wtd_set_quantum_friction(wtd_ctx *c, double alpha, double beta, double gamma, double nreq, double start,
                             double stop, double ramp)
{
    if (!c) return WTD_ERR_ARG;
    const bool on = alpha != 0.0 || beta != 0.0 || gamma != 0.0;
    if (on && !(ramp > 0.0)) return WTD_ERR_ARG;
    if (on && c->line) {
        /* the line path has no friction densities: the run continues on the staged path, which
         * keeps the same state, ring and f_k conventions (FP64 only) */
        if (c->prec != WTD_FP64) return WTD_ERR_UNSUPPORTED;
        WTD_CU(cudaSetDevice(c->dev));
        if (!c->fk_given && c->have_coef) WTD_TRY(ensure_fk(c));
        const size_t n2 = (size_t)2 * c->S * WTD_NUMEL;
        cudaError_t e = cudaSuccess;
        double2 **bufs[5] = {&c->ddx, &c->ddy, &c->ddz, &c->dlap, &c->dalap};
        for (int k = 0; k < 5 && e == cudaSuccess; k++)
            if ((k < 4 || WTD_VAR) && !*bufs[k]) e = cudaMalloc((void **)bufs[k], n2 * sizeof(double2));
        if (e != cudaSuccess) { cudaGetLastError(); return WTD_ERR_NOMEM; }
        c->line = 0;
        c->staged = 1;
    }
    c->qf[0] = alpha; c->qf[1] = beta; c->qf[2] = gamma; c->qf[3] = nreq;
    c->qf[4] = start; c->qf[5] = stop; c->qf[6] = ramp;
    c->sstride = (on ? 16 : 12) * WTD_NUMEL;
    return WTD_OK;
}

int wtd_set_high_k_filter(wtd_ctx *c, int mode, double mu, double T)
{
    if (!c || (mode >= 1 && !(T > 0.0))) return WTD_ERR_ARG;
    c->hkf_mode = mode;
    c->hkf_mu = mu;
    c->hkf_T = T;
    return WTD_OK;
}

int wtd_set_density_exchange(wtd_ctx *c, wtd_exchange_fn fn, void *user)
{
    if (!c) return WTD_ERR_ARG;
    c->xfn = fn;
    c->xuser = user;
    return WTD_OK;
}

} /* extern "C" */

/* ---------------------------------------------------------------------------------------
 * Taylor self-start of the ABM history (pca.c:1086-1330, input selfstart 1), FP64: the q
 * first steps are taken with exp(-i H dt) expanded to exp_iters orders (midpoint potentials
 * from a half step), recording (H - <H>) psi of each start state as the history, so that the
 * predictor-corrector starts from a consistent history instead of the zero one.  The
 * reference keeps the time index at its start value and evaluates potentials and H at time
 * index 0 during these steps; so does this.
 * -------------------------------------------------------------------------------------*/
struct SelfWork {
    double2 *ddx, *ddy, *ddz, *dlap, *dalap, *rec;
    double *qs;
    std::vector<void *> own;
};

static int ss_derivs(wtd_ctx *c, SelfWork &w, const double2 *in, int grads)
{
    const int nf = 2 * c->S;
    double2 *dx = grads ? w.ddx : NULL, *dy = (grads && CODEDIM >= 2) ? w.ddy : NULL, *dz = (grads && CODEDIM >= 3) ? w.ddz : NULL;
    if (WTD_BIG) return big_derivs_sep(in, nf, w.dlap, dx, dy, dz, NULL, NULL, c->tw, c->ktab, c->st);
    if (k_derivs_smem > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
    WTD_ONCE_PER_DEVICE(WTD_CU(cudaFuncSetAttribute(k_derivs<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k_derivs_smem)));
    k_derivs<WG><<<nf, 512, k_derivs_smem, c->st>>>(in, dx, dy, dz, w.dlap, c->tw, c->ktab);
    WTD_LAUNCHED(c);
    return WTD_OK;
}

/* densities of the states in `in` (derivatives from ss_derivs), summed over ranks, tau */
static int ss_densities(wtd_ctx *c, SelfWork &w, const double2 *in, int grads)
{
    constexpr int N = WTD_NUMEL;
    k_dens_compat<<<c->grid, 256, 0, c->st>>>(c->S, in, w.ddx, w.ddy, w.ddz, w.dlap, c->occ, NULL, c->kp2, c->wcnt,
                                              c->dslot, grads);
    WTD_LAUNCHED(c);
    wtd_dens_reduce<<<(12 * N + 255) / 256, 256, 0, c->st>>>(c->dslot, c->grid, c->dens, N, grads, 1.0 / WTD_LPERP);
    WTD_LAUNCHED(c);
    WTD_TRY(exchange(c, c->dens, 12 * (size_t)N));
    if (!grads) return WTD_OK;
    if (WTD_BIG) return big_tau(c->dens, c->stage3d, c->tw, c->ktab, c->st);
    constexpr size_t sm = (size_t)WG::padded * sizeof(double2) + WG::twtotal * sizeof(double2) + sizeof(KTab<WG>);
    WTD_ONCE_PER_DEVICE(WTD_CU(cudaFuncSetAttribute(wtd_tau_kernel<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)));
    wtd_tau_kernel<WG><<<2, 512, sm, c->st>>>(c->dens, c->tw, c->ktab);
    WTD_LAUNCHED(c);
    return WTD_OK;
}

/* lap(alpha psi) for the variable-mass kinetic term (multiply_wf_by_alpha + compute_laplace) */
static int ss_alap(wtd_ctx *c, SelfWork &w, const double2 *in)
{
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
    constexpr size_t N = WTD_NUMEL;
    const size_t M = (size_t)2 * c->S * N;
    if (WTD_BIG)
        return big_derivs_sep(in, 2 * c->S, w.dalap, NULL, NULL, NULL, c->pots + 4 * N, c->pots + 5 * N, c->tw, c->ktab,
                              c->st);
    k_mul_alpha<<<(unsigned)((M + 255) / 256), 256, 0, c->st>>>(c->S, in, w.dalap, c->pots + 4 * N, c->pots + 5 * N);
    WTD_LAUNCHED(c);
    k_derivs<WG><<<2 * c->S, 512, k_derivs_smem, c->st>>>(w.dalap, NULL, NULL, NULL, w.dalap, c->tw, c->ktab);
    WTD_LAUNCHED(c);
#else
    (void)c; (void)w; (void)in;
#endif
    return WTD_OK;
}

/* out = (H - E) in at time index 0; E computed into c->qpe, or the given useqpe.  The
 * fields are filtered first, as at the top of every apply_hamiltonian of the reference. */
static int ss_hamiltonian(wtd_ctx *c, SelfWork &w, const double2 *in, double2 *out, const double *useqpe)
{
    WTD_TRY(filter_h(c));
    WTD_TRY(coef_from_pots(c, 0));
    k_hamiltonian_compat<<<c->S, 256, 0, c->st>>>(c->S, in, out, w.ddx, w.ddy, w.ddz, w.dlap, w.dalap, c->cf, c->kp2,
                                                  c->qpe, useqpe);
    WTD_LAUNCHED(c);
    return WTD_OK;
}

/* the Taylor order `order` of exp(-i H t): contr = (i t/order) h, upd += contr */
static int ss_taylor(wtd_ctx *c, const double2 *h, double2 *upd, double2 *contr, double t, int order)
{
    const size_t M = (size_t)2 * c->S * WTD_NUMEL;
    k_taylor<<<(unsigned)((M + 255) / 256), 256, 0, c->st>>>(M, h, upd, contr, -1.0 * t / (double)order);
    WTD_LAUNCHED(c);
    return WTD_OK;
}

static int selfstart_run(wtd_ctx *c, SelfWork &w)
{
    constexpr int NH = WTD_NHIST;
    constexpr size_t N = WTD_NUMEL;
    const int q = NH, iters = (NH == 3) ? 4 : 5;
    const int grads = WTD_VAR ? 1 : 0;
    const size_t NS = (size_t)2 * c->S * N, bytes = NS * sizeof(double2);
    double2 *y = (double2 *)c->y;
    /* work arrays: the physical history slots, overwritten by the history at the end */
    double2 *f1 = (double2 *)c->hist[0], *f2 = (double2 *)c->hist[1], *f3 = (double2 *)c->hist[2];
    const double dt = c->dt;
    c->qfsw = 0.0; /* no friction during the self-start (pca.c:1113, 1209) */
    for (int step = 0; step < q; step++) {
        /* start state: densities and potentials at time index 0, its (H - <H>) psi recorded */
        WTD_TRY(ss_derivs(c, w, y, grads));
        WTD_TRY(ss_densities(c, w, y, grads));
        WTD_TRY(functional(c, 0));
        WTD_TRY(filter_alpha(c));
        WTD_TRY(ss_alap(c, w, y));
        WTD_CU(cudaMemcpyAsync(f3, y, bytes, cudaMemcpyDeviceToDevice, c->st));
        WTD_TRY(ss_hamiltonian(c, w, f3, f1, NULL));
        WTD_CU(cudaMemcpyAsync(w.qs, c->qpe, c->S * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
        for (int h = q - 1; h > 0; h--)
            WTD_CU(cudaMemcpyAsync(w.rec + h * NS, w.rec + (h - 1) * NS, bytes, cudaMemcpyDeviceToDevice, c->st));
        WTD_CU(cudaMemcpyAsync(w.rec, f1, bytes, cudaMemcpyDeviceToDevice, c->st));
        /* half step into f3 */
        WTD_TRY(ss_taylor(c, f1, f3, f2, 0.5 * dt, 1));
        for (int m = 1; m < iters; m++) {
            WTD_TRY(ss_derivs(c, w, f2, grads));
            WTD_TRY(ss_alap(c, w, f2));
            WTD_TRY(ss_hamiltonian(c, w, f2, f1, w.qs));
            WTD_TRY(ss_taylor(c, f1, f3, f2, 0.5 * dt, m + 1));
        }
        k_normalize<<<c->S, 256, 0, c->st>>>(c->S, f3);
        WTD_LAUNCHED(c);
        /* midpoint potentials */
        WTD_TRY(ss_derivs(c, w, f3, grads));
        WTD_TRY(ss_densities(c, w, f3, grads));
        WTD_TRY(functional(c, 0));
        WTD_TRY(filter_alpha(c));
        /* full step of the state with the midpoint H */
        WTD_TRY(ss_derivs(c, w, y, grads));
        WTD_TRY(ss_alap(c, w, y));
        WTD_TRY(ss_hamiltonian(c, w, y, f1, NULL));
        WTD_CU(cudaMemcpyAsync(w.qs, c->qpe, c->S * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
        WTD_TRY(ss_taylor(c, f1, y, f2, dt, 1));
        for (int m = 1; m < iters; m++) {
            WTD_TRY(ss_derivs(c, w, f2, grads));
            WTD_TRY(ss_alap(c, w, f2));
            WTD_TRY(ss_hamiltonian(c, w, f2, f1, w.qs));
            WTD_TRY(ss_taylor(c, f1, y, f2, dt, m + 1));
        }
        k_normalize<<<c->S, 256, 0, c->st>>>(c->S, y);
        WTD_LAUNCHED(c);
    }
    /* the recorded entries become the history, f1 (newest) the given f_k of the next step */
    void *slot[WTD_NHIST];
    ring_slots(c, slot);
    for (int r = 0; r < q; r++)
        WTD_CU(cudaMemcpyAsync(slot[ring_of_ref_slot(r)], w.rec + r * NS, bytes, cudaMemcpyDeviceToDevice, c->st));
    c->fk_given = 1;
    /* densities and potentials of the new state at the current time index (pca.c:1315-1318) */
    WTD_TRY(ss_derivs(c, w, y, 1));
    WTD_TRY(ss_densities(c, w, y, 1));
    WTD_TRY(functional(c, c->it));
    return coef_from_pots(c, c->it);
}

extern "C" int wtd_selfstart(wtd_ctx *c)
{
    if (!c) return WTD_ERR_ARG;
    if (c->prec != WTD_FP64) return WTD_ERR_UNSUPPORTED;
    WTD_CU(cudaSetDevice(c->dev));
    constexpr size_t N = WTD_NUMEL;
    const size_t NS = (size_t)2 * c->S * N;
    SelfWork w{};
    auto get = [&](double2 **p, size_t n) -> int {
        void *q = NULL;
        if (cudaMalloc(&q, n * sizeof(double2)) != cudaSuccess) { cudaGetLastError(); return WTD_ERR_NOMEM; }
        w.own.push_back(q);
        *p = (double2 *)q;
        return WTD_OK;
    };
    int r = WTD_OK;
    if (c->staged) {
        w.ddx = c->ddx; w.ddy = c->ddy; w.ddz = c->ddz; w.dlap = c->dlap; w.dalap = c->dalap;
    } else {
        r = get(&w.ddx, NS);
        if (!r && CODEDIM >= 2) r = get(&w.ddy, NS);
        if (!r && CODEDIM >= 3) r = get(&w.ddz, NS);
        if (!r) r = get(&w.dlap, NS);
        if (!r && WTD_VAR) r = get(&w.dalap, NS);
    }
    if (!r) r = get(&w.rec, (size_t)WTD_NHIST * NS);
    if (!r) r = get((double2 **)&w.qs, (size_t)c->S);
    if (!r) r = selfstart_run(c, w);
    cudaStreamSynchronize(c->st);
    for (void *q : w.own) cudaFree(q);
    return r ? r : wtd_cuerr(cudaGetLastError());
}

/* densities of a weighted subset of the states (the reference's subset tracking, pca.c:842-870,
 * 1056-1066: weight 1 for quasiparticle energies inside [subsetMinEn, subsetMaxEn] eF): the
 * density sums of calculate_densities with each state's occupation factors multiplied by its
 * weight (pca_dens.cu:46-47), gradients and tau included, summed over ranks */
extern "C" int wtd_subset_densities(wtd_ctx *c, const double *weights, double *host12)
{
    if (!c || !weights || !host12) return WTD_ERR_ARG;
    if (c->prec != WTD_FP64) return WTD_ERR_UNSUPPORTED;
    WTD_CU(cudaSetDevice(c->dev));
    constexpr size_t N = WTD_NUMEL;
    const size_t NS = (size_t)2 * c->S * N;
    SelfWork w{};
    double *dw = NULL, *out = NULL;
    auto get = [&](void **p, size_t bytes) -> int {
        if (cudaMalloc(p, bytes) != cudaSuccess) { cudaGetLastError(); return WTD_ERR_NOMEM; }
        w.own.push_back(*p);
        return WTD_OK;
    };
    int r = WTD_OK;
    if (c->staged) {
        w.ddx = c->ddx; w.ddy = c->ddy; w.ddz = c->ddz; w.dlap = c->dlap;
    } else {
        r = get((void **)&w.ddx, NS * sizeof(double2));
        if (!r && CODEDIM >= 2) r = get((void **)&w.ddy, NS * sizeof(double2));
        if (!r && CODEDIM >= 3) r = get((void **)&w.ddz, NS * sizeof(double2));
        if (!r) r = get((void **)&w.dlap, NS * sizeof(double2));
    }
    if (!r) r = get((void **)&dw, c->S * sizeof(double));
    if (!r) r = get((void **)&out, 12 * N * sizeof(double));
    if (!r) r = wtd_cuerr(cudaMemcpyAsync(dw, weights, c->S * sizeof(double), cudaMemcpyHostToDevice, c->st));
    if (!r) r = ss_derivs(c, w, (const double2 *)c->y, 1);
    if (!r) {
        k_dens_compat<<<c->grid, 256, 0, c->st>>>(c->S, (const double2 *)c->y, w.ddx, w.ddy, w.ddz, w.dlap, c->occ, dw,
                                                  c->kp2, c->wcnt, c->dslot, 1);
        wtd_dens_reduce<<<(12 * (int)N + 255) / 256, 256, 0, c->st>>>(c->dslot, c->grid, out, (int)N, 1, 1.0 / WTD_LPERP);
        r = wtd_cuerr(cudaGetLastError());
        c->launches += 2;
    }
    if (!r) r = exchange(c, out, 12 * N);
    if (!r) {
        if (WTD_BIG) {
            r = big_tau(out, c->stage3d, c->tw, c->ktab, c->st);
        } else {
            constexpr size_t sm = (size_t)WG::padded * sizeof(double2) + WG::twtotal * sizeof(double2) + sizeof(KTab<WG>);
            cudaFuncSetAttribute(wtd_tau_kernel<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            wtd_tau_kernel<WG><<<2, 512, sm, c->st>>>(out, c->tw, c->ktab);
            r = wtd_cuerr(cudaGetLastError());
            c->launches++;
        }
    }
    if (!r) r = wtd_cuerr(cudaMemcpyAsync(host12, out, 12 * N * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    cudaStreamSynchronize(c->st);
    for (void *q : w.own) cudaFree(q);
    return r;
}

/* ---------------------------------------------------------------------------------------
 * adjoint (gradient of a loss of the final pairing field with respect to the parameters of
 * the external potential): forward with checkpoints, the last segment recorded as it runs;
 * reverse sweep over segments, recomputing each earlier segment once with records
 * -------------------------------------------------------------------------------------*/
#include "wtd_adjoint.cuh"

#if defined(WTD_ADJOINT_CONTACT_BDG) && defined(FAST_CONST_EFFECTIVE_MASS_MODE)
/* device allocations of the adjoint workspace, released together */
struct AdjPool {
    cudaStream_t st;
    size_t bytes = 0;
    std::vector<void *> p;
    explicit AdjPool(cudaStream_t s) : st(s) {}
    template <typename T> int get(T **out, size_t count)
    {
        void *q = NULL;
        if (cudaMalloc(&q, count * sizeof(T) + 16) != cudaSuccess) { cudaGetLastError(); return WTD_ERR_NOMEM; }
        p.push_back(q);
        bytes += count * sizeof(T) + 16;
        *out = (T *)q;
        return WTD_OK;
    }
    ~AdjPool()
    {
        cudaStreamSynchronize(st); /* nothing queued may still use the buffers */
        for (void *q : p) cudaFree(q);
    }
};

/* everything a step reads of the context: states, physical history slots, coefficients,
 * densities, potentials, <H> and the ring/time bookkeeping */
struct Checkpoint {
    void *y;
    void *hist[WTD_NHIST];
    double *cf, *dens, *pots, *qpe;
    int head, it, fk_given, have_coef;
};

static int ck_alloc(wtd_ctx *c, AdjPool &pool, Checkpoint &k)
{
    constexpr size_t N = WTD_NUMEL;
    WTD_TRY(pool.get((char **)&k.y, c->ysz));
    for (int h = 0; h < WTD_NHIST; h++) WTD_TRY(pool.get((char **)&k.hist[h], c->hsz));
    WTD_TRY(pool.get(&k.cf, CF_COUNT * N));
    WTD_TRY(pool.get(&k.dens, 12 * N));
    WTD_TRY(pool.get(&k.pots, 12 * N));
    WTD_TRY(pool.get(&k.qpe, (size_t)c->S));
    return WTD_OK;
}

static int ck_copy(wtd_ctx *c, bool save, Checkpoint &k)
{
    constexpr size_t N = WTD_NUMEL;
    auto cp = [&](void *ctxp, void *ckp, size_t bytes) {
        return cudaMemcpyAsync(save ? ckp : ctxp, save ? ctxp : ckp, bytes, cudaMemcpyDeviceToDevice, c->st);
    };
    WTD_CU(cp(c->y, k.y, c->ysz));
    for (int h = 0; h < WTD_NHIST; h++) WTD_CU(cp(c->hist[h], k.hist[h], c->hsz));
    WTD_CU(cp(c->cf, k.cf, CF_COUNT * N * sizeof(double)));
    WTD_CU(cp(c->dens, k.dens, 12 * N * sizeof(double)));
    WTD_CU(cp(c->pots, k.pots, 12 * N * sizeof(double)));
    WTD_CU(cp(c->qpe, k.qpe, (size_t)c->S * sizeof(double)));
    if (save) { k.head = c->head; k.it = c->it; k.fk_given = c->fk_given; k.have_coef = c->have_coef; }
    else { c->head = k.head; c->it = k.it; c->fk_given = k.fk_given; c->have_coef = k.have_coef; }
    return WTD_OK;
}

/* the workspace: capK step records and capCk checkpoints (capK = 0: loss only) */
struct AdjWork {
    AdjPool pool;
    int capK = 0, capCk = 0;
    std::vector<Checkpoint> ck;
    Checkpoint fin;                 /* the forward's final state when segments are recomputed */
    std::vector<StepRecord> rec;
    double2 *ybar = NULL, *ypbar = NULL, *pbar = NULL, *fring[WTD_NHIST] = {};
    double *fields = NULL, *dgrad = NULL, *tpart = NULL, *dloss = NULL, *dmask = NULL;
    /* events of the last forward (start, loss) and of the last reverse sweep (start, end) */
    cudaEvent_t ev[4] = {};
    bool timed_f = false, timed_r = false;
    /* a recorded forward the reverse sweep may follow: its schedule, the time index of each
     * step of the last segment, and the context's counters when it ended (any later launch,
     * upload or setter invalidates it) */
    bool ready = false;
    int K = 0, nsteps = 0, nseg = 0, last0 = 0;
    std::vector<int> itk;
    long long mark_launches = 0, mark_mut = 0;
    explicit AdjWork(cudaStream_t s) : pool(s)
    {
        for (auto &e : ev) cudaEventCreate(&e);
    }
    ~AdjWork()
    {
        for (auto &e : ev) if (e) cudaEventDestroy(e);
    }
};

static size_t adj_record_bytes(const wtd_ctx *c)
{
    return 2 * c->ysz + 2 * CF_COUNT * (size_t)WTD_NUMEL * sizeof(double) + 4 * (size_t)c->S * sizeof(double) + 96;
}
static size_t adj_ck_bytes(const wtd_ctx *c)
{
    return c->ysz + WTD_NHIST * c->hsz + (CF_COUNT + 24) * (size_t)WTD_NUMEL * sizeof(double) + (size_t)c->S * 8 + 112;
}
/* device bytes of a gradient workspace with K records and nck checkpoints */
static size_t adj_bytes(const wtd_ctx *c, int K, int nck)
{
    size_t b = (size_t)K * adj_record_bytes(c) + (size_t)(nck > 0 ? nck + 1 : 0) * adj_ck_bytes(c);
    if (K > 0) b += (3 + WTD_NHIST) * c->ysz;
    return b + 8 * (size_t)WTD_NUMEL * sizeof(double) + (1 << 16);
}

static void adj_release(wtd_ctx *c)
{
    delete (AdjWork *)c->adj;
    c->adj = NULL;
}

/* a workspace for K records and nck checkpoints: the cached one if large enough */
static int adj_workspace(wtd_ctx *c, int K, int nck, AdjWork **out)
{
    AdjWork *w = (AdjWork *)c->adj;
    if (w && w->capK >= K && w->capCk >= nck) { *out = w; return WTD_OK; }
    const int capK = w ? (K > w->capK ? K : w->capK) : K, capCk = w ? (nck > w->capCk ? nck : w->capCk) : nck;
    adj_release(c);
    w = new AdjWork(c->st);
    c->adj = w;
    constexpr size_t N = WTD_NUMEL;
    const size_t NS = (size_t)2 * c->S * N;
    int r = WTD_OK;
    auto get = [&](auto **p, size_t n) { if (r == WTD_OK) r = w->pool.get(p, n); };
    get(&w->dloss, 1);
    get(&w->fields, 4 * N);
    get(&w->dmask, N);
    get(&w->dgrad, (size_t)MAX_USER_PARAMS);
    get(&w->tpart, (size_t)MAX_USER_PARAMS * WTD_THETA_CHUNKS);
    if (capK > 0) {
        get(&w->ybar, NS);
        get(&w->ypbar, NS);
        get(&w->pbar, NS);
        for (int j = 0; j < WTD_NHIST; j++) get(&w->fring[j], NS);
        w->rec.resize(capK);
        for (auto &q : w->rec) {
            get(&q.yk, NS);
            get(&q.yp, NS);
            get(&q.cfA, CF_COUNT * N);
            get(&q.cfB, CF_COUNT * N);
            double *sc = NULL;
            get(&sc, 4 * (size_t)c->S);
            q.EA = sc; q.EB = sc ? sc + c->S : NULL; q.nA = sc ? sc + 2 * c->S : NULL; q.nB = sc ? sc + 3 * c->S : NULL;
        }
    }
    if (capCk > 0) {
        w->ck.resize(capCk);
        for (auto &k : w->ck) if (r == WTD_OK) r = ck_alloc(c, w->pool, k);
        if (r == WTD_OK) r = ck_alloc(c, w->pool, w->fin);
    }
    if (r != WTD_OK) { adj_release(c); return r; }
    w->capK = capK;
    w->capCk = capCk;
    *out = w;
    return WTD_OK;
}

/* checkpoint interval: the caller's, or (0) the largest that fits in free device memory —
 * nsteps itself (one segment, no recompute) when the records of every step fit */
static int adj_choose_K(wtd_ctx *c, int nsteps, int K)
{
    if (K > 0) return K < nsteps ? K : nsteps;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return -1;
    if (c->adj) fr += ((AdjWork *)c->adj)->pool.bytes;
    const size_t margin = ((size_t)1 << 30) + tot / 50;
    const size_t budget = fr > margin ? fr - margin : 0;
    for (int k = nsteps; k >= 1; k--) {
        const int nck = (nsteps + k - 1) / k - 1;
        if (adj_bytes(c, k, nck) <= budget) return k;
    }
    return -1;
}

/* the forward from the uploaded states: initial measurement(it0), nsteps steps and the loss.
 * record: keep a checkpoint every K steps and the last segment's step records, so that
 * adjoint_reverse can follow (K from Kin as adj_choose_K picks it) */
static int adjoint_forward(wtd_ctx *c, int it0, int nsteps, int Kin, const double *mask_h, bool record, double *loss_h)
{
    constexpr int N = WTD_NUMEL;
    constexpr size_t sm = 2 * (size_t)WG::padded * sizeof(double2) + WG::twtotal * sizeof(double2) + sizeof(KTab<WG>) +
                          80 * sizeof(double);
    if (sm > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
    const int K = record ? adj_choose_K(c, nsteps, Kin) : 0;
    if (record && K < 1) return WTD_ERR_NOMEM;
    const int nseg = record ? (nsteps + K - 1) / K : 1;
    const int last0 = (nseg - 1) * K; /* first step of the last segment, recorded by the forward */
    AdjWork *w = NULL;
    WTD_TRY(adj_workspace(c, K, record ? nseg - 1 : 0, &w));
    w->ready = false;
    w->K = K; w->nsteps = nsteps; w->nseg = nseg; w->last0 = last0;
    w->itk.assign(K > 0 ? K : 1, 0);
    double2 *nubar = (double2 *)(w->fields + 2 * (size_t)N);
    if (mask_h) WTD_CU(cudaMemcpyAsync(w->dmask, mask_h, N * sizeof(double), cudaMemcpyHostToDevice, c->st));

    w->timed_f = w->timed_r = false;
    WTD_CU(cudaEventRecord(w->ev[0], c->st));
    WTD_TRY(wtd_initial_measurement(c, it0));
    for (int s = 0; s < nsteps; s++) {
        StepRecord *r = NULL;
        if (record && s < last0 && s % K == 0) WTD_TRY(ck_copy(c, true, w->ck[s / K]));
        double2 *next = NULL;
        if (record && s >= last0) {
            const int j = s - last0;
            r = &w->rec[j];
            w->itk[j] = c->it;
            if (j == 0) WTD_CU(cudaMemcpyAsync(r->yk, c->y, c->ysz, cudaMemcpyDeviceToDevice, c->st));
            if (s + 1 < nsteps) next = w->rec[j + 1].yk;
        }
        WTD_TRY(fused_step(c, s == nsteps - 1, r, next));
    }
    k_adj_loss<<<1, 512, 0, c->st>>>(c->pots, mask_h ? w->dmask : NULL, nubar, w->dloss);
    WTD_LAUNCHED(c);
    WTD_CU(cudaMemcpyAsync(loss_h, w->dloss, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    WTD_CU(cudaEventRecord(w->ev[1], c->st));
    WTD_TRY(wtd_cuerr(cudaStreamSynchronize(c->st)));
    w->timed_f = true;
    w->ready = record;
    w->mark_launches = c->launches;
    w->mark_mut = c->mut;
    return WTD_OK;
}

/* the reverse sweep after a recorded forward: dL/dparams[0..nparam) into grad_h; the context is
 * left where the forward left it */
static int adjoint_reverse(wtd_ctx *c, int nparam, double *grad_h)
{
    constexpr int N = WTD_NUMEL, NH = WTD_NHIST;
    const int S = c->S;
    const size_t NS = (size_t)2 * S * N;
    constexpr size_t sm = 2 * (size_t)WG::padded * sizeof(double2) + WG::twtotal * sizeof(double2) + sizeof(KTab<WG>) +
                          80 * sizeof(double);
    AdjWork *w = (AdjWork *)c->adj;
    if (!w || !w->ready || w->mark_launches != c->launches || w->mark_mut != c->mut) return WTD_ERR_STATE;
    w->ready = false;
    const int K = w->K, nsteps = w->nsteps, nseg = w->nseg;
    std::vector<int> &itk = w->itk;
    double *vbar = w->fields;
    double2 *nubar = (double2 *)(w->fields + 2 * (size_t)N);
    WTD_CU(cudaEventRecord(w->ev[2], c->st));

    /* reverse sweep */
    if (nseg > 1) WTD_TRY(ck_copy(c, true, w->fin));
    for (int j = 0; j < NH; j++) WTD_CU(cudaMemsetAsync(w->fring[j], 0, NS * sizeof(double2), c->st));
    WTD_CU(cudaMemsetAsync(w->ybar, 0, NS * sizeof(double2), c->st));
    WTD_CU(cudaMemsetAsync(w->dgrad, 0, MAX_USER_PARAMS * sizeof(double), c->st));
    auto theta_grad = [&](int it) -> int {
        if (nparam <= 0) return WTD_OK;
        k_theta_grad<<<dim3(nparam, WTD_THETA_CHUNKS), 256, 0, c->st>>>(vbar, it, w->tpart);
        WTD_LAUNCHED(c);
        k_theta_sum<<<1, ((nparam + 31) / 32) * 32, 0, c->st>>>(w->tpart, nparam, WTD_THETA_CHUNKS, w->dgrad);
        WTD_LAUNCHED(c);
        return WTD_OK;
    };
    auto kB = k_adj_B<WG, NH>;
    auto kA = k_adj_A<WG, NH>;
    WTD_ONCE_PER_DEVICE(
        WTD_CU(cudaFuncSetAttribute(kB, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        WTD_CU(cudaFuncSetAttribute(kA, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)));
    /* the reverse kernels: one persistent CTA of 512 threads per SM (two CTAs of 256 per SM
     * measured the same); the slots hold c->grid * 12 N words, so up to 3 * c->grid CTAs of 4 N */
    const int threads = WG::ntot >= 512 ? 512 : ((WG::ntot + 31) / 32) * 32;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->dev);
    int agrid = nsm;
    if (agrid > 3 * c->grid) agrid = 3 * c->grid;
    if (agrid > S) agrid = S;
    const int nb = (N + 255) / 256;
    AdjArgs base;
    memset(&base, 0, sizeof(base));
    base.occ = c->occ; base.kp2 = c->kp2; base.wcnt = c->wcnt;
    base.slots = c->dslot; base.dt = c->dt; base.inv_lperp = 1.0 / WTD_LPERP; base.S = S;
    base.ybar = w->ybar; base.ypbar = w->ypbar; base.pbar = w->pbar;
    double2 *fring[NH];
    for (int q = 0; q < NH; q++) fring[q] = w->fring[q];
    bool pending = true; /* nubar holds the loss seed, the adjoint of nu(y_T) */
    for (int sg = nseg - 1; sg >= 0; sg--) {
        const int len = (sg == nseg - 1) ? nsteps - sg * K : K;
        if (sg < nseg - 1) {
            /* recompute this segment from its checkpoint, recording every step */
            WTD_TRY(ck_copy(c, false, w->ck[sg]));
            WTD_CU(cudaMemcpyAsync(w->rec[0].yk, c->y, c->ysz, cudaMemcpyDeviceToDevice, c->st));
            for (int j = 0; j < len; j++) {
                itk[j] = c->it;
                WTD_TRY(fused_step(c, false, &w->rec[j], j + 1 < len ? w->rec[j + 1].yk : NULL));
            }
        }
        for (int j = len - 1; j >= 0; j--) {
            const StepRecord &r = w->rec[j];
            AdjArgs b = base;
            b.y1 = (j == len - 1) ? (const double2 *)c->y : w->rec[j + 1].yk;
            b.yp = r.yp; b.nubar = pending ? nubar : NULL;
            b.nrm = r.nB; b.E = r.EB; b.cf = r.cfB;
            kB<<<agrid, threads, sm, c->st>>>(b, c->tw, c->ktab);
            WTD_LAUNCHED(c);
            k_adj_reduce<<<nb, 256, 0, c->st>>>(c->dslot, agrid, vbar, nubar);
            WTD_LAUNCHED(c);
            WTD_TRY(exchange(c, w->fields, 4 * (size_t)N));
            WTD_TRY(theta_grad(itk[j] + 1));
            AdjArgs a = base;
            a.y1 = r.yk; a.yp = r.yp; a.nubar = nubar;
            a.nrm = r.nA; a.E = r.EA; a.cf = r.cfA; a.has_h = r.hasH;
            for (int q = 0; q < NH; q++) a.fring[q] = fring[q];
            kA<<<agrid, threads, sm, c->st>>>(a, c->tw, c->ktab);
            WTD_LAUNCHED(c);
            if (r.hasH) {
                k_adj_reduce<<<nb, 256, 0, c->st>>>(c->dslot, agrid, vbar, nubar);
                WTD_LAUNCHED(c);
                WTD_TRY(exchange(c, w->fields, 4 * (size_t)N));
                WTD_TRY(theta_grad(itk[j]));
            }
            pending = r.hasH != 0;
            /* the ring moves one step back: fbar_{k-1} becomes position 0 */
            double2 *f0 = fring[0];
            for (int q = 0; q < NH - 1; q++) fring[q] = fring[q + 1];
            fring[NH - 1] = f0;
            WTD_CU(cudaMemsetAsync(f0, 0, NS * sizeof(double2), c->st));
        }
    }
    if (nseg > 1) WTD_TRY(ck_copy(c, false, w->fin));
    WTD_CU(cudaMemcpyAsync(grad_h, w->dgrad, nparam * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    WTD_CU(cudaEventRecord(w->ev[3], c->st));
    WTD_TRY(wtd_cuerr(cudaStreamSynchronize(c->st)));
    w->timed_r = true;
    return WTD_OK;
}

static int adj_times(wtd_ctx *c, double *ms_forward, double *ms_reverse)
{
    AdjWork *w = (AdjWork *)c->adj;
    if (!w || !w->timed_f) return WTD_ERR_STATE;
    float a = 0.f, b = 0.f;
    WTD_CU(cudaEventElapsedTime(&a, w->ev[0], w->ev[1]));
    if (w->timed_r) WTD_CU(cudaEventElapsedTime(&b, w->ev[2], w->ev[3]));
    *ms_forward = a;
    *ms_reverse = b;
    return WTD_OK;
}
#else
static void adj_release(wtd_ctx *c) { (void)c; }
static int adj_times(wtd_ctx *, double *, double *) { return WTD_ERR_UNSUPPORTED; }
#endif

extern "C" int wtd_adjoint(wtd_ctx *c, int it0, int nsteps, int checkpoint_every, const double *mask, int nparam,
                           double *loss, double *grad)
{
    if (!c || !loss || nsteps < 1 || checkpoint_every < 0 || nparam < 0 || nparam > MAX_USER_PARAMS ||
        (grad && nparam < 1))
        return WTD_ERR_ARG;
#if defined(WTD_ADJOINT_CONTACT_BDG) && defined(FAST_CONST_EFFECTIVE_MASS_MODE) && !defined(SPINSYMMETRY_MODE)
    if (c->prec != WTD_FP64 || c->staged || c->sstride != 12 * WTD_NUMEL) return WTD_ERR_UNSUPPORTED;
    WTD_CU(cudaSetDevice(c->dev));
    int r = adjoint_forward(c, it0, nsteps, checkpoint_every, mask, grad != NULL, loss);
    if (r == WTD_OK && grad) r = adjoint_reverse(c, nparam, grad);
    if (r != WTD_OK) cudaStreamSynchronize(c->st);
    return r;
#else
    (void)it0; (void)mask; (void)grad;
    return WTD_ERR_UNSUPPORTED;
#endif
}

extern "C" int wtd_adjoint_forward(wtd_ctx *c, int it0, int nsteps, int checkpoint_every, const double *mask,
                                   double *loss)
{
    if (!c || !loss || nsteps < 1 || checkpoint_every < 0) return WTD_ERR_ARG;
#if defined(WTD_ADJOINT_CONTACT_BDG) && defined(FAST_CONST_EFFECTIVE_MASS_MODE) && !defined(SPINSYMMETRY_MODE)
    if (c->prec != WTD_FP64 || c->staged || c->sstride != 12 * WTD_NUMEL) return WTD_ERR_UNSUPPORTED;
    WTD_CU(cudaSetDevice(c->dev));
    const int r = adjoint_forward(c, it0, nsteps, checkpoint_every, mask, true, loss);
    if (r != WTD_OK) cudaStreamSynchronize(c->st);
    return r;
#else
    (void)it0; (void)mask;
    return WTD_ERR_UNSUPPORTED;
#endif
}

extern "C" int wtd_adjoint_backward(wtd_ctx *c, int nparam, double *grad)
{
    if (!c || !grad || nparam < 1 || nparam > MAX_USER_PARAMS) return WTD_ERR_ARG;
#if defined(WTD_ADJOINT_CONTACT_BDG) && defined(FAST_CONST_EFFECTIVE_MASS_MODE) && !defined(SPINSYMMETRY_MODE)
    WTD_CU(cudaSetDevice(c->dev));
    const int r = adjoint_reverse(c, nparam, grad);
    if (r != WTD_OK) cudaStreamSynchronize(c->st);
    return r;
#else
    return WTD_ERR_UNSUPPORTED;
#endif
}

extern "C" int wtd_adjoint_times(wtd_ctx *c, double *ms_forward, double *ms_reverse)
{
    if (!c || !ms_forward || !ms_reverse) return WTD_ERR_ARG;
    WTD_CU(cudaSetDevice(c->dev));
    return adj_times(c, ms_forward, ms_reverse);
}

extern "C" int wtd_adjoint_release(wtd_ctx *c)
{
    if (!c) return WTD_ERR_ARG;
    WTD_CU(cudaSetDevice(c->dev));
    adj_release(c);
    return WTD_OK;
}

#endif
