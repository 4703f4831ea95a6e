/*
 * Fused TD step for states that fit in one CTA's shared memory (every 1D and 2D lattice of
 * the reference's configurations and small 3D lattices).
 *
 * One persistent CTA owns one quasiparticle state (u, v) at a time and runs, for that state,
 * everything the reference does in separate whole-array kernels:
 *
 *   pass A  (H y_k, predictor)     hpc-engine/pca.c:1565 (H psi into f1) + pca.c:1407-1410
 *     FFT -> k-space multiply -> inverse FFT  (pca_derivative.cu:217-380)
 *     (H - mu) psi with pairing coupling       (pca_kernels.cu:233-495)
 *     <psi|H|psi> subtraction                  (pca_kernels.cu:806-833)
 *     ABM predictor y_pred, partial corrector P (tdwslda_ode_integrator.h:26-135)
 *     renormalisation                          (pca_kernels.cu:913-976)
 *     density contribution of y_pred           (pca_dens.cu:13-198)
 *   pass B  (H y_pred, corrector)  pca.c:1460-1529
 *     same H, then y_{k+1} = P - i dt c (H - <H>) y_pred (tdwslda_ode_integrator.h:138-220),
 *     renormalisation, density contribution (with tau and j on gradient steps).
 *
 * HBM traffic per state and pass is the compulsory stream: pass A reads y and the q history
 * slots and writes f_k, y_pred and P; pass B reads y_pred and P and writes y_{k+1}.  The
 * density sums of the states a CTA processes accumulate in a private FP64 slot that a second
 * kernel reduces in fixed order.  Every word of a slot is updated by one thread only, as L2
 * reductions (red.add, the thread does not wait for the old value) that take effect in program
 * order: the sum and its rounding are those of a plain read-modify-write loop, deterministic.
 *
 * Precision forms (template arguments): TY = storage of y (double2 or float2), TH = storage
 * of history and P, TC = arithmetic of the FFT and H psi.  The ABM combination, the norms,
 * <H> and all density sums are evaluated in FP64.
 */
#ifndef WTD_STEP_CUH
#define WTD_STEP_CUH

#include "wtd_core.cuh"

/* per-point coefficients prepared once per half-step from the potentials */
enum {
    CF_VA = 0,   /* V_a - mu_a                                   */
    CF_VB,       /* V_b - mu_b                                   */
    CF_DRE,      /* Re(Delta + Delta_ext)                        */
    CF_DIM,      /* Im(Delta + Delta_ext)                        */
    CF_AA,       /* -alpha_a/2 (const mass) or -alpha_a/4         */
    CF_AB,       /* -alpha_b/2 (const mass) or -alpha_b/4         */
    CF_NA,       /* lap(alpha_a)/4            (variable mass)     */
    CF_NB,       /* lap(alpha_b)/4                                */
    CF_CJA,      /* -div(A_a)/2                                   */
    CF_CJB,      /* -div(A_b)/2                                   */
    CF_ALA,      /* alpha_a                                       */
    CF_ALB,      /* alpha_b                                       */
    CF_AAX,      /* A_a x, y, z                                   */
    CF_AAY,
    CF_AAZ,
    CF_ABX,      /* A_b x, y, z                                   */
    CF_ABY,
    CF_ABZ,
    CF_COUNT
};

struct StepArgs {
    void *y;            /* [2S][N] TY */
    void *yout;         /* where the pass writes the updated states (NULL: in place into y) */
    void *slot[5];      /* history ring, [2S][N] TH each, indexed by ring position */
    const double *cf;   /* [CF_COUNT][N] */
    const double *occ;  /* f_n */
    const double *kp2;  /* per-state |k_perp|^2 of the plane-wave factor (1D/2D) */
    const double *wcnt; /* per-state degeneracy weight */
    double *dslot;      /* [grid][12][N] density partial sums */
    double *qpe;        /* [S] <H> of the last H application */
    double *nrm_out;    /* [S] norm of the unnormalised update (nullable; the adjoint records it) */
    double dt;
    int S;
    int fk_given;       /* pass A: f_k is already in ring slot NH-1 */
    int prefetch;       /* bit 0: next state's y; bits 1-3: how many of this state's ABM history
                         * arrays go into L2 ahead of the FFT phase (7: all) */
    int accumulate;     /* add to the density slot (otherwise start from zero) */
    int sstride;        /* density-slot words per CTA: 12 N, or 16 N with quantum friction */
    int qf;             /* accumulate the quantum-friction densities (needs GRAD) */
};

/* ABM coefficients (tdwslda_ode_integrator.h:44-45, 69-70, 94-95, 153, 172, 191) */
template <int NH> struct Abm {
    /* predictor weights of f_k, f_{k-1}, ... */
    __host__ __device__ static constexpr double b(int j)
    {
        return NH == 3 ? (j == 0 ? 23. / 12. : j == 1 ? -16. / 12. : j == 2 ? 5. / 12. : 0.)
             : NH == 4 ? (j == 0 ? 55. / 24. : j == 1 ? -59. / 24. : j == 2 ? 37. / 24. : j == 3 ? -9. / 24. : 0.)
                       : (j == 0 ? 1901. / 720. : j == 1 ? -2774. / 720. : j == 2 ? 2616. / 720. : j == 3 ? -1274. / 720. : 251. / 720.);
    }
    /* partial corrector weights of f_k, f_{k-1}, ... (the AM term of f_{k+1} is c) */
    __host__ __device__ static constexpr double a(int j)
    {
        return NH == 3 ? (j == 0 ? 19. / 24. : j == 1 ? -5. / 24. : j == 2 ? 1. / 24. : 0.)
                       : (j == 0 ? 646. / 720. : j == 1 ? -264. / 720. : j == 2 ? 106. / 720. : j == 3 ? -19. / 720. : 0.);
    }
    static constexpr double c = NH == 3 ? 9. / 24. : 251. / 720.;
    static constexpr int na = NH == 3 ? 3 : 4;
};

template <typename T> __device__ __forceinline__ double2 ld2(const T *p, size_t i) { return to_d(p[i]); }

/* entries per axis of the wave-number tables: the longest lattice axis (at least 128) */
#define WTD_KT_MAXN ((NX) > (NY) ? ((NX) > (NZ) ? (NX) : (NZ)) : ((NY) > (NZ) ? (NY) : (NZ)))
#define WTD_KT (WTD_KT_MAXN > 128 ? ((WTD_KT_MAXN + 31) / 32) * 32 : 128)

/* k-space multiplier tables: per axis, wave numbers of digit-reversed positions */
template <class G> struct KTab {
    double k[6][WTD_KT];   /* rows 0-2: k_d of a digit-reversed position; rows 3-5: same with the
                           Nyquist mode set to 0 (first derivatives) */
};

/* the spectral operator applied in k-space */
enum { OP_LAP = 0, OP_DX = 1, OP_DY = 2, OP_DZ = 3 };

/* multiply a transformed field by the operator OP (1/N folded in): laplacian -|k|^2/N,
 * d/dx_d -> i k_d/N with the Nyquist mode zeroed (pca_derivative.cu:152-171) */
template <class G, int OP, typename C>
__device__ __forceinline__ void kmul(C *buf, const double (*kt)[WTD_KT])
{
    typedef decltype(buf[0].x) R;
    for (int i = threadIdx.x; i < G::ntot; i += blockDim.x) {
        int c0, c1 = 0, c2 = 0;
        if (G::dims == 1) { c0 = i; }
        else if (G::dims == 2) { c0 = i / G::N1; c1 = i - c0 * G::N1; }
        else { c0 = i / (G::N1 * G::N2); int r = i - c0 * G::N1 * G::N2; c1 = r / G::N2; c2 = r - c1 * G::N2; }
        int o = G::off(i);
        C z = buf[o];
        if (OP == OP_LAP) {
            double k2 = kt[0][c0] * kt[0][c0];
            if (G::dims >= 2) k2 += kt[1][c1] * kt[1][c1];
            if (G::dims >= 3) k2 += kt[2][c2] * kt[2][c2];
            R s = (R)(-1.0 * k2 / G::ntot);
            z.x *= s; z.y *= s;
        } else {
            constexpr int ax = OP - 1;
            int cc = ax == 0 ? c0 : ax == 1 ? c1 : c2;
            R s = (R)(kt[3 + ax][cc] / G::ntot);
            C t; t.x = -s * z.y; t.y = s * z.x;
            z = t;
        }
        buf[o] = z;
    }
}

/* ---------------------------------------------------------------------------------------
 * shared-memory layout of the fused kernel
 * -------------------------------------------------------------------------------------*/
template <class G, typename TC, int NBUF> struct FusedSmem {
    typedef typename cplx<TC>::t C;
    static constexpr size_t buf_bytes = (size_t)G::padded * sizeof(C);
    static constexpr size_t tw_bytes = (size_t)G::twtotal * sizeof(C);
    static constexpr size_t bytes = NBUF * buf_bytes + tw_bytes + sizeof(KTab<G>) + 80 * sizeof(double);
};

/* load twiddles (e^{-2 pi i t/n} per axis) and the k tables into shared memory */
template <class G, typename C>
__device__ __forceinline__ void load_tables(C *tw, double (*kt)[WTD_KT], const double2 *gtw, const double *gk)
{
    for (int t = threadIdx.x; t < G::twtotal; t += blockDim.x) {
        double2 w = gtw[t];
        C c; c.x = w.x; c.y = w.y;
        tw[t] = c;
    }
    for (int t = threadIdx.x; t < 6 * WTD_KT; t += blockDim.x) kt[t / WTD_KT][t % WTD_KT] = gk[t];
    __syncthreads();
}

/* ---------------------------------------------------------------------------------------
 * H psi for one state, constant effective mass (FAST_CONST_EFFECTIVE_MASS_MODE / BDG_MODE).
 * On return BU/BV hold (H psi) in natural order (compute precision) and the function returns
 * <psi|H|psi> dV.  pca_kernels.cu:233-391 (const-mass branches) and :393-495 (BdG).
 * -------------------------------------------------------------------------------------*/
template <class G, typename TY, typename TC>
__device__ __forceinline__ double hpsi_const(const TY *yu, const TY *yv, typename cplx<TC>::t *BU,
                                             typename cplx<TC>::t *BV, const typename cplx<TC>::t *tw,
                                             const double (*kt)[WTD_KT], const double *cf, double kp2, double *red)
{
    typedef typename cplx<TC>::t C;
    constexpr int N = G::ntot;
    const uint64_t pol = l2_policy_keep();
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        double2 u = to_d(yu[p]), v = to_d(yv[p]);
        int o = G::off(p);
        BU[o].x = (TC)u.x; BU[o].y = (TC)u.y;
        BV[o].x = (TC)v.x; BV[o].y = (TC)v.y;
    }
    __syncthreads();
    fft_forward<G, 2>(BU, (int)(BV - BU), tw);
    kmul<G, OP_LAP>(BU, kt);
    kmul<G, OP_LAP>(BV, kt);
    __syncthreads();
    fft_inverse<G, 2>(BU, (int)(BV - BU), tw);
    double q = 0.0;
#pragma unroll 2
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        int o = G::off(p);
        TC ur, ui, vr, vi;
        {
            double2 u = to_d(yu[p]), v = to_d(yv[p]);
            ur = (TC)u.x; ui = (TC)u.y; vr = (TC)v.x; vi = (TC)v.y;
        }
        const TC va = (TC)ld_ro_keep(cf + CF_VA * N + p, pol), vb = (TC)ld_ro_keep(cf + CF_VB * N + p, pol);
        const TC dr = (TC)ld_ro_keep(cf + CF_DRE * N + p, pol), di = (TC)ld_ro_keep(cf + CF_DIM * N + p, pol);
        const TC aa = (TC)ld_ro_keep(cf + CF_AA * N + p, pol), ab = (TC)ld_ro_keep(cf + CF_AB * N + p, pol);
        const TC ja = -aa * (TC)kp2, jb = -ab * (TC)kp2;
        C lu = BU[o], lv = BV[o];
        /* u' = (Va-mu_a+ja) u + D v + aa lap u ;  v' = -(Vb-mu_b+jb) v + D* u - ab lap v */
        C hu, hv;
        hu.x = (va + ja) * ur + (dr * vr - di * vi) + aa * lu.x;
        hu.y = (va + ja) * ui + (dr * vi + di * vr) + aa * lu.y;
        hv.x = -(vb + jb) * vr + (dr * ur + di * ui) - ab * lv.x;
        hv.y = -(vb + jb) * vi + (dr * ui - di * ur) - ab * lv.y;
        BU[o] = hu; BV[o] = hv;
        q += (double)ur * (double)hu.x + (double)ui * (double)hu.y + (double)vr * (double)hv.x + (double)vi * (double)hv.y;
    }
    return block_sum(q, red) * WTD_DV;
}

/* ---------------------------------------------------------------------------------------
 * H psi for one state, variable effective mass with current corrections (ASLDA / CUSTOMEDF
 * without SLDA_FORCE_A1).  pca_kernels.cu:233-391:
 *   u' = (Va-mu_a+ja, cja) u + D v + (1/4)lap(alpha_a) u + sum_d (-i A_a,d) d_d u
 *        - (1/4) alpha_a lap u - (1/4) lap(alpha_a u)
 *   v' = -(Vb-mu_b+jb, -cjb) v + D* u - (1/4)lap(alpha_b) v - sum_d (+i A_b,d) d_d v
 *        + (1/4) alpha_b lap v + (1/4) lap(alpha_b v)
 * Buffers: B0 (transform of one component), W (work), HU, HV (results).
 * -------------------------------------------------------------------------------------*/
template <class G, typename TY, typename TC>
__device__ __forceinline__ double hpsi_var(const TY *yu, const TY *yv, typename cplx<TC>::t *B0,
                                           typename cplx<TC>::t *W, typename cplx<TC>::t *HU,
                                           typename cplx<TC>::t *HV, const typename cplx<TC>::t *tw,
                                           const double (*kt)[WTD_KT], const double *cf, double kp2, double *red)
{
    typedef typename cplx<TC>::t C;
    constexpr int N = G::ntot;
    /* local terms into HU/HV */
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        int o = G::off(p);
        double2 u = to_d(yu[p]), v = to_d(yv[p]);
        double va = cf[CF_VA * N + p], vb = cf[CF_VB * N + p];
        double dr = cf[CF_DRE * N + p], di = cf[CF_DIM * N + p];
        double aa = cf[CF_AA * N + p], ab = cf[CF_AB * N + p];
        double na = cf[CF_NA * N + p], nb = cf[CF_NB * N + p];
        double cja = cf[CF_CJA * N + p], cjb = cf[CF_CJB * N + p];
        double ja = -2.0 * aa * kp2, jb = -2.0 * ab * kp2;
        double2 hu, hv;
        /* (va+ja + i cja) u + D v + na u */
        hu.x = (va + ja) * u.x - cja * u.y + (dr * v.x - di * v.y) + na * u.x;
        hu.y = (va + ja) * u.y + cja * u.x + (dr * v.y + di * v.x) + na * u.y;
        /* -(vb+jb - i cjb) v + D* u - nb v */
        hv.x = -((vb + jb) * v.x + cjb * v.y) + (dr * u.x + di * u.y) - nb * v.x;
        hv.y = -((vb + jb) * v.y - cjb * v.x) + (dr * u.y - di * u.x) - nb * v.y;
        HU[o].x = (TC)hu.x; HU[o].y = (TC)hu.y;
        HV[o].x = (TC)hv.x; HV[o].y = (TC)hv.y;
    }
    for (int comp = 0; comp < 2; comp++) {
        const TY *y = comp == 0 ? yu : yv;
        C *H = comp == 0 ? HU : HV;
        const TC sgn = comp == 0 ? (TC)1 : (TC)-1;
        __syncthreads();
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            double2 a = to_d(y[p]);
            C c; c.x = (TC)a.x; c.y = (TC)a.y;
            B0[G::off(p)] = c;
        }
        __syncthreads();
        fft_forward<G, 1>(B0, 0, tw);
        /* laplacian term: sgn * aa * lap */
        for (int op = 0; op <= G::dims; op++) {
            for (int i = threadIdx.x; i < G::padded; i += blockDim.x) W[i] = B0[i];
            __syncthreads();
            if (op == 0) kmul<G, OP_LAP>(W, kt);
            else if (op == 1) kmul<G, OP_DX>(W, kt);
            else if (op == 2) kmul<G, OP_DY>(W, kt);
            else kmul<G, OP_DZ>(W, kt);
            __syncthreads();
            fft_inverse<G, 1>(W, 0, tw);
            for (int p = threadIdx.x; p < N; p += blockDim.x) {
                int o = G::off(p);
                C w = W[o], h = H[o];
                if (op == 0) {
                    TC a = (TC)cf[(comp == 0 ? CF_AA : CF_AB) * N + p];
                    h.x += sgn * a * w.x; h.y += sgn * a * w.y;
                } else {
                    /* u: + (-i A_a) du ; v: - (+i A_b) dv, i.e. the same form (-i A) d for both */
                    TC A = (TC)cf[((comp == 0 ? CF_AAX : CF_ABX) + op - 1) * N + p];
                    h.x += A * w.y;
                    h.y += -A * w.x;
                }
                H[o] = h;
            }
            /* every thread has read W (by point) before the next operator overwrites it (by
             * padded index, another thread's points) */
            __syncthreads();
        }
        /* - (1/4) lap(alpha psi) with the spin's sign */
        __syncthreads();
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            double2 a = to_d(y[p]);
            TC al = (TC)cf[(comp == 0 ? CF_ALA : CF_ALB) * N + p];
            C c; c.x = (TC)a.x * al; c.y = (TC)a.y * al;
            W[G::off(p)] = c;
        }
        __syncthreads();
        fft_forward<G, 1>(W, 0, tw);
        kmul<G, OP_LAP>(W, kt);
        __syncthreads();
        fft_inverse<G, 1>(W, 0, tw);
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            int o = G::off(p);
            C w = W[o], h = H[o];
            h.x += sgn * (TC)(-0.25) * w.x; h.y += sgn * (TC)(-0.25) * w.y;
            H[o] = h;
        }
    }
    __syncthreads();
    double q = 0.0;
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        int o = G::off(p);
        double2 u = to_d(yu[p]), v = to_d(yv[p]);
        C hu = HU[o], hv = HV[o];
        q += u.x * (double)hu.x + u.y * (double)hu.y + v.x * (double)hv.x + v.y * (double)hv.y;
    }
    return block_sum(q, red) * WTD_DV;
}

/* ---------------------------------------------------------------------------------------
 * density contribution of one normalised state (pca_dens.cu:13-198, cpca_dens.cu:14-140,
 * ccpca_dens.cu:14-140).  Limited form: rho_a, rho_b, nu.  The slot has the reference's
 * 12-block layout [nu re/im interleaved, rho_a, tau_a, j_a xyz, rho_b, tau_b, j_b xyz].
 * -------------------------------------------------------------------------------------*/
__device__ __forceinline__ void dens_limited(double *ds, int p, int N, double2 u, double2 v, double f, double w, uint64_t pol)
{
    double fa = f * w, fb = (1.0 - f) * w, fn = (1.0 - 2.0 * f) * 0.5 * w;
    double *a0 = ds + 2 * p, *a1 = ds + 2 * p + 1, *a2 = ds + 2 * (size_t)N + p, *a3 = ds + 7 * (size_t)N + p;
    double s0 = ld_keep(a0, pol), s1 = ld_keep(a1, pol), s2 = ld_keep(a2, pol), s3 = ld_keep(a3, pol);
    st_keep(a0, s0 + (u.x * v.x + u.y * v.y) * fn, pol);
    st_keep(a1, s1 + (u.y * v.x - u.x * v.y) * fn, pol);
    st_keep(a2, s2 + (u.x * u.x + u.y * u.y) * fa, pol);
    st_keep(a3, s3 + (v.x * v.x + v.y * v.y) * fb, pol);
}

/* the same as reductions performed in L2 (red_keep): the thread does not wait for the slot's
 * old values; every word of the slot must be updated by this one thread only */
__device__ __forceinline__ void dens_limited_red(double *ds, int p, int N, double2 u, double2 v, double f, double w,
                                                 uint64_t pol)
{
    double fa = f * w, fb = (1.0 - f) * w, fn = (1.0 - 2.0 * f) * 0.5 * w;
    red_keep(ds + 2 * p, (u.x * v.x + u.y * v.y) * fn, pol);
    red_keep(ds + 2 * p + 1, (u.y * v.x - u.x * v.y) * fn, pol);
    red_keep(ds + 2 * (size_t)N + p, (u.x * u.x + u.y * u.y) * fa, pol);
    red_keep(ds + 7 * (size_t)N + p, (v.x * v.x + v.y * v.y) * fb, pol);
}

/* tau and j contributions of one normalised component (pca_dens.cu:41-108).  B0 holds the
 * component in natural order and is transformed in place; W is work; ysrc gives the stored
 * normalised values.  tau_tmp_s += f_s Re(conj(psi)(lap psi - |k_perp|^2 psi)),
 * j_s,d += (+1 for u, -1 for v) f_s Im(conj(psi) d_d psi). */
template <class G, typename TY, typename TC>
__device__ __forceinline__ void dens_gradients(double *ds, const TY *ysrc, typename cplx<TC>::t *B0,
                                               typename cplx<TC>::t *W, const typename cplx<TC>::t *tw,
                                               const double (*kt)[WTD_KT], double f, double w, double kp2, int comp,
                                               const TY *yother = nullptr)
{
    typedef typename cplx<TC>::t C;
    constexpr int N = G::ntot;
    const double fw = (comp == 0 ? f : (1.0 - f)) * w;
    /* quantum-friction densities when yother (the other component) is given, after the 12 N
     * density words (pca_dens.cu:365-461): U_a += f Im[u* lap u], U_b -= (1-f) Im[v* lap v],
     * D += -1/2 (1-2f) [v* lap u + (lap v)* u], lap including -|k_perp|^2 */
    const double fq = (1.0 - 2.0 * f) * w * -0.5;
    const int tau_q = comp == 0 ? 3 : 8, j_q = comp == 0 ? 4 : 9;
    const double jsgn = comp == 0 ? 1.0 : -1.0;
    /* slot updates as L2 reductions: each word of the CTA's slot is updated by one thread only */
    const uint64_t pol = l2_policy_keep();
    __syncthreads();
    fft_forward<G, 1>(B0, 0, tw);
    for (int op = 0; op <= G::dims; op++) {
        for (int i = threadIdx.x; i < G::padded; i += blockDim.x) W[i] = B0[i];
        __syncthreads();
        if (op == 0) kmul<G, OP_LAP>(W, kt);
        else if (op == 1) kmul<G, OP_DX>(W, kt);
        else if (op == 2) kmul<G, OP_DY>(W, kt);
        else kmul<G, OP_DZ>(W, kt);
        __syncthreads();
        fft_inverse<G, 1>(W, 0, tw);
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            double2 sv = to_d(ysrc[p]);
            C d = W[G::off(p)];
            double dx = d.x, dy = d.y;
            if (op == 0) {
                double lx = dx - sv.x * kp2, ly = dy - sv.y * kp2;
                red_keep(ds + tau_q * (size_t)N + p, (sv.x * lx + sv.y * ly) * fw, pol);
                if (yother) {
                    const double2 o = to_d(yother[p]);
                    const double im = sv.x * ly - sv.y * lx; /* Im[psi* lap psi] */
                    if (comp == 0) {
                        red_keep(ds + 12 * (size_t)N + p, im * fw, pol);
                        /* v* lap u */
                        red_keep(ds + 14 * (size_t)N + 2 * p, (o.x * lx + o.y * ly) * fq, pol);
                        red_keep(ds + 14 * (size_t)N + 2 * p + 1, (o.x * ly - o.y * lx) * fq, pol);
                    } else {
                        red_keep(ds + 13 * (size_t)N + p, -(im * fw), pol);
                        /* (lap v)* u */
                        red_keep(ds + 14 * (size_t)N + 2 * p, (lx * o.x + ly * o.y) * fq, pol);
                        red_keep(ds + 14 * (size_t)N + 2 * p + 1, (lx * o.y - ly * o.x) * fq, pol);
                    }
                }
            } else {
                red_keep(ds + (j_q + op - 1) * (size_t)N + p, jsgn * (sv.x * dy - sv.y * dx) * fw, pol);
            }
        }
        __syncthreads();
    }
}

/* ---------------------------------------------------------------------------------------
 * the fused pass kernel
 *   PASS 0 (A): f_k = (H - <H>) y (or read), predictor, P, renormalise, densities of y_pred
 *   PASS 1 (B): f = (H - <H>) y_pred, y = P - i dt c f, renormalise, densities
 *   PASS 2    : renormalise and densities only (initial measurement, pca.c:939-958)
 *   PASS 3    : f = (H - <H>) y into ring slot NH-1 only — the reference's end-of-step
 *               apply_hamiltonian into f1 (pca.c:1565), formed on demand
 * VAR: variable effective mass; GRAD: tau and j of the output state too.
 * -------------------------------------------------------------------------------------*/
template <class G, typename TY, typename TH, typename TC, int NH, int PASS, bool VAR, bool GRAD, int BS>
__global__ void __launch_bounds__(BS, (sizeof(TC) == 4 && BS == 512) ? 2 : 1) /* FP32 compute: 2 CTAs/SM */
wtd_fused_pass(StepArgs a, const double2 *gtw, const double *gk)
{
    typedef typename cplx<TC>::t C;
    constexpr int N = G::ntot;
    constexpr int NBUF = VAR ? 4 : (GRAD ? 3 : 2);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *BU = (C *)smem_raw;
    C *BV = BU + G::padded;
    C *B2 = BV + G::padded;
    C *B3 = B2 + G::padded;
    C *tw = BU + NBUF * G::padded;
    double (*kt)[WTD_KT] = (double (*)[WTD_KT])(tw + G::twtotal);
    double *red = (double *)(kt + 6);

    load_tables<G>(tw, kt, gtw, gk);

    TY *Y = (TY *)a.y;
    TY *YO = a.yout ? (TY *)a.yout : Y;
    const uint64_t pol = l2_policy_keep();
    double *ds = a.dslot + (size_t)blockIdx.x * a.sstride;
    if (!a.accumulate)
        for (int i = threadIdx.x; i < a.sstride; i += blockDim.x) ds[i] = 0.0;
    const double dt = a.dt;
    const size_t SN = (size_t)a.S * N;

    constexpr int NR = (PASS == 0) ? NH - 1 : (PASS == 1 ? 1 : 0); /* history arrays read per element */
    for (int n = blockIdx.x; n < a.S; n += gridDim.x) {
        TY *yu = Y + (size_t)n * N, *yv = Y + SN + (size_t)n * N;
        TY *ou = YO + (size_t)n * N, *ov = YO + SN + (size_t)n * N;
        const double kp2 = a.kp2[n];
        const bool haveH = (PASS == 1) || (PASS == 3) || (PASS == 0 && !a.fk_given);
        /* bulk L2 prefetch: this state's ABM inputs (used after the FFT phase) and the next
         * state's y (used by the next iteration), so HBM streams while the SM computes */
        if (threadIdx.x == 0) {
            const size_t hb = (size_t)N * sizeof(TH), yb = (size_t)N * sizeof(TY);
            const int nh = (a.prefetch >> 1) & 7;
            if (nh == 0) {
            } else if (PASS == 0) {
                for (int j = 0; j < NH - 1 && j < nh; j++) {
                    prefetch_l2((const TH *)a.slot[j] + (size_t)n * N, hb);
                    prefetch_l2((const TH *)a.slot[j] + SN + (size_t)n * N, hb);
                }
                if (!haveH && nh >= NH) {
                    prefetch_l2((const TH *)a.slot[NH - 1] + (size_t)n * N, hb);
                    prefetch_l2((const TH *)a.slot[NH - 1] + SN + (size_t)n * N, hb);
                }
            } else if (PASS == 1) {
                prefetch_l2((const TH *)a.slot[NH - 2] + (size_t)n * N, hb);
                prefetch_l2((const TH *)a.slot[NH - 2] + SN + (size_t)n * N, hb);
            }
            const int nn = n + gridDim.x;
            if ((a.prefetch & 1) && nn < a.S) {
                prefetch_l2(Y + (size_t)nn * N, yb);
                prefetch_l2(Y + SN + (size_t)nn * N, yb);
            }
        }
        /* results of H land in (HU, HV) */
        C *HU = VAR ? B2 : BU, *HV = VAR ? B3 : BV;
        double E = 0.0;
        if (haveH) {
            if (VAR) E = hpsi_var<G, TY, TC>(yu, yv, BU, BV, HU, HV, tw, kt, a.cf, kp2, red);
            else E = hpsi_const<G, TY, TC>(yu, yv, BU, BV, tw, kt, a.cf, kp2, red);
            if (threadIdx.x == 0) a.qpe[n] = E;
        }
        if (PASS == 3) {
            for (int p = threadIdx.x; p < N; p += blockDim.x) {
                const int o = G::off(p);
#pragma unroll
                for (int comp = 0; comp < 2; comp++) {
                    const size_t gi = (comp ? SN : 0) + (size_t)n * N + p;
                    double2 y0 = to_d(Y[gi]);
                    C h = comp ? HV[o] : HU[o];
                    ((TH *)a.slot[NH - 1])[gi] = from_d<TH>(make_double2((double)h.x - E * y0.x, (double)h.y - E * y0.y));
                }
            }
            __syncthreads();
            continue;
        }
        /* ---- ABM update, unnormalised result into (HU, HV) ---- */
        const TH *__restrict__ hs[NH];
#pragma unroll
        for (int j = 0; j < NH; j++) hs[j] = (const TH *)a.slot[j];
        TH *__restrict__ fk_out = (TH *)a.slot[NH - 1];
        TH *__restrict__ p_out = (TH *)a.slot[NH - 2];
        double nrm = 0.0;
#pragma unroll 2
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            const int o = G::off(p);
            /* all global loads of this point first (both components), then arithmetic */
            double2 y0[2], fr[2][NR > 0 ? NR : 1], fkg[2];
#pragma unroll
            for (int comp = 0; comp < 2; comp++) {
                const size_t gi = (comp ? SN : 0) + (size_t)n * N + p;
                y0[comp] = to_d(Y[gi]);
                if (PASS == 0) {
#pragma unroll
                    for (int j = 0; j < NR; j++) fr[comp][j] = to_d(ld_stream(hs[j] + gi));
                    if (!haveH) fkg[comp] = to_d(ld_stream(hs[NH - 1] + gi));
                } else if (PASS == 1) {
                    fr[comp][0] = to_d(ld_stream(hs[NH - 2] + gi));
                }
            }
#pragma unroll
            for (int comp = 0; comp < 2; comp++) {
                const size_t gi = (comp ? SN : 0) + (size_t)n * N + p;
                double2 fk = make_double2(0.0, 0.0);
                if (PASS != 2) {
                    if (haveH) {
                        C h = comp ? HV[o] : HU[o];
                        fk.x = (double)h.x - E * y0[comp].x;
                        fk.y = (double)h.y - E * y0[comp].y;
                    } else {
                        fk = fkg[comp];
                    }
                }
                double2 out;
                if (PASS == 2) {
                    out = y0[comp];   /* initial measurement: normalise only (pca.c:941) */
                } else if (PASS == 0) {
                    typedef Abm<NH> A;
                    /* sums in the reference's order: f_k*b0 - f_{k-1}*|b1| + ... */
                    double2 sb = make_double2(fk.x * A::b(0), fk.y * A::b(0));
                    double2 sa = make_double2(fk.x * A::a(0), fk.y * A::a(0));
#pragma unroll
                    for (int j = 1; j < NH; j++) {
                        const double2 fj = fr[comp][j - 1];
                        sb.x += fj.x * A::b(j); sb.y += fj.y * A::b(j);
                        if (j < A::na) { sa.x += fj.x * A::a(j); sa.y += fj.y * A::a(j); }
                    }
                    /* y_pred = y + (-i dt) sb ; P = y + (-i dt) sa */
                    out.x = y0[comp].x + dt * sb.y; out.y = y0[comp].y - dt * sb.x;
                    double2 P = make_double2(y0[comp].x + dt * sa.y, y0[comp].y - dt * sa.x);
                    if (haveH) st_stream(fk_out + gi, from_d<TH>(fk));
                    st_stream(p_out + gi, from_d<TH>(P));
                } else {
                    /* y = (-i dt) f c + P */
                    const double2 P = fr[comp][0];
                    const double c = Abm<NH>::c;
                    out.x = dt * fk.y * c + P.x;
                    out.y = -dt * fk.x * c + P.y;
                }
                nrm += out.x * out.x + out.y * out.y;
                C r; r.x = (TC)out.x; r.y = (TC)out.y;
                if (comp) HV[o] = r; else HU[o] = r;
            }
        }
        const double nrm_tot = sqrt(block_sum(nrm, red) * WTD_DV);
        const double c = 1.0 / nrm_tot;
        if (a.nrm_out && threadIdx.x == 0) a.nrm_out[n] = nrm_tot;
        /* ---- normalise, store, densities ---- */
        const double f = a.occ[n], w = a.wcnt[n];
        for (int p = threadIdx.x; p < N; p += 2 * blockDim.x) {
            /* two points per iteration (p, q = p + blockDim.x) so that their density-slot
             * updates share one L2 round trip */
            const int q = p + blockDim.x;
            const bool hq = q < N;
            double2 uu[2], vv[2];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                if (k == 1 && !hq) { uu[1] = vv[1] = make_double2(0.0, 0.0); break; }
                const int pp = k ? q : p, o = G::off(pp);
                C hu = HU[o], hv = HV[o];
                double2 u = make_double2((double)hu.x * c, (double)hu.y * c);
                double2 v = make_double2((double)hv.x * c, (double)hv.y * c);
                TY su = from_d<TY>(u), sv = from_d<TY>(v);
                st_stream(ou + pp, su); st_stream(ov + pp, sv);
                u = to_d(su); v = to_d(sv);
                uu[k] = u; vv[k] = v;
                if (GRAD) {
                    C cu, cv;
                    cu.x = (TC)u.x; cu.y = (TC)u.y; cv.x = (TC)v.x; cv.y = (TC)v.y;
                    HU[o] = cu; HV[o] = cv;
                }
            }
            dens_limited_red(ds, p, N, uu[0], vv[0], f, w, pol);
            if (hq) dens_limited_red(ds, q, N, uu[1], vv[1], f, w, pol);
        }
        if (GRAD) {
            /* const mass: (HU, HV) = (BU, BV) hold the state, B2 is work.
             * variable mass: (HU, HV) = (B2, B3), BU is work. */
            C *Wk = VAR ? BU : B2;
            dens_gradients<G, TY, TC>(ds, ou, HU, Wk, tw, kt, f, w, kp2, 0, a.qf ? ov : nullptr);
            dens_gradients<G, TY, TC>(ds, ov, HV, Wk, tw, kt, f, w, kp2, 1, a.qf ? ou : nullptr);
        }
        __syncthreads();
    }
}

#endif
