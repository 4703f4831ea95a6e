/*
 * The reference's per-kernel C ABI (include/wslda_td_compat.h) on this library's kernels.
 *
 * These entry points keep the reference's buffer-per-stage contract: the caller owns every
 * state, derivative and density array and chains the calls as hpc-engine/pca.c:1401-1571
 * does.  Each call runs on the legacy default stream and returns after completion.  The
 * transforms are the shared-memory FFTs of wtd_core.cuh (one CTA per field), so no cuFFT plan
 * or cuFFT work area exists; create_cufftPlans only sizes the work area the library needs.
 *
 * Work-area layout (bytes from create_cufftPlans, pointer from set_workspace_for_cufftPlan):
 *   [0, S)            quasiparticle energies of the last apply_hamiltonian (pca.c:1575 reads them)
 *   [S', S'+18N)      per-point H coefficients (the CF_* list)
 *   [.., +G*12N)      density partial sums of the G CTAs of calculate_densities
 *   [.., +2S')        per-state |k_perp|^2 and degeneracy weights of the plane-wave factor
 * so calculate_densities and apply_hamiltonian allocate nothing once the work area is set.
 */
#ifndef WTD_COMPAT_CUH
#define WTD_COMPAT_CUH

#include "wslda_td_compat.h"

static void *g_work = NULL;          /* set_workspace_for_cufftPlan */
static int g_nwfip = 0;               /* create_cufftPlans */
static int g_dens_grid = 0;

static size_t compat_spad(void) { return ((size_t)(g_nwfip > 0 ? g_nwfip : 1) + 31) / 32 * 32; }
static double *compat_qpe(void) { return (double *)g_work; }
static double *compat_cf(void) { return (double *)g_work + compat_spad(); }
static double *compat_slots(void) { return (double *)g_work + compat_spad() + (size_t)CF_COUNT * WTD_NUMEL; }
static double *compat_kpw(void) { return compat_slots() + (size_t)g_dens_grid * 12 * WTD_NUMEL; }
static size_t compat_work_words(void)
{
    return compat_spad() + (size_t)CF_COUNT * WTD_NUMEL + (size_t)g_dens_grid * 12 * WTD_NUMEL + 2 * compat_spad();
}

static int cu_sync_status(void)
{
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}

/* ---------------------------------------------------------------------------------------
 * kernels of the compatibility layer
 * -------------------------------------------------------------------------------------*/
/* tdwslda_ode_integrator.h:26-97 */
template <int NH>
__global__ void k_abm_step1(size_t M, double2 *y, double2 *f1, double2 *f2, double2 *f3, double2 *f4, double2 *f5, double dt)
{
    size_t i = threadIdx.x + (size_t)blockIdx.x * blockDim.x;
    if (i >= M) return;
    typedef Abm<NH> A;
    double2 y0 = y[i];
    double2 f[5];
    f[0] = f1[i]; f[1] = f2[i]; f[2] = f3[i];
    if (NH >= 4) f[3] = f4[i];
    if (NH >= 5) f[4] = f5[i];
    double2 sb = make_double2(f[0].x * A::b(0), f[0].y * A::b(0));
    double2 sa = make_double2(f[0].x * A::a(0), f[0].y * A::a(0));
#pragma unroll
    for (int j = 1; j < NH; j++) {
        sb.x += f[j].x * A::b(j); sb.y += f[j].y * A::b(j);
        if (j < A::na) { sa.x += f[j].x * A::a(j); sa.y += f[j].y * A::a(j); }
    }
    y[i] = make_double2(y0.x + dt * sb.y, y0.y - dt * sb.x);
    double2 P = make_double2(y0.x + dt * sa.y, y0.y - dt * sa.x);
    if (NH == 3) f3[i] = P; else if (NH == 4) f4[i] = P; else f5[i] = P;
}

/* tdwslda_ode_integrator.h:138-193 */
__global__ void k_abm_step4(size_t M, const double2 *hy, double2 *yout, const double2 *flast, double dt, double c)
{
    size_t i = threadIdx.x + (size_t)blockIdx.x * blockDim.x;
    if (i >= M) return;
    double2 h = hy[i], P = flast[i];
    yout[i] = make_double2(dt * h.y * c + P.x, -dt * h.x * c + P.y);
}

/* pca_kernels.cu:913-976: one CTA per state */
__global__ void k_normalize(int n, double2 *wf)
{
    __shared__ double red[80];
    constexpr int N = WTD_NUMEL;
    double2 *u = wf + (size_t)blockIdx.x * N, *v = wf + (size_t)n * N + (size_t)blockIdx.x * N;
    double s = 0.0;
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        double2 a = u[p], b = v[p];
        s += a.x * a.x + a.y * a.y + b.x * b.x + b.y * b.y;
    }
    double c = 1.0 / sqrt(block_sum(s, red) * WTD_DV);
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        double2 a = u[p], b = v[p];
        u[p] = make_double2(a.x * c, a.y * c);
        v[p] = make_double2(b.x * c, b.y * c);
    }
}

/* spectral derivatives of one field per CTA (pca_derivative.cu:139-380); any output may be
 * null and any output may alias the input (the field is read into shared memory first) */
template <class G>
__global__ void __launch_bounds__(512) k_derivs(const double2 *in, double2 *odx, double2 *ody, double2 *odz, double2 *olap,
                                                const double2 *gtw, const double *gk)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *B0 = (double2 *)smem_raw;
    double2 *W = B0 + G::padded;
    double2 *tw = W + G::padded;
    double (*kt)[WTD_KT] = (double (*)[WTD_KT])(tw + G::twtotal);
    load_tables<G>(tw, kt, gtw, gk);
    constexpr int N = G::ntot;
    const size_t base = (size_t)blockIdx.x * N;
    for (int p = threadIdx.x; p < N; p += blockDim.x) B0[G::off(p)] = in[base + p];
    __syncthreads();
    fft_forward<G, 1>(B0, 0, tw);
    double2 *outs[4] = {olap, odx, ody, odz};
    for (int op = 0; op < 4; op++) {
        double2 *o = outs[op];
        if (!o || (op == 2 && G::dims < 2) || (op == 3 && G::dims < 3)) continue;
        for (int i = threadIdx.x; i < G::padded; i += blockDim.x) W[i] = B0[i];
        __syncthreads();
        if (op == 0) kmul<G, OP_LAP>(W, kt);
        else if (op == 1) kmul<G, OP_DX>(W, kt);
        else if (op == 2) kmul<G, OP_DY>(W, kt);
        else kmul<G, OP_DZ>(W, kt);
        __syncthreads();
        fft_inverse<G, 1>(W, 0, tw);
        for (int p = threadIdx.x; p < N; p += blockDim.x) o[base + p] = W[G::off(p)];
        __syncthreads();
    }
}

/* real-field derivatives: 'which' selects lap (0) or d/dx_d (1..3), one CTA */
template <class G>
__global__ void __launch_bounds__(512) k_real_deriv(const double *f, double *out, int which, const double2 *gtw, const double *gk)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *B = (double2 *)smem_raw;
    double2 *tw = B + G::padded;
    double (*kt)[WTD_KT] = (double (*)[WTD_KT])(tw + G::twtotal);
    load_tables<G>(tw, kt, gtw, gk);
    constexpr int N = G::ntot;
    for (int p = threadIdx.x; p < N; p += blockDim.x) B[G::off(p)] = make_double2(f[p], 0.0);
    __syncthreads();
    fft_forward<G, 1>(B, 0, tw);
    if (which == 0) kmul<G, OP_LAP>(B, kt);
    else if (which == 1) kmul<G, OP_DX>(B, kt);
    else if (which == 2) kmul<G, OP_DY>(B, kt);
    else kmul<G, OP_DZ>(B, kt);
    __syncthreads();
    fft_inverse<G, 1>(B, 0, tw);
    for (int p = threadIdx.x; p < N; p += blockDim.x) out[p] = B[G::off(p)].x;
}

/* calculate_densities: CTA b accumulates the states b, b+G, ... into its slot
 * (pca_dens.cu:13-198; plane-wave weights of cpca_dens.cu:44-61, ccpca_dens.cu:41-76) */
__global__ void k_dens_compat(int n, const double2 *wf, const double2 *dx, const double2 *dy, const double2 *dz,
                              const double2 *lap, const double *fb, const double *wts, const double *kp2,
                              const double *wcnt, double *slots, int grads)
{
    constexpr int N = WTD_NUMEL;
    double *ds = slots + (size_t)blockIdx.x * 12 * N;
    const uint64_t pol = l2_policy_keep();
    for (int i = threadIdx.x; i < 12 * N; i += blockDim.x) ds[i] = 0.0;
    __syncthreads();
    const size_t SN = (size_t)n * N;
    for (int s = blockIdx.x; s < n; s += gridDim.x) {
        const double f = fb[s];
        const double w = (wts ? wts[s] : 1.0) * wcnt[s];
        const double k2 = kp2[s];
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            const size_t iu = (size_t)s * N + p, iv = SN + iu;
            double2 u = wf[iu], v = wf[iv];
            dens_limited(ds, p, N, u, v, f, w, pol);
            if (grads) {
                const double fa = f * w, fbm = (1.0 - f) * w;
                double2 lu = lap[iu], lv = lap[iv];
                ds[3 * (size_t)N + p] += (u.x * (lu.x - u.x * k2) + u.y * (lu.y - u.y * k2)) * fa;
                ds[8 * (size_t)N + p] += (v.x * (lv.x - v.x * k2) + v.y * (lv.y - v.y * k2)) * fbm;
                const double2 *dd[3] = {dx, dy, dz};
                for (int d = 0; d < CODEDIM; d++) {
                    double2 a = dd[d][iu], b = dd[d][iv];
                    ds[(4 + d) * (size_t)N + p] += (u.x * a.y - u.y * a.x) * fa;
                    ds[(9 + d) * (size_t)N + p] -= (v.x * b.y - v.y * b.x) * fbm;
                }
            }
        }
    }
}

/* the same densities parallel over points, for lattices whose 12 N-word slot per CTA does not
 * stay in L2 (3D 32^3: 3 MB per slot).  CTA (tile, chunk) sums the states of chunk
 * [n*chunk/nchunk, n*(chunk+1)/nchunk) at WTD_DP_T points in registers, in state order, and
 * writes the whole 12-block partial once into slot `chunk`; wtd_dens_reduce then sums the
 * chunks in order (bitwise reproducible for a given nchunk). */
#define WTD_DP_T 128
__global__ void __launch_bounds__(WTD_DP_T) k_dens_points(int n, int nchunk, const double2 *__restrict__ wf,
                                                          const double2 *__restrict__ dx, const double2 *__restrict__ dy,
                                                          const double2 *__restrict__ dz, const double2 *__restrict__ lap,
                                                          const double *__restrict__ fb, const double *__restrict__ kp2,
                                                          const double *__restrict__ wcnt, double *slots, int grads)
{
    constexpr int N = WTD_NUMEL;
    const int p = blockIdx.x * WTD_DP_T + threadIdx.x;
    if (p >= N) return;
    const int chunk = blockIdx.y;
    const int s0 = (int)((long long)n * chunk / nchunk), s1 = (int)((long long)n * (chunk + 1) / nchunk);
    const size_t SN = (size_t)n * N;
    double nre = 0.0, nim = 0.0, ra = 0.0, rb = 0.0, ta = 0.0, tb = 0.0;
    double ja[3] = {0.0, 0.0, 0.0}, jb[3] = {0.0, 0.0, 0.0};
    const double2 *dd[3] = {dx, dy, dz};
#pragma unroll 2
    for (int s = s0; s < s1; s++) {
        const double f = fb[s], w = wcnt[s], k2 = kp2[s];
        const double fa = f * w, fbm = (1.0 - f) * w, fn = (1.0 - 2.0 * f) * 0.5 * w;
        const size_t iu = (size_t)s * N + p, iv = SN + iu;
        const double2 u = wf[iu], v = wf[iv];
        nre += (u.x * v.x + u.y * v.y) * fn;
        nim += (u.y * v.x - u.x * v.y) * fn;
        ra += (u.x * u.x + u.y * u.y) * fa;
        rb += (v.x * v.x + v.y * v.y) * fbm;
        if (grads) {
            const double2 lu = lap[iu], lv = lap[iv];
            ta += (u.x * (lu.x - u.x * k2) + u.y * (lu.y - u.y * k2)) * fa;
            tb += (v.x * (lv.x - v.x * k2) + v.y * (lv.y - v.y * k2)) * fbm;
#pragma unroll
            for (int d = 0; d < CODEDIM; d++) {
                const double2 a = dd[d][iu], b = dd[d][iv];
                ja[d] += (u.x * a.y - u.y * a.x) * fa;
                jb[d] -= (v.x * b.y - v.y * b.x) * fbm;
            }
        }
    }
    double *ds = slots + (size_t)chunk * 12 * N;
    ds[2 * p] = nre;
    ds[2 * p + 1] = nim;
    ds[2 * (size_t)N + p] = ra;
    ds[3 * (size_t)N + p] = ta;
    ds[7 * (size_t)N + p] = rb;
    ds[8 * (size_t)N + p] = tb;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        ds[(4 + d) * (size_t)N + p] = ja[d];
        ds[(9 + d) * (size_t)N + p] = jb[d];
    }
}

/* apply_hamiltonian from caller-provided derivative arrays (pca_kernels.cu:233-495, 806-833):
 * one CTA per state; out may alias lap (each element is read before it is written) */
__global__ void k_hamiltonian_compat(int n, const double2 *in, double2 *out, const double2 *dx, const double2 *dy,
                                     const double2 *dz, const double2 *lap, const double2 *alap, const double *cf,
                                     const double *kp2, double *qpe_out, const double *useqpe)
{
    __shared__ double red[80];
    constexpr int N = WTD_NUMEL;
    const int s = blockIdx.x;
    const size_t SN = (size_t)n * N;
    const double k2 = kp2[s];
    double q = 0.0;
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        const size_t iu = (size_t)s * N + p, iv = SN + iu;
        double2 u = in[iu], v = in[iv], lu = lap[iu], lv = lap[iv];
        double va = cf[CF_VA * N + p], vb = cf[CF_VB * N + p], dr = cf[CF_DRE * N + p], di = cf[CF_DIM * N + p];
        double aa = cf[CF_AA * N + p], ab = cf[CF_AB * N + p];
        double2 hu, hv;
#ifdef FAST_CONST_EFFECTIVE_MASS_MODE
        double ja = -aa * k2, jb = -ab * k2;
        hu.x = (va + ja) * u.x + (dr * v.x - di * v.y) + aa * lu.x;
        hu.y = (va + ja) * u.y + (dr * v.y + di * v.x) + aa * lu.y;
        hv.x = -(vb + jb) * v.x + (dr * u.x + di * u.y) - ab * lv.x;
        hv.y = -(vb + jb) * v.y + (dr * u.y - di * u.x) - ab * lv.y;
#else
        double na = cf[CF_NA * N + p], nb = cf[CF_NB * N + p], cja = cf[CF_CJA * N + p], cjb = cf[CF_CJB * N + p];
        double ja = -2.0 * aa * k2, jb = -2.0 * ab * k2;
        hu.x = (va + ja) * u.x - cja * u.y + (dr * v.x - di * v.y) + na * u.x;
        hu.y = (va + ja) * u.y + cja * u.x + (dr * v.y + di * v.x) + na * u.y;
        hv.x = -((vb + jb) * v.x + cjb * v.y) + (dr * u.x + di * u.y) - nb * v.x;
        hv.y = -((vb + jb) * v.y - cjb * v.x) + (dr * u.y - di * u.x) - nb * v.y;
        const double2 *dd[3] = {dx, dy, dz};
        for (int d = 0; d < CODEDIM; d++) {
            double Aa = cf[(CF_AAX + d) * N + p], Ab = cf[(CF_ABX + d) * N + p];
            double2 a = dd[d][iu], b = dd[d][iv];
            hu.x += Aa * a.y; hu.y += -Aa * a.x;
            hv.x += Ab * b.y; hv.y += -Ab * b.x;
        }
        hu.x += aa * lu.x; hu.y += aa * lu.y;
        hv.x -= ab * lv.x; hv.y -= ab * lv.y;
        double2 au = alap[iu], av = alap[iv];
        hu.x += -0.25 * au.x; hu.y += -0.25 * au.y;
        hv.x -= -0.25 * av.x; hv.y -= -0.25 * av.y;
#endif
        out[iu] = hu; out[iv] = hv;
        q += u.x * hu.x + u.y * hu.y + v.x * hv.x + v.y * hv.y;
    }
    double E = block_sum(q, red) * WTD_DV;
    if (useqpe) E = useqpe[s];
    else if (threadIdx.x == 0) qpe_out[s] = E;
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        const size_t iu = (size_t)s * N + p, iv = SN + iu;
        double2 u = in[iu], v = in[iv], hu = out[iu], hv = out[iv];
        out[iu] = make_double2(hu.x - u.x * E, hu.y - u.y * E);
        out[iv] = make_double2(hv.x - v.x * E, hv.y - v.y * E);
    }
}

/* multiply_wf_by_alpha (pca_kernels.cu:981-1005) */
__global__ void k_mul_alpha(int n, const double2 *in, double2 *out, const double *aa, const double *ab)
{
    constexpr int N = WTD_NUMEL;
    size_t i = threadIdx.x + (size_t)blockIdx.x * blockDim.x;
    if (i >= (size_t)2 * n * N) return;
    int p = (int)(i % N);
    double a = (i < (size_t)n * N) ? aa[p] : ab[p];
    double2 z = in[i];
    out[i] = make_double2(z.x * a, z.y * a);
}

/* taylor_expansion_contribution (pca_kernels.cu:1032-1062) */
__global__ void k_taylor(size_t M, const double2 *h, double2 *upd, double2 *contr, double t)
{
    size_t i = threadIdx.x + (size_t)blockIdx.x * blockDim.x;
    if (i >= M) return;
    double2 z = h[i];
    double2 c = make_double2(-t * z.y, t * z.x); /* z * (0, t) */
    contr[i] = c;
    double2 u = upd[i];
    upd[i] = make_double2(u.x + c.x, u.y + c.y);
}

/* n sums of length m into tmp (one CTA each) */
__global__ void k_sum_many(const double *in, int m, double *tmp)
{
    __shared__ double red[80];
    double s = 0.0;
    const double *a = in + (size_t)blockIdx.x * m;
    for (int i = threadIdx.x; i < m; i += blockDim.x) s += a[i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) tmp[blockIdx.x] = s;
}

/* <wf1_n|wf2_n> dV (pca_kernels.cu:853-907), one CTA per state */
__global__ void k_overlap(int n, const double2 *a, const double2 *b, double *re, double *im)
{
    __shared__ double red[80];
    constexpr int N = WTD_NUMEL;
    const size_t SN = (size_t)n * N;
    double sr = 0.0, si = 0.0;
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        const size_t iu = (size_t)blockIdx.x * N + p, iv = SN + iu;
        double2 x = a[iu], y = b[iu], z = a[iv], w = b[iv];
        sr += x.x * y.x + x.y * y.y + z.x * w.x + z.y * w.y;
        si += x.x * y.y - x.y * y.x + z.x * w.y - z.y * w.x;
    }
    double2 t = block_sum2(sr, si, red);
    if (threadIdx.x == 0) {
        if (re) re[blockIdx.x] = t.x * WTD_DV;
        if (im) im[blockIdx.x] = t.y * WTD_DV;
    }
}

/* calculate_quantum_friction_densities (pca_dens.cu:365-461; cpca_dens.cu:385-450; ccpca): one
 * thread per point, states in order; out = [U_a, U_b, D (complex)] */
__global__ void k_qf_dens_compat(int n, const double2 *wf, const double2 *lap, const double *fb, const double *wts,
                                 const double *kp2, const double *wcnt, double *out, double inv_lperp)
{
    constexpr int N = WTD_NUMEL;
    const int p = threadIdx.x + blockIdx.x * blockDim.x;
    if (p >= N) return;
    const size_t SN = (size_t)n * N;
    double ua = 0.0, ub = 0.0, dre = 0.0, dim = 0.0;
    for (int s = 0; s < n; s++) {
        double f = fb[s], fm = 1.0 - f;
        if (wts) { f *= wts[s]; fm *= wts[s]; }
        const double wc = wcnt[s], k2 = kp2[s];
        const size_t iu = (size_t)s * N + p, iv = SN + iu;
        const double2 u = wf[iu], v = wf[iv];
        const double2 lu = make_double2(lap[iu].x - u.x * k2, lap[iu].y - u.y * k2);
        const double2 lv = make_double2(lap[iv].x - v.x * k2, lap[iv].y - v.y * k2);
        ua += (u.x * lu.y - u.y * lu.x) * f * wc;
        ub -= (v.x * lv.y - v.y * lv.x) * fm * wc;
        /* v* lu + lv* u */
        dre += ((v.x * lu.x + v.y * lu.y) + (lv.x * u.x + lv.y * u.y)) * (fm - f) * wc;
        dim += ((v.x * lu.y - v.y * lu.x) + (lv.x * u.y - lv.y * u.x)) * (fm - f) * wc;
    }
#ifdef SPINSYMMETRY_MODE
    /* spin-symmetric system (pca_dens.cu:411-420): U_a = U_b = both sums, D counted twice */
    ua += ub; ub = ua; dre *= 2.0; dim *= 2.0;
#endif
    out[p] = ua * inv_lperp;
    out[N + p] = ub * inv_lperp;
    out[2 * (size_t)N + 2 * p] = -0.5 * dre * inv_lperp;
    out[2 * (size_t)N + 2 * p + 1] = -0.5 * dim * inv_lperp;
}

/* out += a (+ b) */
__global__ void k_add_fields(double *out, const double *a, const double *b, int n)
{
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i < n) out[i] += a[i] + (b ? b[i] : 0.0);
}

__global__ void k_get_vext(int it, int spin, double *out)
{
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= WTD_NUMEL) return;
    int ix, iy, iz; wtd_decode(i, ix, iy, iz);
    out[i] = WTD_U_EXT(ix, iy, iz, it, spin);
}
__global__ void k_get_dext(int it, const Complex *din, Complex *out)
{
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= WTD_NUMEL) return;
    int ix, iy, iz; wtd_decode(i, ix, iy, iz);
    out[i] = WTD_D_EXT(ix, iy, iz, it, din[i]);
}

/* the external velocity field, x, y, z blocks of N */
__global__ void k_get_velext(int it, int spin, double *out)
{
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= WTD_NUMEL) return;
    int ix, iy, iz; wtd_decode(i, ix, iy, iz);
    /* the user's hook, whether or not the field acts (pca_kernels.cu:1149-1160) */
    out[i] = velocity_ext(ix, iy, iz, it, spin, XAXIS, dc_params, dc_extra_data_size, dc_extra_data);
    out[WTD_NUMEL + i] = velocity_ext(ix, iy, iz, it, spin, YAXIS, dc_params, dc_extra_data_size, dc_extra_data);
    out[2 * WTD_NUMEL + i] = velocity_ext(ix, iy, iz, it, spin, ZAXIS, dc_params, dc_extra_data_size, dc_extra_data);
}

static __device__ double g_sum_tmp[1 << 16];   /* outputs of k_sum_many before they are moved */

/* the spectral tables every compatibility call uses (built once per process) */
static double2 *g_tw = NULL;
static double *g_ktab = NULL;
static int compat_tables(void)
{
    if (g_tw) return 0;
    double2 tw[WG::twtotal];
    double kt[6 * WTD_KT];
    wtd_make_tables(tw, kt);
    if (cudaMalloc((void **)&g_tw, sizeof(tw)) != cudaSuccess) return WTD_ERR_NOMEM;
    if (cudaMalloc((void **)&g_ktab, sizeof(kt)) != cudaSuccess) return WTD_ERR_NOMEM;
    cudaMemcpy(g_tw, tw, sizeof(tw), cudaMemcpyHostToDevice);
    cudaMemcpy(g_ktab, kt, sizeof(kt), cudaMemcpyHostToDevice);
    return 0;
}


static double2 *g_stage3d = NULL;
static int compat_stage(void)
{
    if (g_stage3d) return 0;
    return cudaMalloc((void **)&g_stage3d, 2 * sizeof(double2) * WTD_NUMEL) == cudaSuccess ? 0 : WTD_ERR_NOMEM;
}

static int compat_real_deriv(const double *f, double *out, int which)
{
    if (WTD_BIG) {
        WTD_TRY(compat_tables());
        WTD_TRY(compat_stage());
        WTD_TRY(big_real_deriv(f, out, which, 1.0, 0, g_stage3d, g_tw, g_ktab, 0));
        return cu_sync_status();
    }
    if (k_field_smem > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
    int r = compat_tables();
    if (r) return r;
    cudaFuncSetAttribute(k_real_deriv<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k_field_smem);
    k_real_deriv<WG><<<1, 512, k_field_smem>>>(f, out, which, g_tw, g_ktab);
    return cu_sync_status();
}

/* per-point coefficients from the potentials (+ lap alpha, div A for variable mass) */
static int compat_coefficients(int it, double *pots, const double *fld = NULL)
{
    wslda_potential P = convert_into_wslda_potential(pots, WTD_NUMEL, NULL);
    if (fld) { /* V_a, V_b, delta with the friction terms */
        P.V_a = (double *)fld;
        P.V_b = (double *)fld + WTD_NUMEL;
        P.delta = (Complex *)(fld + 2 * (size_t)WTD_NUMEL);
    }
    double *cf = compat_cf();
    wtd_prep_coef<<<(WTD_NUMEL + 127) / 128, 128>>>(it, P, cf);
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
    int r = compat_tables();
    if (r) return r;
    if (WTD_BIG) {
        WTD_TRY(compat_stage());
        WTD_TRY(big_prep_var(cf, g_stage3d, g_tw, g_ktab, 0));
    } else {
        if (k_field_smem > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
        cudaFuncSetAttribute(wtd_prep_var<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k_field_smem);
        wtd_prep_var<WG><<<2, 256, k_field_smem>>>(cf, g_tw, g_ktab);
    }
#endif
    return cu_sync_status();
}

/* per-state |k_perp|^2 and degeneracy weight from the reference's plane-wave arrays */
__global__ void k_planewave(int n, const double *kky, const double *kkz, const int *cnt, double *kp2, double *wcnt)
{
    int s = threadIdx.x + blockIdx.x * blockDim.x;
    if (s >= n) return;
    double ky = kky ? kky[s] : 0.0, kz = kkz ? kkz[s] : 0.0;
#if CODEDIM == 2
    kp2[s] = kz * kz;
    double w = (fabs(kz) < 1.0e-12) ? 1.0 : 2.0;
#ifdef USE_CUBIC_CUTOFF
    if (fabs(kz + M_PI / DZ) < 1.0e-12) w = 1.0;
#endif
    wcnt[s] = w;
#elif CODEDIM == 1
    kp2[s] = ky * ky + kz * kz;
    wcnt[s] = cnt ? (double)cnt[s] : 1.0;
#else
    kp2[s] = 0.0;
    wcnt[s] = 1.0;
#endif
}

/* the per-state plane-wave arrays of the current call: in the work area for the calls that
 * require it anyway (calculate_densities, apply_hamiltonian: in_work); otherwise
 * (calculate_quantum_friction_densities, which needs no work area) in a library-owned pair that
 * is allocated when it first has to grow */
static double *g_kp2 = NULL, *g_wcnt = NULL;
static double *g_kp2_own = NULL, *g_wcnt_own = NULL;
static int g_kp_own_n = 0;
static int compat_planewave(int n, const double *kky, const double *kkz, const int *cnt, bool in_work)
{
    if (in_work && g_work && n <= g_nwfip) {
        g_kp2 = compat_kpw();
        g_wcnt = g_kp2 + compat_spad();
    } else {
        if (g_kp_own_n < n) {
            if (g_kp2_own) cudaFree(g_kp2_own);
            if (g_wcnt_own) cudaFree(g_wcnt_own);
            g_kp2_own = g_wcnt_own = NULL;
            g_kp_own_n = 0;
            if (cudaMalloc((void **)&g_kp2_own, n * sizeof(double)) != cudaSuccess) return WTD_ERR_NOMEM;
            if (cudaMalloc((void **)&g_wcnt_own, n * sizeof(double)) != cudaSuccess) return WTD_ERR_NOMEM;
            g_kp_own_n = n;
        }
        g_kp2 = g_kp2_own;
        g_wcnt = g_wcnt_own;
    }
    k_planewave<<<(n + 127) / 128, 128>>>(n, kky, kkz, cnt, g_kp2, g_wcnt);
    return 0;
}

/* ---------------------------------------------------------------------------------------
 * calculate_densities without any allocation
 *
 * Some callers cannot call cudaMalloc: hosts whose device memory is owned by another
 * allocator (a pool reserved once at start-up, as the reference's driver sizes every device
 * buffer up front at pca.c:749-765 and treats any later allocation as fatal) and embedding
 * runtimes that forbid a library from allocating device memory on their behalf.  For them
 * calculate_densities_noalloc computes the same densities as calculate_densities without a
 * work area: the per-CTA FP64 partial sums live in the file-scope array below, which every
 * GPU that loads this library holds until the process exits.
 *
 * Limit: WTD_NOALLOC_BYTES (8 MiB) of scratch, i.e. lattices with 12*N doubles <= 1 Mi words
 * (N <= 87381 points); larger lattices are rejected with WTD_ERR_NOALLOC_SIZE before any
 * work is issued.  The number of CTAs is min(2 per SM, n, 8 MiB / (12*N*8)).
 * Every call shares the array and leaves its partial sums in it; each call clears the part it
 * uses first.  Calls that overlap on the GPU (other host threads, other streams) race on it.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress); make
 * it before any stream capture on that device.
 * -------------------------------------------------------------------------------------*/
#define WTD_NOALLOC_BYTES (8u << 20)
static __device__ __align__(256) double wtd_noalloc_scratch[WTD_NOALLOC_BYTES / sizeof(double)];
static double *g_noalloc_scratch[64];   /* device address of wtd_noalloc_scratch, per device */

/* the array's name is a host-side stand-in, not a device address: resolve it once per
 * device, with that device current, and pass the resolved pointer to the kernels */
static int noalloc_scratch(double **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return WTD_ERR_CUDA;
    if (dev < 0 || dev >= 64) return WTD_ERR_ARG;
    /* host threads may race on the first call; each stores the same address (atomic access
     * keeps every read whole) */
    double *p = __atomic_load_n(&g_noalloc_scratch[dev], __ATOMIC_ACQUIRE);
    if (!p) {
        if (cudaGetSymbolAddress((void **)&p, wtd_noalloc_scratch) != cudaSuccess || !p) return WTD_ERR_CUDA;
        __atomic_store_n(&g_noalloc_scratch[dev], p, __ATOMIC_RELEASE);
    }
    *out = p;
    return WTD_OK;
}

/* k_dens_compat with the per-state plane-wave weights formed in the kernel (so no per-state
 * arrays are needed) */
__global__ void k_dens_noalloc(int n, const double2 *wf, const double2 *dx, const double2 *dy, const double2 *dz,
                               const double2 *lap, const double *fb, const double *wts, const double *kky,
                               const double *kkz, const int *cnt, double *slots, int grads)
{
    constexpr int N = WTD_NUMEL;
    double *ds = slots + (size_t)blockIdx.x * 12 * N;
    const uint64_t pol = l2_policy_keep();
    for (int i = threadIdx.x; i < 12 * N; i += blockDim.x) ds[i] = 0.0;
    __syncthreads();
    const size_t SN = (size_t)n * N;
    for (int s = blockIdx.x; s < n; s += gridDim.x) {
        double ky = kky ? kky[s] : 0.0, kz = kkz ? kkz[s] : 0.0, k2 = 0.0, wc = 1.0;
#if CODEDIM == 2
        k2 = kz * kz;
        wc = (fabs(kz) < 1.0e-12) ? 1.0 : 2.0;
#ifdef USE_CUBIC_CUTOFF
        if (fabs(kz + M_PI / DZ) < 1.0e-12) wc = 1.0;
#endif
#elif CODEDIM == 1
        k2 = ky * ky + kz * kz;
        wc = cnt ? (double)cnt[s] : 1.0;
#endif
        (void)ky; (void)kz;
        const double f = fb[s];
        const double w = (wts ? wts[s] : 1.0) * wc;
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            const size_t iu = (size_t)s * N + p, iv = SN + iu;
            double2 u = wf[iu], v = wf[iv];
            dens_limited(ds, p, N, u, v, f, w, pol);
            if (grads) {
                const double fa = f * w, fbm = (1.0 - f) * w;
                double2 lu = lap[iu], lv = lap[iv];
                ds[3 * (size_t)N + p] += (u.x * (lu.x - u.x * k2) + u.y * (lu.y - u.y * k2)) * fa;
                ds[8 * (size_t)N + p] += (v.x * (lv.x - v.x * k2) + v.y * (lv.y - v.y * k2)) * fbm;
                const double2 *dd[3] = {dx, dy, dz};
                for (int d = 0; d < CODEDIM; d++) {
                    double2 a = dd[d][iu], b = dd[d][iv];
                    ds[(4 + d) * (size_t)N + p] += (u.x * a.y - u.y * a.x) * fa;
                    ds[(9 + d) * (size_t)N + p] -= (v.x * b.y - v.y * b.x) * fbm;
                }
            }
        }
    }
}

static int calculate_densities_noalloc_impl(int n, wtd_z *wf, wtd_z *dx, wtd_z *dy, wtd_z *dz, wtd_z *lap,
                                            const double *kky, const double *kkz, const int *cnt, double *fb,
                                            double *w, double *dens, int grads)
{
    const size_t per_cta = (size_t)12 * WTD_NUMEL;
    const size_t cap = WTD_NOALLOC_BYTES / sizeof(double);
    if (per_cta > cap) return WTD_ERR_NOALLOC_SIZE;
    if (n <= 0 || !wf || !fb || !dens || (grads && !lap)) return WTD_ERR_ARG;
    double *slots = NULL;
    int r = noalloc_scratch(&slots);
    if (r) return r;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int G = 2 * nsm;
    if (G > n) G = n;
    if ((size_t)G > cap / per_cta) G = (int)(cap / per_cta);
    k_dens_noalloc<<<G, 256>>>(n, (const double2 *)wf, (const double2 *)dx, (const double2 *)dy, (const double2 *)dz,
                               (const double2 *)lap, fb, w, kky, kkz, cnt, slots, grads);
    wtd_dens_reduce<<<(12 * WTD_NUMEL + 255) / 256, 256>>>(slots, G, dens, WTD_NUMEL, grads ? 1 : 0, 1.0 / WTD_LPERP);
    return cu_sync_status();
}

/* ---------------------------------------------------------------------------------------
 * entry points
 * -------------------------------------------------------------------------------------*/
extern "C" {

/* host forms of the energy-density-functional pieces (pca_kernels.h:11-30 and the 2D/1D
 * headers; pca_edf.h:46-350): the uniform-solution start of the drivers (pca_uniform.h) calls
 * them on the host.  Same published formulas as the device functional (edf:: above). */
double polarization_h(double n_a, double n_b) { return edf::pol(n_a, n_b); }
double der_polarization__der_na_h(double n_a, double n_b) { return edf::dpol(n_a, n_b, true); }
double der_polarization__der_nb_h(double n_a, double n_b) { return edf::dpol(n_a, n_b, false); }
double alpha_h(double p) { return edf::alpha(p); }
double alpha_a_h(double p) { return edf::alpha(p); }
double alpha_b_h(double p) { return edf::alpha(-p); }
double alpha_plus_h(double p) { return edf::alpha_plus(p); }
double alpha_minus_h(double p) { return edf::alpha_minus(p); }
double der_alpha_plus__der_na_h(double n_a, double n_b)
{
    return edf::dap_core(edf::pol(n_a, n_b)) * edf::dpol(n_a, n_b, true);
}
double der_alpha_plus__der_nb_h(double n_a, double n_b)
{
    return edf::dap_core(edf::pol(n_a, n_b)) * edf::dpol(n_a, n_b, false);
}
double der_alpha_minus__der_na_h(double n_a, double n_b)
{
    return edf::dam_core(edf::pol(n_a, n_b)) * edf::dpol(n_a, n_b, true);
}
double der_alpha_minus__der_nb_h(double n_a, double n_b)
{
    return edf::dam_core(edf::pol(n_a, n_b)) * edf::dpol(n_a, n_b, false);
}
double funG_h(double p) { return edf::funG(p); }
double funD_h(double n_a, double n_b) { return edf::funD(n_a, n_b); }
double der_funD__der_na_h(double n_a, double n_b) { return edf::dD(n_a, n_b, true); }
double der_funD__der_nb_h(double n_a, double n_b) { return edf::dD(n_a, n_b, false); }
double tildeC_h(double n_a, double n_b) { return edf::tildeC(n_a, n_b); }
double der_tildeC__der_na_h(double n_a, double n_b) { return edf::dtildeC(n_a, n_b, true); }
double der_tildeC__der_nb_h(double n_a, double n_b) { return edf::dtildeC(n_a, n_b, false); }

int memcopy_const(double mu_a, double mu_b, double ec, double t0, double dt, double kF)
{
    double eF = kF * kF / 2., nF = kF * kF * kF / (3. * M_PI * M_PI);
    if (cudaMemcpyToSymbol(dc_mu_a, &mu_a, sizeof(double)) != cudaSuccess) return 1;
    if (cudaMemcpyToSymbol(dc_mu_b, &mu_b, sizeof(double)) != cudaSuccess) return 2;
    if (cudaMemcpyToSymbol(dc_ec, &ec, sizeof(double)) != cudaSuccess) return 3;
    if (cudaMemcpyToSymbol(dc_t0, &t0, sizeof(double)) != cudaSuccess) return 4;
    if (cudaMemcpyToSymbol(dc_dt, &dt, sizeof(double)) != cudaSuccess) return 5;
    if (cudaMemcpyToSymbol(dc_kF, &kF, sizeof(double)) != cudaSuccess) return 6;
    if (cudaMemcpyToSymbol(dc_eF, &eF, sizeof(double)) != cudaSuccess) return 7;
    if (cudaMemcpyToSymbol(dc_nF, &nF, sizeof(double)) != cudaSuccess) return 7;
    hc_mu_a = mu_a; hc_mu_b = mu_b; hc_ec = ec; hc_t0 = t0; hc_dt = dt; hc_kF = kF; hc_eF = eF; hc_nF = nF;
    md.dt = dt; md.ec = ec;
    return 0;
}
int memcopy_const_params(double *params)
{
    if (cudaMemcpyToSymbol(dc_params, params, MAX_USER_PARAMS * sizeof(double)) != cudaSuccess) return 1;
    memcpy(md.params, params, MAX_USER_PARAMS * sizeof(double));
    return 0;
}
int memcopy_const_sclgth(double a)
{
    if (cudaMemcpyToSymbol(dc_sclgth, &a, sizeof(double)) != cudaSuccess) return 1;
    hc_sclgth = a; md.sclgth = a;
    return 0;
}
int memcopy_extra_data(size_t extra_data_size, void *extra_data)
{
    if (cudaMemcpyToSymbol(dc_extra_data, &extra_data, sizeof(void *)) != cudaSuccess) return 1;
    if (cudaMemcpyToSymbol(dc_extra_data_size, &extra_data_size, sizeof(size_t)) != cudaSuccess) return 2;
    return 0;
}
int set_gpu(int device) { return (int)cudaSetDevice(device); }
int gpu_malloc(size_t size, void **pointer) { return (int)cudaMalloc(pointer, size); }
int gpu_free(void *pointer) { return (int)cudaFree(pointer); }
int host_malloc_pl(size_t size, void **pointer) { return (int)cudaHostAlloc(pointer, size, cudaHostAllocDefault); }
int host_free_pl(void *pointer) { return (int)cudaFreeHost(pointer); }
int memcopy_host2gpu(void *host, void *gpu, size_t size) { return (int)cudaMemcpy(gpu, host, size, cudaMemcpyHostToDevice); }
int memcopy_gpu2host(void *gpu, void *host, size_t size) { return (int)cudaMemcpy(host, gpu, size, cudaMemcpyDeviceToHost); }
int memcopy_gpu2gpu(void *gpusrc, void *gpudst, size_t size) { return (int)cudaMemcpy(gpudst, gpusrc, size, cudaMemcpyDeviceToDevice); }

int create_cufftPlans(int batch_size, int nwfip, size_t *workSize)
{
    if (nwfip <= 0 || !workSize) return WTD_ERR_ARG;
    g_nwfip = nwfip;
    int nsm = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    g_dens_grid = nsm * 2 < nwfip ? nsm * 2 : nwfip;
    size_t need = compat_work_words();
    size_t ref = (size_t)(24 + 8) * WTD_NUMEL;  /* PCA_WORKSPACE_SHIFT + PCA_DERIVATIVE_SHIFT */
    *workSize = sizeof(double) * (need > ref ? need : ref);
    return compat_tables();
}
int set_workspace_for_cufftPlan(void *workArea)
{
    if (!workArea) return WTD_ERR_ARG;
    g_work = workArea;
    return 0;
}
size_t mm_get_size_of_kernels_workspace(size_t n) { return sizeof(double) * n * 24; }
size_t mm_get_size_of_derivatives_workspace(size_t n) { return sizeof(double) * n * 8; }
size_t mm_get_size_of_total_workspace(size_t n) { return sizeof(double) * n * 32; }
void *mm_get_pointer_to_kernels_workspace(size_t n) { return g_work; }
void *mm_get_pointer_to_derivatives_workspace(size_t n) { return g_work ? (void *)((double *)g_work + 24 * n) : NULL; }
void *mm_get_pointer_to_total_workspace(size_t n) { return g_work; }

int abm_step1(int n, wtd_z *y, wtd_z *f1, wtd_z *f2, wtd_z *f3, wtd_z *f4, wtd_z *f5, int scheme, int nthreads)
{
    size_t M = (size_t)2 * n * WTD_NUMEL;
    unsigned nb = (unsigned)((M + 255) / 256);
    double dt = hc_dt;
    if (scheme == AB3AM4) k_abm_step1<3><<<nb, 256>>>(M, (double2 *)y, (double2 *)f1, (double2 *)f2, (double2 *)f3, NULL, NULL, dt);
    else if (scheme == AB4AM5) k_abm_step1<4><<<nb, 256>>>(M, (double2 *)y, (double2 *)f1, (double2 *)f2, (double2 *)f3, (double2 *)f4, NULL, dt);
    else if (scheme == AB5AM5) k_abm_step1<5><<<nb, 256>>>(M, (double2 *)y, (double2 *)f1, (double2 *)f2, (double2 *)f3, (double2 *)f4, (double2 *)f5, dt);
    else return -999999; /* the reference's code for an unknown scheme */
    return cu_sync_status();
}
int abm_step4(int n, wtd_z *yin, wtd_z *yout, wtd_z *flast, int scheme, int nthreads)
{
    size_t M = (size_t)2 * n * WTD_NUMEL;
    double c;
    if (scheme == AB3AM4) c = 9. / 24.;
    else if (scheme == AB4AM5 || scheme == AB5AM5) c = 251. / 720.;
    else return -999999;
    k_abm_step4<<<(unsigned)((M + 255) / 256), 256>>>(M, (const double2 *)yin, (double2 *)yout, (const double2 *)flast, hc_dt, c);
    return cu_sync_status();
}
int normalize_wf(int n, wtd_z *wf, int nthreads)
{
    k_normalize<<<n, 256>>>(n, (double2 *)wf);
    return cu_sync_status();
}
int compute_derivatives(int n, wtd_z *wf, wtd_z *dx, wtd_z *dy, wtd_z *dz, wtd_z *lap, int nthreads)
{
    int r = compat_tables();
    if (r) return r;
    if (WTD_BIG) {
        WTD_TRY(big_derivs((double2 *)wf, n, (double2 *)lap, (double2 *)dx, (double2 *)dy,
                           CODEDIM >= 3 ? (double2 *)dz : NULL, g_tw, g_ktab, 0));
        return cu_sync_status();
    }
    if (k_derivs_smem > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
    cudaFuncSetAttribute(k_derivs<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k_derivs_smem);
    k_derivs<WG><<<n, 512, k_derivs_smem>>>((const double2 *)wf, (double2 *)dx, CODEDIM >= 2 ? (double2 *)dy : NULL,
                                             CODEDIM >= 3 ? (double2 *)dz : NULL, (double2 *)lap, g_tw, g_ktab);
    return cu_sync_status();
}
int compute_laplace(int n, wtd_z *wf, wtd_z *lap, int nthreads)
{
    int r = compat_tables();
    if (r) return r;
    if (WTD_BIG) {
        WTD_TRY(big_derivs((double2 *)wf, n, (double2 *)lap, NULL, NULL, NULL, g_tw, g_ktab, 0));
        return cu_sync_status();
    }
    if (k_derivs_smem > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
    cudaFuncSetAttribute(k_derivs<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k_derivs_smem);
    k_derivs<WG><<<n, 512, k_derivs_smem>>>((const double2 *)wf, NULL, NULL, NULL, (double2 *)lap, g_tw, g_ktab);
    return cu_sync_status();
}
int compute_laplace_real_f(double *f, double *laplace_f, int nthreads) { return compat_real_deriv(f, laplace_f, 0); }
int compute_gradient_real_f(double *f, double *dfx, double *dfy, double *dfz, int nthreads)
{
    int r = compat_real_deriv(f, dfx, 1);
    if (!r && CODEDIM >= 2 && dfy) r = compat_real_deriv(f, dfy, 2);
    if (!r && CODEDIM >= 3 && dfz) r = compat_real_deriv(f, dfz, 3);
    return r;
}
int compute_derivative_real_vector_f(double *fx, double *fy, double *fz, double *dfx_dx, double *dfy_dy, double *dfz_dz, int nthreads)
{
    int r = compat_real_deriv(fx, dfx_dx, 1);
    if (!r && CODEDIM >= 2 && fy) r = compat_real_deriv(fy, dfy_dy, 2);
    if (!r && CODEDIM >= 3 && fz) r = compat_real_deriv(fz, dfz_dz, 3);
    return r;
}
/* scratch of the divergence: a library-owned array of 2 N words, allocated on the first such
 * call and kept (the call needs no work area, so it must not depend on one being alive) */
static double *g_divtmp_own = NULL;
int compute_divergence_real_vector_f(double *fx, double *fy, double *fz, double *divf, int nthreads)
{
    if (!g_divtmp_own && cudaMalloc((void **)&g_divtmp_own, 2 * sizeof(double) * WTD_NUMEL) != cudaSuccess) {
        g_divtmp_own = NULL;
        return WTD_ERR_NOMEM;
    }
    double *t = g_divtmp_own;
    int r = compat_real_deriv(fx, divf, 1);
    if (!r && CODEDIM >= 2) { r = compat_real_deriv(fy, t, 2); }
    if (!r && CODEDIM >= 3) { r = compat_real_deriv(fz, t + WTD_NUMEL, 3); }
    if (!r && CODEDIM >= 2) {
        k_add_fields<<<(WTD_NUMEL + 255) / 256, 256>>>(divf, t, CODEDIM >= 3 ? t + WTD_NUMEL : NULL, WTD_NUMEL);
        r = cu_sync_status();
    }
    return r;
}

/* high-k filters (pca_derivative.cu:829-859, 906-935, 950-963): in -> IFFT[FD(k^2/2) FFT in];
 * out may alias in */
int high_frequency_filter_massive_d(int n, double *in, double *out, double fd_mu, double fd_T, int nthreads)
{
    if (n < 0 || !(fd_T > 0.0)) return WTD_ERR_ARG;
    if (n == 0) return 0;
    int r = compat_tables();
    if (r) return r;
    if (out != in) cudaMemcpy(out, in, (size_t)n * WTD_NUMEL * sizeof(double), cudaMemcpyDeviceToDevice);
    if (WTD_BIG) {
        WTD_TRY(compat_stage());
        WTD_TRY(big_filter_real(out, n, fd_mu, fd_T, g_stage3d, g_tw, g_ktab, 0));
        return cu_sync_status();
    }
    if (k_field_smem > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
    cudaFuncSetAttribute(wtd_hkf_kernel<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k_field_smem);
    wtd_hkf_kernel<WG><<<n, 512, k_field_smem>>>(out, fd_mu, fd_T, g_tw, g_ktab);
    return cu_sync_status();
}
int high_frequency_filter_d(double *in, double *out, double fd_mu, double fd_T, int nthreads)
{
    return high_frequency_filter_massive_d(1, in, out, fd_mu, fd_T, nthreads);
}
int high_frequency_filter_c(wtd_z *in, wtd_z *out, double fd_mu, double fd_T, int nthreads)
{
    if (!(fd_T > 0.0)) return WTD_ERR_ARG;
    int r = compat_tables();
    if (r) return r;
    if (WTD_BIG) {
        WTD_TRY(compat_stage());
        WTD_TRY(big_derivs((double2 *)in, 1, (double2 *)out, NULL, NULL, NULL, g_tw, g_ktab, 0, 1, fd_mu, fd_T));
        return cu_sync_status();
    }
    if (k_field_smem > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
    cudaFuncSetAttribute(wtd_hkf_c_kernel<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k_field_smem);
    wtd_hkf_c_kernel<WG><<<1, 512, k_field_smem>>>((const double2 *)in, (double2 *)out, fd_mu, fd_T, g_tw, g_ktab);
    return cu_sync_status();
}

static int calculate_densities_impl(int n, wtd_z *wf, wtd_z *dx, wtd_z *dy, wtd_z *dz, wtd_z *lap, const double *kky,
                                    const double *kkz, const int *cnt, double *fb, double *w, double *dens, int grads)
{
    if (!g_work || g_nwfip < n || g_dens_grid <= 0) return WTD_ERR_STATE;
    int r = compat_planewave(n, kky, kkz, cnt, true);
    if (r) return r;
    double *slots = compat_slots();
    int G = g_dens_grid < n ? g_dens_grid : n;
    k_dens_compat<<<G, 256>>>(n, (const double2 *)wf, (const double2 *)dx, (const double2 *)dy, (const double2 *)dz,
                              (const double2 *)lap, fb, w, g_kp2, g_wcnt, slots, grads);
    wtd_dens_reduce<<<(12 * WTD_NUMEL + 255) / 256, 256>>>(slots, G, dens, WTD_NUMEL, grads ? 1 : 0, 1.0 / WTD_LPERP);
    return cu_sync_status();
}

#if CODEDIM == 3
int calculate_densities(int n, wtd_z *wf, wtd_z *dx, wtd_z *dy, wtd_z *dz, wtd_z *lap, double *fb, double *w, double *dens, int grads, int nthreads)
{
    return calculate_densities_impl(n, wf, dx, dy, dz, lap, NULL, NULL, NULL, fb, w, dens, grads);
}
#elif CODEDIM == 2
int calculate_densities(int n, wtd_z *wf, wtd_z *dx, wtd_z *dy, wtd_z *lap, double *kkz, double *fb, double *w, double *dens, int grads, int nthreads)
{
    return calculate_densities_impl(n, wf, dx, dy, NULL, lap, NULL, kkz, NULL, fb, w, dens, grads);
}
#else
int calculate_densities(int n, wtd_z *wf, wtd_z *dx, wtd_z *lap, double *kkyz, double *fb, double *w, int *cnt, double *dens, int grads, int nthreads)
{
    return calculate_densities_impl(n, wf, dx, NULL, NULL, lap, kkyz, kkyz ? kkyz + n : NULL, cnt, fb, w, dens, grads);
}
#endif

#if CODEDIM == 3
int calculate_densities_noalloc(int n, wtd_z *wf, wtd_z *dx, wtd_z *dy, wtd_z *dz, wtd_z *lap, double *fb, double *w,
                                double *dens, int grads, int nthreads)
{
    return calculate_densities_noalloc_impl(n, wf, dx, dy, dz, lap, NULL, NULL, NULL, fb, w, dens, grads);
}
#elif CODEDIM == 2
int calculate_densities_noalloc(int n, wtd_z *wf, wtd_z *dx, wtd_z *dy, wtd_z *lap, double *kkz, double *fb, double *w,
                                double *dens, int grads, int nthreads)
{
    return calculate_densities_noalloc_impl(n, wf, dx, dy, NULL, lap, NULL, kkz, NULL, fb, w, dens, grads);
}
#else
int calculate_densities_noalloc(int n, wtd_z *wf, wtd_z *dx, wtd_z *lap, double *kkyz, double *fb, double *w, int *cnt,
                                double *dens, int grads, int nthreads)
{
    return calculate_densities_noalloc_impl(n, wf, dx, NULL, NULL, lap, kkyz, kkyz ? kkyz + n : NULL, cnt, fb, w, dens, grads);
}
#endif

int density_caculate_tau(double *dens, int nthreads)
{
    int r = compat_tables();
    if (r) return r;
    if (WTD_BIG) {
        WTD_TRY(compat_stage());
        WTD_TRY(big_tau(dens, g_stage3d, g_tw, g_ktab, 0));
        return cu_sync_status();
    }
    if (k_field_smem > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
    cudaFuncSetAttribute(wtd_tau_kernel<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k_field_smem);
    wtd_tau_kernel<WG><<<2, 512, k_field_smem>>>(dens, g_tw, g_ktab);
    return cu_sync_status();
}
int symmetrize_densities_device(double *dens) { return 0; /* spin-symmetric mode is not provided */ }

int compute_potentials(int it, double *dens, double *pots, double cccoeff, int nthreads)
{
    wslda_density D = convert_into_wslda_density(dens, WTD_NUMEL);
    wslda_potential P = convert_into_wslda_potential(pots, WTD_NUMEL, NULL);
    wtd_potentials_kernel<<<(WTD_NUMEL + 127) / 128, 128>>>(it, D, P, cccoeff);
#ifdef ENABLE_MODIFY_POTENTIALS
    modify_potentials<<<(WTD_NUMEL + 127) / 128, 128>>>(it, D, P);
#endif
    return cu_sync_status();
}
int multiply_wf_by_alpha(int n, wtd_z *in, wtd_z *out, double *pots, int nthreads)
{
    wslda_potential P = convert_into_wslda_potential(pots, WTD_NUMEL, NULL);
    size_t M = (size_t)2 * n * WTD_NUMEL;
    k_mul_alpha<<<(unsigned)((M + 255) / 256), 256>>>(n, (const double2 *)in, (double2 *)out, P.alpha_a, P.alpha_b);
    return cu_sync_status();
}

/* the friction-modified V_a, V_b, delta (4 N) and the control coefficient on the device */
static double *g_qfld = NULL, *g_pcc = NULL;

static int apply_hamiltonian_impl(int it, int n, wtd_z *in, wtd_z *out, wtd_z *dx, wtd_z *dy, wtd_z *dz, wtd_z *lap,
                                  wtd_z *alap, const double *kky, const double *kkz, double *dens, double *pots,
                                  double qfswitch, double *useqpe, double pccoeff)
{
    if (!g_work || g_nwfip < n) return WTD_ERR_STATE;
    /* quantum friction (pca_kernels.cu:497-539): H from V, delta plus the friction terms, the
     * potentials left as they are; the V and delta filters then act on that copy only */
    double *fld = pots;
    if (qfswitch > 0.0) {
        if (!dens) return WTD_ERR_ARG;
        if (!g_qfld) {
            if (cudaMalloc((void **)&g_qfld, 4 * sizeof(double) * WTD_NUMEL) != cudaSuccess) return WTD_ERR_NOMEM;
            if (cudaMalloc((void **)&g_pcc, sizeof(double)) != cudaSuccess) return WTD_ERR_NOMEM;
        }
        cudaMemcpy(g_pcc, &pccoeff, sizeof(double), cudaMemcpyHostToDevice);
        wtd_qf_fields<<<(WTD_NUMEL + 255) / 256, 256>>>(pots, dens + 12 * (size_t)WTD_NUMEL, g_pcc, md.qfalpha * qfswitch,
                                                        md.qfbeta * qfswitch, md.qfgamma * qfswitch, hc_nF, g_qfld, WTD_NUMEL);
        fld = g_qfld;
    }
    /* high-k filters of the fields, in place, as the reference's apply_hamiltonian: V_a, V_b
     * (hkf_mode >= 1, pca_kernels.cu:700-704), delta (>= 2, :758-762), the A components
     * (>= 1 with current corrections outside BdG, :791-795) */
    if (md.hkf_mode >= 1) {
        int rf = high_frequency_filter_massive_d(2, fld, fld, md.hkf_mu, md.hkf_T, 512);
        if (rf) return rf;
    }
    if (md.hkf_mode >= 2) {
        wtd_z *delta = (wtd_z *)(fld + 2 * (size_t)WTD_NUMEL);
        int rf = high_frequency_filter_c(delta, delta, md.hkf_mu, md.hkf_T, 512);
        if (rf) return rf;
    }
#if defined(CURRENT_CORRECTIONS) && !defined(BDG_MODE)
    if (md.hkf_mode >= 1) {
        double *A = pots + 6 * (size_t)WTD_NUMEL;
        int rf = high_frequency_filter_massive_d(6, A, A, md.hkf_mu, md.hkf_T, 512);
        if (rf) return rf;
    }
#endif
    int r = compat_coefficients(it, pots, fld == pots ? NULL : fld);
    if (r) return r;
    r = compat_planewave(n, kky, kkz, NULL, true);
    if (r) return r;
    k_hamiltonian_compat<<<n, 256>>>(n, (const double2 *)in, (double2 *)out, (const double2 *)dx, (const double2 *)dy,
                                     (const double2 *)dz, (const double2 *)lap, (const double2 *)alap, compat_cf(), g_kp2,
                                     compat_qpe(), useqpe);
#if CODEDIM == 2
    if (fld != pots) {
        /* the 2D engine does not remove the friction terms (cpca_kernels.cu:846 commented out):
         * the potentials keep the modified fields, the friction densities the originals */
        cudaMemcpy(dens + 12 * (size_t)WTD_NUMEL, pots, 4 * sizeof(double) * WTD_NUMEL, cudaMemcpyDeviceToDevice);
        cudaMemcpy(pots, fld, 4 * sizeof(double) * WTD_NUMEL, cudaMemcpyDeviceToDevice);
    }
#endif
    return cu_sync_status();
}

#if CODEDIM == 3
int apply_hamiltonian(int it, int n, wtd_z *in, wtd_z *out, wtd_z *dx, wtd_z *dy, wtd_z *dz, wtd_z *lap, wtd_z *alap,
                      double *dens, double *pots, double qfswitch, double *useqpe, double pccoeff, int nthreads)
{
    return apply_hamiltonian_impl(it, n, in, out, dx, dy, dz, lap, alap, NULL, NULL, dens, pots, qfswitch, useqpe, pccoeff);
}
#elif CODEDIM == 2
int apply_hamiltonian(int it, int n, wtd_z *in, wtd_z *out, wtd_z *dx, wtd_z *dy, double *kkz, wtd_z *lap, wtd_z *alap,
                      double *dens, double *pots, double qfswitch, double *useqpe, double pccoeff, int nthreads)
{
    return apply_hamiltonian_impl(it, n, in, out, dx, dy, NULL, lap, alap, NULL, kkz, dens, pots, qfswitch, useqpe, pccoeff);
}
#else
int apply_hamiltonian(int it, int n, wtd_z *in, wtd_z *out, wtd_z *dx, double *kkyz, wtd_z *lap, wtd_z *alap,
                      double *dens, double *pots, double qfswitch, double *useqpe, double pccoeff, int nthreads)
{
    return apply_hamiltonian_impl(it, n, in, out, dx, NULL, NULL, lap, alap, kkyz, kkyz ? kkyz + n : NULL, dens, pots, qfswitch,
                                  useqpe, pccoeff);
}
#endif

static int calculate_qf_densities_impl(int n, const wtd_z *wf, const wtd_z *lap, const double *kky, const double *kkz,
                                const int *cnt, const double *fb, const double *w, double *qf)
{
    if (n <= 0 || !wf || !lap || !fb || !qf) return WTD_ERR_ARG;
    int r = compat_planewave(n, kky, kkz, cnt, false);
    if (r) return r;
    k_qf_dens_compat<<<(WTD_NUMEL + 255) / 256, 256>>>(n, (const double2 *)wf, (const double2 *)lap, fb, w, g_kp2, g_wcnt,
                                                       qf, 1.0 / WTD_LPERP);
    return cu_sync_status();
}
#if CODEDIM == 3
int calculate_quantum_friction_densities(int n, wtd_z *wf, wtd_z *lap, double *fb, double *w, double *qf, int nthreads)
{
    return calculate_qf_densities_impl(n, wf, lap, NULL, NULL, NULL, fb, w, qf);
}
#elif CODEDIM == 2
int calculate_quantum_friction_densities(int n, wtd_z *wf, wtd_z *lap, double *kkz, double *fb, double *w, double *qf,
                                         int nthreads)
{
    return calculate_qf_densities_impl(n, wf, lap, NULL, kkz, NULL, fb, w, qf);
}
#else
int calculate_quantum_friction_densities(int n, wtd_z *wf, wtd_z *lap, double *kkyz, double *fb, double *w, int *cnt,
                                         double *qf, int nthreads)
{
    return calculate_qf_densities_impl(n, wf, lap, kkyz, kkyz ? kkyz + n : NULL, cnt, fb, w, qf);
}
#endif

int local_reductions_many(int n, int m, double *d_in, double *d_out)
{
    if (n <= 0 || m <= 0) return -1;
    if (n > (1 << 16)) return -2;
    double *tmp = NULL;
    if (cudaGetSymbolAddress((void **)&tmp, g_sum_tmp) != cudaSuccess) return -1;
    k_sum_many<<<n, 256>>>(d_in, m, tmp);
    if (cudaMemcpy(d_out, tmp, n * sizeof(double), cudaMemcpyDeviceToDevice) != cudaSuccess) return -1;
    return cu_sync_status();
}

int compute_energy(int it, double *dens, double *pots, double *work, int nthreads)
{
    constexpr int N = WTD_NUMEL;
    wslda_density D = convert_into_wslda_density(dens, N);
    wslda_potential P = convert_into_wslda_potential(pots, N, NULL);
    int pb = (N + 127) / 128;
    wtd_energy_kernel<<<pb, 128>>>(it, D, P, work + EKIN * (size_t)N, work + EPOT * (size_t)N, work + EPAIR * (size_t)N,
                                   work + ECURRENT * (size_t)N);
    wtd_energy_ext_kernel<<<pb, 128>>>(it, D, P, work);
#ifdef ENABLE_MODIFY_ENERGIES
    modify_energies<<<pb, 128>>>(it, D, P, work);
#endif
    double *tmp = NULL;
    if (cudaGetSymbolAddress((void **)&tmp, g_sum_tmp) != cudaSuccess) return -1;
    wtd_sum_items<<<TDWSLDAITEMS, 256>>>(work, N, tmp, WTD_VOLEL);
    if (cudaMemcpy(work, tmp, TDWSLDAITEMS * sizeof(double), cudaMemcpyDeviceToDevice) != cudaSuccess) return -100;
    return cu_sync_status();
}

int compute_ovelap(int n, wtd_z *wf1, wtd_z *wf2, double *re, double *im, double *workarea, int nthreads)
{
    k_overlap<<<n, 256>>>(n, (const double2 *)wf1, (const double2 *)wf2, re, im);
    return cu_sync_status();
}

int taylor_expansion_contribution(int it, double dt, int n, wtd_z *hpsi, wtd_z *upd, wtd_z *contr, int nthreads)
{
    size_t M = (size_t)2 * n * WTD_NUMEL;
    k_taylor<<<(unsigned)((M + 255) / 256), 256>>>(M, (const double2 *)hpsi, (double2 *)upd, (double2 *)contr, -1.0 * dt / (double)it);
    return cu_sync_status();
}

int get_v_ext(int datadim, int spin, int it, double *data)
{
    double *t = NULL;
    if (cudaMalloc((void **)&t, sizeof(double) * WTD_NUMEL) != cudaSuccess) return 1;
    k_get_vext<<<(WTD_NUMEL + 127) / 128, 128>>>(it, spin, t);
    int r = cudaMemcpy(data, t, sizeof(double) * WTD_NUMEL, cudaMemcpyDeviceToHost) != cudaSuccess;
    cudaFree(t);
    return r;
}
/* velocity_ext on the lattice, x, y, z blocks into data (3 N host doubles; wslda_writevars.c:80) */
int get_velocity_ext(int datadim, int spin, int it, double *data)
{
    double *t = NULL;
    if (cudaMalloc((void **)&t, sizeof(double) * 3 * WTD_NUMEL) != cudaSuccess) return 1;
    k_get_velext<<<(WTD_NUMEL + 127) / 128, 128>>>(it, spin, t);
    int r = cudaMemcpy(data, t, sizeof(double) * 3 * WTD_NUMEL, cudaMemcpyDeviceToHost) != cudaSuccess;
    cudaFree(t);
    return r;
}
int get_delta_ext(int datadim, int it, void *deltain, void *data)
{
    Complex *t = NULL;
    if (cudaMalloc((void **)&t, sizeof(Complex) * WTD_NUMEL) != cudaSuccess) return 1;
    k_get_dext<<<(WTD_NUMEL + 127) / 128, 128>>>(it, (const Complex *)deltain, t);
    int r = cudaMemcpy(data, t, sizeof(Complex) * WTD_NUMEL, cudaMemcpyDeviceToHost) != cudaSuccess;
    cudaFree(t);
    return r;
}

} /* extern "C" */

#endif
