/*
 * Hand-written adjoint of the fused TD step (constant effective mass, FP64) for gradients of
 *   L = sum_r |Delta(r, T)|^2 mask(r) dV
 * with respect to the user parameters params[0..np) of the external potential v_ext, for the
 * contact-BdG functional Delta = -g nu, V_a,b = v_ext (a CUSTOMEDF project that defines
 * WTD_ADJOINT_CONTACT_BDG to the params index of g).  The reference has no adjoint.
 *
 * Adjoint convention: for a real L and complex z, zbar = dL/dRe z + i dL/dIm z, so
 * dL = Re sum conj(zbar) dz.  Per operation of the forward step (wtd_step.cuh):
 *   normalisation y = yt/n, n^2 = dV |yt|^2      ytbar = (ybar - dV Re<ybar,y> y) / n
 *   f = (H - E) psi, E = dV Re<psi|H psi>         psibar = H(fbar - 2 s dV psi) - E fbar,
 *                                                 s = Re<fbar, psi>; the potentials see
 *                                                 wbar = fbar - s dV psi:
 *       Deltabar += wbar_u conj(v) + conj(wbar_v) u,  Vabar += Re(conj(wbar_u) u),
 *       Vbbar -= Re(conj(wbar_v) v)            (H is Hermitian; one H application)
 *   predictor yt = y - i dt sum b_j f_{k-j}, P = y - i dt sum a_j f_{k-j}
 *                                                 ybar += ytbar + Pbar,
 *                                                 fbar_{k-j} += i dt (b_j ytbar + a_j Pbar)
 *   corrector yh = P - i dt c f_p                 Pbar = yhbar, fbar_p = i dt c yhbar
 *   Delta = -g nu, nu = sum_n c_n u conj(v)       nubar = -g Deltabar,
 *                                                 ubar += c_n nubar v, vbar += c_n conj(nubar) u
 *   V_s = v_ext(theta, t)                         thetabar += sum_r Vbar_s dV_s/dtheta (central
 *                                                 differences of the user's v_ext hook)
 * The forward is checkpointed every K steps (state, ABM history ring, coefficients) and each
 * segment is recomputed once in the reverse sweep, storing y_k, y_pred, the per-state norms
 * and <H> of both half steps.  Per reverse step: two H applications (one per half step).
 */
#ifndef WTD_ADJOINT_CUH
#define WTD_ADJOINT_CUH

struct AdjArgs {
    const double2 *y1;      /* RB: state after the step; RA: y_k */
    const double2 *yp;      /* predictor state y_pred (normalised) */
    double2 *ybar;          /* RB: in (ybar_{k+1}); RA: out (ybar_k) */
    double2 *ypbar;         /* RB: out; RA: in */
    double2 *pbar;          /* RB: out; RA: in */
    double2 *fring[5];      /* RA: fbar_k, fbar_{k-1}, ... */
    const double2 *nubar;   /* pending density adjoint field (N complex) or null */
    const double *nrm;      /* per-state norm of the unnormalised update of this half step */
    const double *E;        /* per-state <H> of this half step */
    const double *cf;       /* H coefficients of this half step */
    const double *occ, *kp2, *wcnt;
    double *slots;          /* [grid][4][N]: Deltabar re/im interleaved (2N), Vabar, Vbbar */
    double dt, inv_lperp;
    int S, has_h;
};

/* H x at point p, constant effective mass (same arithmetic as hpsi_const) */
__device__ __forceinline__ void h_apply_point(const double *cf, int N, int p, double kp2, double2 xu, double2 xv,
                                              double2 lu, double2 lv, double2 &hu, double2 &hv)
{
    const double va = cf[CF_VA * N + p], vb = cf[CF_VB * N + p], dr = cf[CF_DRE * N + p], di = cf[CF_DIM * N + p];
    const double aa = cf[CF_AA * N + p], ab = cf[CF_AB * N + p];
    const double ja = -aa * kp2, jb = -ab * kp2;
    hu.x = (va + ja) * xu.x + (dr * xv.x - di * xv.y) + aa * lu.x;
    hu.y = (va + ja) * xu.y + (dr * xv.y + di * xv.x) + aa * lu.y;
    hv.x = -(vb + jb) * xv.x + (dr * xu.x + di * xu.y) - ab * lv.x;
    hv.y = -(vb + jb) * xv.y + (dr * xu.y - di * xu.x) - ab * lv.y;
}

/* the potentials' adjoint at one point: Deltabar, Vabar, Vbbar — L2 reductions into the CTA's
 * slot, every word of which is updated by one thread only (program order, deterministic) */
__device__ __forceinline__ void field_adjoint(double *ds, int N, int p, double2 wu, double2 wv, double2 u, double2 v)
{
    const uint64_t pol = l2_policy_keep();
    red_keep(ds + 2 * p, (wu.x * v.x + wu.y * v.y) + (wv.x * u.x + wv.y * u.y), pol);
    red_keep(ds + 2 * p + 1, (wu.y * v.x - wu.x * v.y) + (wv.x * u.y - wv.y * u.x), pol);
    red_keep(ds + 2 * (size_t)N + p, wu.x * u.x + wu.y * u.y, pol);
    red_keep(ds + 3 * (size_t)N + p, -(wv.x * v.x + wv.y * v.y), pol);
}

/* density adjoint of nu = sum_n c_n u conj(v): ubar += c nubar v, vbar += c conj(nubar) u */
__device__ __forceinline__ void nu_adjoint(double2 &gu, double2 &gv, double2 nb, double cn, double2 u, double2 v)
{
    gu.x += cn * (nb.x * v.x - nb.y * v.y);
    gu.y += cn * (nb.x * v.y + nb.y * v.x);
    gv.x += cn * (nb.x * u.x + nb.y * u.y);
    gv.y += cn * (nb.x * u.y - nb.y * u.x);
}

/* laplacian of the two fields in (BU, BV), in place */
template <class G>
__device__ __forceinline__ void lap2(double2 *BU, double2 *BV, const double2 *tw, const double (*kt)[WTD_KT])
{
    __syncthreads();
    fft_forward<G, 2>(BU, (int)(BV - BU), tw);
    kmul<G, OP_LAP>(BU, kt);
    kmul<G, OP_LAP>(BV, kt);
    __syncthreads();
    fft_inverse<G, 2>(BU, (int)(BV - BU), tw);
}

/* reverse of pass B (corrector half step), persistent CTAs over states */
template <class G, int NH>
__global__ void __launch_bounds__(512, 1) k_adj_B(AdjArgs a, const double2 *gtw, const double *gk)
{
    constexpr int N = G::ntot;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *BU = (double2 *)smem_raw;
    double2 *BV = BU + G::padded;
    double2 *tw = BV + G::padded;
    double (*kt)[WTD_KT] = (double (*)[WTD_KT])(tw + G::twtotal);
    double *red = (double *)(kt + 6);
    load_tables<G>(tw, kt, gtw, gk);
    double *ds = a.slots + (size_t)blockIdx.x * 4 * N;
    for (int i = threadIdx.x; i < 4 * N; i += blockDim.x) ds[i] = 0.0;
    const size_t SN = (size_t)a.S * N;
    const double cAM = Abm<NH>::c, dV = WTD_DV, dc = a.dt * cAM;
    for (int n = blockIdx.x; n < a.S; n += gridDim.x) {
        const size_t bu = (size_t)n * N, bv = SN + bu;
        const double cn = (1.0 - 2.0 * a.occ[n]) * 0.5 * a.wcnt[n] * a.inv_lperp;
        const double kp2 = a.kp2[n];
        /* ybar_{k+1} (+ the pending density adjoint of nu(y_{k+1})), r1 = Re<ybar, y1> */
        double r1 = 0.0;
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            double2 u = a.y1[bu + p], v = a.y1[bv + p], gu = a.ybar[bu + p], gv = a.ybar[bv + p];
            if (a.nubar) nu_adjoint(gu, gv, a.nubar[p], cn, u, v);
            BU[G::off(p)] = gu;
            BV[G::off(p)] = gv;
            r1 += gu.x * u.x + gu.y * u.y + gv.x * v.x + gv.y * v.y;
        }
        r1 = block_sum(r1, red);
        const double inv_n = 1.0 / a.nrm[n];
        /* Pbar = yhbar = (ybar - dV r1 y1)/n;  fbar_p = i dt c Pbar;  s = Re<fbar_p, y_p> */
        double s = 0.0;
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            const int o = G::off(p);
            double2 u = a.y1[bu + p], v = a.y1[bv + p], gu = BU[o], gv = BV[o];
            double2 pu = make_double2((gu.x - dV * r1 * u.x) * inv_n, (gu.y - dV * r1 * u.y) * inv_n);
            double2 pv = make_double2((gv.x - dV * r1 * v.x) * inv_n, (gv.y - dV * r1 * v.y) * inv_n);
            a.pbar[bu + p] = pu;
            a.pbar[bv + p] = pv;
            double2 yu = a.yp[bu + p], yv = a.yp[bv + p];
            s += (-dc * pu.y) * yu.x + (dc * pu.x) * yu.y + (-dc * pv.y) * yv.x + (dc * pv.x) * yv.y;
        }
        s = block_sum(s, red);
        /* x = fbar_p - 2 s dV y_p, its laplacian in shared memory */
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            const int o = G::off(p);
            double2 pu = a.pbar[bu + p], pv = a.pbar[bv + p], yu = a.yp[bu + p], yv = a.yp[bv + p];
            BU[o] = make_double2(-dc * pu.y - 2.0 * s * dV * yu.x, dc * pu.x - 2.0 * s * dV * yu.y);
            BV[o] = make_double2(-dc * pv.y - 2.0 * s * dV * yv.x, dc * pv.x - 2.0 * s * dV * yv.y);
        }
        lap2<G>(BU, BV, tw, kt);
        const double E = a.E[n];
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            const int o = G::off(p);
            double2 pu = a.pbar[bu + p], pv = a.pbar[bv + p], yu = a.yp[bu + p], yv = a.yp[bv + p];
            double2 fu = make_double2(-dc * pu.y, dc * pu.x), fv = make_double2(-dc * pv.y, dc * pv.x);
            double2 xu = make_double2(fu.x - 2.0 * s * dV * yu.x, fu.y - 2.0 * s * dV * yu.y);
            double2 xv = make_double2(fv.x - 2.0 * s * dV * yv.x, fv.y - 2.0 * s * dV * yv.y);
            double2 hu, hv;
            h_apply_point(a.cf, N, p, kp2, xu, xv, BU[o], BV[o], hu, hv);
            a.ypbar[bu + p] = make_double2(hu.x - E * fu.x, hu.y - E * fu.y);
            a.ypbar[bv + p] = make_double2(hv.x - E * fv.x, hv.y - E * fv.y);
            double2 wu = make_double2(fu.x - s * dV * yu.x, fu.y - s * dV * yu.y);
            double2 wv = make_double2(fv.x - s * dV * yv.x, fv.y - s * dV * yv.y);
            field_adjoint(ds, N, p, wu, wv, yu, yv);
        }
        __syncthreads();
    }
}

/* reverse of pass A (predictor half step).  has_h: f_k was formed from y_k with H of this
 * half step, so its completed adjoint (ring position 0) flows into ybar_k and the potentials */
template <class G, int NH>
__global__ void __launch_bounds__(512, 1) k_adj_A(AdjArgs a, const double2 *gtw, const double *gk)
{
    typedef Abm<NH> AB;
    constexpr int N = G::ntot;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *BU = (double2 *)smem_raw;
    double2 *BV = BU + G::padded;
    double2 *tw = BV + G::padded;
    double (*kt)[WTD_KT] = (double (*)[WTD_KT])(tw + G::twtotal);
    double *red = (double *)(kt + 6);
    load_tables<G>(tw, kt, gtw, gk);
    double *ds = a.slots + (size_t)blockIdx.x * 4 * N;
    if (a.has_h)
        for (int i = threadIdx.x; i < 4 * N; i += blockDim.x) ds[i] = 0.0;
    const size_t SN = (size_t)a.S * N;
    const double dV = WTD_DV, dt = a.dt;
    for (int n = blockIdx.x; n < a.S; n += gridDim.x) {
        const size_t bu = (size_t)n * N, bv = SN + bu;
        const double cn = (1.0 - 2.0 * a.occ[n]) * 0.5 * a.wcnt[n] * a.inv_lperp;
        const double kp2 = a.kp2[n];
        /* ybar_pred (+ density adjoint of nu(y_pred)), r2 = Re<ybar_pred, y_pred> */
        double r2 = 0.0;
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            double2 u = a.yp[bu + p], v = a.yp[bv + p], gu = a.ypbar[bu + p], gv = a.ypbar[bv + p];
            if (a.nubar) nu_adjoint(gu, gv, a.nubar[p], cn, u, v);
            BU[G::off(p)] = gu;
            BV[G::off(p)] = gv;
            r2 += gu.x * u.x + gu.y * u.y + gv.x * v.x + gv.y * v.y;
        }
        r2 = block_sum(r2, red);
        const double inv_n = 1.0 / a.nrm[n];
        /* ytbar = (ybar_pred - dV r2 y_pred)/n;  ybar_k = ytbar + Pbar;
         * fbar_{k-j} += i dt (b_j ytbar + a_j Pbar);  s = Re<fbar_k, y_k> */
        double s = 0.0;
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            const int o = G::off(p);
#pragma unroll
            for (int comp = 0; comp < 2; comp++) {
                const size_t gi = (comp ? bv : bu) + p;
                const double2 y = a.yp[gi], g = comp ? BV[o] : BU[o], P = a.pbar[gi];
                const double2 t = make_double2((g.x - dV * r2 * y.x) * inv_n, (g.y - dV * r2 * y.y) * inv_n);
                a.ybar[gi] = make_double2(t.x + P.x, t.y + P.y);
#pragma unroll
                for (int j = 0; j < NH; j++) {
                    const double cb = AB::b(j), ca = (j < AB::na) ? AB::a(j) : 0.0;
                    const double zx = cb * t.x + ca * P.x, zy = cb * t.y + ca * P.y;
                    double2 f = a.fring[j][gi];
                    f.x -= dt * zy;
                    f.y += dt * zx;
                    a.fring[j][gi] = f;
                    if (j == 0 && a.has_h) {
                        const double2 yk = a.y1[gi];
                        s += f.x * yk.x + f.y * yk.y;
                    }
                }
            }
        }
        if (a.has_h) {
            s = block_sum(s, red);
            for (int p = threadIdx.x; p < N; p += blockDim.x) {
                const int o = G::off(p);
                double2 fu = a.fring[0][bu + p], fv = a.fring[0][bv + p], yu = a.y1[bu + p], yv = a.y1[bv + p];
                BU[o] = make_double2(fu.x - 2.0 * s * dV * yu.x, fu.y - 2.0 * s * dV * yu.y);
                BV[o] = make_double2(fv.x - 2.0 * s * dV * yv.x, fv.y - 2.0 * s * dV * yv.y);
            }
            lap2<G>(BU, BV, tw, kt);
            const double E = a.E[n];
            for (int p = threadIdx.x; p < N; p += blockDim.x) {
                const int o = G::off(p);
                double2 fu = a.fring[0][bu + p], fv = a.fring[0][bv + p], yu = a.y1[bu + p], yv = a.y1[bv + p];
                double2 xu = make_double2(fu.x - 2.0 * s * dV * yu.x, fu.y - 2.0 * s * dV * yu.y);
                double2 xv = make_double2(fv.x - 2.0 * s * dV * yv.x, fv.y - 2.0 * s * dV * yv.y);
                double2 hu, hv;
                h_apply_point(a.cf, N, p, kp2, xu, xv, BU[o], BV[o], hu, hv);
                double2 gu = a.ybar[bu + p], gv = a.ybar[bv + p];
                a.ybar[bu + p] = make_double2(gu.x + hu.x - E * fu.x, gu.y + hu.y - E * fu.y);
                a.ybar[bv + p] = make_double2(gv.x + hv.x - E * fv.x, gv.y + hv.y - E * fv.y);
                double2 wu = make_double2(fu.x - s * dV * yu.x, fu.y - s * dV * yu.y);
                double2 wv = make_double2(fv.x - s * dV * yv.x, fv.y - s * dV * yv.y);
                field_adjoint(ds, N, p, wu, wv, yu, yv);
            }
        }
        __syncthreads();
    }
}

#ifdef WTD_ADJOINT_CONTACT_BDG
/* second stage of the potentials' adjoint: fixed-order sum over the per-CTA slots.
 * vbar[0..N) = Vabar, vbar[N..2N) = Vbbar; nubar = -g Deltabar */
__global__ void k_adj_reduce(const double *slots, int nslots, double *vbar, double2 *nubar)
{
    constexpr int N = WTD_NUMEL;
    int p = threadIdx.x + blockIdx.x * blockDim.x;
    if (p >= N) return;
    double dr = 0.0, di = 0.0, va = 0.0, vb = 0.0;
    for (int k = 0; k < nslots; k++) {
        const double *s = slots + (size_t)k * 4 * N;
        dr += s[2 * p]; di += s[2 * p + 1]; va += s[2 * N + p]; vb += s[3 * N + p];
    }
    const double g = dc_params[WTD_ADJOINT_CONTACT_BDG];
    vbar[p] = va;
    vbar[N + p] = vb;
    nubar[p] = make_double2(-g * dr, -g * di);
}

/* part[j][chunk] = sum over this chunk of the points of (Vabar dv_ext_a/dtheta_j + Vbbar
 * dv_ext_b/dtheta_j) at time index it, the derivative by central differences of the user's
 * v_ext hook with step h = 1e-6 max(1, |theta_j|); grid (parameter, point chunk) */
#define WTD_THETA_CHUNKS 16
__global__ void __launch_bounds__(256) k_theta_grad(const double *vbar, int it, double *part)
{
    constexpr int N = WTD_NUMEL;
    __shared__ double red[80];
    const int j = blockIdx.x;
    double lp[MAX_USER_PARAMS], lm[MAX_USER_PARAMS];
    for (int q = 0; q < MAX_USER_PARAMS; q++) lp[q] = lm[q] = dc_params[q];
    const double h = 1.0e-6 * fmax(1.0, fabs(dc_params[j]));
    lp[j] += h;
    lm[j] -= h;
    const double ih = 1.0 / (lp[j] - lm[j]);
    double acc = 0.0;
    for (int p = threadIdx.x + blockIdx.y * blockDim.x; p < N; p += blockDim.x * gridDim.y) {
        int ix, iy, iz;
        wtd_decode(p, ix, iy, iz);
        const double da = (v_ext(ix, iy, iz, it, SPINA, lp, dc_extra_data_size, dc_extra_data) -
                           v_ext(ix, iy, iz, it, SPINA, lm, dc_extra_data_size, dc_extra_data)) * ih;
        const double db = (v_ext(ix, iy, iz, it, SPINB, lp, dc_extra_data_size, dc_extra_data) -
                           v_ext(ix, iy, iz, it, SPINB, lm, dc_extra_data_size, dc_extra_data)) * ih;
        acc += vbar[p] * da + vbar[N + p] * db;
    }
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) part[j * gridDim.y + blockIdx.y] = acc;
}

/* grad[j] += sum over chunks of part[j][.] (fixed order) */
__global__ void k_theta_sum(const double *part, int nparam, int nchunk, double *grad)
{
    const int j = threadIdx.x;
    if (j >= nparam) return;
    double s = 0.0;
    for (int k = 0; k < nchunk; k++) s += part[j * nchunk + k];
    grad[j] += s;
}

/* L = sum_r |Delta(r)|^2 mask(r) dV of the current potentials and the seed of the reverse
 * sweep, nubar = -g dL/dDelta* = -g 2 Delta mask dV (one CTA) */
__global__ void __launch_bounds__(512) k_adj_loss(const double *pots, const double *mask, double2 *nubar, double *loss)
{
    constexpr int N = WTD_NUMEL;
    __shared__ double red[80];
    const double2 *D = (const double2 *)(pots + 2 * (size_t)N);
    const double g = dc_params[WTD_ADJOINT_CONTACT_BDG], dV = WTD_DV;
    double acc = 0.0;
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        const double m = mask ? mask[p] : 1.0;
        const double2 d = D[p];
        acc += (d.x * d.x + d.y * d.y) * m;
        nubar[p] = make_double2(-g * 2.0 * d.x * m * dV, -g * 2.0 * d.y * m * dV);
    }
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) *loss = acc * dV;
}
#endif

#endif
