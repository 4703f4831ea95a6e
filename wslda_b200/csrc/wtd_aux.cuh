/*
 * O(N) kernels that sit between the two stream passes of a step: second-stage reduction of
 * the density slots, tau from the laplacian of rho, the per-point coefficients H psi reads,
 * and the energy integrals.  All FP64.
 */
#ifndef WTD_AUX_CUH
#define WTD_AUX_CUH

#include "wtd_step.cuh"

/* dens[i] = sum_s slot[s][i] / L_perp over the 12N density words (fixed slot order, so the
 * result is bitwise reproducible).  Limited mode keeps nu, rho_a, rho_b and zeroes the rest,
 * as kernel_calculate_densities_limited does (pca_dens.cu:133-198). */
__global__ void wtd_dens_reduce(const double *slots, int nslots, double *dens, int N, int full, double inv_lperp,
                                size_t stride = 0, int words = 0)
{
    /* words: 12 N, or 16 N with the quantum-friction densities [U_a, U_b, D] after them;
     * stride: slot words per CTA */
    if (!stride) stride = 12 * (size_t)N;
    if (!words) words = 12 * N;
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= words) return;
    int q = (i < 2 * N) ? 0 : 1 + (i - 2 * N) / N; /* 0: nu, 1: rho_a, 2: tau_a, ..., 6: rho_b ... */
    bool needed = full || q == 0 || q == 1 || q == 6 || i >= 12 * N;
    double s = 0.0;
#ifdef SPINSYMMETRY_MODE
    /* spin-symmetric system (pca_dens.cu:55-124, 365-461; symmetrize_densities_device): both
     * spin channels take the sum of the u (f) and v (1 - f) contributions, nu and the friction
     * pairing density D count twice.  The sum is linear, so it is taken here, over the slots,
     * before the exchange between ranks. */
    if (needed) {
        size_t j = (size_t)i;
        double mul = 1.0;
        if (q == 0 || i >= 14 * N) mul = 2.0, j = (size_t)-1;
        else if (i >= 13 * N) j = (size_t)i - N;                /* U_b <- U_a + U_b */
        else if (i >= 12 * N) j = (size_t)i + N;                /* U_a <- U_a + U_b */
        else if (q >= 6) j = (size_t)i - 5 * (size_t)N;          /* b <- a + b */
        else j = (size_t)i + 5 * (size_t)N;                      /* a <- a + b */
        if (j == (size_t)-1)
            for (int k = 0; k < nslots; k++) s += slots[(size_t)k * stride + i];
        else
            for (int k = 0; k < nslots; k++) s += slots[(size_t)k * stride + i] + slots[(size_t)k * stride + j];
        s *= mul;
    }
#else
    if (needed)
        for (int k = 0; k < nslots; k++) s += slots[(size_t)k * stride + i];
#endif
    dens[i] = s * inv_lperp;
}

/* the quantum-friction particle-control coefficient (N - N_req) / N_req, N = volel *
 * sum(rho_a + rho_b), N_req kept >= 1 (pca_utils.c:1063-1072; the reference reads an
 * uninitialised divisor there, this takes the guard it intends) -> out[0] */
__global__ void __launch_bounds__(512) wtd_qf_pccoeff(const double *dens, int N, double volel, double nreq, double *out)
{
    __shared__ double red[80];
    double s = 0.0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) s += dens[2 * (size_t)N + i] + dens[7 * (size_t)N + i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) out[0] = (s * volel - nreq) / (nreq < 1.0 ? 1.0 : nreq);
}

/* the fields H is built from while quantum friction acts (kernel_add_quantum_friction,
 * pca_kernels.cu:497-527), into fld = [V_a, V_b, delta (complex)] without touching the
 * potentials: V_s - U_s qa / nF, delta + qb |delta| e^{i phi} sin(phi - phi_D) + i qg pcc delta */
__global__ void wtd_qf_fields(const double *pots, const double *qfd, const double *pcc, double qa, double qb, double qg,
                              double nF, double *fld, int N)
{
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= N) return;
    const double *Ua = qfd, *Ub = qfd + N;
    const Complex *Dq = (const Complex *)(qfd + 2 * (size_t)N);
    const Complex d0 = ((const Complex *)(pots + 2 * (size_t)N))[i];
    fld[i] = pots[i] - Ua[i] * qa / nF;
    fld[N + i] = pots[N + i] - Ub[i] * qa / nF;
    const double phd = thrust::arg(d0), phn = thrust::arg(Dq[i]);
    Complex d = d0 + qb * thrust::abs(d0) * Complex(cos(phd), sin(phd)) * sin(phd - phn);
    d += Complex(0.0, qg * pcc[0]) * d0;
    ((Complex *)(fld + 2 * (size_t)N))[i] = d;
}

/* ---------------------------------------------------------------------------------------
 * single-CTA spectral operations on O(N) real fields (lattices whose field fits in smem)
 * -------------------------------------------------------------------------------------*/
template <class G>
__device__ __forceinline__ void field_to_smem(double2 *B, const double *f)
{
    for (int p = threadIdx.x; p < G::ntot; p += blockDim.x) B[G::off(p)] = make_double2(f[p], 0.0);
    __syncthreads();
}

/* tau_s = max(0, lap(rho_s)/2 - tau_s)  (pca_dens.cu:275-338); blockIdx.x = spin */
template <class G>
__global__ void __launch_bounds__(512) wtd_tau_kernel(double *dens, const double2 *gtw, const double *gk)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *B = (double2 *)smem_raw;
    double2 *tw = B + G::padded;
    double (*kt)[WTD_KT] = (double (*)[WTD_KT])(tw + G::twtotal);
    load_tables<G>(tw, kt, gtw, gk);
    constexpr int N = G::ntot;
    double *rho = dens + (blockIdx.x == 0 ? 2 : 7) * (size_t)N;
    double *tau = dens + (blockIdx.x == 0 ? 3 : 8) * (size_t)N;
    field_to_smem<G>(B, rho);
    fft_forward<G, 1>(B, 0, tw);
    kmul<G, OP_LAP>(B, kt);
    __syncthreads();
    fft_inverse<G, 1>(B, 0, tw);
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        double t = 0.5 * B[G::off(p)].x - tau[p];
        if (t < 0.0) t = 0.0;
        tau[p] = t;
    }
}

/* per-point coefficients of H psi (see the CF_* list) from the potentials at time index it.
 * Delta includes Delta_ext (pca_kernels.cu:271-276); constant mass uses -alpha/2, variable
 * mass -alpha/4 (pca_kernels.cu:296-309); BdG uses -1/2 (pca_kernels.cu:478-482). */
__global__ void wtd_prep_coef(int it, wslda_potential P, double *cf)
{
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    constexpr int N = WTD_NUMEL;
    if (i >= N) return;
    int ix, iy, iz; wtd_decode(i, ix, iy, iz);
    Complex D = P.delta[i];
#ifdef ENABLE_DELTA_EXT
    D = D + WTD_D_EXT(ix, iy, iz, it, D);
#endif
    cf[CF_VA * N + i] = P.V_a[i] - dc_mu_a;
    cf[CF_VB * N + i] = P.V_b[i] - dc_mu_b;
    cf[CF_DRE * N + i] = D.real();
    cf[CF_DIM * N + i] = D.imag();
#if defined(BDG_MODE) && defined(FAST_CONST_EFFECTIVE_MASS_MODE)
    cf[CF_AA * N + i] = -0.5;
    cf[CF_AB * N + i] = -0.5;
#elif defined(FAST_CONST_EFFECTIVE_MASS_MODE)
    cf[CF_AA * N + i] = P.alpha_a[i] * -0.5;
    cf[CF_AB * N + i] = P.alpha_b[i] * -0.5;
#else
#ifdef BDG_MODE
    /* BdG with a velocity field: -1/2 lap, gradient terms only (pca_kernels.cu:393-495) */
    const double ala = 1.0, alb = 1.0;
    double Aa[3] = {0.0, 0.0, 0.0}, Ab[3] = {0.0, 0.0, 0.0};
#else
    const double ala = P.alpha_a[i], alb = P.alpha_b[i];
    double Aa[3] = {P.A_a_x[i], (CODEDIM >= 2) ? P.A_a_y[i] : 0.0, (CODEDIM >= 3) ? P.A_a_z[i] : 0.0};
    double Ab[3] = {P.A_b_x[i], (CODEDIM >= 2) ? P.A_b_y[i] : 0.0, (CODEDIM >= 3) ? P.A_b_z[i] : 0.0};
#endif
#ifdef ENABLE_VELOCITY_EXT
    /* the external velocity enters as A - v: gradient coefficient i v and +div(v)/2
     * (pca_kernels.cu:315-327, the divergence taken spectrally like div A) */
    for (int d = 0; d < CODEDIM; d++) {
        Aa[d] -= WTD_VEL_EXT(ix, iy, iz, it, SPINA, d);
        Ab[d] -= WTD_VEL_EXT(ix, iy, iz, it, SPINB, d);
    }
#endif
    cf[CF_AA * N + i] = ala * -0.25;
    cf[CF_AB * N + i] = alb * -0.25;
    cf[CF_ALA * N + i] = ala;
    cf[CF_ALB * N + i] = alb;
    cf[CF_AAX * N + i] = Aa[0];
    cf[CF_ABX * N + i] = Ab[0];
    cf[CF_AAY * N + i] = Aa[1];
    cf[CF_ABY * N + i] = Ab[1];
    cf[CF_AAZ * N + i] = Aa[2];
    cf[CF_ABZ * N + i] = Ab[2];
#endif
}

/* variable mass: lap(alpha_s)/4 and -div(A_s)/2 by spectral derivatives of real fields
 * (pca_kernels.cu:778-795; pca_derivative.cu:490-700).  blockIdx.x = spin. */
template <class G>
__global__ void __launch_bounds__(256) wtd_prep_var(double *cf, const double2 *gtw, const double *gk)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *B = (double2 *)smem_raw;
    double2 *tw = B + G::padded;
    double (*kt)[WTD_KT] = (double (*)[WTD_KT])(tw + G::twtotal);
    load_tables<G>(tw, kt, gtw, gk);
    constexpr int N = G::ntot;
    const int s = blockIdx.x;
    /* lap(alpha) */
    field_to_smem<G>(B, cf + (s == 0 ? CF_ALA : CF_ALB) * (size_t)N);
    fft_forward<G, 1>(B, 0, tw);
    kmul<G, OP_LAP>(B, kt);
    __syncthreads();
    fft_inverse<G, 1>(B, 0, tw);
    for (int p = threadIdx.x; p < N; p += blockDim.x) cf[(s == 0 ? CF_NA : CF_NB) * (size_t)N + p] = 0.25 * B[G::off(p)].x;
    __syncthreads();
    /* div A = sum_d d_d A_d */
    double acc[64];
    const int per = (N + blockDim.x - 1) / blockDim.x;
    for (int k = 0; k < per && k < 64; k++) acc[k] = 0.0;
    for (int d = 0; d < G::dims; d++) {
        field_to_smem<G>(B, cf + ((s == 0 ? CF_AAX : CF_ABX) + d) * (size_t)N);
        fft_forward<G, 1>(B, 0, tw);
        if (d == 0) kmul<G, OP_DX>(B, kt);
        else if (d == 1) kmul<G, OP_DY>(B, kt);
        else kmul<G, OP_DZ>(B, kt);
        __syncthreads();
        fft_inverse<G, 1>(B, 0, tw);
        for (int k = 0, p = threadIdx.x; p < N && k < 64; p += blockDim.x, k++) acc[k] += B[G::off(p)].x;
        __syncthreads();
    }
    for (int k = 0, p = threadIdx.x; p < N && k < 64; p += blockDim.x, k++)
        cf[(s == 0 ? CF_CJA : CF_CJB) * (size_t)N + p] = -0.5 * acc[k];
}

/* Fermi-Dirac high-k filter of real fields (high_frequency_filter_d, pca_derivative.cu:784-859;
 * 2D cpca_derivative.cu:709-736, 1D ccpca_derivative.cu:640-662): f -> IFFT[FD(k^2/2) FFT f],
 * FD(e) = 1 / (exp((e - mu) / T) + 1), the Nyquist mode counted with |k| = pi/dx.
 * blockIdx.x = field (consecutive fields of N doubles, filtered in place). */
template <class G>
__global__ void __launch_bounds__(512) wtd_hkf_kernel(double *f, double mu, double T, const double2 *gtw, const double *gk)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *B = (double2 *)smem_raw;
    double2 *tw = B + G::padded;
    double (*kt)[WTD_KT] = (double (*)[WTD_KT])(tw + G::twtotal);
    load_tables<G>(tw, kt, gtw, gk);
    constexpr int N = G::ntot;
    double *a = f + (size_t)blockIdx.x * N;
    field_to_smem<G>(B, a);
    fft_forward<G, 1>(B, 0, tw);
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        int c0, c1 = 0, c2 = 0;
        if (G::dims == 1) { c0 = i; }
        else if (G::dims == 2) { c0 = i / G::N1; c1 = i - c0 * G::N1; }
        else { c0 = i / (G::N1 * G::N2); int r = i - c0 * G::N1 * G::N2; c1 = r / G::N2; c2 = r - c1 * G::N2; }
        double k2 = kt[0][c0] * kt[0][c0];
        if (G::dims >= 2) k2 += kt[1][c1] * kt[1][c1];
        if (G::dims >= 3) k2 += kt[2][c2] * kt[2][c2];
        const double w = 1.0 / (exp((0.5 * k2 - mu) / T) + 1.0) / N;
        const int o = G::off(i);
        B[o].x *= w;
        B[o].y *= w;
    }
    __syncthreads();
    fft_inverse<G, 1>(B, 0, tw);
    for (int p = threadIdx.x; p < N; p += blockDim.x) a[p] = B[G::off(p)].x;
}

/* the same filter of complex fields (high_frequency_filter_c, pca_derivative.cu:861-935) */
template <class G>
__global__ void __launch_bounds__(512) wtd_hkf_c_kernel(const double2 *in, double2 *out, double mu, double T,
                                                        const double2 *gtw, const double *gk)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *B = (double2 *)smem_raw;
    double2 *tw = B + G::padded;
    double (*kt)[WTD_KT] = (double (*)[WTD_KT])(tw + G::twtotal);
    load_tables<G>(tw, kt, gtw, gk);
    constexpr int N = G::ntot;
    for (int p = threadIdx.x; p < N; p += blockDim.x) B[G::off(p)] = in[p];
    __syncthreads();
    fft_forward<G, 1>(B, 0, tw);
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        int c0, c1 = 0, c2 = 0;
        if (G::dims == 1) { c0 = i; }
        else if (G::dims == 2) { c0 = i / G::N1; c1 = i - c0 * G::N1; }
        else { c0 = i / (G::N1 * G::N2); int r = i - c0 * G::N1 * G::N2; c1 = r / G::N2; c2 = r - c1 * G::N2; }
        double k2 = kt[0][c0] * kt[0][c0];
        if (G::dims >= 2) k2 += kt[1][c1] * kt[1][c1];
        if (G::dims >= 3) k2 += kt[2][c2] * kt[2][c2];
        const double w = 1.0 / (exp((0.5 * k2 - mu) / T) + 1.0) / N;
        const int o = G::off(i);
        B[o].x *= w;
        B[o].y *= w;
    }
    __syncthreads();
    fft_inverse<G, 1>(B, 0, tw);
    for (int p = threadIdx.x; p < N; p += blockDim.x) out[p] = B[G::off(p)];
}

/* sum of each of the TDWSLDAITEMS integrand arrays (one CTA per item) */
__global__ void wtd_sum_items(const double *e, int N, double *out, double volel)
{
    __shared__ double red[80];
    double s = 0.0;
    const double *a = e + (size_t)blockIdx.x * N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) s += a[i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) out[blockIdx.x] = (blockIdx.x == NPARTA || blockIdx.x == NPARTB) ? s * volel : s;
}

/* FP64 <-> storage conversion of state arrays */
template <typename T>
__global__ void wtd_convert_in(const double2 *src, T *dst, size_t n)
{
    size_t i = threadIdx.x + (size_t)blockIdx.x * blockDim.x;
    if (i < n) dst[i] = from_d<T>(src[i]);
}
template <typename T>
__global__ void wtd_convert_out(const T *src, double2 *dst, size_t n)
{
    size_t i = threadIdx.x + (size_t)blockIdx.x * blockDim.x;
    if (i < n) dst[i] = to_d(src[i]);
}

#endif
