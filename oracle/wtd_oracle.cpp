/*
 * ORACLE — TEST INFRASTRUCTURE ONLY.
 *
 * CPU (FP64, host C++) restatement of one real-time step of W-SLDA's TD-(A)SLDA/BdG engine,
 * used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg to check and time
 * the CUDA library.  It is never linked into, imported by or called from the product path.
 *
 * Built once per project, like the reference (`make -C oracle PROJECT=<name>`): the project's
 * predefines.h and problem-definition.h are compiled in through oracle_surface.h, so the user
 * hooks (v_ext, delta_ext, scattering_length, CUSTOMEDF kernels) run here unchanged.
 *
 * Every routine restates the reference function cited beside it, in the same arithmetic order
 * where the order matters for rounding (ABM combinations, the 1e4 DENS_FACTOR_M scaling of the
 * density weights).  FFTs are this file's own mixed-radix Cooley-Tukey transform with the
 * cuFFT/FFTW sign convention (forward e^{-2 pi i k n / N}, inverse unnormalised).
 *
 * Parity pins: tests/golden/ holds outputs of the reference's own CUDA kernels
 * (oracle/ref_harness.cu linked against hpc-engine/*.cu) on small seeded cases; the oracle
 * is checked against them in tests/test_oracle_golden.py.
 */
#include "oracle_surface.h"
#include "predefines.h"
#include "wtd_settings.h"
static double dc_params[MAX_USER_PARAMS];
#include "oracle_edf.h"
#include "problem-definition.h"

#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#if defined(ENABLE_V_EXT)
#define ORC_U_EXT(ix, iy, iz, it, spin) v_ext(ix, iy, iz, it, spin, dc_params, dc_extra_data_size, dc_extra_data)
#else
#define ORC_U_EXT(ix, iy, iz, it, spin) 0.0
#endif
#if defined(ENABLE_VELOCITY_EXT)
#define ORC_VEL_EXT(ix, iy, iz, it, spin, ax) velocity_ext(ix, iy, iz, it, spin, ax, dc_params, dc_extra_data_size, dc_extra_data)
#endif
#if defined(ENABLE_DELTA_EXT)
#define ORC_D_EXT(ix, iy, iz, it, d) delta_ext(ix, iy, iz, it, d, dc_params, dc_extra_data_size, dc_extra_data)
#else
#define ORC_D_EXT(ix, iy, iz, it, d) Complex(0.0, 0.0)
#endif

namespace orc {

static const int N = WTD_NUMEL;
static const int AXN[3] = {NX, (CODEDIM >= 2) ? NY : 1, (CODEDIM >= 3) ? NZ : 1};
static const double AXL[3] = {LX, LY, LZ};
static const int NHIST = WTD_NHIST;

static int S = 0;             /* number of (u,v) quasiparticle states */
static int it_global = 0;
static std::vector<Complex> y, fk[5], ddx, ddy, ddz, dlap, dalap;
static std::vector<double> dens, pots, fb, kky, kkz, qpe, work;
static std::vector<int> cnt;
static std::vector<unsigned char> extra;
static int last_gradients = 0;
/* state-sharded runs: sum of the density partials over ranks, after each density reduction
 * (the reference's MPI_Allreduce of the densities, pca.c:948, 1433, 1505) */
typedef int (*exchange_fn)(void *user, double *dens, size_t count);
static exchange_fn xfn = nullptr;
/* quantum friction (input qfalpha, qfbeta, qfgamma, qfNreq and the qfstart/qfstop/qfswitch
 * times in units of 1/eF) and its value in the current step */
static double qf_alpha = 0.0, qf_beta = 0.0, qf_gamma = 0.0, qf_Nreq = 0.0, qf_start = 0.0, qf_stop = 0.0, qf_ramp = 0.0;
static double qfsw = 0.0, pccoeff = 0.0;
static void *xuser = nullptr;
static void exchange_densities()
{
    if (xfn) xfn(xuser, dens.data(), dens.size());
}

/* point coordinates of linear index i (pca_macro.h:134-160) */
static inline void decode(int i, int &ix, int &iy, int &iz)
{
#if CODEDIM == 3
    ix = i / (NY * NZ); int r = i - ix * NY * NZ; iy = r / NZ; iz = r - iy * NZ;
#elif CODEDIM == 2
    ix = i / NY; iy = i - ix * NY; iz = 0;
#else
    ix = i; iy = 0; iz = 0;
#endif
}

/* ----------------------------------------------------------------------------------------
 * FFT: recursive mixed-radix decimation in time, radices 4, 2, 3, then generic DFT.
 * sign = -1 forward, +1 inverse (unnormalised), as cuFFT CUFFT_FORWARD / CUFFT_INVERSE.
 * --------------------------------------------------------------------------------------*/
struct Plan1D {
    int n = 0;
    std::vector<Complex> wf, wi; /* e^{-2 pi i j/n}, e^{+2 pi i j/n} */
};
static Plan1D plans[3];

static void make_plan(Plan1D &p, int n)
{
    p.n = n;
    p.wf.resize(n); p.wi.resize(n);
    for (int j = 0; j < n; j++) {
        /* exact symmetric angle reduction keeps the table to libm accuracy */
        long double a = 2.0L * (long double)M_PI * (long double)j / (long double)n;
        double c = (double)std::cos(a), s = (double)std::sin(a);
        p.wf[j] = Complex(c, -s);
        p.wi[j] = Complex(c, s);
    }
}

static void fft_rec(const Complex *in, Complex *out, int n, int stride, const Complex *w, int wstep)
{
    if (n == 1) { out[0] = in[0]; return; }
    int r = (n % 4 == 0) ? 4 : (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : n;
    int m = n / r;
    if (r == n) { /* generic DFT */
        for (int k = 0; k < n; k++) {
            Complex s(0.0, 0.0);
            for (int q = 0; q < n; q++) s += in[q * stride] * w[((long)q * k % n) * wstep];
            out[k] = s;
        }
        return;
    }
    for (int q = 0; q < r; q++) fft_rec(in + q * stride, out + q * m, m, stride * r, w, wstep * r);
    Complex t[4];
    std::vector<Complex> tmp(n);
    for (int k = 0; k < m; k++) {
        for (int q = 0; q < r; q++) t[q] = out[q * m + k] * w[(long)q * k * wstep];
        for (int j = 0; j < r; j++) {
            Complex s(0.0, 0.0);
            for (int q = 0; q < r; q++) s += t[q] * w[((long)q * j * m % n) * wstep];
            tmp[k + j * m] = s;
        }
    }
    for (int i = 0; i < n; i++) out[i] = tmp[i];
}

/* in-place FFT of one lattice field (row-major, x slowest) along every lattice axis */
static void fftn(Complex *a, int sign)
{
    std::vector<Complex> line, res;
    int dims = CODEDIM;
    for (int ax = 0; ax < dims; ax++) {
        int n = AXN[ax];
        if (n == 1) continue;
        int inner = 1;
        for (int b = ax + 1; b < dims; b++) inner *= AXN[b];
        int outer = N / (n * inner);
        line.resize(n); res.resize(n);
        const Complex *w = (sign < 0) ? plans[ax].wf.data() : plans[ax].wi.data();
        for (int o = 0; o < outer; o++)
            for (int in = 0; in < inner; in++) {
                Complex *base = a + (size_t)o * n * inner + in;
                for (int j = 0; j < n; j++) line[j] = base[(size_t)j * inner];
                fft_rec(line.data(), res.data(), n, 1, w, 1);
                for (int j = 0; j < n; j++) base[(size_t)j * inner] = res[j];
            }
    }
}

/* wave number of index i on axis ax (pca_derivative.cu:152-160) */
static inline double kval(int ax, int i)
{
    int n = AXN[ax];
    return (i < n / 2) ? 2. * M_PI / AXL[ax] * (double)i : 2. * M_PI / AXL[ax] * (double)(i - n);
}

#ifdef ORACLE_WDERIV
/* Host-core baseline build (make -C oracle wderiv): the spectral derivatives of the states come
 * from the reference's own CPU library, lib/wderiv/c/wderiv.c, compiled unmodified over the
 * FFTW3-API shim of oracle/fftw_shim (FFTW is not installed).  wderiv_*_c take C99 double
 * complex arrays, which have std::complex<double>'s layout. */
extern "C" {
int wderiv_init_3d(int nx, int ny, int nz, double dx, double dy, double dz);
int wderiv_init_2d(int nx, int ny, double dx, double dy);
int wderiv_init_1d(int nx, double dx);
int wderiv_gradient_3d_c(void *f, void *dfdx, void *dfdy, void *dfdz);
int wderiv_gradient_2d_c(void *f, void *dfdx, void *dfdy);
int wderiv_gradient_1d_c(void *f, void *dfdx);
int wderiv_laplace_3d_c(void *f, void *laplace);
int wderiv_laplace_2d_c(void *f, void *laplace);
int wderiv_laplace_1d_c(void *f, void *laplace);
int wderiv_dfdx_3d_c(void *f, void *d);
int wderiv_dfdy_3d_c(void *f, void *d);
int wderiv_dfdz_3d_c(void *f, void *d);
int wderiv_dfdx_2d_c(void *f, void *d);
int wderiv_dfdy_2d_c(void *f, void *d);
int wderiv_dfdx_1d_c(void *f, void *d);
}
static int wderiv_ready = [] {
#if CODEDIM == 3
    return wderiv_init_3d(NX, NY, NZ, DX, DY, DZ);
#elif CODEDIM == 2
    return wderiv_init_2d(NX, NY, DX, DY);
#else
    return wderiv_init_1d(NX, DX);
#endif
}();

/* compute_derivatives for one complex field through wderiv: d/dx_d (odd derivative, Nyquist
 * mode zeroed) and the laplacian as the sum of the second derivatives, each 1/N normalised
 * (wderiv.c:503-567, the same multipliers as pca_derivative.cu:139-277) */
static void derivs_one(const Complex *f, Complex *dx, Complex *dy, Complex *dz, Complex *lap)
{
    (void)wderiv_ready;
    void *in = (void *)f;
#if CODEDIM == 3
    if (dx) wderiv_dfdx_3d_c(in, dx);
    if (dy) wderiv_dfdy_3d_c(in, dy);
    if (dz) wderiv_dfdz_3d_c(in, dz);
    if (lap) wderiv_laplace_3d_c(in, lap);
#elif CODEDIM == 2
    (void)dz;
    if (dx) wderiv_dfdx_2d_c(in, dx);
    if (dy) wderiv_dfdy_2d_c(in, dy);
    if (lap) wderiv_laplace_2d_c(in, lap);
#else
    (void)dy; (void)dz;
    if (dx) wderiv_dfdx_1d_c(in, dx);
    if (lap) wderiv_laplace_1d_c(in, lap);
#endif
}
#else
/* compute_derivatives for one complex field (pca_derivative.cu:139-277): d/dx_d with the
 * Nyquist mode zeroed, laplacian without; 1/N folded into the k factors. Any output may be
 * null. */
static void derivs_one(const Complex *f, Complex *dx, Complex *dy, Complex *dz, Complex *lap)
{
    std::vector<Complex> F(f, f + N);
    fftn(F.data(), -1);
    Complex *outs[3] = {dx, dy, dz};
    std::vector<Complex> G(N);
    for (int d = 0; d < CODEDIM; d++) {
        if (!outs[d]) continue;
        for (int i = 0; i < N; i++) {
            int c[3]; decode(i, c[0], c[1], c[2]);
            double k = kval(d, c[d]) / N;
            if (c[d] == AXN[d] / 2) k = 0.0;
            G[i] = Complex(-k * F[i].imag(), k * F[i].real());
        }
        fftn(G.data(), +1);
        std::copy(G.begin(), G.end(), outs[d]);
    }
    if (lap) {
        for (int i = 0; i < N; i++) {
            int c[3]; decode(i, c[0], c[1], c[2]);
            double k2 = 0.0;
            for (int d = 0; d < CODEDIM; d++) { double k = kval(d, c[d]); k2 += k * k; }
            k2 = -1.0 * k2 / N;
            G[i] = Complex(k2 * F[i].real(), k2 * F[i].imag());
        }
        fftn(G.data(), +1);
        std::copy(G.begin(), G.end(), lap);
    }
}
#endif

/* laplacian / d f_d/dx_d of real fields (pca_derivative.cu:490-700, D2Z/Z2D); the complex
 * transform of a real field gives the same real result. */
static void lap_real(const double *f, double *out)
{
    std::vector<Complex> F(N), L(N);
    for (int i = 0; i < N; i++) F[i] = Complex(f[i], 0.0);
    derivs_one(F.data(), nullptr, nullptr, nullptr, L.data());
    for (int i = 0; i < N; i++) out[i] = L[i].real();
}
/* high_frequency_filter_d (pca_derivative.cu:784-859; cpca_derivative.cu:709-736;
 * ccpca_derivative.cu:640-662): f -> IFFT[FD(k^2/2) FFT f] / N with FD(e) = 1/(exp((e-mu)/T)+1),
 * k of index i as kval (the Nyquist mode counted with k = -pi/dx) */
static int hkf_mode = 0;
static double hkf_mu = 0.0, hkf_T = 1.0;
static void high_k_filter(double *f)
{
    std::vector<Complex> F(N);
    for (int i = 0; i < N; i++) F[i] = Complex(f[i], 0.0);
    fftn(F.data(), -1);
    for (int i = 0; i < N; i++) {
        int c[3]; decode(i, c[0], c[1], c[2]);
        double k2 = 0.0;
        for (int d = 0; d < CODEDIM; d++) { double k = kval(d, c[d]); k2 += k * k; }
        const double w = 1.0 / (std::exp((0.5 * k2 - hkf_mu) / hkf_T) + 1.0) / N;
        F[i] *= w;
    }
    fftn(F.data(), +1);
    for (int i = 0; i < N; i++) f[i] = F[i].real();
}
/* high_frequency_filter_c (pca_derivative.cu:861-935): the same filter of a complex field */
static void high_k_filter_c(Complex *f)
{
    std::vector<Complex> F(f, f + N);
    fftn(F.data(), -1);
    for (int i = 0; i < N; i++) {
        int c[3]; decode(i, c[0], c[1], c[2]);
        double k2 = 0.0;
        for (int d = 0; d < CODEDIM; d++) { double k = kval(d, c[d]); k2 += k * k; }
        F[i] *= 1.0 / (std::exp((0.5 * k2 - hkf_mu) / hkf_T) + 1.0) / N;
    }
    fftn(F.data(), +1);
    std::copy(F.begin(), F.end(), f);
}
static void dcomp_real(const double *f, int d, double *out)
{
    std::vector<Complex> F(N), D(N);
    for (int i = 0; i < N; i++) F[i] = Complex(f[i], 0.0);
    Complex *o[3] = {nullptr, nullptr, nullptr};
    o[d] = D.data();
    derivs_one(F.data(), o[0], o[1], o[2], nullptr);
    for (int i = 0; i < N; i++) out[i] = D[i].real();
}

/* ---------------------------------------------------------------------------------------
 * field views
 * -------------------------------------------------------------------------------------*/
static inline Complex *U(std::vector<Complex> &a, int n) { return a.data() + (size_t)n * N; }
static inline Complex *V(std::vector<Complex> &a, int n) { return a.data() + (size_t)S * N + (size_t)n * N; }
static wslda_density dens_view(double *d)
{
    wslda_density r;
    r.nx = NX; r.ny = AXN[1]; r.nz = AXN[2]; r.datadim = CODEDIM; r.blocklength = N;
    r.nu = (Complex *)d;
    r.rho_a = d + 2 * N; r.tau_a = d + 3 * N; r.j_a_x = d + 4 * N; r.j_a_y = d + 5 * N; r.j_a_z = d + 6 * N;
    r.rho_b = d + 7 * N; r.tau_b = d + 8 * N; r.j_b_x = d + 9 * N; r.j_b_y = d + 10 * N; r.j_b_z = d + 11 * N;
    return r;
}
static wslda_potential pots_view(double *d)
{
    wslda_potential r;
    r.nx = NX; r.ny = AXN[1]; r.nz = AXN[2]; r.datadim = CODEDIM; r.blocklength = N;
    r.V_a = d; r.V_b = d + N; r.delta = (Complex *)(d + 2 * N); r.alpha_a = d + 4 * N; r.alpha_b = d + 5 * N;
    r.A_a_x = d + 6 * N; r.A_a_y = d + 7 * N; r.A_a_z = d + 8 * N;
    r.A_b_x = d + 9 * N; r.A_b_y = d + 10 * N; r.A_b_z = d + 11 * N;
    r.mu = nullptr;
    return r;
}

/* ---------------------------------------------------------------------------------------
 * ABM predictor / corrector (tdwslda_ode_integrator.h:26-220)
 * -------------------------------------------------------------------------------------*/
static void abm_step1(Complex *yv, Complex *f1, Complex *f2, Complex *f3, Complex *f4, Complex *f5)
{
    const Complex dti(0.0, -1.0 * dc_dt);
    const size_t M = (size_t)2 * S * N;
#pragma omp parallel for
    for (long i = 0; i < (long)M; i++) {
        Complex y0 = yv[i];
#if INTEGRATION_SCHEME == AB3AM4
        Complex a = f1[i], b = f2[i], c = f3[i];
        yv[i] = y0 + dti * (a * (23. / 12.) - b * (16. / 12.) + c * (5. / 12.));
        f3[i] = y0 + dti * (a * (19. / 24.) - b * (5. / 24.) + c * (1. / 24.));
#elif INTEGRATION_SCHEME == AB4AM5
        Complex a = f1[i], b = f2[i], c = f3[i], d = f4[i];
        yv[i] = y0 + dti * (a * (55. / 24.) - b * (59. / 24.) + c * (37. / 24.) - d * (9. / 24.));
        f4[i] = y0 + dti * (a * (646. / 720.) - b * (264. / 720.) + c * (106. / 720.) - d * (19. / 720.));
#else
        Complex a = f1[i], b = f2[i], c = f3[i], d = f4[i], e = f5[i];
        yv[i] = y0 + dti * (a * (1901. / 720.) - b * (2774. / 720.) + c * (2616. / 720.) - d * (1274. / 720.) + e * (251. / 720.));
        f5[i] = y0 + dti * (a * (646. / 720.) - b * (264. / 720.) + c * (106. / 720.) - d * (19. / 720.));
#endif
    }
}
static void abm_step4(const Complex *hy, Complex *yout, const Complex *flast)
{
    const Complex dti(0.0, -1.0 * dc_dt);
#if INTEGRATION_SCHEME == AB3AM4
    const double c = 9. / 24.;
#else
    const double c = 251. / 720.;
#endif
    const size_t M = (size_t)2 * S * N;
#pragma omp parallel for
    for (long i = 0; i < (long)M; i++) yout[i] = dti * hy[i] * c + flast[i];
}

/* normalize_wf (pca_kernels.cu:913-976): psi_n /= sqrt(sum_x (|u|^2+|v|^2) dV) */
static void normalize(std::vector<Complex> &w)
{
#pragma omp parallel for
    for (int n = 0; n < S; n++) {
        Complex *u = U(w, n), *v = V(w, n);
        double s = 0.0;
        for (int i = 0; i < N; i++) s += (std::norm(u[i]) + std::norm(v[i])) * WTD_DV;
        double c = 1.0 / std::sqrt(s);
        for (int i = 0; i < N; i++) { u[i] *= c; v[i] *= c; }
    }
}

/* derivatives of all 2S component fields (compute_derivatives / compute_laplace) */
static void derivatives(std::vector<Complex> &w, int grads)
{
#pragma omp parallel for schedule(dynamic)
    for (long m = 0; m < 2L * S; m++) {
        size_t o = (size_t)m * N;
        if (grads)
            derivs_one(w.data() + o, ddx.data() + o, CODEDIM >= 2 ? ddy.data() + o : nullptr,
                       CODEDIM >= 3 ? ddz.data() + o : nullptr, dlap.data() + o);
        else
            derivs_one(w.data() + o, nullptr, nullptr, nullptr, dlap.data() + o);
    }
}

/* calculate_densities (pca_dens.cu:13-198; cpca_dens.cu:14-140; ccpca_dens.cu:14-140) */
static void calculate_densities(std::vector<Complex> &w, int grads, const double *weights = nullptr,
                                double *into = nullptr)
{
    /* weights: per-state factors of the subset densities (pca_dens.cu:46-47), into: output */
    wslda_density D = dens_view(into ? into : dens.data());
    const double DF = 10000.;
#pragma omp parallel for
    for (int i = 0; i < N; i++) {
        double na = 0, nb = 0, taua = 0, taub = 0, jax = 0, jay = 0, jaz = 0, jbx = 0, jby = 0, jbz = 0;
        Complex nu(0.0, 0.0);
        for (int n = 0; n < S; n++) {
            double fbEn = fb[n] * DF, fbmEn = DF - fbEn;
            if (weights) { fbEn *= weights[n]; fbmEn *= weights[n]; }
            double wcnt = 1.0, kp2 = 0.0;
#if CODEDIM == 2
            double kz = kkz[n];
            kp2 = kz * kz;
            wcnt = (std::fabs(kz) < 1.0e-12) ? 1.0 : 2.0;
#ifdef USE_CUBIC_CUTOFF
            if (std::fabs(kz + M_PI / DZ) < 1.0e-12) wcnt = 1.0;
#endif
#elif CODEDIM == 1
            kp2 = kkz[n] * kkz[n] + kky[n] * kky[n];
            wcnt = (double)cnt[n];
#endif
            Complex u = U(w, n)[i], v = V(w, n)[i];
#ifdef SPINSYMMETRY_MODE
            /* spin-symmetric system (pca_dens.cu:55-62): the u and v contributions go to one
             * channel, taken for both spins below; nu without the factor 1/2 */
            nb += (std::norm(v) * fbmEn + std::norm(u) * fbEn) * wcnt;
            nu += u * std::conj(v) * (fbmEn - fbEn) * wcnt;
            double &tu = taub, &jux = jbx, &juy = jby, &juz = jbz;
#else
            na += std::norm(u) * fbEn * wcnt;
            nb += std::norm(v) * fbmEn * wcnt;
            nu += u * std::conj(v) * (fbmEn - fbEn) / 2.0 * wcnt;
            double &tu = taua, &jux = jax, &juy = jay, &juz = jaz;
#endif
            (void)juy; (void)juz;
            if (grads) {
                Complex lu = U(dlap, n)[i], lv = V(dlap, n)[i];
                tu += (std::conj(u) * (lu - u * kp2)).real() * fbEn * wcnt;
                taub += (std::conj(v) * (lv - v * kp2)).real() * fbmEn * wcnt;
                jux += (std::conj(u) * U(ddx, n)[i]).imag() * fbEn * wcnt;
                jbx -= (std::conj(v) * V(ddx, n)[i]).imag() * fbmEn * wcnt;
#if CODEDIM >= 2
                juy += (std::conj(u) * U(ddy, n)[i]).imag() * fbEn * wcnt;
                jby -= (std::conj(v) * V(ddy, n)[i]).imag() * fbmEn * wcnt;
#endif
#if CODEDIM >= 3
                juz += (std::conj(u) * U(ddz, n)[i]).imag() * fbEn * wcnt;
                jbz -= (std::conj(v) * V(ddz, n)[i]).imag() * fbmEn * wcnt;
#endif
            }
        }
#ifdef SPINSYMMETRY_MODE
        na = nb; taua = taub; jax = jbx; jay = jby; jaz = jbz;
#endif
        const double L = WTD_LPERP;
        D.rho_a[i] = na / DF / L; D.rho_b[i] = nb / DF / L;
        D.tau_a[i] = taua / DF / L; D.tau_b[i] = taub / DF / L;
        D.nu[i] = nu / DF / L;
        D.j_a_x[i] = jax / DF / L; D.j_a_y[i] = jay / DF / L; D.j_a_z[i] = jaz / DF / L;
        D.j_b_x[i] = jbx / DF / L; D.j_b_y[i] = jby / DF / L; D.j_b_z[i] = jbz / DF / L;
    }
}

/* calculate_quantum_friction_densities (pca_dens.cu:365-461; cpca_dens.cu:385-450, ccpca with
 * |k_perp|^2 and the degeneracy weight): U_a = sum f Im[u* lap u], U_b = -sum (1-f) Im[v* lap v],
 * D = -1/2 sum (1-2f) [v* lap u + (lap v)* u], lap including -|k_perp|^2, divided by L_perp;
 * stored after the 12 N densities as [U_a, U_b, D (complex)] */
static void calculate_qf_densities(std::vector<Complex> &w)
{
    double *Ua = dens.data() + 12 * (size_t)N, *Ub = Ua + N;
    Complex *Dq = (Complex *)(Ua + 2 * (size_t)N);
#pragma omp parallel for
    for (int i = 0; i < N; i++) {
        double ua = 0.0, ub = 0.0;
        Complex d(0.0, 0.0);
        for (int n = 0; n < S; n++) {
            double f = fb[n], fm = 1.0 - f, wcnt = 1.0, kp2 = 0.0;
#if CODEDIM == 2
            kp2 = kkz[n] * kkz[n];
            wcnt = (std::fabs(kkz[n]) < 1.0e-12) ? 1.0 : 2.0;
#elif CODEDIM == 1
            kp2 = kkz[n] * kkz[n] + kky[n] * kky[n];
            wcnt = (double)cnt[n];
#endif
            Complex u = U(w, n)[i], v = V(w, n)[i];
            Complex lu = U(dlap, n)[i] - u * kp2, lv = V(dlap, n)[i] - v * kp2;
#ifdef SPINSYMMETRY_MODE
            /* pca_dens.cu:411-414 */
            ub += ((std::conj(u) * lu).imag() * f - (std::conj(v) * lv).imag() * fm) * wcnt;
            d += (std::conj(v) * lu + std::conj(lv) * u) * (fm - f) * wcnt * 2.0;
#else
            ua += (std::conj(u) * lu).imag() * f * wcnt;
            ub -= (std::conj(v) * lv).imag() * fm * wcnt;
            d += (std::conj(v) * lu + std::conj(lv) * u) * (fm - f) * wcnt;
#endif
        }
#ifdef SPINSYMMETRY_MODE
        ua = ub;
#endif
        const double L = WTD_LPERP;
        Ua[i] = ua / L;
        Ub[i] = ub / L;
        Dq[i] = -0.5 * d / L;
    }
}

/* the smooth switch of the friction (pca_utils.c:779-790): 0 outside (start, stop), 1 inside
 * (start + ramp, stop - ramp), (1 + tanh(tan(pi/2 (2 s/ramp - 1))))/2 on the ramps */
static double smooth_ramp(double s, double ramp) { return 0.5 * (1.0 + std::tanh(std::tan(M_PI_2 * (2.0 * s / ramp - 1.0)))); }
static double smooth_step(double t, double a, double b, double ramp)
{
    if (t <= a || t >= b) return 0.0;
    if (t >= a + ramp && t <= b - ramp) return 1.0;
    if (t > a && t < a + ramp) return smooth_ramp(t - a, ramp);
    return 1.0 - smooth_ramp(t - b + ramp, ramp);
}
static double qf_switch(double t)
{
    if (qf_alpha == 0.0 && qf_beta == 0.0 && qf_gamma == 0.0) return 0.0;
    return smooth_step(t, qf_start / dc_eF, qf_stop / dc_eF, qf_ramp / dc_eF);
}
/* particle-number control coefficient (N - N_req) / N_req with N_req kept >= 1 (the reference
 * intends this guard, pca_utils.c:1063-1072, but reads an uninitialised variable) */
static double qf_pccoeff()
{
    wslda_density D = dens_view(dens.data());
    double n = 0.0;
    for (int i = 0; i < N; i++) n += D.rho_a[i];
    for (int i = 0; i < N; i++) n += D.rho_b[i];
    n *= WTD_VOLEL;
    const double req = qf_Nreq < 1.0 ? 1.0 : qf_Nreq;
    return (n - qf_Nreq) / req;
}

/* density_caculate_tau (pca_dens.cu:275-338): tau = max(0, lap(rho)/2 - tau_tmp) */
static void density_tau(double *into = nullptr)
{
    wslda_density D = dens_view(into ? into : dens.data());
    std::vector<double> lr(N);
    double *rho[2] = {D.rho_b, D.rho_a}, *tau[2] = {D.tau_b, D.tau_a};
    for (int s = 0; s < 2; s++) {
        lap_real(rho[s], lr.data());
        for (int i = 0; i < N; i++) {
            double t = 0.5 * lr[i] - tau[s][i];
            if (t < 0.0) t = 0.0;
            tau[s][i] = t;
        }
    }
}

/* ---------------------------------------------------------------------------------------
 * compute_potentials (pca_kernels.cu:81-94 -> tdwslda_functionals.h)
 * -------------------------------------------------------------------------------------*/
#if FUNCTIONAL == SLDA || FUNCTIONAL == ASLDA
/* tdwslda_functionals.h:47-306 */
static void potentials_point(int it, int i, wslda_density Dn, wslda_potential P, double cccoeff)
{
    using namespace oedf;
    int ix, iy, iz; decode(i, ix, iy, iz);
    double Va_const = ORC_U_EXT(ix, iy, iz, it, SPINA);
    double Vb_const = ORC_U_EXT(ix, iy, iz, it, SPINB);
    double na = Dn.rho_a[i], nb = Dn.rho_b[i];
    double t1 = pol(na, nb);
    double aplus = alpha_plus(t1);
    double dam_a, dam_b, dap_a, dap_b;
#ifdef CURRENT_CORRECTIONS
    double aminus = alpha_minus(t1);
    double t2 = alpha(t1), t3 = alpha(-t1);
    P.alpha_a[i] = t2; P.alpha_b[i] = t3;
    double *Aa[3] = {P.A_a_x, P.A_a_y, P.A_a_z}, *Ab[3] = {P.A_b_x, P.A_b_y, P.A_b_z};
    double *ja[3] = {Dn.j_a_x, Dn.j_a_y, Dn.j_a_z}, *jb[3] = {Dn.j_b_x, Dn.j_b_y, Dn.j_b_z};
    double t4 = p_reg(na) * cccoeff;
    for (int d = 0; d < CODEDIM; d++) Aa[d][i] = (t4 == 0.0) ? 0.0 : t4 * (1. - t2) * ja[d][i] / na;
    t4 = p_reg(nb) * cccoeff;
    for (int d = 0; d < CODEDIM; d++) Ab[d][i] = (t4 == 0.0) ? 0.0 : t4 * (1. - t3) * jb[d][i] / nb;
#endif
#ifdef FAST_CONST_EFFECTIVE_MASS_MODE
    dam_a = dam_b = dap_a = dap_b = 0.0;
#else
    {
        double ta = Dn.tau_a[i], tb = Dn.tau_b[i];
        double tm = ta - tb;
        dam_a = oedf::dam_da(na, nb); dam_b = oedf::dam_db(na, nb);
        Va_const += dam_a * tm / 2.0; Vb_const += dam_b * tm / 2.0;
        double tp = ta + tb;
        dap_a = oedf::dap_da(na, nb); dap_b = oedf::dap_db(na, nb);
        Va_const += dap_a * tp / 2.0; Vb_const += dap_b * tp / 2.0;
    }
#endif
    Va_const += dD_da(na, nb);
    Vb_const += dD_db(na, nb);
#ifdef CURRENT_CORRECTIONS
    {
        double jx = Dn.j_a_x[i], kx = Dn.j_b_x[i];
        double jy = (CODEDIM >= 2) ? Dn.j_a_y[i] : 0.0, ky = (CODEDIM >= 2) ? Dn.j_b_y[i] : 0.0;
        double jz = (CODEDIM >= 3) ? Dn.j_a_z[i] : 0.0, kz = (CODEDIM >= 3) ? Dn.j_b_z[i] : 0.0;
        double t7 = p_reg(na) * cccoeff;
        if (t7 != 0.0) {
            t7 = t7 * (jx * jx + jy * jy + jz * jz) / (2.0 * na);
            Va_const += ((aplus + aminus - 1.0) / na - (dap_a + dam_a)) * t7;
            Va_const -= cccoeff * dp_reg(na) * (aplus + aminus - 1.0) * (jx * jx + jy * jy + jz * jz) / (2.0 * na);
            Vb_const -= (dap_b + dam_b) * t7;
        }
        t7 = p_reg(nb) * cccoeff;
        if (t7 != 0.0) {
            t7 = t7 * (kx * kx + ky * ky + kz * kz) / (2.0 * nb);
            Va_const -= (dap_a - dam_a) * t7;
            Vb_const += ((aplus - aminus - 1.0) / nb - (dap_b - dam_b)) * t7;
            Vb_const -= cccoeff * dp_reg(nb) * (aplus - aminus - 1.0) * (kx * kx + ky * ky + kz * kz) / (2.0 * nb);
        }
    }
#endif
    double c1 = dap_a / aplus, c2 = dap_b / aplus;
    double c3 = dtC_da(na, nb) / aplus, c4 = dtC_db(na, nb) / aplus;
    double tC = tildeC(na, nb);
    double Va = P.V_a[i], Vb = P.V_b[i];
    Complex lnu = Dn.nu[i], ldelta(0.0, 0.0), Zone(1.0, 0.0), p0, kc, wz;
#ifdef INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
    double lkF = std::pow(3.0 * M_PI * M_PI * (na + nb), 1.0 / 3.0);
#endif
    for (int k = 0; k < UD_SCITERS; k++) {
        double t7 = (dc_mu_a - Va + dc_mu_b - Vb) / 2.0;
        p0 = std::sqrt(Complex(2.0 * t7 / aplus, 0.0));
        if (p0.imag() < 0.) p0 *= -1.;
#ifdef USE_CUBIC_CUTOFF
        kc = Complex(M_PI / DX, 0.0);
#else
        kc = std::sqrt(Complex(2.0 * (dc_ec + t7) / aplus, 0.0));
        if (kc.imag() < 0.) kc *= -1.;
#endif
        wz = std::log((kc + p0) / (kc - p0));
        if (wz.imag() < 0.) wz += Complex(0.0, 2. * M_PI);
        wz = kc * REG_COEFF_R0 * (1. - (p0 / kc) * REG_COEFF_R1 * wz);
        wz = Zone * aplus / (Zone * tC - wz);
        ldelta = lnu * (-1.0 * wz.real());
        double t6 = (std::conj(ldelta) * lnu).real();
        double tn = std::norm(ldelta);
        double Vanew = Va_const - c1 * t6 - c3 * tn;
        double Vbnew = Vb_const - c2 * t6 - c4 * tn;
#ifdef INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
        {
            double bcoeff = (p0 / (lkF + 1.0e-12)).real();
            double lx = bcoeff * lkF * DX / M_PI;
            if (wz.real() < -1.0e-10 && lx > 1.0e-10) {
                double L0 = bcoeff * REG_COEFF_R0 / lx * (1.0 - REG_COEFF_R1 * lx * std::log((1.0 + lx) / (1.0 - lx)));
                double dL0 = (-2. * bcoeff * REG_COEFF_R0 * REG_COEFF_R1) / (1. - lx * lx) - bcoeff * REG_COEFF_R0 / lx / lx;
                double dLdn = (lkF / (3. * (na + nb) * aplus)) * (L0 + dL0 * bcoeff * DX * lkF / M_PI);
                Vanew += dLdn * tn;
                Vbnew += dLdn * tn;
            }
        }
#endif
        Va = UD_MIX_COEFF * Vanew + (1.0 - UD_MIX_COEFF) * Va;
        Vb = UD_MIX_COEFF * Vbnew + (1.0 - UD_MIX_COEFF) * Vb;
    }
    P.V_a[i] = Va; P.V_b[i] = Vb; P.delta[i] = ldelta;
}
#elif FUNCTIONAL == BDG
/* tdwslda_functionals.h:373-452 */
static void potentials_point(int it, int i, wslda_density Dn, wslda_potential P, double cccoeff)
{
    int ix, iy, iz; decode(i, ix, iy, iz);
    double Va = ORC_U_EXT(ix, iy, iz, it, SPINA);
    double Vb = ORC_U_EXT(ix, iy, iz, it, SPINB);
    double aplus = 0.5 * (P.alpha_a[i] + P.alpha_b[i]);
    double t5 = 1.0 / (4.0 * M_PI * scattering_length(ix, iy, iz, it, dc_params, dc_extra_data_size, dc_extra_data) * aplus);
    Complex lnu = Dn.nu[i], Zone(1.0, 0.0), p0, kc, wz;
#ifdef INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
    double nab = Dn.rho_a[i] + Dn.rho_b[i];
    double lkF = std::pow(3.0 * M_PI * M_PI * nab, 1.0 / 3.0);
#endif
    double t7 = (dc_mu_a - P.V_a[i] + dc_mu_b - P.V_b[i]) / 2.0;
    p0 = std::sqrt(Complex(2.0 * t7, 0.0));
    if (p0.imag() < 0.) p0 *= -1.;
#ifdef USE_CUBIC_CUTOFF
    kc = Complex(M_PI / DX, 0.0);
#else
    kc = std::sqrt(Complex(2.0 * (dc_ec + t7), 0.0));
    if (kc.imag() < 0.) kc *= -1.;
#endif
    wz = std::log((kc + p0) / (kc - p0));
    if (wz.imag() < 0.) wz += Complex(0.0, 2. * M_PI);
    wz = kc * REG_COEFF_R0 / aplus * (1. - (p0 / kc) * REG_COEFF_R1 * wz);
    wz = Zone / (Zone * t5 - wz);
    Complex ldelta = lnu * (-1.0 * wz.real());
#ifdef INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
    {
        double bcoeff = (p0 / (lkF + 1.0e-12)).real();
        double lx = bcoeff * lkF * DX / M_PI;
        if (wz.real() < -1.0e-10 && lx > 1.0e-10) {
            double L0 = bcoeff * REG_COEFF_R0 / lx * (1.0 - REG_COEFF_R1 * lx * std::log((1.0 + lx) / (1.0 - lx)));
            double dL0 = (-2. * bcoeff * REG_COEFF_R0 * REG_COEFF_R1) / (1. - lx * lx) - bcoeff * REG_COEFF_R0 / lx / lx;
            double dLdn = (lkF / (3. * nab * aplus)) * (L0 + dL0 * bcoeff * DX * lkF / M_PI);
            double tn = std::norm(ldelta);
            Va += dLdn * tn;
            Vb += dLdn * tn;
        }
    }
#endif
    P.V_a[i] = Va; P.V_b[i] = Vb; P.delta[i] = ldelta;
}
#elif FUNCTIONAL == SLDAE
/* tdwslda_functionals.h:530-812 */
static void potentials_point(int it, int i, wslda_density Dn, wslda_potential P, double cccoeff)
{
    using namespace oedf;
    using namespace osldae;
    int ix, iy, iz; decode(i, ix, iy, iz);
    double Va_const = ORC_U_EXT(ix, iy, iz, it, SPINA);
    double Vb_const = ORC_U_EXT(ix, iy, iz, it, SPINB);
    double na = Dn.rho_a[i], nb = Dn.rho_b[i];
    double taua = Dn.tau_a[i], taub = Dn.tau_b[i];
    Complex lnu = Dn.nu[i];
    double Va = P.V_a[i], Vb = P.V_b[i];
    Complex ldelta = P.delta[i];
    double nt = na + nb;
    double nt_1o3 = std::pow(nt, 1. / 3.), nt_2o3 = std::pow(nt, 2. / 3.);
    double kF = std::pow(3. * std::pow(M_PI, 2) * nt, 1. / 3.);
    double eF = std::pow(kF, 2) / 2.;
    double as = scattering_length(ix, iy, iz, it, dc_params, dc_extra_data_size, dc_extra_data);
    double x = std::fabs(as * kF);
    double nt_reg = p_reg(nt);
    double dx_dnt = (nt_reg > 0.0) ? nt_reg * x / (3. * nt) : 0.0;
    double beta = beta_d0(x), inverse_gamma = inverse_gamma_d0(x);
    double alpha_p = dx_dnt * alpha_d1(x);
    double af = a_functional_d0(x), cf = c_functional_d0(x);
    double af_p = 0.0, cf_p = 0.0;
    if (nt_reg > 0.0) {
        af_p = alpha_p;
        cf_p = nt_reg * cf / (3. * nt) * (1. - cf * inverse_gamma);
    }
    double ctilde = af * nt_1o3 / cf;
    double inverse_gamma_eff = (1 / cf) * (1. - 3. * nt / cf * cf_p);
    double ctilde_p = (nt_reg > 0.) ? std::pow(nt_reg, 2. / 3.) * inverse_gamma_eff * af / (3. * nt_2o3) : 0.;
    ctilde_p += af_p * nt_1o3 / cf;
#ifdef CURRENT_CORRECTIONS
    P.alpha_a[i] = af; P.alpha_b[i] = af;
    double *Aa[3] = {P.A_a_x, P.A_a_y, P.A_a_z}, *Ab[3] = {P.A_b_x, P.A_b_y, P.A_b_z};
    double *ja[3] = {Dn.j_a_x, Dn.j_a_y, Dn.j_a_z}, *jb[3] = {Dn.j_b_x, Dn.j_b_y, Dn.j_b_z};
    double t4 = p_reg(na) * cccoeff;
    for (int d = 0; d < CODEDIM; d++) Aa[d][i] = (t4 == 0.0) ? 0.0 : t4 * (1. - af) * ja[d][i] / na;
    t4 = p_reg(nb) * cccoeff;
    for (int d = 0; d < CODEDIM; d++) Ab[d][i] = (t4 == 0.0) ? 0.0 : t4 * (1. - af) * jb[d][i] / nb;
#endif
    /* kinetic (Galilean) and mean-field contributions */
    Va_const += af_p * (taua + taub) / 2.;
    Vb_const += af_p * (taua + taub) / 2.;
    Va_const += beta * eF;
    Vb_const += beta * eF;
#ifdef CURRENT_CORRECTIONS
    {
        double ja2 = 0.0, jb2 = 0.0;
        for (int d = 0; d < CODEDIM; d++) { ja2 += ja[d][i] * ja[d][i]; jb2 += jb[d][i] * jb[d][i]; }
        double t7 = p_reg(na) * cccoeff;
        if (t7 != 0.0) {
            t7 = t7 * ja2 / (2.0 * na);
            Va_const += ((af - 1.0) / na - af_p) * t7;
            Va_const -= cccoeff * dp_reg(na) * (af - 1.0) * ja2 / (2.0 * na);
            Vb_const -= af_p * t7;
        }
        t7 = p_reg(nb) * cccoeff;
        if (t7 != 0.0) {
            t7 = t7 * jb2 / (2.0 * nb);
            Va_const -= af_p * t7;
            Vb_const += ((af - 1.0) / nb - af_p) * t7;
            Vb_const -= cccoeff * dp_reg(nb) * (af - 1.0) * jb2 / (2.0 * nb);
        }
    }
#endif
#ifdef INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
    double lkF = std::pow(3.0 * M_PI * M_PI * (na + nb), 1.0 / 3.0);
#endif
    for (int k = 0; k < UD_SCITERS; k++) {
        double lmu_sc = (dc_mu_a - Va + dc_mu_b - Vb) / 2.;
        Complex p0 = std::sqrt(Complex(2.0 * lmu_sc / af, 0.0));
        if (p0.imag() < 0.) p0 *= -1.;
#ifdef USE_CUBIC_CUTOFF
        Complex kc = Complex(M_PI / DX, 0.0);
#else
        Complex kc = std::sqrt(Complex(2.0 * (dc_ec + lmu_sc) / af, 0.0));
        if (kc.imag() < 0.) kc *= -1.;
#endif
        Complex wz = std::log((kc + p0) / (kc - p0));
        if (wz.imag() < 0.) wz += Complex(0.0, 2. * M_PI);
        wz = kc * REG_COEFF_R0 * (1. - (p0 / kc) * REG_COEFF_R1 * wz);
        double lambda = wz.real();
        double g_eff = af / (ctilde - lambda);
        ldelta = -lnu * g_eff;
        double ddn = (std::conj(ldelta) * lnu).real();
        double das = ldelta.real() * ldelta.real() + ldelta.imag() * ldelta.imag();
        double Vanew = Va_const - (af_p / af) * ddn - ctilde_p / af * das;
        double Vbnew = Vb_const - (af_p / af) * ddn - ctilde_p / af * das;
#ifdef INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
        {
            double bcoeff = (p0 / (lkF + 1.0e-12)).real();
            double lx = bcoeff * lkF * DX / M_PI;
            if (g_eff < -1.0e-10 && lx > 1.0e-10) {
                double L0 = bcoeff * REG_COEFF_R0 / lx * (1.0 - REG_COEFF_R1 * lx * std::log((1.0 + lx) / (1.0 - lx)));
                double dL0 = (-2. * bcoeff * REG_COEFF_R0 * REG_COEFF_R1) / (1. - lx * lx) - bcoeff * REG_COEFF_R0 / lx / lx;
                double dLdn = (lkF / (3. * (na + nb) * af)) * (L0 + dL0 * bcoeff * DX * lkF / M_PI);
                Vanew += dLdn * das;
                Vbnew += dLdn * das;
            }
        }
#endif
        Va = UD_MIX_COEFF * Vanew + (1. - UD_MIX_COEFF) * Va;
        Vb = UD_MIX_COEFF * Vbnew + (1. - UD_MIX_COEFF) * Vb;
    }
    P.V_a[i] = Va; P.V_b[i] = Vb; P.delta[i] = ldelta;
}
#endif

static void compute_potentials(int it)
{
    wslda_density Dn = dens_view(dens.data());
    wslda_potential P = pots_view(pots.data());
#if FUNCTIONAL == CUSTOMEDF
    blockIdx.x = 0; blockDim.x = 1;
    for (int i = 0; i < N; i++) { threadIdx.x = i; tdwslda_compute_potentials(it, Dn, P, 1.0); }
#else
#pragma omp parallel for
    for (int i = 0; i < N; i++) potentials_point(it, i, Dn, P, 1.0);
#endif
#ifdef ENABLE_MODIFY_POTENTIALS
    blockIdx.x = 0; blockDim.x = 1;
    for (int i = 0; i < N; i++) { threadIdx.x = i; modify_potentials(it, Dn, P); }
#endif
}

/* multiply_wf_by_alpha + compute_laplace (pca_kernels.cu:981-1026, pca.c:1455-1456) */
static void alpha_laplace(std::vector<Complex> &w)
{
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
    wslda_potential P = pots_view(pots.data());
#pragma omp parallel for schedule(dynamic)
    for (long m = 0; m < 2L * S; m++) {
        const double *al = (m < S) ? P.alpha_a : P.alpha_b;
        std::vector<Complex> t(N);
        const Complex *src = w.data() + (size_t)m * N;
        for (int i = 0; i < N; i++) t[i] = src[i] * al[i];
        derivs_one(t.data(), nullptr, nullptr, nullptr, dalap.data() + (size_t)m * N);
    }
#else
    (void)w;
#endif
}

/* apply_hamiltonian (pca_kernels.cu:233-495, 674-848; cpca_kernels.cu:231-490;
 * ccpca_kernels.cu:209-448): out = (H - <H>) w.  out may alias the laplacian buffer. */
static void filter_h_fields();
static void apply_hamiltonian(int it, std::vector<Complex> &w, Complex *out, const double *useqpe = nullptr)
{
    wslda_potential P = pots_view(pots.data());
    /* quantum friction added to V_a, V_b, delta for this H only (kernel_add_quantum_friction,
     * pca_kernels.cu:497-527; restored at the end, :530-539) */
    std::vector<double> keep_va, keep_vb;
    std::vector<Complex> keep_d;
    if (qfsw > 0.0) {
        const double qa = qf_alpha * qfsw, qb = qf_beta * qfsw, qg = qf_gamma * qfsw * pccoeff;
        const double *Ua = dens.data() + 12 * (size_t)N, *Ub = Ua + N;
        const Complex *Dq = (const Complex *)(Ua + 2 * (size_t)N);
        keep_va.assign(P.V_a, P.V_a + N);
        keep_vb.assign(P.V_b, P.V_b + N);
        keep_d.assign(P.delta, P.delta + N);
        for (int i = 0; i < N; i++) {
            const double phd = std::arg(P.delta[i]), phn = std::arg(Dq[i]);
            P.V_a[i] -= Ua[i] * qa / dc_nF;
            P.V_b[i] -= Ub[i] * qa / dc_nF;
            const Complex d0 = P.delta[i];
            P.delta[i] += qb * std::abs(P.delta[i]) * Complex(std::cos(phd), std::sin(phd)) * std::sin(phd - phn);
            P.delta[i] += Complex(0.0, qg) * d0;
        }
    }
    /* the high-k filters at the top of apply_hamiltonian (pca_kernels.cu:700-704, 758-762, 791-795) */
    filter_h_fields();
#ifdef CURRENT_CORRECTIONS
    std::vector<double> dA[2][3], lal[2];
#endif
#if !defined(FAST_CONST_EFFECTIVE_MASS_MODE)
    std::vector<double> lapal_a(N), lapal_b(N);
    lap_real(P.alpha_a, lapal_a.data());
    lap_real(P.alpha_b, lapal_b.data());
#endif
#ifdef CURRENT_CORRECTIONS
    double *Aa[3] = {P.A_a_x, P.A_a_y, P.A_a_z}, *Ab[3] = {P.A_b_x, P.A_b_y, P.A_b_z};
    for (int d = 0; d < CODEDIM; d++) {
        dA[0][d].resize(N); dA[1][d].resize(N);
        dcomp_real(Aa[d], d, dA[0][d].data());
        dcomp_real(Ab[d], d, dA[1][d].data());
    }
#endif
#ifdef ENABLE_VELOCITY_EXT
    /* kernel_get_vector_vext + compute_divergence_real_vector_f (pca_kernels.cu:623-640, 743-757) */
    std::vector<double> vel[2][3], divv[2];
    for (int sp = 0; sp < 2; sp++) {
        divv[sp].assign(N, 0.0);
        for (int d = 0; d < 3; d++) vel[sp][d].assign(N, 0.0);
        for (int i = 0; i < N; i++) {
            int ix, iy, iz; decode(i, ix, iy, iz);
            for (int d = 0; d < CODEDIM; d++) vel[sp][d][i] = ORC_VEL_EXT(ix, iy, iz, it, sp == 0 ? SPINA : SPINB, d);
        }
        std::vector<double> t(N);
        for (int d = 0; d < CODEDIM; d++) {
            dcomp_real(vel[sp][d].data(), d, t.data());
            for (int i = 0; i < N; i++) divv[sp][i] += t[i];
        }
    }
#endif
    std::vector<Complex> Dt(N);
    for (int i = 0; i < N; i++) {
        int ix, iy, iz; decode(i, ix, iy, iz);
        Complex D = P.delta[i];
#ifdef ENABLE_DELTA_EXT
        D = D + ORC_D_EXT(ix, iy, iz, it, D);
#endif
        Dt[i] = D;
    }
#pragma omp parallel for
    for (int n = 0; n < S; n++) {
        double kp2 = 0.0;
#if CODEDIM == 2
        kp2 = kkz[n] * kkz[n];
#elif CODEDIM == 1
        kp2 = kky[n] * kky[n] + kkz[n] * kkz[n];
#endif
        for (int i = 0; i < N; i++) {
            Complex tu = U(w, n)[i], tv = V(w, n)[i];
            Complex lu = U(dlap, n)[i], lv = V(dlap, n)[i];
            double Va = P.V_a[i], Vb = P.V_b[i];
            Complex D = Dt[i];
            Complex u(0.0, 0.0), v(0.0, 0.0);
            double cja = 0.0, cjb = 0.0;
#ifdef BDG_MODE
            double p = 0.5 * kp2;
#ifdef ENABLE_VELOCITY_EXT
            /* kernel_apply_hamiltonian_bdg with the velocity terms (pca_kernels.cu:432-480) */
            Complex gav[3], gbv[3];
            for (int d = 0; d < 3; d++) {
                gav[d] = Complex(0.0, 1.0 * vel[0][d][i]);
                gbv[d] = Complex(0.0, -1.0 * vel[1][d][i]);
            }
            cja = 0.5 * divv[0][i];
            cjb = 0.5 * divv[1][i];
#endif
            u += tu * Complex(Va - dc_mu_a + p, cja);
            v -= tv * Complex(Vb - dc_mu_b + p, -1.0 * cjb);
            u += tv * D;
            v += tu * std::conj(D);
#ifdef ENABLE_VELOCITY_EXT
            {
                std::vector<Complex> *dd[3] = {&ddx, &ddy, &ddz};
                for (int d = 0; d < CODEDIM; d++) {
                    u += U(*dd[d], n)[i] * gav[d];
                    v -= V(*dd[d], n)[i] * gbv[d];
                }
            }
#endif
            u += lu * (-0.5);
            v -= lv * (-0.5);
#else
#ifdef FAST_CONST_EFFECTIVE_MASS_MODE
            double aa = P.alpha_a[i] * -0.5, ab = P.alpha_b[i] * -0.5;
            double ja = -1.0 * aa * kp2, jb = -1.0 * ab * kp2;
#else
            double aa = P.alpha_a[i] * -0.25, ab = P.alpha_b[i] * -0.25;
            double na = 0.25 * lapal_a[i], nb = 0.25 * lapal_b[i];
            double ja = -2.0 * aa * kp2, jb = -2.0 * ab * kp2;
#endif
#ifdef CURRENT_CORRECTIONS
            Complex ga[3], gb[3];
            for (int d = 0; d < 3; d++) { ga[d] = Complex(0, 0); gb[d] = Complex(0, 0); }
            for (int d = 0; d < CODEDIM; d++) {
                cja += -0.5 * dA[0][d][i];
                cjb += -0.5 * dA[1][d][i];
                ga[d] += Complex(0.0, -1. * Aa[d][i]);
                gb[d] += Complex(0.0, 1. * Ab[d][i]);
            }
#ifdef ENABLE_VELOCITY_EXT
            /* pca_kernels.cu:315-327 */
            for (int d = 0; d < CODEDIM; d++) {
                ga[d] += Complex(0.0, 1.0 * vel[0][d][i]);
                gb[d] += Complex(0.0, -1.0 * vel[1][d][i]);
            }
            cja += 0.5 * divv[0][i];
            cjb += 0.5 * divv[1][i];
#endif
#endif
            u += tu * Complex(Va - dc_mu_a + ja, cja);
            v -= tv * Complex(Vb - dc_mu_b + jb, -1.0 * cjb);
            u += tv * D;
            v += tu * std::conj(D);
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
            u += tu * na;
            v -= tv * nb;
#endif
#ifdef CURRENT_CORRECTIONS
            {
                std::vector<Complex> *dd[3] = {&ddx, &ddy, &ddz};
                for (int d = 0; d < CODEDIM; d++) {
                    u += U(*dd[d], n)[i] * ga[d];
                    v -= V(*dd[d], n)[i] * gb[d];
                }
            }
#endif
            u += lu * aa;
            v -= lv * ab;
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
            u += U(dalap, n)[i] * (-0.25);
            v -= V(dalap, n)[i] * (-0.25);
#endif
#endif
            out[(size_t)n * N + i] = u;
            out[(size_t)S * N + (size_t)n * N + i] = v;
        }
    }
    /* quasiparticle energies and subtraction (pca_kernels.cu:806-833) */
#pragma omp parallel for
    for (int n = 0; n < S; n++) {
        double e = 0.0;
        if (useqpe) {
            e = useqpe[n]; /* given energies (useqpe, pca_kernels.cu:806-833) */
        } else {
            for (int i = 0; i < N; i++) {
                Complex p = std::conj(U(w, n)[i]) * out[(size_t)n * N + i] +
                            std::conj(V(w, n)[i]) * out[(size_t)S * N + (size_t)n * N + i];
                e += p.real() * WTD_DV;
            }
            qpe[n] = e;
        }
        for (int i = 0; i < N; i++) {
            out[(size_t)n * N + i] -= U(w, n)[i] * e;
            out[(size_t)S * N + (size_t)n * N + i] -= V(w, n)[i] * e;
        }
    }
    if (qfsw > 0.0) {
#if CODEDIM == 2
        /* the 2D engine does not remove the friction terms again (cpca_kernels.cu:846 is
         * commented out): the potentials keep the modified, filtered fields and the friction
         * density arrays hold the saved originals (kernel_add_quantum_friction, :521-525) */
        double *Ua = dens.data() + 12 * (size_t)N, *Ub = Ua + N;
        Complex *Dq = (Complex *)(Ua + 2 * (size_t)N);
        std::copy(keep_va.begin(), keep_va.end(), Ua);
        std::copy(keep_vb.begin(), keep_vb.end(), Ub);
        std::copy(keep_d.begin(), keep_d.end(), Dq);
#else
        std::copy(keep_va.begin(), keep_va.end(), P.V_a);
        std::copy(keep_vb.begin(), keep_vb.end(), P.V_b);
        std::copy(keep_d.begin(), keep_d.end(), P.delta);
#endif
    }
}

/* the fields apply_hamiltonian filters in place before building H, at every call: V_a, V_b
 * (pca_kernels.cu:700-704), delta (mode 2, :758-762), the A components with current
 * corrections outside BdG (:791-795) */
static void filter_h_fields()
{
    if (hkf_mode < 1) return;
    wslda_potential P = pots_view(pots.data());
    high_k_filter(P.V_a);
    high_k_filter(P.V_b);
    if (hkf_mode >= 2) high_k_filter_c(P.delta);
#if defined(CURRENT_CORRECTIONS) && !defined(BDG_MODE)
    double *A[6] = {P.A_a_x, P.A_a_y, P.A_a_z, P.A_b_x, P.A_b_y, P.A_b_z};
    for (int k = 0; k < 6; k++) high_k_filter(A[k]);
#endif
}

/* densities -> potentials block shared by both half steps (pca.c:1424-1457) */
static void half_step_densities(int it_next, int grads)
{
    derivatives(y, grads);
    calculate_densities(y, grads);
    if (qfsw > 0.0) calculate_qf_densities(y); /* pca.c:1426-1430 */
    exchange_densities();
    if (grads) density_tau();
    compute_potentials(it_next);
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
    if (hkf_mode >= 1) { /* effective-mass filtering (pca.c:1448-1453) */
        wslda_potential P = pots_view(pots.data());
        high_k_filter(P.alpha_a);
        high_k_filter(P.alpha_b);
    }
#endif
    alpha_laplace(y);
    if (qfsw > 0.0) pccoeff = qf_pccoeff(); /* pca.c:1458 */
}

static int scheme_slots() { return NHIST; }

} // namespace orc

using namespace orc;

extern "C" {

int orc_numel(void) { return N; }
int orc_codedim(void) { return CODEDIM; }
int orc_nhist(void) { return NHIST; }
int orc_dims(int *d) { d[0] = AXN[0]; d[1] = AXN[1]; d[2] = AXN[2]; return 0; }
int orc_functional(void) { return FUNCTIONAL; }
/* the user's host hook process_params (pca.c:903), as the reference's driver calls it */
int orc_process_params(double *params, double *kF, double *mu)
{
    process_params(params, kF, mu, 0, NULL);
    return 0;
}
int orc_const_mass(void)
{
#ifdef FAST_CONST_EFFECTIVE_MASS_MODE
    return 1;
#else
    return 0;
#endif
}

/* constants (memcopy_const / memcopy_const_params / memcopy_const_sclgth / memcopy_extra_data;
 * wslda_cuda_utils.h:47-105) */
int orc_set_constants(double mu_a, double mu_b, double ec, double t0, double dt, double kF, double sclgth)
{
    dc_mu_a = mu_a; dc_mu_b = mu_b; dc_ec = ec; dc_t0 = t0; dc_dt = dt; dc_kF = kF;
    dc_eF = kF * kF / 2.; dc_nF = kF * kF * kF / (3. * M_PI * M_PI); dc_sclgth = sclgth;
    md.sclgth = sclgth; md.dt = dt; md.ec = ec;
    return 0;
}
int orc_set_params(const double *p)
{
    for (int k = 0; k < MAX_USER_PARAMS; k++) { dc_params[k] = p[k]; md.params[k] = p[k]; }
    return 0;
}
int orc_set_extra_data(const void *d, size_t size)
{
    extra.assign((const unsigned char *)d, (const unsigned char *)d + size);
    dc_extra_data = size ? extra.data() : nullptr;
    dc_extra_data_size = size;
    return 0;
}

/* states: y = [u_0..u_{S-1}, v_0..v_{S-1}] as interleaved (re, im) doubles; pots: 12N */
int orc_setup(int nwf, const double *yin, const double *potsin, const double *fbeta,
              const double *kyin, const double *kzin, const int *cntin, int it0)
{
    S = nwf;
    for (int d = 0; d < 3; d++) make_plan(plans[d], AXN[d]);
    size_t M = (size_t)2 * S * N;
    y.assign((const Complex *)yin, (const Complex *)yin + M);
    for (int h = 0; h < 5; h++) fk[h].assign(h < NHIST ? M : 0, Complex(0.0, 0.0));
    ddx.assign(M, Complex(0, 0));
    ddy.assign(CODEDIM >= 2 ? M : 0, Complex(0, 0));
    ddz.assign(CODEDIM >= 3 ? M : 0, Complex(0, 0));
    dlap.assign(M, Complex(0, 0));
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
    dalap.assign(M, Complex(0, 0));
#endif
    dens.assign((size_t)16 * N, 0.0); /* 12 N densities + 4 N quantum-friction densities */
    pots.assign(potsin, potsin + (size_t)12 * N);
    fb.assign(fbeta, fbeta + S);
    kky.assign(S, 0.0); kkz.assign(S, 0.0); cnt.assign(S, 1);
    if (kyin) kky.assign(kyin, kyin + S);
    if (kzin) kkz.assign(kzin, kzin + S);
    if (cntin) cnt.assign(cntin, cntin + S);
    qpe.assign(S, 0.0);
    it_global = it0;
    return 0;
}

/* initial measurement (pca.c:939-958): normalise, derivatives, all densities, tau */
int orc_initial_measurement(void)
{
    normalize(y);
    derivatives(y, 1);
    calculate_densities(y, 1);
    exchange_densities();
    density_tau();
    last_gradients = 1;
    return 0;
}

/* nsteps ABM steps as one measurement block (pca.c:1401-1571); gradients are formed on the
 * last step (const mass) or on every step (variable mass). */
int orc_steps(int nsteps)
{
    Complex *f[5];
    for (int h = 0; h < 5; h++) f[h] = fk[h].empty() ? nullptr : fk[h].data();
    for (int s = 0; s < nsteps; s++) {
        int last = (s == nsteps - 1);
        int it = it_global;
        qfsw = qf_switch(dc_t0 + (it + 1) * dc_dt); /* pca.c:1405, 1467 */
        /* predictor */
        abm_step1(y.data(), f[0], f[1], f[2], f[3], f[4]);
        normalize(y);
        int grads = orc_const_mass() ? (qfsw > 0.0 ? 1 : 0) : 1;
        half_step_densities(it + 1, grads);
        apply_hamiltonian(it + 1, y, dlap.data());
        /* corrector */
        abm_step4(dlap.data(), y.data(), f[NHIST - 1]);
        normalize(y);
        grads = orc_const_mass() ? ((last || qfsw > 0.0) ? 1 : 0) : 1;
        half_step_densities(it + 1, grads);
        last_gradients = grads;
        Complex *tmp = f[NHIST - 1];
        for (int h = NHIST - 1; h > 0; h--) f[h] = f[h - 1];
        f[0] = tmp;
        apply_hamiltonian(it + 1, y, f[0]);
        it_global++;
    }
    qfsw = 0.0; /* friction acts inside steps only */
    /* keep the rotated order visible to getters */
    std::vector<std::vector<Complex>> nv(5);
    for (int h = 0; h < NHIST; h++) nv[h].assign(f[h], f[h] + (size_t)2 * S * N);
    for (int h = 0; h < NHIST; h++) fk[h].swap(nv[h]);
    return 0;
}

/* Taylor self-start of the ABM history (pca.c:1086-1330, selfstart 1): each of the q first
 * steps records (H - <H>) psi of its start state as the newest history entry, takes a half step
 * exp(-i H dt/2) psi by a Taylor series of exp_iters terms to build midpoint potentials, then
 * the full step exp(-i H_mid dt) psi the same way and renormalises.  Potentials and H use time
 * index 0 throughout ("potential is constant during first steps"), and the time index does not
 * advance.  Afterwards the history holds the recorded entries (f1 newest) and densities and
 * potentials are recomputed at the current time index. */
static void taylor_term(int order, double dt, const std::vector<Complex> &h, std::vector<Complex> &upd,
                        std::vector<Complex> &contr)
{
    /* taylor_expansion_contribution (pca_kernels.cu:1032-1062): contr = h * (i t), upd += contr,
     * t = -dt/order */
    const double t = -1.0 * dt / (double)order;
    for (size_t i = 0; i < h.size(); i++) {
        Complex c = h[i] * Complex(0.0, t);
        contr[i] = c;
        upd[i] += c;
    }
}

static void selfstart()
{
    const int q = NHIST;
    const int iters = (NHIST == 3) ? 4 : 5;
#ifdef FAST_CONST_EFFECTIVE_MASS_MODE
    const int grads = 0;
#else
    const int grads = 1;
#endif
    const size_t M = (size_t)2 * S * N;
    std::vector<Complex> f1(M), f2(M), f3(M);
    std::vector<std::vector<Complex>> rec(q, std::vector<Complex>(M, Complex(0.0, 0.0)));
    std::vector<double> qs(S);
    for (int step = 0; step < q; step++) {
        /* densities and potentials of the start state (time index 0) */
        derivatives(y, grads);
        calculate_densities(y, grads);
        exchange_densities();
        if (grads) density_tau();
        compute_potentials(0);
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
        if (hkf_mode >= 1) {
            wslda_potential P = pots_view(pots.data());
            high_k_filter(P.alpha_a);
            high_k_filter(P.alpha_b);
        }
#endif
        alpha_laplace(y);
        /* H psi of the start state, recorded as the newest history entry */
        f3 = y;
        apply_hamiltonian(0, f3, f1.data());
        qs = qpe;
        for (int h = q - 1; h > 0; h--) rec[h] = rec[h - 1];
        rec[0] = f1;
        /* half step: f3 = exp(-i H dt/2) psi, Taylor series */
        taylor_term(1, 0.5 * md.dt, f1, f3, f2);
        for (int m = 1; m < iters; m++) {
            derivatives(f2, grads);
            alpha_laplace(f2);
            apply_hamiltonian(0, f2, f1.data(), qs.data());
            taylor_term(m + 1, 0.5 * md.dt, f1, f3, f2);
        }
        normalize(f3);
        /* midpoint densities and potentials */
        derivatives(f3, grads);
        calculate_densities(f3, grads);
        exchange_densities();
        if (grads) density_tau();
        compute_potentials(0);
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
        if (hkf_mode >= 1) {
            wslda_potential P = pots_view(pots.data());
            high_k_filter(P.alpha_a);
            high_k_filter(P.alpha_b);
        }
#endif
        /* full step from the start state with the midpoint H */
        derivatives(y, grads);
        alpha_laplace(y);
        apply_hamiltonian(0, y, f1.data());
        qs = qpe;
        taylor_term(1, md.dt, f1, y, f2);
        for (int m = 1; m < iters; m++) {
            derivatives(f2, grads);
            alpha_laplace(f2);
            apply_hamiltonian(0, f2, f1.data(), qs.data());
            taylor_term(m + 1, md.dt, f1, y, f2);
        }
        normalize(y);
    }
    for (int h = 0; h < q; h++) fk[h] = rec[h];
    /* densities and potentials of the new state at the current time index (pca.c:1315-1318) */
    derivatives(y, 1);
    calculate_densities(y, 1);
    exchange_densities();
    density_tau();
    compute_potentials(it_global);
    last_gradients = 1;
}

/* compute_energy (tdwslda_energy_generic.h:21-111 and the functional energy kernels) */
int orc_energy(double *E)
{
    using namespace oedf;
    int it = it_global;
    wslda_density Dn = dens_view(dens.data());
    wslda_potential P = pots_view(pots.data());
    std::vector<double> e(11 * (size_t)N, 0.0);
    const double VOL = WTD_VOLEL;
    for (int i = 0; i < N; i++) {
        int ix, iy, iz; decode(i, ix, iy, iz);
        double na = Dn.rho_a[i], nb = Dn.rho_b[i];
        double x1 = Dn.j_a_x[i], x2 = Dn.j_b_x[i];
        double y1 = (CODEDIM >= 2) ? Dn.j_a_y[i] : 0.0, y2 = (CODEDIM >= 2) ? Dn.j_b_y[i] : 0.0;
        double z1 = (CODEDIM >= 3) ? Dn.j_a_z[i] : 0.0, z2 = (CODEDIM >= 3) ? Dn.j_b_z[i] : 0.0;
#if FUNCTIONAL == CUSTOMEDF
        blockIdx.x = 0; blockDim.x = 1; threadIdx.x = i;
        tdwslda_compute_energy(it, Dn, P, &e[EKIN * (size_t)N], &e[EPOT * (size_t)N], &e[EPAIR * (size_t)N], &e[ECURRENT * (size_t)N]);
#else
        double taua = Dn.tau_a[i], taub = Dn.tau_b[i];
        taua -= p_reg(na) * (x1 * x1 + y1 * y1 + z1 * z1) / na;
        taub -= p_reg(nb) * (x2 * x2 + y2 * y2 + z2 * z2) / nb;
#if FUNCTIONAL == BDG
        e[EKIN * (size_t)N + i] = 0.5 * (P.alpha_a[i] * taua + P.alpha_b[i] * taub) * VOL;
        e[EPOT * (size_t)N + i] = 0.0;
#elif FUNCTIONAL == SLDAE
        /* tdwslda_functionals.h:815-884 */
        {
            double nt = na + nb;
            double kF = std::pow(3. * std::pow(M_PI, 2) * nt, 1. / 3.);
            double eF = std::pow(kF, 2) / 2.;
            double x = std::fabs(scattering_length(ix, iy, iz, it, dc_params, dc_extra_data_size, dc_extra_data) * kF);
            double af = osldae::a_functional_d0(x), bf = osldae::b_functional_d0(x);
            e[EKIN * (size_t)N + i] = af * (taua + taub) / 2. * VOL;
            e[EPOT * (size_t)N + i] = (3. / 5.) * bf * eF * nt * VOL;
        }
#else
        double p = pol(na, nb);
        e[EKIN * (size_t)N + i] = 0.5 * (alpha(p) * taua + alpha(-p) * taub) * VOL;
        e[EPOT * (size_t)N + i] = funD(na, nb) * VOL;
#endif
        e[EPAIR * (size_t)N + i] = (P.delta[i] * std::conj(Dn.nu[i])).real() * (-1.0) * VOL;
        e[ECURRENT * (size_t)N + i] = p_reg(na) * (x1 * x1 + y1 * y1 + z1 * z1) / (2. * na) * VOL +
                                      p_reg(nb) * (x2 * x2 + y2 * y2 + z2 * z2) / (2. * nb) * VOL;
#endif
#ifdef ENABLE_V_EXT
        e[EPOTEXT * (size_t)N + i] = (na * ORC_U_EXT(ix, iy, iz, it, SPINA) + nb * ORC_U_EXT(ix, iy, iz, it, SPINB)) * VOL;
#endif
#ifdef ENABLE_DELTA_EXT
        e[EPAIREXT * (size_t)N + i] = (std::conj(Dn.nu[i]) * ORC_D_EXT(ix, iy, iz, it, P.delta[i])).real() * (-2.0) * VOL;
#endif
#ifdef ENABLE_VELOCITY_EXT
        /* kernel_compute_energy_velocity_ext (pca_kernels.cu:163-187; 2D/1D over their axes) */
        {
            const double *ja[3] = {Dn.j_a_x, Dn.j_a_y, Dn.j_a_z}, *jb[3] = {Dn.j_b_x, Dn.j_b_y, Dn.j_b_z};
            double sv = 0.0;
            for (int d = 0; d < CODEDIM; d++)
                sv += ja[d][i] * ORC_VEL_EXT(ix, iy, iz, it, SPINA, d) + jb[d][i] * ORC_VEL_EXT(ix, iy, iz, it, SPINB, d);
            e[EVELEXT * (size_t)N + i] = sv * (-1.0) * VOL;
        }
#endif
        e[NPARTA * (size_t)N + i] = na;
        e[NPARTB * (size_t)N + i] = nb;
#if CODEDIM >= 2
        double xx = (double)(ix - NX / 2) * DX, yy = (double)(iy - NY / 2) * DY;
        e[LZA * (size_t)N + i] = (xx * y1 - yy * x1) * VOL;
        e[LZB * (size_t)N + i] = (xx * y2 - yy * x2) * VOL;
#endif
    }
#ifdef ENABLE_MODIFY_ENERGIES
    blockIdx.x = 0; blockDim.x = 1;
    for (int i = 0; i < N; i++) { threadIdx.x = i; modify_energies(it, Dn, P, e.data()); }
#endif
    for (int k = 0; k < TDWSLDAITEMS; k++) {
        double s = 0.0;
        for (int i = 0; i < N; i++) s += e[(size_t)k * N + i];
        E[k] = s;
    }
    E[NPARTA] *= VOL;
    E[NPARTB] *= VOL;
    return 0;
}

int orc_get_states(double *out) { std::memcpy(out, y.data(), y.size() * sizeof(Complex)); return 0; }
int orc_get_densities(double *out) { std::memcpy(out, dens.data(), (size_t)12 * N * sizeof(double)); return 0; }
int orc_get_potentials(double *out) { std::memcpy(out, pots.data(), pots.size() * sizeof(double)); return 0; }
int orc_get_qpe(double *out) { std::memcpy(out, qpe.data(), qpe.size() * sizeof(double)); return 0; }
int orc_get_history(int slot, double *out)
{
    if (slot < 0 || slot >= NHIST) return -1;
    std::memcpy(out, fk[slot].data(), fk[slot].size() * sizeof(Complex));
    return 0;
}
int orc_get_it(void) { return it_global; }
/* the quantum-friction densities of the current states (4 N: U_a, U_b, D complex) */
int orc_qf_densities(double *out)
{
    derivatives(y, 0);
    calculate_qf_densities(y);
    std::memcpy(out, dens.data() + 12 * (size_t)N, (size_t)4 * N * sizeof(double));
    return 0;
}
/* densities of a weighted subset of the current states, with gradients and tau (pca.c:1056-1066,
 * the subset tracking of md.subsetMinEn/subsetMaxEn) into out (12 N); summed over ranks */
int orc_subset_densities(const double *weights, double *out)
{
    std::vector<double> d((size_t)16 * N, 0.0);
    derivatives(y, 1);
    calculate_densities(y, 1, weights, d.data());
    if (xfn) xfn(xuser, d.data(), (size_t)12 * N);
    density_tau(d.data());
    std::memcpy(out, d.data(), (size_t)12 * N * sizeof(double));
    return 0;
}
int orc_set_quantum_friction(double alpha, double beta, double gamma, double nreq, double start, double stop, double ramp)
{
    qf_alpha = alpha; qf_beta = beta; qf_gamma = gamma; qf_Nreq = nreq;
    qf_start = start; qf_stop = stop; qf_ramp = ramp;
    return 0;
}
int orc_selfstart(void)
{
    selfstart();
    return 0;
}
int orc_set_high_k_filter(int mode, double mu, double T)
{
    hkf_mode = mode; hkf_mu = mu; hkf_T = T;
    return 0;
}
int orc_filter_field(double *f)
{
    for (int d = 0; d < 3; d++) if (plans[d].n != AXN[d]) make_plan(plans[d], AXN[d]);
    high_k_filter(f);
    return 0;
}
int orc_set_density_exchange(exchange_fn fn, void *user)
{
    xfn = fn;
    xuser = user;
    return 0;
}
int orc_set_threads(int n)
{
#ifdef _OPENMP
    omp_set_num_threads(n);
#endif
    return n;
}

/* standalone transform of one lattice field, for checking the FFT against numpy */
int orc_fft_field(double *data, int sign)
{
    for (int d = 0; d < 3; d++) if (plans[d].n != AXN[d]) make_plan(plans[d], AXN[d]);
    fftn((Complex *)data, sign);
    return 0;
}
/* spectral derivatives of one complex field: outputs dx, dy, dz, lap (N complex each) */
int orc_derivatives_field(const double *f, double *dx, double *dy, double *dz, double *lap)
{
    for (int d = 0; d < 3; d++) if (plans[d].n != AXN[d]) make_plan(plans[d], AXN[d]);
    derivs_one((const Complex *)f, (Complex *)dx, CODEDIM >= 2 ? (Complex *)dy : nullptr,
               CODEDIM >= 3 ? (Complex *)dz : nullptr, (Complex *)lap);
    return 0;
}
}
