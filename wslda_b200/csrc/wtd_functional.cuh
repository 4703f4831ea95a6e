/*
 * Local energy density functionals on the device: potentials from densities (one thread per
 * lattice point, FP64 always) and the energy integrands.
 *
 *   SLDA / ASLDA  hpc-engine/tdwslda_functionals.h:47-306 (potentials), :308-366 (energy),
 *                 EDF pieces hpc-engine/pca_edf.h:17-350
 *   BDG           hpc-engine/tdwslda_functionals.h:373-452 (potentials), :455-503 (energy)
 *   SLDAE         hpc-engine/tdwslda_functionals.h:530-812 (potentials), :815-884 (energy),
 *                 parameter fits hpc-engine/sldae_functional.c:68-330
 *   CUSTOMEDF     the user's tdwslda_compute_potentials / tdwslda_compute_energy kernels from
 *                 problem-definition.h, launched unchanged
 *
 * The 15-iteration local self-consistency with 0.75 mixing, the spherical/cubic cut-off
 * regularisation with complex sqrt/log and the optional mean-field correction of the
 * regularisation scheme follow the reference formula by formula; the published functional
 * constants (A0..A2, G0, G1, GAMMA0, P_NMIN/P_NMAX) come from wtd_settings.h.
 */
#ifndef WTD_FUNCTIONAL_CUH
#define WTD_FUNCTIONAL_CUH

#if defined(ENABLE_V_EXT)
#define WTD_U_EXT(ix, iy, iz, it, spin) v_ext(ix, iy, iz, it, spin, dc_params, dc_extra_data_size, dc_extra_data)
#else
#define WTD_U_EXT(ix, iy, iz, it, spin) 0.0
#endif
#if defined(ENABLE_VELOCITY_EXT)
#define WTD_VEL_EXT(ix, iy, iz, it, spin, axis) velocity_ext(ix, iy, iz, it, spin, axis, dc_params, dc_extra_data_size, dc_extra_data)
#else
#define WTD_VEL_EXT(ix, iy, iz, it, spin, axis) 0.0
#endif
#if defined(ENABLE_DELTA_EXT)
#define WTD_D_EXT(ix, iy, iz, it, d) delta_ext(ix, iy, iz, it, d, dc_params, dc_extra_data_size, dc_extra_data)
#else
#define WTD_D_EXT(ix, iy, iz, it, d) Complex(0.0, 0.0)
#endif

__device__ __forceinline__ void wtd_decode(int i, int &ix, int &iy, int &iz)
{
#if CODEDIM == 3
    ix = i / (NY * NZ); int r = i - ix * NY * NZ; iy = r / NZ; iz = r - iy * NZ;
#elif CODEDIM == 2
    ix = i / NY; iy = i - ix * NY; iz = 0;
#else
    ix = i; iy = 0; iz = 0;
#endif
}

namespace edf {
/* pca_edf.h:17-33 */
__host__ __device__ __forceinline__ double p_reg(double n)
{
    if (n <= P_NMIN) return 0.0;
    if (n >= P_NMAX) return 1.0;
    return 0.5 + 0.5 * tanh(P_ALPHA * tan((M_PI * (n - P_NMIN)) / (P_NMAX - P_NMIN) - M_PI / 2.0));
}
__host__ __device__ __forceinline__ double dp_reg(double n)
{
    if (n <= P_NMIN || n >= P_NMAX) return 0.0;
    double a = (M_PI * (n - P_NMIN)) / (P_NMAX - P_NMIN) - M_PI / 2.0;
    double c = cosh(P_ALPHA * tan(a)) * cos(a);
    return 0.5 * P_ALPHA * M_PI / (c * c) / (P_NMAX - P_NMIN);
}
/* pca_edf.h:39-97 */
__host__ __device__ __forceinline__ double pol(double a, double b)
{
    double pr = p_reg(a + b);
    return pr == 0.0 ? 0.0 : pr * (a - b) / (a + b);
}
__host__ __device__ __forceinline__ double dpol(double a, double b, bool wrt_a)
{
    double np = a + b, pr = p_reg(np), dpr = dp_reg(np), r = 0.0;
    if (pr != 0.0) r += pr * (wrt_a ? 2.0 * b : -2.0 * a) / (np * np);
    if (dpr != 0.0) r += dpr * (a - b) / np;
    return r;
}
/* pca_edf.h:102-211 */
__host__ __device__ __forceinline__ double alpha(double p)
{
    double p2 = p * p, p4 = p2 * p2;
    return A0 + A1 * p * (1.0 - (2.0 / 3.0) * p2 + (1.0 / 5.0) * p4) + A2 * p2 * (1.0 - p2 + (1.0 / 3.0) * p4);
}
__host__ __device__ __forceinline__ double alpha_plus(double p) { return 0.5 * (alpha(p) + alpha(-p)); }
__host__ __device__ __forceinline__ double alpha_minus(double p) { return 0.5 * (alpha(p) - alpha(-p)); }
__host__ __device__ __forceinline__ double dap_core(double p)
{
    double p2 = p * p, p4 = p2 * p2;
    return 2.0 * A2 * p * (1.0 - p2 + (1.0 / 3.0) * p4) - 2.0 * A2 * p * p2 * (1.0 - (2.0 / 3.0) * p2);
}
__host__ __device__ __forceinline__ double dam_core(double p)
{
    double p2 = p * p, p4 = p2 * p2;
    return A1 * (1.0 - (2.0 / 3.0) * p2 + (1.0 / 5.0) * p4) - 4.0 * A1 * p2 * ((1.0 / 3.0) - (1.0 / 5.0) * p2);
}
/* pca_edf.h:216-311 */
__host__ __device__ __forceinline__ double funG(double p) { return G0 + G1 * p * p; }
__host__ __device__ __forceinline__ double funD(double a, double b)
{
    double p = pol(a, b);
    return (1.0 / (20.0 * M_PI * M_PI)) * pow(6.0 * M_PI * M_PI * (a + b), 5.0 / 3.0) *
           (funG(p) - alpha(p) * pow((1.0 + p) / 2.0, 5.0 / 3.0) - alpha(-p) * pow((1.0 - p) / 2.0, 5.0 / 3.0));
}
__host__ __device__ __forceinline__ double dD(double a, double b, bool wrt_a)
{
    double p = pol(a, b);
    double dA = dam_core(p), dB = dap_core(p);
    double brk = funG(p) - alpha(p) * pow((1.0 + p) / 2.0, 5.0 / 3.0) - alpha(-p) * pow((1.0 - p) / 2.0, 5.0 / 3.0);
    double t1 = 0.5 * pow(6.0 * M_PI * M_PI * (a + b), 2.0 / 3.0) * brk;
    double t2 = (1.0 / (20.0 * M_PI * M_PI)) * pow(6.0 * M_PI * M_PI * (a + b), 5.0 / 3.0) *
                (2.0 * G1 * p - (dA + dB) * pow((1.0 + p) / 2.0, 5.0 / 3.0) - (5.0 / 6.0) * alpha(p) * pow((1.0 + p) / 2.0, 2.0 / 3.0)
                 - (-dA + dB) * pow((1.0 - p) / 2.0, 5.0 / 3.0) + (5.0 / 6.0) * alpha(-p) * pow((1.0 - p) / 2.0, 2.0 / 3.0)) *
                dpol(a, b, wrt_a);
    return t1 + t2;
}
/* pca_edf.h:316-350 */
__host__ __device__ __forceinline__ double tildeC(double a, double b)
{
    return alpha_plus(pol(a, b)) * pow(a + b + DENSEPSILON, 1.0 / 3.0) / GAMMA0;
}
__host__ __device__ __forceinline__ double dtildeC(double a, double b, bool wrt_a)
{
    return (dap_core(pol(a, b)) * dpol(a, b, wrt_a) * pow(a + b + DENSEPSILON, 1.0 / 3.0) +
            (1.0 / 3.0) * alpha_plus(pol(a, b)) * pow(a + b + DENSEPSILON, -2.0 / 3.0)) / GAMMA0;
}
} // namespace edf

#if FUNCTIONAL == SLDAE
namespace sldae {
/* Pade[4/4] form P(x) = N(x)/D(x) of the SLDAE parameter fits and its first derivative
 * (sldae_functional.c:68-80), evaluated in Horner form */
__device__ __forceinline__ double pade0(double x, double a1, double a2, double a3, double a4,
                                        double b1, double b2, double b3, double b4)
{
    double num = x * (a1 + x * (a2 + x * (a3 + x * a4)));
    double den = 1.0 + x * (b1 + x * (b2 + x * (b3 + x * b4)));
    return num / den;
}
__device__ __forceinline__ double pade1(double x, double a1, double a2, double a3, double a4,
                                        double b1, double b2, double b3, double b4)
{
    double num = x * (a1 + x * (a2 + x * (a3 + x * a4)));
    double dnum = a1 + x * (2.0 * a2 + x * (3.0 * a3 + x * (4.0 * a4)));
    double den = 1.0 + x * (b1 + x * (b2 + x * (b3 + x * b4)));
    double dden = b1 + x * (2.0 * b2 + x * (3.0 * b3 + x * (4.0 * b4)));
    return (dnum * den - num * dden) / (den * den);
}
#define WTD_SLDAE_ALPHA_SET 0.0, WTD_SLDAE_ALPHA_A2, WTD_SLDAE_ALPHA_A3, WTD_SLDAE_ALPHA_A4, \
    WTD_SLDAE_ALPHA_B1, WTD_SLDAE_ALPHA_B2, WTD_SLDAE_ALPHA_B3, WTD_SLDAE_ALPHA_B4
#define WTD_SLDAE_SET(p) p##_a1, p##_a2, p##_a3, p##_c, p##_b1, p##_b2, p##_b3, p##_c
/* effective mass alpha(x) = a(x) (sldae_functional.c:93-166, 264-284) */
__device__ __forceinline__ double a_functional(double x)
{
#ifdef SLDA_FORCE_A1
    return 1.0;
#else
    return 1.0 + pade0(x, WTD_SLDAE_ALPHA_SET);
#endif
}
__device__ __forceinline__ double a_functional_d1(double x)
{
#ifdef SLDA_FORCE_A1
    return 0.0;
#else
    return pade1(x, WTD_SLDAE_ALPHA_SET);
#endif
}
/* beta, 1/gamma, b and c (sldae_functional.c:168-262, 286-330) */
__device__ __forceinline__ double beta(double x) { return BF_APS_UFG * pade0(x, WTD_SLDAE_SET(SLDAE_beta)); }
__device__ __forceinline__ double inverse_gamma(double x)
{
    return (1. / CF_APS_UFG) * pade0(x, WTD_SLDAE_SET(SLDAE_inverse_gamma));
}
__device__ __forceinline__ double b_functional(double x) { return BF_APS_UFG * pade0(x, WTD_SLDAE_SET(SLDAE_b_functional)); }
__device__ __forceinline__ double c_functional(double x) { return CF_APS_UFG * pade0(x, WTD_SLDAE_SET(SLDAE_c_functional)); }
/* x = |a kF| at one point, kF = (3 pi^2 n)^(1/3) */
__device__ __forceinline__ double kfermi(double nt) { return pow(3. * (M_PI * M_PI) * nt, 1. / 3.); }
} // namespace sldae
#endif

#if FUNCTIONAL == SLDA || FUNCTIONAL == ASLDA
/* tdwslda_functionals.h:47-306 */
__global__ void wtd_potentials_kernel(int it, wslda_density Dn, wslda_potential P, double cccoeff)
{
    using namespace edf;
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= WTD_NUMEL) return;
    int ix, iy, iz; wtd_decode(i, ix, iy, iz);
    double Va_c = WTD_U_EXT(ix, iy, iz, it, SPINA);
    double Vb_c = WTD_U_EXT(ix, iy, iz, it, SPINB);
    double na = Dn.rho_a[i], nb = Dn.rho_b[i];
    double p = pol(na, nb);
    double ap = alpha_plus(p);
    double dam_a = 0.0, dam_b = 0.0, dap_a = 0.0, dap_b = 0.0;
#ifdef CURRENT_CORRECTIONS
    double am = alpha_minus(p);
    double aa = alpha(p), ab = alpha(-p);
    P.alpha_a[i] = aa; P.alpha_b[i] = ab;
    double jx = Dn.j_a_x[i], kx = Dn.j_b_x[i];
    double jy = (CODEDIM >= 2) ? Dn.j_a_y[i] : 0.0, ky = (CODEDIM >= 2) ? Dn.j_b_y[i] : 0.0;
    double jz = (CODEDIM >= 3) ? Dn.j_a_z[i] : 0.0, kz = (CODEDIM >= 3) ? Dn.j_b_z[i] : 0.0;
    {
        double t4 = p_reg(na) * cccoeff;
        P.A_a_x[i] = (t4 == 0.0) ? 0.0 : t4 * (1. - aa) * jx / na;
        if (CODEDIM >= 2) P.A_a_y[i] = (t4 == 0.0) ? 0.0 : t4 * (1. - aa) * jy / na;
        if (CODEDIM >= 3) P.A_a_z[i] = (t4 == 0.0) ? 0.0 : t4 * (1. - aa) * jz / na;
        t4 = p_reg(nb) * cccoeff;
        P.A_b_x[i] = (t4 == 0.0) ? 0.0 : t4 * (1. - ab) * kx / nb;
        if (CODEDIM >= 2) P.A_b_y[i] = (t4 == 0.0) ? 0.0 : t4 * (1. - ab) * ky / nb;
        if (CODEDIM >= 3) P.A_b_z[i] = (t4 == 0.0) ? 0.0 : t4 * (1. - ab) * kz / nb;
    }
#endif
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
    {
        double ta = Dn.tau_a[i], tb = Dn.tau_b[i];
        double dpa = dpol(na, nb, true), dpb = dpol(na, nb, false);
        dam_a = dam_core(p) * dpa; dam_b = dam_core(p) * dpb;
        Va_c += dam_a * (ta - tb) / 2.0; Vb_c += dam_b * (ta - tb) / 2.0;
        dap_a = dap_core(p) * dpa; dap_b = dap_core(p) * dpb;
        Va_c += dap_a * (ta + tb) / 2.0; Vb_c += dap_b * (ta + tb) / 2.0;
    }
#endif
    Va_c += dD(na, nb, true);
    Vb_c += dD(na, nb, false);
#ifdef CURRENT_CORRECTIONS
    {
        double t7 = p_reg(na) * cccoeff;
        if (t7 != 0.0) {
            double j2 = jx * jx + jy * jy + jz * jz;
            t7 = t7 * j2 / (2.0 * na);
            Va_c += ((ap + am - 1.0) / na - (dap_a + dam_a)) * t7;
            Va_c -= cccoeff * dp_reg(na) * (ap + am - 1.0) * j2 / (2.0 * na);
            Vb_c -= (dap_b + dam_b) * t7;
        }
        t7 = p_reg(nb) * cccoeff;
        if (t7 != 0.0) {
            double k2 = kx * kx + ky * ky + kz * kz;
            t7 = t7 * k2 / (2.0 * nb);
            Va_c -= (dap_a - dam_a) * t7;
            Vb_c += ((ap - am - 1.0) / nb - (dap_b - dam_b)) * t7;
            Vb_c -= cccoeff * dp_reg(nb) * (ap - am - 1.0) * k2 / (2.0 * nb);
        }
    }
#endif
    double c1 = dap_a / ap, c2 = dap_b / ap;
    double c3 = dtildeC(na, nb, true) / ap, c4 = dtildeC(na, nb, false) / ap;
    double tC = tildeC(na, nb);
    double Va = P.V_a[i], Vb = P.V_b[i];
    Complex lnu = Dn.nu[i], ld(0.0, 0.0), one(1.0, 0.0), p0, kc, wz;
#ifdef INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
    double lkF = pow(3.0 * M_PI * M_PI * (na + nb), 1.0 / 3.0);
#endif
    for (int k = 0; k < UD_SCITERS; k++) {
        double t7 = (dc_mu_a - Va + dc_mu_b - Vb) / 2.0;
        p0 = thrust::sqrt(Complex(2.0 * t7 / ap, 0.0));
        if (p0.imag() < 0.) p0 *= -1.;
#ifdef USE_CUBIC_CUTOFF
        kc = Complex(M_PI / DX, 0.0);
#else
        kc = thrust::sqrt(Complex(2.0 * (dc_ec + t7) / ap, 0.0));
        if (kc.imag() < 0.) kc *= -1.;
#endif
        wz = thrust::log((kc + p0) / (kc - p0));
        if (wz.imag() < 0.) wz += Complex(0.0, 2. * M_PI);
        wz = kc * REG_COEFF_R0 * (1. - (p0 / kc) * REG_COEFF_R1 * wz);
        wz = one * ap / (one * tC - wz);
        ld = lnu * (-1.0 * wz.real());
        double t6 = (thrust::conj(ld) * lnu).real();
        double tn = thrust::norm(ld);
        double Van = Va_c - c1 * t6 - c3 * tn;
        double Vbn = Vb_c - c2 * t6 - c4 * tn;
#ifdef INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
        {
            double bc = (p0 / (lkF + 1.0e-12)).real();
            double lx = bc * lkF * DX / M_PI;
            if (wz.real() < -1.0e-10 && lx > 1.0e-10) {
                double L0 = bc * REG_COEFF_R0 / lx * (1.0 - REG_COEFF_R1 * lx * log((1.0 + lx) / (1.0 - lx)));
                double dL0 = (-2. * bc * REG_COEFF_R0 * REG_COEFF_R1) / (1. - lx * lx) - bc * REG_COEFF_R0 / lx / lx;
                double dLdn = (lkF / (3. * (na + nb) * ap)) * (L0 + dL0 * bc * DX * lkF / M_PI);
                Van += dLdn * tn;
                Vbn += dLdn * tn;
            }
        }
#endif
        Va = UD_MIX_COEFF * Van + (1.0 - UD_MIX_COEFF) * Va;
        Vb = UD_MIX_COEFF * Vbn + (1.0 - UD_MIX_COEFF) * Vb;
    }
    P.V_a[i] = Va; P.V_b[i] = Vb; P.delta[i] = ld;
}

/* tdwslda_functionals.h:308-366 */
__global__ void wtd_energy_kernel(int it, wslda_density Dn, wslda_potential P, double *Ek, double *Ep, double *Epair, double *Ec)
{
    using namespace edf;
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= WTD_NUMEL) return;
    double na = Dn.rho_a[i], nb = Dn.rho_b[i];
    double p = pol(na, nb);
    double ta = Dn.tau_a[i], tb = Dn.tau_b[i];
    double x1 = Dn.j_a_x[i], x2 = Dn.j_b_x[i];
    double y1 = (CODEDIM >= 2) ? Dn.j_a_y[i] : 0.0, y2 = (CODEDIM >= 2) ? Dn.j_b_y[i] : 0.0;
    double z1 = (CODEDIM >= 3) ? Dn.j_a_z[i] : 0.0, z2 = (CODEDIM >= 3) ? Dn.j_b_z[i] : 0.0;
    ta -= p_reg(na) * (x1 * x1 + y1 * y1 + z1 * z1) / na;
    tb -= p_reg(nb) * (x2 * x2 + y2 * y2 + z2 * z2) / nb;
    Ek[i] = 0.5 * (alpha(p) * ta + alpha(-p) * tb) * WTD_VOLEL;
    Ep[i] = funD(na, nb) * WTD_VOLEL;
    Epair[i] = (P.delta[i] * thrust::conj(Dn.nu[i])).real() * (-1.0) * WTD_VOLEL;
    Ec[i] = p_reg(na) * (x1 * x1 + y1 * y1 + z1 * z1) / (2. * na) * WTD_VOLEL +
            p_reg(nb) * (x2 * x2 + y2 * y2 + z2 * z2) / (2. * nb) * WTD_VOLEL;
}
#elif FUNCTIONAL == BDG
/* tdwslda_functionals.h:373-452 */
__global__ void wtd_potentials_kernel(int it, wslda_density Dn, wslda_potential P, double cccoeff)
{
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= WTD_NUMEL) return;
    int ix, iy, iz; wtd_decode(i, ix, iy, iz);
    double Va = WTD_U_EXT(ix, iy, iz, it, SPINA);
    double Vb = WTD_U_EXT(ix, iy, iz, it, SPINB);
    double ap = 0.5 * (P.alpha_a[i] + P.alpha_b[i]);
    double t5 = 1.0 / (4.0 * M_PI * scattering_length(ix, iy, iz, it, dc_params, dc_extra_data_size, dc_extra_data) * ap);
    Complex lnu = Dn.nu[i], one(1.0, 0.0), p0, kc, wz;
#ifdef INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
    double nab = Dn.rho_a[i] + Dn.rho_b[i];
    double lkF = pow(3.0 * M_PI * M_PI * nab, 1.0 / 3.0);
#endif
    double t7 = (dc_mu_a - P.V_a[i] + dc_mu_b - P.V_b[i]) / 2.0;
    p0 = thrust::sqrt(Complex(2.0 * t7, 0.0));
    if (p0.imag() < 0.) p0 *= -1.;
#ifdef USE_CUBIC_CUTOFF
    kc = Complex(M_PI / DX, 0.0);
#else
    kc = thrust::sqrt(Complex(2.0 * (dc_ec + t7), 0.0));
    if (kc.imag() < 0.) kc *= -1.;
#endif
    wz = thrust::log((kc + p0) / (kc - p0));
    if (wz.imag() < 0.) wz += Complex(0.0, 2. * M_PI);
    wz = kc * REG_COEFF_R0 / ap * (1. - (p0 / kc) * REG_COEFF_R1 * wz);
    wz = one / (one * t5 - wz);
    Complex ld = lnu * (-1.0 * wz.real());
#ifdef INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
    {
        double bc = (p0 / (lkF + 1.0e-12)).real();
        double lx = bc * lkF * DX / M_PI;
        if (wz.real() < -1.0e-10 && lx > 1.0e-10) {
            double L0 = bc * REG_COEFF_R0 / lx * (1.0 - REG_COEFF_R1 * lx * log((1.0 + lx) / (1.0 - lx)));
            double dL0 = (-2. * bc * REG_COEFF_R0 * REG_COEFF_R1) / (1. - lx * lx) - bc * REG_COEFF_R0 / lx / lx;
            double dLdn = (lkF / (3. * nab * ap)) * (L0 + dL0 * bc * DX * lkF / M_PI);
            double tn = thrust::norm(ld);
            Va += dLdn * tn;
            Vb += dLdn * tn;
        }
    }
#endif
    P.V_a[i] = Va; P.V_b[i] = Vb; P.delta[i] = ld;
}

/* tdwslda_functionals.h:455-503 */
__global__ void wtd_energy_kernel(int it, wslda_density Dn, wslda_potential P, double *Ek, double *Ep, double *Epair, double *Ec)
{
    using namespace edf;
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= WTD_NUMEL) return;
    double na = Dn.rho_a[i], nb = Dn.rho_b[i];
    double ta = Dn.tau_a[i], tb = Dn.tau_b[i];
    double x1 = Dn.j_a_x[i], x2 = Dn.j_b_x[i];
    double y1 = (CODEDIM >= 2) ? Dn.j_a_y[i] : 0.0, y2 = (CODEDIM >= 2) ? Dn.j_b_y[i] : 0.0;
    double z1 = (CODEDIM >= 3) ? Dn.j_a_z[i] : 0.0, z2 = (CODEDIM >= 3) ? Dn.j_b_z[i] : 0.0;
    ta -= p_reg(na) * (x1 * x1 + y1 * y1 + z1 * z1) / na;
    tb -= p_reg(nb) * (x2 * x2 + y2 * y2 + z2 * z2) / nb;
    Ek[i] = 0.5 * (P.alpha_a[i] * ta + P.alpha_b[i] * tb) * WTD_VOLEL;
    Ep[i] = 0.0;
    Epair[i] = (P.delta[i] * thrust::conj(Dn.nu[i])).real() * (-1.0) * WTD_VOLEL;
    Ec[i] = p_reg(na) * (x1 * x1 + y1 * y1 + z1 * z1) / (2. * na) * WTD_VOLEL +
            p_reg(nb) * (x2 * x2 + y2 * y2 + z2 * z2) / (2. * nb) * WTD_VOLEL;
}
#elif FUNCTIONAL == SLDAE
/* tdwslda_functionals.h:530-812: spin-symmetric parameters a, b, c of x = |a kF|, the
 * current-correction terms with alpha_a = alpha_b = a(x), and the local self-consistent
 * solution for U and Delta with g_eff = a / (c~ - Lambda) */
__global__ void wtd_potentials_kernel(int it, wslda_density Dn, wslda_potential P, double cccoeff)
{
    using namespace edf;
    using namespace sldae;
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= WTD_NUMEL) return;
    int ix, iy, iz; wtd_decode(i, ix, iy, iz);
    double Va_c = WTD_U_EXT(ix, iy, iz, it, SPINA);
    double Vb_c = WTD_U_EXT(ix, iy, iz, it, SPINB);
    double na = Dn.rho_a[i], nb = Dn.rho_b[i];
    double ta = Dn.tau_a[i], tb = Dn.tau_b[i];
    double nt = na + nb;
    double n13 = pow(nt, 1. / 3.), n23 = pow(nt, 2. / 3.);
    double kF = kfermi(nt), eF = kF * kF / 2.;
    double x = fabs(scattering_length(ix, iy, iz, it, dc_params, dc_extra_data_size, dc_extra_data) * kF);
    double nreg = p_reg(nt);
    double bet = beta(x), ig = inverse_gamma(x);
    double af = a_functional(x), cf = c_functional(x);
    double af_p = 0.0, cf_p = 0.0;
    if (nreg > 0.0) {
        af_p = nreg * x / (3. * nt) * a_functional_d1(x);
        cf_p = nreg * cf / (3. * nt) * (1. - cf * ig);
    }
    double ct = af * n13 / cf;
    double igeff = (1 / cf) * (1. - 3. * nt / cf * cf_p);
    double ct_p = (nreg > 0.) ? pow(nreg, 2. / 3.) * igeff * af / (3. * n23) : 0.;
    ct_p += af_p * n13 / cf;
#ifdef CURRENT_CORRECTIONS
    P.alpha_a[i] = af; P.alpha_b[i] = af;
    double jx = Dn.j_a_x[i], kx = Dn.j_b_x[i];
    double jy = (CODEDIM >= 2) ? Dn.j_a_y[i] : 0.0, ky = (CODEDIM >= 2) ? Dn.j_b_y[i] : 0.0;
    double jz = (CODEDIM >= 3) ? Dn.j_a_z[i] : 0.0, kz = (CODEDIM >= 3) ? Dn.j_b_z[i] : 0.0;
    {
        double t4 = p_reg(na) * cccoeff;
        P.A_a_x[i] = (t4 == 0.0) ? 0.0 : t4 * (1. - af) * jx / na;
        if (CODEDIM >= 2) P.A_a_y[i] = (t4 == 0.0) ? 0.0 : t4 * (1. - af) * jy / na;
        if (CODEDIM >= 3) P.A_a_z[i] = (t4 == 0.0) ? 0.0 : t4 * (1. - af) * jz / na;
        t4 = p_reg(nb) * cccoeff;
        P.A_b_x[i] = (t4 == 0.0) ? 0.0 : t4 * (1. - af) * kx / nb;
        if (CODEDIM >= 2) P.A_b_y[i] = (t4 == 0.0) ? 0.0 : t4 * (1. - af) * ky / nb;
        if (CODEDIM >= 3) P.A_b_z[i] = (t4 == 0.0) ? 0.0 : t4 * (1. - af) * kz / nb;
    }
#endif
    Va_c += af_p * (ta + tb) / 2.;
    Vb_c += af_p * (ta + tb) / 2.;
    Va_c += bet * eF;
    Vb_c += bet * eF;
#ifdef CURRENT_CORRECTIONS
    {
        double t7 = p_reg(na) * cccoeff;
        if (t7 != 0.0) {
            double j2 = jx * jx + jy * jy + jz * jz;
            t7 = t7 * j2 / (2.0 * na);
            Va_c += ((af - 1.0) / na - af_p) * t7;
            Va_c -= cccoeff * dp_reg(na) * (af - 1.0) * j2 / (2.0 * na);
            Vb_c -= af_p * t7;
        }
        t7 = p_reg(nb) * cccoeff;
        if (t7 != 0.0) {
            double k2 = kx * kx + ky * ky + kz * kz;
            t7 = t7 * k2 / (2.0 * nb);
            Va_c -= af_p * t7;
            Vb_c += ((af - 1.0) / nb - af_p) * t7;
            Vb_c -= cccoeff * dp_reg(nb) * (af - 1.0) * k2 / (2.0 * nb);
        }
    }
#endif
    double Va = P.V_a[i], Vb = P.V_b[i];
    Complex lnu = Dn.nu[i], ld = P.delta[i], p0, kc, wz;
#ifdef INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
    double lkF = pow(3.0 * M_PI * M_PI * (na + nb), 1.0 / 3.0);
#endif
    for (int k = 0; k < UD_SCITERS; k++) {
        double lmu = (dc_mu_a - Va + dc_mu_b - Vb) / 2.;
        p0 = thrust::sqrt(Complex(2.0 * lmu / af, 0.0));
        if (p0.imag() < 0.) p0 *= -1.;
#ifdef USE_CUBIC_CUTOFF
        kc = Complex(M_PI / DX, 0.0);
#else
        kc = thrust::sqrt(Complex(2.0 * (dc_ec + lmu) / af, 0.0));
        if (kc.imag() < 0.) kc *= -1.;
#endif
        wz = thrust::log((kc + p0) / (kc - p0));
        if (wz.imag() < 0.) wz += Complex(0.0, 2. * M_PI);
        wz = kc * REG_COEFF_R0 * (1. - (p0 / kc) * REG_COEFF_R1 * wz);
        double geff = af / (ct - wz.real());
        ld = lnu * (-geff);
        double dn = (thrust::conj(ld) * lnu).real();
        double d2 = ld.real() * ld.real() + ld.imag() * ld.imag();
        double Van = Va_c - (af_p / af) * dn - ct_p / af * d2;
        double Vbn = Vb_c - (af_p / af) * dn - ct_p / af * d2;
#ifdef INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
        {
            double bc = (p0 / (lkF + 1.0e-12)).real();
            double lx = bc * lkF * DX / M_PI;
            if (geff < -1.0e-10 && lx > 1.0e-10) {
                double L0 = bc * REG_COEFF_R0 / lx * (1.0 - REG_COEFF_R1 * lx * log((1.0 + lx) / (1.0 - lx)));
                double dL0 = (-2. * bc * REG_COEFF_R0 * REG_COEFF_R1) / (1. - lx * lx) - bc * REG_COEFF_R0 / lx / lx;
                double dLdn = (lkF / (3. * (na + nb) * af)) * (L0 + dL0 * bc * DX * lkF / M_PI);
                Van += dLdn * d2;
                Vbn += dLdn * d2;
            }
        }
#endif
        Va = UD_MIX_COEFF * Van + (1. - UD_MIX_COEFF) * Va;
        Vb = UD_MIX_COEFF * Vbn + (1. - UD_MIX_COEFF) * Vb;
    }
    P.V_a[i] = Va; P.V_b[i] = Vb; P.delta[i] = ld;
}

/* tdwslda_functionals.h:815-884 */
__global__ void wtd_energy_kernel(int it, wslda_density Dn, wslda_potential P, double *Ek, double *Ep, double *Epair, double *Ec)
{
    using namespace edf;
    using namespace sldae;
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= WTD_NUMEL) return;
    int ix, iy, iz; wtd_decode(i, ix, iy, iz);
    double na = Dn.rho_a[i], nb = Dn.rho_b[i];
    double ta = Dn.tau_a[i], tb = Dn.tau_b[i];
    double x1 = Dn.j_a_x[i], x2 = Dn.j_b_x[i];
    double y1 = (CODEDIM >= 2) ? Dn.j_a_y[i] : 0.0, y2 = (CODEDIM >= 2) ? Dn.j_b_y[i] : 0.0;
    double z1 = (CODEDIM >= 3) ? Dn.j_a_z[i] : 0.0, z2 = (CODEDIM >= 3) ? Dn.j_b_z[i] : 0.0;
    ta -= p_reg(na) * (x1 * x1 + y1 * y1 + z1 * z1) / na;
    tb -= p_reg(nb) * (x2 * x2 + y2 * y2 + z2 * z2) / nb;
    double nt = na + nb;
    double kF = kfermi(nt), eF = kF * kF / 2.;
    double x = fabs(scattering_length(ix, iy, iz, it, dc_params, dc_extra_data_size, dc_extra_data) * kF);
    double af = a_functional(x), bf = b_functional(x);
    Ek[i] = af * (ta + tb) / 2. * WTD_VOLEL;
    Ep[i] = (3. / 5.) * bf * eF * nt * WTD_VOLEL;
    Epair[i] = (P.delta[i] * thrust::conj(Dn.nu[i])).real() * (-1.0) * WTD_VOLEL;
    Ec[i] = p_reg(na) * (x1 * x1 + y1 * y1 + z1 * z1) / (2. * na) * WTD_VOLEL +
            p_reg(nb) * (x2 * x2 + y2 * y2 + z2 * z2) / (2. * nb) * WTD_VOLEL;
}
#elif FUNCTIONAL == CUSTOMEDF
/* the user's kernels from problem-definition.h (hpc-engine/tdwslda_functionals.h:891-897) */
#define wtd_potentials_kernel tdwslda_compute_potentials
#define wtd_energy_kernel tdwslda_compute_energy
#endif

/* threads per CTA of the potentials kernel: the built-in functionals are a few hundred FP64
 * operations per point on a lattice of a few thousand points, so one warp per CTA spreads them
 * over more SMs; the user's CUSTOMEDF kernel keeps the reference's launch shape */
#if FUNCTIONAL == CUSTOMEDF
#define WTD_POT_THREADS 128
#else
#define WTD_POT_THREADS 32
#endif

/* external-field energies, particle number and L_z integrands
 * (pca_kernels.cu:121-209; cpca_kernels.cu:121-209; tdwslda_energy_generic.h:40-92) */
__global__ void wtd_energy_ext_kernel(int it, wslda_density Dn, wslda_potential P, double *e)
{
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= WTD_NUMEL) return;
    int ix, iy, iz; wtd_decode(i, ix, iy, iz);
    const size_t N = WTD_NUMEL;
    double na = Dn.rho_a[i], nb = Dn.rho_b[i];
#ifdef ENABLE_V_EXT
    e[EPOTEXT * N + i] = (na * WTD_U_EXT(ix, iy, iz, it, SPINA) + nb * WTD_U_EXT(ix, iy, iz, it, SPINB)) * WTD_VOLEL;
#else
    e[EPOTEXT * N + i] = 0.0;
#endif
#ifdef ENABLE_DELTA_EXT
    e[EPAIREXT * N + i] = (thrust::conj(Dn.nu[i]) * WTD_D_EXT(ix, iy, iz, it, P.delta[i])).real() * (-2.0) * WTD_VOLEL;
#else
    e[EPAIREXT * N + i] = 0.0;
#endif
#ifdef ENABLE_VELOCITY_EXT
    /* -(j_a . v_a + j_b . v_b) (pca_kernels.cu:163-187; cpca/ccpca over their axes) */
    {
        const double *ja[3] = {Dn.j_a_x, Dn.j_a_y, Dn.j_a_z}, *jb[3] = {Dn.j_b_x, Dn.j_b_y, Dn.j_b_z};
        double s = 0.0;
        for (int d = 0; d < CODEDIM; d++)
            s += ja[d][i] * WTD_VEL_EXT(ix, iy, iz, it, SPINA, d) + jb[d][i] * WTD_VEL_EXT(ix, iy, iz, it, SPINB, d);
        e[EVELEXT * N + i] = s * (-1.0) * WTD_VOLEL;
    }
#else
    e[EVELEXT * N + i] = 0.0;
#endif
    e[NPARTA * N + i] = na;
    e[NPARTB * N + i] = nb;
#if CODEDIM >= 2
    double x = (double)(ix - NX / 2) * DX, y = (double)(iy - NY / 2) * DY;
    e[LZA * N + i] = (x * Dn.j_a_y[i] - y * Dn.j_a_x[i]) * WTD_VOLEL;
    e[LZB * N + i] = (x * Dn.j_b_y[i] - y * Dn.j_b_x[i]) * WTD_VOLEL;
#else
    e[LZA * N + i] = 0.0;
    e[LZB * N + i] = 0.0;
#endif
}

#endif
