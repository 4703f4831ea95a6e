/*
 * ORACLE (test infrastructure only).  SLDA/ASLDA energy density functional pieces, restated
 * from hpc-engine/pca_edf.h (line numbers cited per function), and the SLDAE parameter fits.  A0..A2, G0, G1, GAMMA0,
 * P_NMIN/P_NMAX/P_ALPHA come from the project's settings (wtd_settings.h).
 */
#ifndef ORACLE_EDF_H
#define ORACLE_EDF_H

namespace oedf {

/* regularisation function and its derivative (pca_edf.h:17-33) */
static inline double p_reg(double n)
{
    if (n <= P_NMIN) return 0.0;
    if (n >= P_NMAX) return 1.0;
    double a = (M_PI * (n - P_NMIN)) / (P_NMAX - P_NMIN) - M_PI / 2.0;
    return 0.5 + 0.5 * std::tanh(P_ALPHA * std::tan(a));
}
static inline double dp_reg(double n)
{
    if (n <= P_NMIN || n >= P_NMAX) return 0.0;
    double a = (M_PI * (n - P_NMIN)) / (P_NMAX - P_NMIN) - M_PI / 2.0;
    double c = std::cosh(P_ALPHA * std::tan(a)) * std::cos(a);
    return 0.5 * P_ALPHA * M_PI / (c * c) / (P_NMAX - P_NMIN);
}
/* polarisation and its derivatives (pca_edf.h:39-97) */
static inline double pol(double a, double b)
{
    double pr = p_reg(a + b);
    return pr == 0.0 ? 0.0 : pr * (a - b) / (a + b);
}
static inline double dpol_da(double a, double b)
{
    double np = a + b, pr = p_reg(np), dpr = dp_reg(np), r = 0.0;
    if (pr != 0.0) r += pr * (2.0 * b) / (np * np);
    if (dpr != 0.0) r += dpr * (a - b) / np;
    return r;
}
static inline double dpol_db(double a, double b)
{
    double np = a + b, pr = p_reg(np), dpr = dp_reg(np), r = 0.0;
    if (pr != 0.0) r += pr * (-2.0 * a) / (np * np);
    if (dpr != 0.0) r += dpr * (a - b) / np;
    return r;
}
/* effective mass alpha(p) (pca_edf.h:102-160) */
static inline double alpha(double p)
{
    double p2 = p * p, p4 = p2 * p2;
    return A0 + A1 * p * (1.0 - (2.0 / 3.0) * p2 + (1.0 / 5.0) * p4) + A2 * p2 * (1.0 - p2 + (1.0 / 3.0) * p4);
}
static inline double alpha_plus(double p) { return 0.5 * (alpha(p) + alpha(-p)); }
static inline double alpha_minus(double p) { return 0.5 * (alpha(p) - alpha(-p)); }
/* d alpha_plus / d n_s and d alpha_minus / d n_s (pca_edf.h:165-211) */
static inline double dap_core(double p)
{
    double p2 = p * p, p4 = p2 * p2;
    return 2.0 * A2 * p * (1.0 - p2 + (1.0 / 3.0) * p4) - 2.0 * A2 * p * p2 * (1.0 - (2.0 / 3.0) * p2);
}
static inline double dam_core(double p)
{
    double p2 = p * p, p4 = p2 * p2;
    return A1 * (1.0 - (2.0 / 3.0) * p2 + (1.0 / 5.0) * p4) - 4.0 * A1 * p2 * ((1.0 / 3.0) - (1.0 / 5.0) * p2);
}
static inline double dap_da(double a, double b) { return dap_core(pol(a, b)) * dpol_da(a, b); }
static inline double dap_db(double a, double b) { return dap_core(pol(a, b)) * dpol_db(a, b); }
static inline double dam_da(double a, double b) { return dam_core(pol(a, b)) * dpol_da(a, b); }
static inline double dam_db(double a, double b) { return dam_core(pol(a, b)) * dpol_db(a, b); }
/* normal-phase energy D(n_a, n_b) and its derivatives (pca_edf.h:216-311) */
static inline double funG(double p) { return G0 + G1 * p * p; }
static inline double funD(double a, double b)
{
    double p = pol(a, b);
    return (1.0 / (20.0 * M_PI * M_PI)) * std::pow(6.0 * M_PI * M_PI * (a + b), 5.0 / 3.0) *
           (funG(p) - alpha(p) * std::pow((1.0 + p) / 2.0, 5.0 / 3.0) - alpha(-p) * std::pow((1.0 - p) / 2.0, 5.0 / 3.0));
}
static inline double dD_common(double a, double b, double dp)
{
    double p = pol(a, b), p2 = p * p, p4 = p2 * p2;
    double dA = A1 * (1.0 - (2.0 / 3.0) * p2 + (1.0 / 5.0) * p4) - 4.0 * A1 * p2 * ((1.0 / 3.0) - (1.0 / 5.0) * p2);
    double dB = 2.0 * A2 * p * (1.0 - p2 + (1.0 / 3.0) * p4) - 2.0 * A2 * p * p2 * (1.0 - (2.0 / 3.0) * p2);
    double t1 = 0.5 * std::pow(6.0 * M_PI * M_PI * (a + b), 2.0 / 3.0) *
                (funG(p) - alpha(p) * std::pow((1.0 + p) / 2.0, 5.0 / 3.0) - alpha(-p) * std::pow((1.0 - p) / 2.0, 5.0 / 3.0));
    double t2 = (1.0 / (20.0 * M_PI * M_PI)) * std::pow(6.0 * M_PI * M_PI * (a + b), 5.0 / 3.0) *
                (2.0 * G1 * p
                 - (dA + dB) * std::pow((1.0 + p) / 2.0, 5.0 / 3.0)
                 - (5.0 / 6.0) * alpha(p) * std::pow((1.0 + p) / 2.0, 2.0 / 3.0)
                 - (-dA + dB) * std::pow((1.0 - p) / 2.0, 5.0 / 3.0)
                 + (5.0 / 6.0) * alpha(-p) * std::pow((1.0 - p) / 2.0, 2.0 / 3.0)) * dp;
    return t1 + t2;
}
static inline double dD_da(double a, double b) { return dD_common(a, b, dpol_da(a, b)); }
static inline double dD_db(double a, double b) { return dD_common(a, b, dpol_db(a, b)); }
/* pairing coupling tilde C and its derivatives (pca_edf.h:316-350) */
static inline double tildeC(double a, double b)
{
    return alpha_plus(pol(a, b)) * std::pow(a + b + DENSEPSILON, 1.0 / 3.0) / GAMMA0;
}
static inline double dtC_da(double a, double b)
{
    return (dap_da(a, b) * std::pow(a + b + DENSEPSILON, 1.0 / 3.0) +
            (1.0 / 3.0) * alpha_plus(pol(a, b)) * std::pow(a + b + DENSEPSILON, -2.0 / 3.0)) / GAMMA0;
}
static inline double dtC_db(double a, double b)
{
    return (dap_db(a, b) * std::pow(a + b + DENSEPSILON, 1.0 / 3.0) +
            (1.0 / 3.0) * alpha_plus(pol(a, b)) * std::pow(a + b + DENSEPSILON, -2.0 / 3.0)) / GAMMA0;
}
} // namespace oedf

#if FUNCTIONAL == SLDAE
/* SLDAE parameter fits (hpc-engine/sldae_functional.c:68-330): Pade[4/4] forms in x = |a kF|,
 * written term by term as the reference does; the coefficient tables come from wtd_settings.h */
namespace osldae {
static inline double pade_num(double x, const double *a) { return a[0] * x + a[1] * x * x + a[2] * std::pow(x, 3) + a[3] * std::pow(x, 4); }
static inline double pade_den(double x, const double *b) { return 1. + b[0] * x + b[1] * x * x + b[2] * std::pow(x, 3) + b[3] * std::pow(x, 4); }
/* sldae_functional.c:68-72 */
static inline double pade_d0(double x, const double *a, const double *b) { return pade_num(x, a) / pade_den(x, b); }
/* sldae_functional.c:74-80 */
static inline double pade_d1(double x, const double *a, const double *b)
{
    double dn = a[0] + 2. * a[1] * x + 3. * a[2] * x * x + 4. * a[3] * std::pow(x, 3);
    double dd = b[0] + 2. * b[1] * x + 3. * b[2] * x * x + 4. * b[3] * std::pow(x, 3);
    double d = pade_den(x, b);
    return -(dd * pade_num(x, a)) / (d * d) + dn / d;
}
static const double AL_A[4] = {0.0, WTD_SLDAE_ALPHA_A2, WTD_SLDAE_ALPHA_A3, WTD_SLDAE_ALPHA_A4};
static const double AL_B[4] = {WTD_SLDAE_ALPHA_B1, WTD_SLDAE_ALPHA_B2, WTD_SLDAE_ALPHA_B3, WTD_SLDAE_ALPHA_B4};
static const double BE_A[4] = {SLDAE_beta_a1, SLDAE_beta_a2, SLDAE_beta_a3, SLDAE_beta_c};
static const double BE_B[4] = {SLDAE_beta_b1, SLDAE_beta_b2, SLDAE_beta_b3, SLDAE_beta_c};
static const double IG_A[4] = {SLDAE_inverse_gamma_a1, SLDAE_inverse_gamma_a2, SLDAE_inverse_gamma_a3, SLDAE_inverse_gamma_c};
static const double IG_B[4] = {SLDAE_inverse_gamma_b1, SLDAE_inverse_gamma_b2, SLDAE_inverse_gamma_b3, SLDAE_inverse_gamma_c};
static const double BF_A[4] = {SLDAE_b_functional_a1, SLDAE_b_functional_a2, SLDAE_b_functional_a3, SLDAE_b_functional_c};
static const double BF_B[4] = {SLDAE_b_functional_b1, SLDAE_b_functional_b2, SLDAE_b_functional_b3, SLDAE_b_functional_c};
static const double CF_A[4] = {SLDAE_c_functional_a1, SLDAE_c_functional_a2, SLDAE_c_functional_a3, SLDAE_c_functional_c};
static const double CF_B[4] = {SLDAE_c_functional_b1, SLDAE_c_functional_b2, SLDAE_c_functional_b3, SLDAE_c_functional_c};
#ifdef SLDA_FORCE_A1
static inline double alpha_d0(double) { return 1.; }
static inline double alpha_d1(double) { return 0.; }
#else
static inline double alpha_d0(double x) { return 1. + pade_d0(x, AL_A, AL_B); }
static inline double alpha_d1(double x) { return pade_d1(x, AL_A, AL_B); }
#endif
static inline double beta_d0(double x) { return BF_APS_UFG * pade_d0(x, BE_A, BE_B); }
static inline double inverse_gamma_d0(double x) { return (1. / CF_APS_UFG) * pade_d0(x, IG_A, IG_B); }
static inline double a_functional_d0(double x) { return alpha_d0(x); }
static inline double b_functional_d0(double x) { return BF_APS_UFG * pade_d0(x, BF_A, BF_B); }
static inline double c_functional_d0(double x) { return CF_APS_UFG * pade_d0(x, CF_A, CF_B); }
} // namespace osldae
#endif
#endif
