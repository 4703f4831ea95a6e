/*
 * ORACLE (test infrastructure only).  SLDA/ASLDA energy density functional pieces, restated
 * from hpc-engine/pca_edf.h (line numbers cited per function).  A0..A2, G0, G1, GAMMA0,
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
#endif
