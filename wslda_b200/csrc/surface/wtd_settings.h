/*
 * Compile-time configuration of a project: derives the evolution mode from the user's
 * predefines.h exactly as hpc-engine/pca_settings.h:36-95,143-241 does, and defines the
 * names user hook code relies on (NXYZ, DXYZ, LX, SPINA, XAXIS, energy slots, ...).
 *
 * Names and numeric values are kept identical to the reference because they are part of the
 * plugin surface: problem-definition.h files written for W-SLDA test them (FUNCTIONAL==SLDA,
 * CODEDIM, SPINA, ...) and the functional constants (A0..A2, G0, G1, GAMMA0, regularisation)
 * are the published parameters of the SLDA/ASLDA energy density functional.
 *
 * Include after predefines.h.  CODEDIM (1, 2 or 3) is given on the compiler command line.
 */
#ifndef WTD_SETTINGS_H
#define WTD_SETTINGS_H

#ifndef CODEDIM
#error "CODEDIM must be defined (1, 2 or 3)"
#endif

/* functional selectors (pca_settings.h:69-73) */
#define SLDA 111
#define ASLDA 112
#define BDG 113
#define CUSTOMEDF 114
#define SLDAE 115

/* integration schemes (pca_settings.h:203-205) */
#define AB3AM4 34
#define AB4AM5 45
#define AB5AM5 55
#ifndef INTEGRATION_SCHEME
#define INTEGRATION_SCHEME AB4AM5
#endif

/* regularisation schemes (pca_settings.h:224-225) */
#define SPHERICAL_CUTOFF 88
#define CUBIC_CUTOFF 89

/* self-consistent local solve of U and Delta (pca_settings.h:36-38) */
#define UD_SCITERS 15
#define UD_MIX_COEFF 0.75

/* legacy spellings (pca_settings.h:52-63) */
#ifdef SLDAE_FORCE_A1
#define SLDA_FORCE_A1
#endif
#ifdef ASLDA_STABILIZATION_RETAIN_ABOVE_DENSITY
#define SLDA_STABILIZATION_RETAIN_ABOVE_DENSITY ASLDA_STABILIZATION_RETAIN_ABOVE_DENSITY
#endif
#ifdef ASLDA_STABILIZATION_EXCLUDE_BELOW_DENISTY
#define SLDA_STABILIZATION_EXCLUDE_BELOW_DENISTY ASLDA_STABILIZATION_EXCLUDE_BELOW_DENISTY
#endif

#if FUNCTIONAL==SLDAE
/* SLDAE: the published Pade[4/4] fits of the extended SLDA functional of Boulet et al.
 * (hpc-engine/sldae_parameters.h, sldae_parameters_A1.h, sldae_functional.c:93-330).  Each
 * parameter is P(x) = s * (a1 x + a2 x^2 + a3 x^3 + a4 x^4) / (1 + b1 x + b2 x^2 + b3 x^3 + b4 x^4)
 * of x = |a kF|, with a4 = b4 = c for the fitted sets.  The effective-mass fit alpha(x) =
 * 1 + P(x) is the same for both sets and becomes alpha = 1 under SLDA_FORCE_A1. */
#define WTD_SLDAE_ALPHA_A2 (-0.2081560)
#define WTD_SLDAE_ALPHA_A3 (-0.1358830)
#define WTD_SLDAE_ALPHA_A4 (-0.0162071)
#define WTD_SLDAE_ALPHA_B1 (2.09838000)
#define WTD_SLDAE_ALPHA_B2 (1.73800000)
#define WTD_SLDAE_ALPHA_B3 (0.66854900)
#define WTD_SLDAE_ALPHA_B4 (0.10150800)
#ifdef SLDA_FORCE_A1
#define SLDAE_beta_a1 +0.797400
#define SLDAE_beta_a2 +0.943961
#define SLDAE_beta_a3 +1.037043
#define SLDAE_beta_b1 +1.227062
#define SLDAE_beta_b2 +2.126210
#define SLDAE_beta_b3 +1.734795
#define SLDAE_beta_c  +0.523445
#define SLDAE_b_functional_a1 +0.698112
#define SLDAE_b_functional_a2 +0.034678
#define SLDAE_b_functional_a3 +0.455138
#define SLDAE_b_functional_b1 +0.353905
#define SLDAE_b_functional_b2 +0.806444
#define SLDAE_b_functional_b3 +0.403679
#define SLDAE_b_functional_c  -0.031327
#define SLDAE_inverse_gamma_a1 +2.713374
#define SLDAE_inverse_gamma_a2 +1.441196
#define SLDAE_inverse_gamma_a3 +3.700251
#define SLDAE_inverse_gamma_b1 +0.634303
#define SLDAE_inverse_gamma_b2 +3.522427
#define SLDAE_inverse_gamma_b3 +3.701347
#define SLDAE_inverse_gamma_c  +1.877961
#define SLDAE_c_functional_a1 +0.370145
#define SLDAE_c_functional_a2 +1.041299
#define SLDAE_c_functional_a3 +1.737347
#define SLDAE_c_functional_b1 +2.458364
#define SLDAE_c_functional_b2 +5.604947
#define SLDAE_c_functional_b3 +3.828124
#define SLDAE_c_functional_c  +1.085400
#define AF_APS_UFG +1.000000
#define BF_APS_UFG -0.481506
#define CF_APS_UFG -10.532397
#else
#define SLDAE_beta_a1 +1.58442
#define SLDAE_beta_a2 +17.2973
#define SLDAE_beta_a3 +0.820671
#define SLDAE_beta_b1 +13.9448
#define SLDAE_beta_b2 +10.1914
#define SLDAE_beta_b3 +11.9429
#define SLDAE_beta_c  +3.48966
#define SLDAE_b_functional_a1 +1.29871
#define SLDAE_b_functional_a2 +6.02212
#define SLDAE_b_functional_a3 +0.376541
#define SLDAE_b_functional_b1 +6.47079
#define SLDAE_b_functional_b2 +3.73389
#define SLDAE_b_functional_b3 +3.47301
#define SLDAE_b_functional_c  +0.810972
#define SLDAE_inverse_gamma_a1 +6.15853
#define SLDAE_inverse_gamma_a2 +0.156722
#define SLDAE_inverse_gamma_a3 +0.76668
#define SLDAE_inverse_gamma_b1 +1.48431
#define SLDAE_inverse_gamma_b2 +2.07468
#define SLDAE_inverse_gamma_b3 +0.737836
#define SLDAE_inverse_gamma_c  +0.0823379
#define SLDAE_c_functional_a1 +0.267952
#define SLDAE_c_functional_a2 +0.754923
#define SLDAE_c_functional_a3 +0.330699
#define SLDAE_c_functional_b1 +2.61695
#define SLDAE_c_functional_b2 +2.71855
#define SLDAE_c_functional_b3 +0.550587
#define SLDAE_c_functional_c  +0.0900897
#define AF_APS_UFG (0.8403360)
#define BF_APS_UFG (-0.281863)
#define CF_APS_UFG (-14.95950)
#endif
#endif

/* mode derivation (pca_settings.h:75-95, 186-222) */
#if FUNCTIONAL==BDG
#define BDG_MODE
#define SLDA_FORCE_A1
#endif
#if FUNCTIONAL==SLDA
#define SLDA_FORCE_A1
#endif

#ifdef SLDA_FORCE_A1
#define A0 1.000
#define A1 0.0
#define A2 0.0
#define FAST_CONST_EFFECTIVE_MASS_MODE
#else
#define A0 1.094
#define A1 0.156
#define A2 -0.532
#define CURRENT_CORRECTIONS
#endif

#define G0 0.357
#define G1 0.642

#ifdef SLDA_STABILIZATION_EXCLUDE_BELOW_DENISTY
#define P_NMIN SLDA_STABILIZATION_EXCLUDE_BELOW_DENISTY
#else
#define P_NMIN 1.0e-7
#endif
#ifdef SLDA_STABILIZATION_RETAIN_ABOVE_DENSITY
#define P_NMAX SLDA_STABILIZATION_RETAIN_ABOVE_DENSITY
#else
#define P_NMAX 1.0e-5
#endif
#define P_ALPHA 1.0

#ifdef ENABLE_MODIFY_POTENTIALS
#undef BDG_MODE
#endif
#ifdef SLDA_FORCE_A1
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
#define FAST_CONST_EFFECTIVE_MASS_MODE
#endif
#endif
#ifdef FAST_CONST_EFFECTIVE_MASS_MODE
#undef CURRENT_CORRECTIONS
#endif
#ifdef BDG_MODE
#undef CURRENT_CORRECTIONS
#ifndef FAST_CONST_EFFECTIVE_MASS_MODE
#define FAST_CONST_EFFECTIVE_MASS_MODE
#endif
#endif
/* an external velocity field needs the gradient (current) terms of H: variable-mass path
 * (pca_settings.h:217-220) */
#ifdef ENABLE_VELOCITY_EXT
#define CURRENT_CORRECTIONS
#undef FAST_CONST_EFFECTIVE_MASS_MODE
#endif

#if REGULARIZATION_SCHEME==CUBIC_CUTOFF
#define USE_CUBIC_CUTOFF
#define GAMMA0 -11.11
#define REG_COEFF_K 2.442749607806335
#define REG_COEFF_R0 (REG_COEFF_K/(4.0*M_PI*M_PI))
#define REG_COEFF_R1 0.31786000
#else
#define GAMMA0 -11.11
#define REG_COEFF_R0 (1./(2.0*M_PI*M_PI))
#define REG_COEFF_R1 0.5
#endif

#ifndef DENSEPSILON
#define DENSEPSILON 1.0e-8
#endif
#ifndef MAX_USER_PARAMS
#define MAX_USER_PARAMS 32
#endif

/* lattice helpers (pca_settings.h:123-139) */
#define NUMERICAL_ZERO 1.0e-16
#define DXYZ (DX*DY*DZ)
#define DXY (DX*DY)
#define LX (DX*NX)
#define LY (DY*NY)
#define LZ (DZ*NZ)
#define LXYZ (LX*LY*LZ)
#define NXYZ (NX*NY*NZ)
#define NXY (NX*NY)
#define LXY (LX*LY)

#define SPINA 0
#define SPINB 1
#define XAXIS 0
#define YAXIS 1
#define ZAXIS 2

/* observable slots written by compute_energy (pca_settings.h:143-158) */
#define ENERGYITEMS 7
#define EKIN 0
#define EPOT 1
#define EPAIR 2
#define ECURRENT 3
#define EPOTEXT 4
#define EPAIREXT 5
#define EVELEXT 6
#define TDWSLDAITEMS (ENERGYITEMS+4)
#define NPARTA 7
#define NPARTB 8
#define LZA 9
#define LZB 10

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#ifndef M_PI_2
#define M_PI_2 1.570796326794896558
#endif
#ifndef API_VERSION
#define API_VERSION 20220218
#endif

/* ---- derived per-dimension quantities used by this library ---- */
#if CODEDIM==1
#define WTD_NUMEL (NX)
#define WTD_DV (DX)                 /* measure of one lattice point in norms and <psi|H|psi> */
#define WTD_LPERP ((double)(LY*LZ)) /* plane-wave normalisation divided out of densities */
#define WTD_VOLEL (DXYZ*NY*NZ)     /* VOLUME_ELEMENT of the energy kernels */
#elif CODEDIM==2
#define WTD_NUMEL (NX*NY)
#define WTD_DV (DX*DY)
#define WTD_LPERP ((double)(LZ))
#define WTD_VOLEL (DXYZ*NZ)
#else
#define WTD_NUMEL (NX*NY*NZ)
#define WTD_DV (DXYZ)
#define WTD_LPERP (1.0)
#define WTD_VOLEL (DXYZ)
#endif

#if INTEGRATION_SCHEME==AB3AM4
#define WTD_NHIST 3
#elif INTEGRATION_SCHEME==AB4AM5
#define WTD_NHIST 4
#elif INTEGRATION_SCHEME==AB5AM5
#define WTD_NHIST 5
#else
#error "INTEGRATION_SCHEME must be AB3AM4, AB4AM5 or AB5AM5"
#endif

#endif /* WTD_SETTINGS_H */
