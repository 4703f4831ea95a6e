/*
 * The subset of the FFTW3 API that the reference's spectral-derivative library uses
 * (lib/wderiv/c/wderiv.c: fftw_plan_dft_{1d,2d,3d}, fftw_plan_dft_{r2c,c2r}_{1d,2d,3d},
 * fftw_execute, fftw_destroy_plan), implemented over this repository's own CPU FFT
 * (fftw_shim.c).  FFTW itself is not installed here; this header lets wderiv.c compile
 * unmodified so that the host-core baseline runs the reference's own derivative code.
 * Test infrastructure only: nothing in the product links it.
 *
 * Conventions are FFTW's: row-major arrays (last index fastest), FFTW_FORWARD = -1 is
 * e^{-2 pi i k n / N}, every transform unnormalised, r2c writes n_last/2 + 1 complex numbers
 * per row, c2r reads them (Hermitian symmetry implied) and may overwrite its input.
 */
#ifndef WTD_FFTW_SHIM_H
#define WTD_FFTW_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

/* as FFTW: the C99 complex type when <complex.h> was included first, else double[2] */
#if !defined(__cplusplus) && defined(_Complex_I) && defined(complex) && defined(I)
typedef double _Complex fftw_complex;
#else
typedef double fftw_complex[2];
#endif

typedef struct wtd_fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif
#endif
