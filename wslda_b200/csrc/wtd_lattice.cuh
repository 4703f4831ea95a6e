/*
 * Host-side facts of the compiled lattice shared by the fused ABI, the staged large-lattice
 * path and the reference-named ABI: the geometry type, the mass mode and the error helpers.
 */
#ifndef WTD_LATTICE_CUH
#define WTD_LATTICE_CUH

#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "wtd.h"
#include "wtd_aux.cuh"

#if CODEDIM == 1
typedef Geo<NX, 1, 1> WG;
#elif CODEDIM == 2
typedef Geo<NX, NY, 1> WG;
#else
typedef Geo<NX, NY, NZ> WG;
#endif

#ifdef FAST_CONST_EFFECTIVE_MASS_MODE
#define WTD_VAR false
#else
#define WTD_VAR true
#endif

static constexpr size_t WTD_SMEM_MAX = 232448;
/* shared memory of one field + tables: the single-CTA spectral kernels fit below this */
static constexpr size_t k_field_smem = (size_t)WG::padded * sizeof(double2) + WG::twtotal * sizeof(double2) + sizeof(KTab<WG>);
static constexpr size_t k_derivs_smem = 2 * (size_t)WG::padded * sizeof(double2) + WG::twtotal * sizeof(double2) + sizeof(KTab<WG>);
/* lattices whose fields exceed one CTA's shared memory take the plane/pencil transforms */
static constexpr bool WTD_BIG = (CODEDIM >= 2) && (k_derivs_smem > WTD_SMEM_MAX);

static inline int wtd_cuerr(cudaError_t e) { return e == cudaSuccess ? WTD_OK : WTD_ERR_CUDA; }
#define WTD_TRY(x) do { int _r = (x); if (_r) return _r; } while (0)
#define WTD_CU(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) return WTD_ERR_CUDA; } while (0)

/* statements run once per device (kernel attributes such as the dynamic shared-memory size are
 * per-device settings, and contexts may live on different devices of one process); devices
 * beyond WTD_MAXDEV run them on every call */
#define WTD_MAXDEV 64
#define WTD_ONCE_PER_DEVICE(...)                                                  \
    do {                                                                          \
        static bool _wtd_once[WTD_MAXDEV];                                        \
        int _wtd_dev = -1;                                                        \
        if (cudaGetDevice(&_wtd_dev) != cudaSuccess) return WTD_ERR_CUDA;         \
        const bool _wtd_slot = _wtd_dev >= 0 && _wtd_dev < WTD_MAXDEV;            \
        if (!_wtd_slot || !_wtd_once[_wtd_dev]) {                                 \
            __VA_ARGS__;                                                          \
            if (_wtd_slot) _wtd_once[_wtd_dev] = true;                            \
        }                                                                         \
    } while (0)

/* FFT twiddles e^{-2 pi i t/n} per axis and wave-number tables of digit-reversed positions
 * (rows 0-2 k_d, rows 3-5 k_d with the Nyquist mode zeroed) for this lattice */
static void wtd_make_tables(double2 *tw, double *kt)
{
    memset(kt, 0, 6 * WTD_KT * sizeof(double));
    const double Lax[3] = {LX, LY, LZ};
    for (int a = 0; a < 3; a++) {
        int n = WG::n(a);
        for (int t = 0; t < n; t++) {
            long double ang = 2.0L * 3.14159265358979323846264338327950288L * (long double)t / (long double)n;
            tw[WG::twoff(a) + t] = make_double2((double)cosl(ang), -(double)sinl(ang));
        }
        for (int p = 0; p < n && p < WTD_KT; p++) {
            int f = dif_freq(n, p);
            double k = (f < n / 2) ? 2. * M_PI / Lax[a] * (double)f : 2. * M_PI / Lax[a] * (double)(f - n);
            kt[a * WTD_KT + p] = (n > 1) ? k : 0.0;
            kt[(3 + a) * WTD_KT + p] = (n > 1 && f != n / 2) ? k : 0.0;
        }
    }
}

#endif
