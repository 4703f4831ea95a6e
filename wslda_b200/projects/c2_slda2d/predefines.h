/* 2D TD-SLDA: 64x64, dx=1 (periodic), harmonic trap omega=0.04, vortex Delta_ext. */
#define NX (64)
#define NY (64)
#define NZ (1)
#define DX (1.0)
#define DY (1.0)
#define DZ (1.0)

#define FUNCTIONAL SLDA

#define ENABLE_V_EXT
#define ENABLE_DELTA_EXT

#define MAX_USER_PARAMS 32
#define DENSEPSILON 1.0e-8
#define REGULARIZATION_SCHEME SPHERICAL_CUTOFF
#define SLDA_STABILIZATION_RETAIN_ABOVE_DENSITY  1.0e-5
#define SLDA_STABILIZATION_EXCLUDE_BELOW_DENISTY 1.0e-7
#define INTEGRATION_SCHEME AB5AM5

#include "machine.h"
#define API_VERSION 20240131
