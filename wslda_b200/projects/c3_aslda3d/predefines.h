/* 3D TD-ASLDA: 32^3, dx=1 (periodic), spin imbalance via mu_a=0.55, mu_b=0.45,
 * Delta_ext = 0.2 with 1% seeded noise (extra_data). */
#define NX (32)
#define NY (32)
#define NZ (32)
#define DX (1.0)
#define DY (1.0)
#define DZ (1.0)

#define FUNCTIONAL ASLDA

#define ENABLE_DELTA_EXT

#define MAX_USER_PARAMS 32
#define DENSEPSILON 1.0e-8
#define REGULARIZATION_SCHEME SPHERICAL_CUTOFF
#define SLDA_STABILIZATION_RETAIN_ABOVE_DENSITY  1.0e-5
#define SLDA_STABILIZATION_EXCLUDE_BELOW_DENISTY 1.0e-7
#define INTEGRATION_SCHEME AB5AM5

#include "machine.h"
#define API_VERSION 20240131
