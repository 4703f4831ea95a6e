/* Parity project for large 2D lattices: 160x96 (radix-5 axis, axis longer than 128, state larger than one CTA: plane/pencil path), ASLDA, AB4AM5. */
#define NX (160)
#define NY (96)
#define NZ (1)
#define DX (1.0)
#define DY (1.0)
#define DZ (1.0)

#define FUNCTIONAL ASLDA

#define ENABLE_V_EXT
#define ENABLE_DELTA_EXT

#define MAX_USER_PARAMS 32
#define DENSEPSILON 1.0e-8
#define REGULARIZATION_SCHEME SPHERICAL_CUTOFF
#define INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
#define SLDA_STABILIZATION_RETAIN_ABOVE_DENSITY  1.0e-5
#define SLDA_STABILIZATION_EXCLUDE_BELOW_DENISTY 1.0e-7
#define INTEGRATION_SCHEME AB4AM5

#include "machine.h"
#define API_VERSION 20240131
