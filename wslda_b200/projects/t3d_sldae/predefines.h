/* Small-lattice parity project: 8x6x10, SLDAE (variable mass, current corrections), AB5AM5. */
#define NX (8)
#define NY (6)
#define NZ (10)
#define DX (1.0)
#define DY (1.0)
#define DZ (1.0)

#define FUNCTIONAL SLDAE

#define ENABLE_V_EXT
#define ENABLE_DELTA_EXT

#define MAX_USER_PARAMS 32
#define DENSEPSILON 1.0e-8
#define REGULARIZATION_SCHEME SPHERICAL_CUTOFF
#define INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
#define SLDA_STABILIZATION_RETAIN_ABOVE_DENSITY  1.0e-5
#define SLDA_STABILIZATION_EXCLUDE_BELOW_DENISTY 1.0e-7
#define INTEGRATION_SCHEME AB5AM5

#include "machine.h"
#define API_VERSION 20240131
