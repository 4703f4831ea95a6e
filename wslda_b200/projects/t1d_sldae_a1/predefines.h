/* Small-lattice parity project: 18x1x1, SLDAE with the legacy SLDAE_FORCE_A1 (alpha = 1), cubic cut-off, AB3AM4. */
#define NX (18)
#define NY (1)
#define NZ (1)
#define DX (1.0)
#define DY (1.0)
#define DZ (1.0)

#define FUNCTIONAL SLDAE
#define SLDAE_FORCE_A1

#define ENABLE_V_EXT
#define ENABLE_DELTA_EXT

#define MAX_USER_PARAMS 32
#define DENSEPSILON 1.0e-8
#define REGULARIZATION_SCHEME CUBIC_CUTOFF
#define INCLUDE_MF_CORRECTION_FROM_REG_SCHEME
#define SLDA_STABILIZATION_RETAIN_ABOVE_DENSITY  1.0e-5
#define SLDA_STABILIZATION_EXCLUDE_BELOW_DENISTY 1.0e-7
#define INTEGRATION_SCHEME AB3AM4

#include "machine.h"
#define API_VERSION 20240131
