/* 3D TD-SLDA: 48^3, dx=1 (periodic), vortex line along z, circling Gaussian stirrer. */
#define NX (48)
#define NY (48)
#define NZ (48)
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
#define INTEGRATION_SCHEME AB3AM4

#include "machine.h"
#define API_VERSION 20240131
