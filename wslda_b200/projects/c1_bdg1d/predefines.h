/* 1D TD-BdG: NX=128, dx=1 (periodic). Pairing Delta = -g*nu (+ seeded Delta_ext), V = V_ext. */
#define NX (128)
#define NY (1)
#define NZ (1)
#define DX (1.0)
#define DY (1.0)
#define DZ (1.0)

#define FUNCTIONAL CUSTOMEDF
#define SLDA_FORCE_A1

#define ENABLE_V_EXT
#define ENABLE_DELTA_EXT

#define MAX_USER_PARAMS 32
#define DENSEPSILON 1.0e-8
#define REGULARIZATION_SCHEME SPHERICAL_CUTOFF
#define INTEGRATION_SCHEME AB3AM4

#include "machine.h"
#define API_VERSION 20240131
