/* 2D TD-BdG (Delta = -g*nu, g=-0.5), 48x48, dx=1 (periodic), 14-parameter Gaussian stirrer. */
#define NX (48)
#define NY (48)
#define NZ (1)
#define DX (1.0)
#define DY (1.0)
#define DZ (1.0)

#define FUNCTIONAL CUSTOMEDF
#define SLDA_FORCE_A1

#define ENABLE_V_EXT

#define MAX_USER_PARAMS 32
#define DENSEPSILON 1.0e-8
#define REGULARIZATION_SCHEME SPHERICAL_CUTOFF
#define INTEGRATION_SCHEME AB3AM4
/* Delta = -params[14]*nu, V_a = V_b = v_ext: the adjoint (wtd_adjoint) applies */
#define WTD_ADJOINT_CONTACT_BDG 14

#include "machine.h"
#define API_VERSION 20240131
