/* td-gauss replay project: SLDAE, 2D engine on a 12^3 lattice (spacing 1.15), spin-symmetric, Gaussian stirrer, AB4AM5. */
#define NX 12
#define NY 12
#define NZ 12
#define DX 1.15
#define DY 1.15
#define DZ 1.15

#define FUNCTIONAL SLDAE
#define SPINSYMMETRY_MODE
#define ENABLE_V_EXT
#define MAX_USER_PARAMS 32
#define DENSEPSILON 1.0e-8
#define REGULARIZATION_SCHEME SPHERICAL_CUTOFF
#define SLDA_STABILIZATION_RETAIN_ABOVE_DENSITY  1.0e-5
#define SLDA_STABILIZATION_EXCLUDE_BELOW_DENISTY 1.0e-7
#define UNIFORM_TEST_MODE

#include "machine.h"
#define API_VERSION 20240131
