/* The td-gauss Gaussian stirrer (see gauss_stirrer.h). */
#include "../gauss_common/gauss_stirrer.h"
