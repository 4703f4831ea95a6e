/*
 * ORACLE (test infrastructure only).  The host forms (*_h) of the reference's SLDA/ASLDA
 * energy-density functional, hpc-engine/pca_edf.h compiled where it lies, for the uniform
 * solver that oracle/uniform_init.c drives.
 */
#include <math.h>
#include "predefines.h"
#include "pca_settings.h"
#include "pca_edf.h"
