/*
 * The translation unit of one project's library (libwtd.so): the project's predefines.h and
 * problem-definition.h are compiled together with the kernels, exactly as the reference
 * compiles them into td-wslda-{1d,2d,3d} (hpc-engine/pca_kernels.cu:30, mk.td:114-138), so the
 * user hooks are inlined into the device code.  Built by wslda_b200/build.py with
 * -DCODEDIM=<1|2|3> -I<project dir>.
 *
 * Exports: the fused ABI (include/wtd.h) and the reference-named per-kernel ABI
 * (include/wslda_td_compat.h).
 */
#include <vector>
#include "predefines.h"
#include "wtd_settings.h"
#include "wtd_surface.h"
#include "problem-definition.h"
#include "wtd_functional.cuh"
#include "wtd_lattice.cuh"
#include "wtd_fft3d.cuh"
#include "wtd_path3d.cuh"
#define WTD_CODEDIM CODEDIM
#include "wtd_compat.cuh"
#include "wtd_api.cuh"
#include "wtd_checkpoint.cuh"
#include "wtd_wdata.cuh"
