/* gpu_funcs.h -- included by src/csbend.c:22 and src/do_tracking.c:24 under
 * HAVE_GPU; the hooks they call are declared in gpu_base.h and the per-element
 * headers. */
#ifndef TRK_ELEGANT_GPU_FUNCS_H
#define TRK_ELEGANT_GPU_FUNCS_H
#include "gpu_base.h"
#endif
