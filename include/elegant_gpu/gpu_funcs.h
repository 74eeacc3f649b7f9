/* gpu_funcs.h -- included by src/csbend.c:22 and src/do_tracking.c:24 under
 * HAVE_GPU; the element hooks are declared in gpu_base.h and the per-element
 * headers, the whole-beam steps of do_tracking here. */
#ifndef TRK_ELEGANT_GPU_FUNCS_H
#define TRK_ELEGANT_GPU_FUNCS_H
#include "gpu_base.h"

#ifdef __cplusplus
extern "C" {
#endif

/* do_match_energy on the device beam (src/do_tracking.c:3404) */
void gpu_do_match_energy(long np, double *P_central, long change_beam);
/* the trajectory centroids of the surviving particles (src/do_tracking.c:2598) */
void gpu_collect_trajectory_data(double *centroid, long n);
/* survivors in increasing particle ID (src/do_tracking.c:943, :3053) */
void sortByPID(long n);

#ifdef __cplusplus
}
#endif
#endif
