/*
 * gpu_compute_centroids.h -- included by src/compute_centroids.c:25 under
 * HAVE_GPU: the beam observers on the device beam, implemented over
 * libtrkgpu.so (trk_beam_centroids, trk_accumulate_beam_sums) by
 * elegant_b200/hooks/trk_elegant_hooks.c.  Include after elegant's track.h.
 * The reference does not ship this header; the signatures are those of its
 * call sites.
 */
#ifndef TRK_ELEGANT_GPU_COMPUTE_CENTROIDS_H
#define TRK_ELEGANT_GPU_COMPUTE_CENTROIDS_H
#include "gpu_base.h"

#ifdef __cplusplus
extern "C" {
#endif

/* compute_centroids on the device beam (src/compute_centroids.c:64-76) */
void gpu_compute_centroids(double *centroid, long n_part);
/* accumulate_beam_sums on the device beam (src/compute_centroids.c:313-327);
 * timeValue must be NULL (elegant's time array follows its host row order,
 * which the device beam does not keep) */
void gpu_accumulate_beam_sums(BEAM_SUMS *sums, long n_part, double p_central, double mp_charge, double *timeValue,
                              double tMin, double tMax, long startPID, long endPID, unsigned long flags);

#ifdef __cplusplus
}
#endif
#endif
