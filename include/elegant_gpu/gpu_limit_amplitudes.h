/* gpu_limit_amplitudes.h -- aperture hooks (src/limit_amplitudes.c:14-15; calls at
 * :207, :298, :510; collimators, scrapers and aperture files at :44, :353, :638,
 * :1237 are outside the GPU path). */
#ifndef TRK_ELEGANT_GPU_LIMIT_AMPLITUDES_H
#define TRK_ELEGANT_GPU_LIMIT_AMPLITUDES_H
#include "gpu_base.h"
#ifdef __cplusplus
extern "C" {
#endif
long gpu_limit_amplitudes(double xmax, double ymax, long np, double **accepted, double z, double Po,
                          long extrapolate_z, long openCode);
long gpu_elimit_amplitudes(double xmax, double ymax, long np, double **accepted, double z, double Po,
                           long extrapolate_z, long openCode, long exponent, long yexponent, ELEMENT_LIST *eptr);
long gpu_removeInvalidParticles(long np, double **accepted, double z, double Po);
long gpu_imposeApertureData(long np, double **accepted, double z, double Po, APERTURE_DATA *apData);
long gpu_rectangular_collimator(RCOL *rcol, long np, double **accepted, double z, double Po);
long gpu_elliptical_collimator(ECOL *ecol, long np, double **accepted, double z, double Po);
long gpu_beam_scraper(SCRAPER *scraper, long np, double **accepted, double z, double Po);
#ifdef __cplusplus
}
#endif
#endif
