/* gpu_csbend.h -- CSBEND, EDRIFT hooks (src/csbend.c:20-21; calls at :692, :3799;
 * the CSR variants at :1979, :3228 and :5405 are outside the GPU path and report
 * an error if reached). */
#ifndef TRK_ELEGANT_GPU_CSBEND_H
#define TRK_ELEGANT_GPU_CSBEND_H
#include "gpu_base.h"
#ifdef __cplusplus
extern "C" {
#endif
long gpu_track_through_csbend(long n_part, CSBEND *csbend, double p_error, double Po, double **accepted,
                              double z_start, double *sigmaDelta2, char *rootname, MAXAMP *maxamp,
                              APCONTOUR *apContour, APERTURE_DATA *apFileData, long iSlice, ELEMENT_LIST *eptr);
void gpu_exactDrift(long np, double length);
long gpu_track_through_csbendCSR(long n_part, CSRCSBEND *csbend, double p_error, double Po, double **accepted,
                                 double z_start, double z_end, CHARGE *charge, char *rootname, MAXAMP *maxamp,
                                 APCONTOUR *apContour, APERTURE_DATA *apFileData, ELEMENT_LIST *eptr);
long gpu_track_through_driftCSR(long np, CSRDRIFT *csrDrift, double Po, double **accepted, double zStart,
                                double revolutionLength, CHARGE *charge, char *rootname);
void gpu_addCorrectorRadiationKick(long np, ELEMENT_LIST *elem, long type, double Po, double *sigmaDelta2,
                                   long disableISR);
#ifdef __cplusplus
}
#endif
#endif
