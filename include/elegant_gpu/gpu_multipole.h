/* gpu_multipole.h -- KQUAD/KSEXT/KOCT hook (src/multipole.c:18-19, call at :701). */
#ifndef TRK_ELEGANT_GPU_MULTIPOLE_H
#define TRK_ELEGANT_GPU_MULTIPOLE_H
#include "gpu_base.h"
#ifdef __cplusplus
extern "C" {
#endif
long gpu_multipole_tracking2(long n_part, ELEMENT_LIST *elem, double p_error, double Po, double **accepted,
                             double z_start, MAXAMP *maxamp, APCONTOUR *apContour, APERTURE_DATA *apFileData,
                             double *sigmaDelta2, long iSlice);
#ifdef __cplusplus
}
#endif
#endif
