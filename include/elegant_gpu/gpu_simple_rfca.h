/* gpu_simple_rfca.h -- RFCA hook (src/simple_rfca.c:17-18, call at :275; RFCW
 * at :1042 is outside the GPU path). */
#ifndef TRK_ELEGANT_GPU_SIMPLE_RFCA_H
#define TRK_ELEGANT_GPU_SIMPLE_RFCA_H
#include "gpu_base.h"
#ifdef __cplusplus
extern "C" {
#endif
long gpu_trackRfCavityWithWakes(long np, RFCA *rfca, double **accepted, double *P_central, double zEnd, long iPass,
                                RUN *run, CHARGE *charge, WAKE *wake, TRWAKE *trwake, LSCKICK *LSCKick,
                                long wakesAtEnd);
long gpu_track_through_rfcw(long np, RFCW *rfcw, double **accepted, double *P_central, double zEnd, RUN *run,
                            long i_pass, CHARGE *charge);
double gpu_findFiducialTime(long np, double s0, double sOffset, double p0, unsigned long mode);
#ifdef __cplusplus
}
#endif
#endif
