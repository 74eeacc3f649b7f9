/* gpu_wake.h -- WAKE hook (src/wake.c:14-15, call at :51). */
#ifndef TRK_ELEGANT_GPU_WAKE_H
#define TRK_ELEGANT_GPU_WAKE_H
#include "gpu_base.h"
#ifdef __cplusplus
extern "C" {
#endif
void gpu_track_through_wake(long np0, WAKE *wakeData, double *PoInput, RUN *run, long i_pass, CHARGE *charge);
#ifdef __cplusplus
}
#endif
#endif
