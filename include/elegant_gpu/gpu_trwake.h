/* gpu_trwake.h -- TRWAKE hook (src/trwake.c:18-21, call at :46). */
#ifndef TRK_ELEGANT_GPU_TRWAKE_H
#define TRK_ELEGANT_GPU_TRWAKE_H
#include "gpu_base.h"
#ifdef __cplusplus
extern "C" {
#endif
void gpu_track_through_trwake(long np0, TRWAKE *wakeData, double Po, RUN *run, long i_pass, CHARGE *charge);
#ifdef __cplusplus
}
#endif
#endif
