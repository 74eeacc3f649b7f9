/* gpu_matrix.h -- matrix tracking hook (src/matrix.c:28-29, call at :233):
 * first- and second-order transport matrices (DRIF and every other
 * matrix-tracked element). */
#ifndef TRK_ELEGANT_GPU_MATRIX_H
#define TRK_ELEGANT_GPU_MATRIX_H
#include "gpu_base.h"
#ifdef __cplusplus
extern "C" {
#endif
void gpu_track_particles(VMATRIX *M, long n_part);
#ifdef __cplusplus
}
#endif
#endif
