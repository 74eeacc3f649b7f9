/*
 * trk_lattice.h -- internal representation of a lattice (host side), shared
 * by the library and the CPU oracle.
 */
#ifndef TRK_LATTICE_H
#define TRK_LATTICE_H

#include "trk.h"
#include "trk_params.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int type;
  char name[48];
  double p[TRK_MAX_PARAMS];
  /* Green functions of WAKE (w0) / TRWAKE (w0 = Wx, w1 = Wy) */
  double *wake_t, *wake_w0, *wake_w1;
  long wake_points;
} trk_elem;

struct trk_lattice {
  int n, cap;
  trk_elem *e;
};

/* thread-local error message helpers */
int trk_set_error(int code, const char *fmt, ...);

/* Parameter value by enum index (no checks). */
#define TRK_P(elem, idx) ((elem)->p[P_##idx])

/* Element length as do_tracking accumulates z (HAS_LENGTH types). */
double trk_elem_length(const trk_elem *e);

#ifdef __cplusplus
}
#endif
#endif
