/*
 * trk_oracle.h -- TEST INFRASTRUCTURE ONLY: the CPU oracle for the tracking
 * path (a C restatement of elegant's element functions and do_tracking pass
 * loop).  Used by tests, smoke() and bench.py's CPU baseline as the checker;
 * the product library never links it.
 */
#ifndef TRK_ORACLE_H
#define TRK_ORACLE_H

#include "trk.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Rows of the oracle beam: x, xp, y, yp, s, delta, id, loss pass, loss element. */
#define ORC_STRIDE 9

typedef struct {
  long n_left;
  long particle_passes;
  double p_central;
} orc_result;

/* Track np particles (rows of ORC_STRIDE doubles, modified in place; lost
 * particles are swapped behind the survivors as the reference does) through
 * n_passes passes starting at pass index pass_offset.  *p_central in/out. */
int orc_track(const trk_lattice *lattice, double *coord, long np, long n_passes, long pass_offset,
              double *p_central, orc_result *result);

/* One element (index `element`), as do_tracking's switch plus the
 * after-element aperture and NaN filters.  z_start is the arc length at the
 * element entrance; maxamp state is taken from the lattice (sticky MAXAMP). */
int orc_track_element(const trk_lattice *lattice, int element, double *coord, long np, long pass,
                      double *p_central, long *n_left);

/* 0: beam averages summed as the reference does; 1: double-double sums
 * rounded once (the GPU path's value) for bit-level checks. */
void orc_set_exact_sums(int on);

/* Seed of the incoherent-radiation deviates (ISR), drawn as the library
 * draws them (elegant_b200/csrc/trk_philox.h). */
void orc_set_isr_seed(unsigned long long seed);

/* 0: libm sin/cos/asin; 1: correctly rounded ones (what the GPU parity build computes). */
void orc_set_cr_math(int on);
double orc_cr_sin(double x);
double orc_cr_cos(double x);
double orc_cr_asin(double x);
double orc_cr_tan(double x);
double orc_cr_slow(int kind, double x);
int orc_cr_parts(int kind, double x, double *out);

/* Sharded runs (test of the multi-GPU decomposition on CPU ranks): gather
 * n doubles from every rank into recv[rank * n ...]; sum n doubles over
 * ranks in place.  world <= 1 or NULL callbacks: a single process. */
typedef void (*orc_gather_fn)(const double *send, double *recv, long n);
typedef void (*orc_sum_fn)(double *buf, long n);
void orc_set_collective(int world, orc_gather_fn gather, orc_sum_fn sum);

/* Field-expansion table of a CSBEND as the oracle builds it (for tests):
 * Fx, Fy are 11x11 row-major, coefficient of x^i y^j at [i*11+j]. */
int orc_csbend_field_table(const trk_lattice *lattice, int element, double *Fx, double *Fy, int *expansionOrder1,
                           int *hasNormal, int *hasSkew);

/* Beam observers on rows of ORC_STRIDE doubles, survivors first (np). */
typedef struct {
  double centroid[7];
  double sigma[7][7];
  double sigman[7][7];
  double maxabs[7], min[7], max[7];
  long n_part;
  double p0;
  double charge;
} orc_beam_sums;
void orc_beam_centroids(const double *coord, long np, double *centroid);
void orc_accumulate_beam_sums(const double *coord, long np, orc_beam_sums *sums, double p_central, double mp_charge,
                              const double *time_value, double t_min, double t_max, long start_pid, long end_pid,
                              unsigned flags);
void orc_match_energy(double *coord, long np, double *p_central, int change_beam);

#ifdef __cplusplus
}
#endif
#endif
