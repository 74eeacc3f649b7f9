/*
 * trk_kernels.h -- launch arguments and launchers of the tracking kernels.
 * trk_kernels.cu is compiled twice (namespaces trk_exact and trk_fast); the
 * host code in trk_host.cu picks one per run.
 */
#ifndef TRK_KERNELS_H
#define TRK_KERNELS_H

#include <cuda_runtime.h>
#include <stdint.h>

#include "trk_ops.h"

#define TRK_BLOCK 128

/* launch shapes of the tracking kernel (trk_run.variant):
 * 0 (128 threads, 1 block/SM min), 1 (128, 4), 2 (256, 2), 3 (64, 8), 4 (128, 5),
 * 5 and 6: two particles per thread (128, 3) / (128, 2), lean lattices in the fast build,
 * 7 (128, 6), 8 (256, 3) */
#define TRK_N_VARIANTS 9

/* device status word bits (a kernel records a problem and returns; the host
 * turns the word into a trk_error after the launch sequence) */
#define TRK_STATUS_LONG_BEAM 1      /* beam longer than the wake table (src/wake.c:134-140) */
#define TRK_STATUS_TOO_MANY_BINS 2  /* autoscaled bin count above the allocated histogram */
#define TRK_STATUS_NO_PARTICLES 4   /* RF fiducial with no particles (src/simple_rfca.c:228) */

struct TrackArgs {
  double *x, *xp, *y, *yp, *s, *dp;
  int32_t *lost_pass, *lost_elem;
  const trk_op *ops;
  const trk_aperture *aps;
  const double *field;
  const double *rf_phase;
  const double *rf_tave; /* mean arrival time per RF slot, this pass (LOCK_PHASE / LINEARIZE) */
  long n;
  int op_begin, op_end;
  long pass_begin, pass_end;
  long fresh_pass; /* pass that sees the MAXAMP state of a fresh do_tracking call */
  double Po;
  int element_only; /* 1: the element body only, no after-element aperture or NaN filter */
  /* ensembles: variant offsets (n_variants + 1), records per variant; null for one lattice */
  const long *ens_offsets;
  int ens_variants, ens_ops;
  /* incoherent synchrotron radiation: particle IDs (the deviates are keyed
   * by ID), the run's seed and the truncation of the normal deviates */
  const double *id;
  unsigned long long isr_seed;
  double isr_limit;
  /* survivor compaction: when `live` is set the kernel tracks particles
   * live[0 .. *live_n) (indices into the beam, ascending) instead of 0..n */
  const long *live;
  const long *live_n;
};

struct TimeStatsArgs {
  const double *s, *dp;
  const int32_t *lost_pass;
  long n;
  long chunk;
  int mode;        /* 0: wake time s*sqrt(P^2+1)/(c P); 1: RF fiducial (s+sOffset)/(c beta) */
  double Po, sOffset;
  double *part_hi, *part_lo, *part_min, *part_max;
  long long *part_n;
  double *out;     /* {sum, n, min, max, sum_hi, sum_lo} */
};

struct WakeState {
  long nb;
  double tmin;
  double ramp;
  double macro;
};

struct WakeArgs {
  double *x, *xp, *y, *yp, *s, *dp;
  int32_t *lost_pass, *lost_elem;
  long n;
  double Po;
  const double *stats;    /* from time stats: {sum, n, min, max} */
  WakeState *state;
  int *status;
  /* geometry */
  double dt, wake_span;
  long wake_points, i0;
  long n_bins, max_bins;
  int smem_bins;
  int allow_long_beam;
  long pass, ramp_passes;
  double macro_charge;    /* used when macro_mode == 0 */
  int macro_mode;         /* 0: macro_charge given; 1: charge / survivors (pass 0, no CHARGE element); 2: keep */
  double charge;          /* element CHARGE parameter for macro_mode 1 */
  double factor, xfactor, yfactor;
  int interpolate;
  int transverse;
  int active_planes;
  int x_power, y_power, x_probe, y_probe;
  double tdx, tdy;
  int untilt;             /* TRWAKE TILT: rotate back by (tilt_c, tilt_s) before the filters */
  double tilt_c, tilt_s;
  /* buffers */
  const double *W, *W_y;
  unsigned long long *counts;
  double *hist_x, *hist_y;
  double *V, *V_y;
  /* after-element filters */
  const trk_aperture *aps;
  int ap_post;
  double z_end;
  int elem;
  int element_only; /* 1: no NaN filter after the kick (per-element entry points) */
};

/* reverse-mode adjoint of the fast build's element maps (DRIF, EDRIFT,
 * single-order multipoles, pure-dipole CSBEND) */
struct AdjArgs {
  const double *ck;      /* checkpoint of the pass being reversed: x, xp, y, yp columns of n */
  double *entry;         /* element entry states: [op][4][n] */
  double *lam;           /* adjoint of x, xp, y, yp, delta: 5 columns of n */
  double *grad;          /* gradient accumulators, one per parameter */
  const int *op_param;   /* parameter index of each op, -1 if none */
  const double *op_dk;   /* per variant and op: d(kick strength)/d(parameter) of kick steps 0..2 */
  const int *op_dfield;  /* per op: offset in dfield of a CSBEND's field derivatives (-1 none) */
  const double *dfield;  /* d(Fx, Fy)/dK1 and d(Fx, Fy)/dK2 tables, 4 x 121 doubles per CSBEND op */
  int n_ops;             /* ops per variant */
  int n_params;          /* parameters per variant (grad holds n_variants x n_params) */
};

#define TRK_DECLARE_LAUNCHERS(NS)                                                                            \
  namespace NS {                                                                                             \
  int track_variant_block(int variant);                                                                      \
  void launch_track(const TrackArgs &a, int variant, int lean, long n, int max_blocks, cudaStream_t st);     \
  void launch_time_stats(const TimeStatsArgs &a, int grid, cudaStream_t st);                                 \
  void launch_rf_fiducial(const double *stats, double omega, double t_reference, double *rf_phase, int slot, \
                          int *status, cudaStream_t st);                                                     \
  void launch_rf_tave(const double *stats, double *rf_tave, int slot, cudaStream_t st);                      \
  void launch_wake(const WakeArgs &a, int grid, cudaStream_t st);                                            \
  void launch_wake_bin(const WakeArgs &a, int grid, cudaStream_t st);                                        \
  void launch_wake_apply(const WakeArgs &a, int grid, cudaStream_t st);                                      \
  void launch_stats_combine(const double *gathered, int ranks, double *out, cudaStream_t st);                \
  void launch_rotate(const TrackArgs &a, double ca, double sa, int grid, cudaStream_t st);                   \
  void launch_limit(const TrackArgs &a, const trk_aperture &ap, int mode, int extrapolate, double z, long pass,  \
                    int elem, int grid, cudaStream_t st);                                                    \
  void launch_matrix(const TrackArgs &a, const double *m, int order, int grid, cudaStream_t st);             \
  int ensemble_variant_ok(int variant);                                                                      \
  void launch_adjoint_record(const TrackArgs &a, const AdjArgs &g, cudaStream_t st);                         \
  void launch_adjoint_reverse(const TrackArgs &a, const AdjArgs &g, cudaStream_t st);                        \
  void launch_track_ensemble(const TrackArgs &a, const long *offsets, int n_variants, int ops_per_variant,   \
                             int variant, int lean, long n, int max_blocks, cudaStream_t st);               \
  cudaError_t set_coefficients(const double *coef10);                                                        \
  }

TRK_DECLARE_LAUNCHERS(trk_exact)
TRK_DECLARE_LAUNCHERS(trk_fast)

#endif
