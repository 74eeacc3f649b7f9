/*
 * trk.h -- C ABI of the B200 particle-tracking library (libtrkgpu.so).
 *
 * The library replaces the per-particle element loops of elegant's
 * do_tracking() pass loop (src/do_tracking.c:498 pass loop, :829 element loop,
 * :1352 element switch) for the elements
 *   DRIF, EDRIFT, KQUAD, KSEXT, KOCT, CSBEND, RFCA, WAKE, TRWAKE, MAXAMP, CHARGE, MARK.
 * Particles live on the device as an FP64 structure of arrays for a whole run.
 *
 * Conventions shared with the reference:
 *   - a particle is (x [m], x' , y [m], y', s [m], delta = dp/p0, id)
 *     (src/track.h:82-100, particleIDIndex = 6);
 *   - a host beam is an array-of-structures of `stride` doubles per particle
 *     (stride >= 7), the layout of elegant's `double **coord` rows;
 *   - element parameters are set by the reference's parameter names with the
 *     reference's defaults (src/track_data.c *_param[] tables);
 *   - particle loss is not an error: lost particles are reported through
 *     survivor counts, loss pass and loss element, and their coordinates are
 *     overwritten as the reference does (coord[4] = loss position,
 *     coord[5] = P*(1+delta) or gamma, src/multipole.c:1044-1045,
 *     src/limit_amplitudes.c:279-280, :580-581).
 *
 * Every function returns TRK_OK (0) or a negative trk_error code and never
 * exits the process (the reference aborts through bombElegant(),
 * src/bombElegant.c:9-18).  trk_last_error() gives a message for the last
 * failure on the calling thread.
 *
 * Thread model: a trk_context is driven by one host thread and owns one CUDA
 * stream on one device; calls on a context are stream-ordered.
 */
#ifndef TRK_H
#define TRK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TRK_ABI_VERSION 1

/* ---------------------------------------------------------------- errors */
typedef enum {
  TRK_OK = 0,
  TRK_ERR_ARG = -1,          /* bad argument (null pointer, size out of range) */
  TRK_ERR_UNKNOWN_TYPE = -2, /* element type name not known */
  TRK_ERR_UNKNOWN_PARAM = -3,/* parameter name not known for that element type */
  TRK_ERR_UNSUPPORTED = -4,  /* element feature outside the implemented path */
  TRK_ERR_CUDA = -5,         /* CUDA runtime error (message has the CUDA text) */
  TRK_ERR_NOMEM = -6,        /* host or device allocation failed */
  TRK_ERR_DEVICE = -7,       /* a kernel reported an error in the device status word */
  TRK_ERR_PHYSICS = -8,      /* input the reference rejects (e.g. beam longer than wake) */
  TRK_ERR_STATE = -9,        /* call out of order (e.g. tracking with no beam loaded) */
  TRK_ERR_NCCL = -10         /* collective failed */
} trk_error;

const char *trk_last_error(void);
int trk_abi_version(void);

/* ---------------------------------------------------------- element types */
/* Type codes; names are the reference's element names (src/track_data.c:60-).*/
typedef enum {
  TRK_MARK = 0,
  TRK_DRIF = 1,
  TRK_EDRIFT = 2,
  TRK_KQUAD = 3,
  TRK_KSEXT = 4,
  TRK_KOCT = 5,
  TRK_CSBEND = 6,
  TRK_RFCA = 7,
  TRK_WAKE = 8,
  TRK_TRWAKE = 9,
  TRK_MAXAMP = 10,
  TRK_CHARGE = 11,
  TRK_N_TYPES = 12
} trk_type;

/* Type name <-> code ("KQUAD" <-> TRK_KQUAD).  Returns -1 / NULL if unknown. */
int trk_type_code(const char *name);
const char *trk_type_name(int type);
/* Number of parameters of a type and the name / default of parameter i. */
int trk_param_count(int type);
const char *trk_param_name(int type, int index);
double trk_param_default(int type, int index);
/* Index of a named parameter of a type, or TRK_ERR_UNKNOWN_PARAM. Aliases
 * (CSBEND N_KICKS == N_SLICES, src/track_data.c:1943-1944) resolve to the
 * same index. */
int trk_param_index(int type, const char *name);

/* -------------------------------------------------------------- lattices */
/* A lattice is an ordered list of elements (one pass of do_tracking's element
 * loop).  Element parameters are doubles addressed by the reference's names;
 * integer parameters (N_KICKS, ORDER, ...) are stored as doubles too. */
typedef struct trk_lattice trk_lattice;

int trk_lattice_create(trk_lattice **lattice);
void trk_lattice_destroy(trk_lattice *lattice);
/* Append an element with default parameters; *index receives its position. */
int trk_lattice_add(trk_lattice *lattice, int type, const char *name, int *index);
int trk_lattice_set(trk_lattice *lattice, int index, const char *param, double value);
int trk_lattice_get(const trk_lattice *lattice, int index, const char *param, double *value);
int trk_lattice_length(const trk_lattice *lattice);
int trk_lattice_type(const trk_lattice *lattice, int index);
/* Green-function table of a WAKE (W = longitudinal, Wy ignored) or TRWAKE
 * (W = Wx, Wy) element: `points` samples at times t[] (seconds, uniform
 * spacing), in V/C (WAKE) or V/C/m (TRWAKE).  This replaces the INPUTFILE /
 * TCOLUMN / WCOLUMN SDDS read of set_up_wake (src/wake.c:340-478) and
 * set_up_trwake (src/trwake.c:325-517).  The arrays are copied. */
int trk_lattice_set_wake(trk_lattice *lattice, int index, const double *t, const double *W,
                         const double *Wy, long points);
/* Parse elegant lattice-file text (the subset "NAME: TYPE, P=V, ..." and
 * "NAME: LINE=(A, B, 2*C, -D...)"), then expand `line` into the lattice.
 * Wake tables must be supplied with trk_lattice_set_wake afterwards. */
int trk_lattice_parse(trk_lattice *lattice, const char *text, const char *line);
/* Design arc length of one pass (sum of element lengths). */
double trk_lattice_total_length(const trk_lattice *lattice);

/* ---------------------------------------------------------- run settings */
typedef struct {
  double p_central;      /* reference momentum beta*gamma (p_central_mev / me_mev) */
  long n_passes;         /* passes (turns) to track */
  long pass_offset;      /* index of the first pass (wake ramps, RF fiducial on pass 0) */
  int32_t fast_math;     /* 0: reference operation order, no FMA contraction (parity build);
                            1: transcendental-free CSBEND drift and FMA (fast build) */
  int32_t block_size;    /* unused, kept 0 (block shape comes with the variant) */
  int32_t compact_every; /* fused multi-pass runs (one-segment lattices, ensembles): track the survivors
                            compacted into an index list, re-formed every N passes, so lost particles
                            hold no lanes (0 = never; trk_run_defaults sets 64) */
  int32_t variant;       /* tracking-kernel variant (block size x occupancy); -1 = autotuned choice */
  int32_t time_kernels;  /* 1: bracket every tracking-kernel launch with CUDA events (trk_stats.track_ms) */
  uint64_t isr_seed;     /* seed of the incoherent-radiation (ISR) deviates; each deviate is a function of
                            (seed, particle ID, pass, element, kick), so runs repeat exactly */
} trk_run;

void trk_run_defaults(trk_run *run);

/* Test hook, no counterpart in the reference: the next `after` growing
 * device allocations of the library succeed and the one after them is
 * refused as if cudaMalloc had failed (TRK_ERR_NOMEM, nothing allocated);
 * the hook then disarms.  after < 0 disarms it.  Process-wide.  Lets tests
 * check that a failed call leaves its context usable. */
int trk_test_fail_allocation(int after);

typedef struct {
  long n_total;          /* particles loaded */
  long n_left;           /* survivors after the run */
  long particle_passes;  /* sum over passes of particles entering the pass (elegant's `effort`) */
  double device_ms;      /* device time of the tracking kernels (CUDA events) */
  long kernel_launches;  /* kernels launched by the library during the call */
  double p_central;      /* reference momentum after the run */
  double track_ms;       /* with trk_run.time_kernels: summed device time of the tracking-kernel launches */
  long track_launches;   /* with trk_run.time_kernels: tracking-kernel launches timed */
} trk_stats;

/* ------------------------------------------------------------- contexts */
typedef struct trk_context trk_context;

/* Create a context on CUDA device `device` (current device if < 0). */
int trk_context_create(trk_context **ctx, int device);
void trk_context_destroy(trk_context *ctx);
/* The CUDA stream (cudaStream_t) all work of the context is ordered on. */
void *trk_context_stream(trk_context *ctx);

/* Sharded tracking across GPUs (one process per GPU, each rank holding its
 * own block of particles), replacing Pelegant's MPI exchanges
 * (src/wake.c:226-233, src/trwake.c:195-204, src/simple_rfca.c:222-230,
 * src/findGlobalMinMax.c:10) with NCCL collectives on the context's stream:
 * beam time statistics are all-gathered and combined in rank order, wake
 * histograms summed, the CHARGE element's particle count summed.
 * trk_comm_get_unique_id is called on one rank and its 128 bytes passed to
 * every rank's trk_context_set_comm (nranks <= 0 removes the communicator;
 * nranks = 1 runs the exchanges on a one-rank communicator).
 * Every rank must then call trk_track with the same lattice and pass range.
 * NCCL (libnccl.so.2) is loaded at run time; TRK_ERR_NCCL if it is absent. */
int trk_comm_get_unique_id(void *id128);
int trk_context_set_comm(trk_context *ctx, const void *id128, int nranks, int rank);
int trk_context_comm(const trk_context *ctx, int *rank, int *nranks);

/* The same sharded run over the caller's own host-side collectives instead
 * of NCCL: the route of a Pelegant-style host that already runs MPI (the
 * reference's MPI_Allreduce / MPI_Allgather over host buffers,
 * src/wake.c:226-233, src/trwake.c:195-204, src/simple_rfca.c:222-230)
 * and has no NCCL.  At each exchange the library copies the device buffer
 * to host memory, synchronizes the context's stream, calls the callback
 * (which must perform the collective over all ranks and return 0, or
 * nonzero to fail the call with TRK_ERR_NCCL), and copies the result back.
 * The callbacks are called from the thread that drives the context, in the
 * same order on every rank.  `ex` must stay valid while it is set;
 * trk_context_set_comm (either form) replaces it. */
typedef struct {
  void *user;
  /* in-place element-wise sum over ranks of n values */
  int (*sum_f64)(void *user, double *buf, size_t n);
  int (*sum_u64)(void *user, uint64_t *buf, size_t n);
  int (*sum_i64)(void *user, int64_t *buf, size_t n);
  /* recv[r * n + k] = rank r's send[k] */
  int (*gather_f64)(void *user, const double *send, double *recv, size_t n);
} trk_exchange;
int trk_context_set_exchange(trk_context *ctx, const trk_exchange *ex, int nranks, int rank);

/* Copy a host AoS beam (np particles, `stride` doubles each, stride >= 7,
 * column 6 = particle id) to the device SoA.  Replaces gpuBaseInit's copy
 * (src/do_tracking.c:411-414). */
int trk_beam_load(trk_context *ctx, const double *coord, long np, long stride);
/* Copy a device SoA beam: 7 columns of `ld` doubles each (x, xp, y, yp, s,
 * delta, id) starting at d_soa; device-to-device, no host traffic. */
int trk_beam_load_device(trk_context *ctx, const double *d_soa, long np, long ld);
/* Copy the beam back to host AoS rows: survivors first (in their original
 * order), then lost particles (in original order).  Replaces
 * forceParticlesToCpu (src/do_tracking.c:864 et al.).  n_left receives the
 * survivor count.  lost_pass / lost_element (optional, np entries, aligned
 * with the rows written) receive the pass and element index of each loss
 * (-1 for survivors). */
int trk_beam_store(trk_context *ctx, double *coord, long stride, long *n_left,
                   long *lost_pass, int32_t *lost_element);
/* Device pointers of the SoA columns (x, xp, y, yp, s, delta, id) and the
 * per-particle loss word; valid until the next trk_beam_load*. */
int trk_beam_device_columns(trk_context *ctx, double **columns, long *np, int32_t **loss);
/* Survivor count of the device beam. */
int trk_beam_count(trk_context *ctx, long *n_left);

/* Track the device beam through n_passes passes of the lattice.
 * *p_central is read and updated (RFCA CHANGE_P0, WAKE CHANGE_P0). */
int trk_track(trk_context *ctx, const trk_lattice *lattice, const trk_run *run, trk_stats *stats);

/* ------------------------------------------------ per-element entry points
 * What the reference's HAVE_GPU hooks call (src/multipole.c:698-709,
 * src/csbend.c:689-701, src/csbend.c:3796-3800, src/simple_rfca.c:267-290,
 * src/wake.c:47-56, src/trwake.c:43-50, src/limit_amplitudes.c:204-214,
 * :296-300, :508-516, src/matrix.c:227-240): one element's body at a time,
 * the after-element filters as separate calls, losses recorded with the
 * given pass and element index.  *n_left receives the survivor count (the
 * hooks' `long` return); the device beam keeps lost particles in place
 * (trk_beam_store returns survivors first). */

/* The sticky MAXAMP state that in-element aperture checks use (the `maxamp`
 * argument of multipole_tracking2 / track_through_csbend). */
typedef struct {
  double x_max, y_max;
  int32_t elliptical, exponent, y_exponent, reserved;
} trk_maxamp;

/* State of one element kept by the caller between calls: the RFCA fiducial
 * phase (set on the first call, src/simple_rfca.c:412-471) and the
 * macroparticle charge a WAKE/TRWAKE uses (CHARGE element, or the element's
 * CHARGE / particles on pass 0: src/wake.c:346-372). */
typedef struct {
  double rf_phase_fiducial;
  int32_t rf_fiducial_seen, reserved;
  double macro_charge;
} trk_element_state;

/* Element `element` of `lattice` (any path type but MAXAMP/CHARGE/MARK, which
 * do nothing here) on the surviving particles; z_start is the arc length at
 * the element entrance; losses are recorded with `pass` and `loss_element`;
 * maxamp may be NULL; state may be NULL for elements other than
 * RFCA/WAKE/TRWAKE.  run supplies p_central, fast_math, variant. */
int trk_track_element(trk_context *ctx, const trk_lattice *lattice, int element, long pass, int loss_element,
                      double z_start, const trk_maxamp *maxamp, trk_element_state *state, const trk_run *run,
                      long *n_left);

/* limit_amplitudes / elimit_amplitudes (src/limit_amplitudes.c:197-288,
 * 487-620) on the surviving particles; x_max = y_max = DBL_MAX is
 * removeInvalidParticles' NaN/inf filter (:289-317).  Open sides (openCode)
 * are not supported. */
int trk_limit_amplitudes(trk_context *ctx, double x_max, double y_max, int elliptical, int exponent, int y_exponent,
                         int extrapolate_z, double z, double p_central, long pass, int element, long *n_left);

/* removeInvalidParticles (src/limit_amplitudes.c:289-331): particles with a
 * NaN coordinate or delta <= -1 are lost at z. */
int trk_remove_invalid(trk_context *ctx, double z, double p_central, long pass, int element, long *n_left);

/* track_particles (src/matrix.c:212-469) for a first- or second-order matrix:
 * C[6], R[36] row-major, T[6*21] with T[i][j][k] (k <= j) at i*21 + j(j+1)/2 + k
 * (ignored for order 1). */
int trk_track_matrix(trk_context *ctx, int order, const double *C, const double *R, const double *T, int fast_math,
                     long *n_left);

/* ------------------------------------------------------- beam observers */
/* Whole-beam readings and operations between elements, on the device beam
 * (survivors only), so observers do not force the beam to the host.  Sums
 * the reference forms with Kahan's summation are formed in double-double. */

/* compute_centroids (src/compute_centroids.c:53-160): means of x, x', y, y',
 * s, delta over the surviving particles (all zero with none); *n (may be
 * NULL) receives their count.  Also the trajectory centroids of do_tracking
 * (src/do_tracking.c:2585-2610). */
int trk_beam_centroids(trk_context *ctx, double *centroid, long *n);

/* The reference's BEAM_SUMS with its BEAM_SUMS2 (src/track.h:281-297);
 * index 6 is the time coordinate.  Zero it (and set min to +DBL_MAX, max to
 * -DBL_MAX) before the first accumulation, as zero_beam_sums does. */
typedef struct {
  double centroid[7];
  double sigma[7][7];
  double sigman[7][7];
  double maxabs[7], min[7], max[7];
  long n_part;
  double p0;
  double charge;
} trk_beam_sums;
#define TRK_SUMS_SPARSE 0x1u         /* BEAM_SUMS_SPARSE: diagonal blocks and dispersive terms only */
#define TRK_SUMS_NOMINMAX 0x2u       /* BEAM_SUMS_NOMINMAX */
#define TRK_SUMS_EXACT_NORMEMIT 0x4u /* exactNormalizedEmittance: sigman with px, py */
#define TRK_SUMS_SECOND_ORDER 0x8u   /* the BEAM_SUMS2 part is kept (sigma, min, max, maxabs) */
/* accumulate_beam_sums (src/compute_centroids.c:286-461): adds the surviving
 * particles with start_pid <= id <= end_pid (both < 0: all) and, if
 * t_min < t_max, t_min <= t <= t_max, to *sums.  time_value (host, one per
 * loaded particle in load order) replaces the computed time coordinates
 * when not NULL. */
int trk_accumulate_beam_sums(trk_context *ctx, trk_beam_sums *sums, double p_central, double mp_charge,
                             const double *time_value, double t_min, double t_max, long start_pid, long end_pid,
                             unsigned int flags);

/* do_match_energy (src/do_tracking.c:3376-3546): change_beam = 0 moves
 * *p_central to the survivors' mean momentum and rescales delta;
 * change_beam = 1 shifts every momentum so the mean is *p_central, keeping
 * each particle's time of flight. */
int trk_match_energy(trk_context *ctx, double *p_central, int change_beam);

/* The particle-ID sort of do_tracking (src/do_tracking.c:935-950, sortByPID
 * on the GPU path): survivors in increasing ID, lost particles after them in
 * their present order. */
int trk_sort_by_id(trk_context *ctx);

/* ----------------------------------------------------- aperture search */
/* The line modes of elegant's aperture search (one-, two-, three- and
 * n-line: do_aperture_search_line, src/aperture_search.c:985-1234). */
typedef struct {
  int32_t lines;          /* 1, 2, 3 (fixed directions) or more (evenly spread over the half or full plane) */
  int32_t full_plane;     /* lines spread over 2 pi instead of pi */
  int32_t slope_mode;     /* search in x', y' instead of x, y */
  int32_t n_splits;       /* refinement sweeps after the first */
  long nx;                /* points of the first sweep along each line (>= 2) */
  double xmax, ymax;      /* extent of the first sweep (positions) */
  double xpmax, ypmax;    /* extent of the first sweep (slopes, slope_mode) */
  double split_fraction;  /* step reduction per refinement sweep, in (0, 1) */
  double orbit[6];        /* added to every particle (offset_by_orbit; zeros otherwise) */
} trk_aperture_search;
/* For each of n_variants lattices (error seeds; one lattice: n_variants = 1)
 * the largest surviving point along every line after run->n_passes passes,
 * the search the reference does particle by particle, with every point of a
 * sweep of every line and variant tracked in one launch.  Outputs, per
 * variant v and line l at [v * lines + l]: x_limit, y_limit (the surviving
 * point); x_clipped, y_clipped (the same after the reference's island
 * clipping, trimApertureSearchResult); x_lost, y_lost, s_lost (the last
 * loss seen on the line, DBL_MAX if none); area[v] (0 if the origin is lost
 * or lines = 1).  Any output but x_limit, y_limit may be NULL.  The loaded
 * beam is replaced. */
int trk_aperture_search_lines(trk_context *ctx, const trk_lattice *const *lattices, int n_variants,
                              const trk_aperture_search *search, const trk_run *run, double *x_limit,
                              double *y_limit, double *x_clipped, double *y_clipped, double *x_lost, double *y_lost,
                              double *s_lost, double *area);

/* The grid mode of elegant's aperture search (do_aperture_search_grid,
 * src/aperture_search.c:1236-1521): a grid of u (x or delta) by v (y or x)
 * tracked for run->n_passes passes, once for v >= 0 and, when vmin < 0, once
 * more for v <= 0. */
typedef struct {
  int32_t delta_mode; /* 0: u = x, v = y; 1: u = delta, v = x; 2: u = delta, v = y */
  int32_t reserved;
  long nx, ny, ndelta; /* points per axis (the two the mode uses, each >= 2) */
  double xmin, xmax, ymin, ymax, deltamin, deltamax;
  double orbit[6]; /* added to every particle (offset_by_orbit; zeros otherwise) */
} trk_aperture_grid;
/* For each of n_variants lattices, every grid point of a side tracked in one
 * launch.  Per variant v, side (0: v >= 0; 1: v <= 0, only if vmin < 0) and
 * u column iu, at [(v * 2 + side) * nu + iu]: u_limit (the column's u),
 * v_limit (the largest |v| below the first loss of the column, as the
 * reference reduces it), and the coordinates of that first lost particle at
 * its loss, x_lost, y_lost, s_lost, delta_lost (its momentum p, as the
 * reference's lost rows hold it; DBL_MAX where nothing was lost); rows of a
 * side not searched are zero with lost coordinates DBL_MAX.  area[v] = sum
 * over sides that kept a survivor of |v_limit du|.  Any output but v_limit
 * may be NULL.  Particle IDs count up over the whole launch.  The loaded
 * beam is replaced. */
int trk_aperture_search_grid(trk_context *ctx, const trk_lattice *const *lattices, int n_variants,
                             const trk_aperture_grid *grid, const trk_run *run, double *u_limit, double *v_limit,
                             double *x_lost, double *y_lost, double *s_lost, double *delta_lost, double *area);

/* ------------------------------------------------------ batched ensembles */
/* Track `n_variants` lattices that differ only in element parameter values
 * (error seeds, grids) in one launch.  `lattices` holds n_variants lattices of
 * identical structure; variant v owns particles [offsets[v], offsets[v+1]) of
 * the device beam (offsets[0] = 0, offsets[n_variants] = particles loaded).
 * All passes run in chunked launches of the fused tracking kernel, captured
 * into a CUDA graph; each particle reads its own variant's element records.
 * Collective elements (WAKE, TRWAKE, RFCA) are not allowed in ensembles.
 * The batched error-seed and dynamic-aperture studies of the reference run
 * do_tracking once per variant (src/error.c, src/aperture_search.c:456). */
int trk_track_ensemble(trk_context *ctx, const trk_lattice *const *lattices, int n_variants,
                       const long *offsets, const trk_run *run, trk_stats *stats);
/* Launch shape (trk_run.variant value) the last trk_track_ensemble used: the
 * caller's, or the autotuner's choice, which times each candidate shape on a
 * scratch copy of the beam over the first passes of the first call for a
 * given element count, particle count and build, and keeps the fastest. */
int trk_ensemble_variant(const trk_context *ctx);

/* ------------------------------------------------- allocation-free wake */
/* No counterpart in the reference: elegant's WAKE (src/wake.c:23-304)
 * allocates its histograms on every call.
 *
 * One WAKE element (time statistics, histogram of N bins, convolution with
 * the Green function, energy kick; the same kernels as a WAKE in trk_track)
 * applied to a beam the caller owns on the current device, for callers that
 * cannot allocate device memory where they track (device memory handed out by
 * their own pool allocator, or pipelines that cannot take the device-wide
 * synchronization of cudaMalloc/cudaFree).  It allocates nothing: its scratch
 * is one static device array of TRK_NOALLOC_SCRATCH_BYTES per GPU that loads
 * the library, kept until the process exits.  The first call on each device
 * looks up that array's address (make it before any stream capture).  All
 * calls share the array and it keeps the last call's contents; calls that
 * overlap on the GPU race on it.
 *
 *   columns[0..5]  device pointers x, x', y, y', s, delta (np each, in/out)
 *   lost_pass, lost_element  device int32[np] (in/out; < 0 marks survivors);
 *                  particles that become non-finite are marked with `pass`
 *   wake_W         device pointer: W(t) at t = i*wake_dt, i < wake_points (V/C)
 *   n_bins         2..TRK_NOALLOC_MAX_BINS (larger values are rejected)
 *   macro_charge   charge per macroparticle (C); factor = WAKE FACTOR
 *   fast_math      0 parity build, 1 fast build; stream = cudaStream_t
 * Returns TRK_ERR_PHYSICS if the beam is longer than the wake (unless
 * allow_long_beam), TRK_ERR_ARG for sizes beyond the static limits.  The
 * beam-time reduction uses trk_track's block count (one block per 4096
 * particles, at most 8 per SM) capped at TRK_NOALLOC_MAX_BLOCKS; the result
 * equals trk_track's bit for bit while the two block counts agree (always
 * on GPUs of up to 148 SMs). */
#define TRK_NOALLOC_MAX_BINS 8192
#define TRK_NOALLOC_MAX_BLOCKS 1184
#define TRK_NOALLOC_SCRATCH_BYTES (256 * 1024)
int trk_wake_noalloc(double *const *columns, int32_t *lost_pass, int32_t *lost_element, long np, double p_central,
                     const double *wake_W, long wake_points, double wake_dt, long n_bins, double macro_charge,
                     double factor, int interpolate, int allow_long_beam, long pass, int fast_math, void *stream);

/* ------------------------------------------------------------- gradients */
/* Reverse-mode adjoint through the fused element chain (no counterpart in
 * the reference, which offers only finite differences through repeated
 * tracking).  Tracks the loaded beam n_passes passes (fast build), keeping
 * the beam at the start of every pass on the device, then sweeps back pass
 * by pass: each pass is recomputed from its checkpoint with every element's
 * entry state recorded, and the elements' hand-written adjoints carry
 * d(loss)/d(coordinates) backwards while the kick-strength sensitivities are
 * summed into the gradient.  Loss function over the surviving particles:
 *   loss = mean_i (x_i^2 + y_i^2) + w_c ((mean_i x_i)^2 + (mean_i y_i)^2)
 * (particles lost during the run are left out: loss events are not
 * differentiable).  Parameters: K1 of every KQUAD and K2 of every KSEXT, in
 * lattice order.  Elements allowed: DRIF, EDRIFT, single-order
 * KQUAD/KSEXT/KOCT without tilt or misalignment, CSBEND (pure dipole, or a
 * K1/K2 field expansion) without misalignment or edge kick, MARK, MAXAMP.
 * grad may be NULL (loss only).  The device beam is left at its final state. */
int trk_adjoint(trk_context *ctx, const trk_lattice *lattice, const trk_run *run,
                double centroid_weight, double *loss, double *grad, int n_grad);
/* The batched form: n_variants lattices of one structure (error seeds) over
 * particle ranges [offsets[v], offsets[v+1]) of the loaded beam, as in
 * trk_track_ensemble, in one forward and one reverse sweep.  loss[v] is
 * variant v's loss over its own survivors; grad[v * P + p] its gradient
 * with respect to parameter p (P = trk_adjoint_param_count of a variant;
 * n_grad = n_variants * P). */
int trk_adjoint_ensemble(trk_context *ctx, const trk_lattice *const *lattices, int n_variants, const long *offsets,
                         const trk_run *run, double centroid_weight, double *loss, double *grad, int n_grad);
/* The same loss function on the device beam as it is (for finite
 * differences against trk_adjoint). */
int trk_objective(trk_context *ctx, double centroid_weight, double *loss);
/* Number of gradient parameters (KQUAD K1 + KSEXT K2) of a lattice. */
int trk_adjoint_param_count(const trk_lattice *lattice);

#ifdef __cplusplus
}
#endif
#endif /* TRK_H */
