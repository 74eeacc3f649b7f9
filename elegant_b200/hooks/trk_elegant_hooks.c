/*
 * trk_elegant_hooks.c -- elegant's HAVE_GPU hooks implemented over
 * libtrkgpu.so.  This file belongs to an elegant build: it is compiled with
 * elegant's own headers (track.h and what it includes) plus the hook headers
 * in include/elegant_gpu/, elegant's tracking sources are compiled with
 * -DHAVE_GPU, and the program links libtrkgpu.so.  Each element function of
 * the path then sends its particles through the device beam:
 *
 *   gpuBaseInit / forceParticlesToCpu / gpuBaseDealloc   beam on the device
 *   setElementGpuData / getElementOnGpu                  which elements run there
 *   gpu_multipole_tracking2      KQUAD, KSEXT, KOCT      (src/multipole.c:701)
 *   gpu_track_through_csbend     CSBEND                  (src/csbend.c:692)
 *   gpu_exactDrift               EDRIFT                  (src/csbend.c:3799)
 *   gpu_track_particles          DRIF and other matrices (src/matrix.c:233)
 *   gpu_trackRfCavityWithWakes   RFCA                    (src/simple_rfca.c:275)
 *   gpu_track_through_wake       WAKE                    (src/wake.c:51)
 *   gpu_track_through_trwake     TRWAKE                  (src/trwake.c:46)
 *   gpu_limit_amplitudes, gpu_elimit_amplitudes, gpu_removeInvalidParticles
 *                                after-element filters   (src/limit_amplitudes.c:207, :510, :298)
 *   gpu_compute_centroids, gpu_accumulate_beam_sums
 *                                beam observers          (src/compute_centroids.c:64-76, :313-327)
 *   gpu_collect_trajectory_data, gpu_do_match_energy, sortByPID
 *                                whole-beam steps        (src/do_tracking.c:2598, :3404, :943)
 *
 * Element parameters are read from elegant's element structures through
 * elegant's own parameter tables (entity_description[], by name), so the
 * library sees exactly the values elegant tracks with.  Library errors end
 * the run through bombElegant, as elegant's own errors do.  The parity build
 * of the library is used unless TRK_HOOKS_FAST=1 is set in the environment.
 */
#include <float.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mdb.h"
#include "track.h"

#include "gpu_base.h"
#include "gpu_compute_centroids.h"
#include "gpu_csbend.h"
#include "gpu_funcs.h"
#include "gpu_limit_amplitudes.h"
#include "gpu_matrix.h"
#include "gpu_multipole.h"
#include "gpu_simple_rfca.h"
#include "gpu_trwake.h"
#include "gpu_wake.h"
#include "trk.h"

void set_up_wake(WAKE *wakeData, RUN *run, long pass, long particles, CHARGE *charge);
void set_up_trwake(TRWAKE *wakeData, RUN *run, long pass, long particles, CHARGE *charge);

static trk_context *g_ctx = NULL;
static GPUBASE g_base;
static long g_pass = 0, g_elem = -1, g_np = 0;
/* the pass the next run starts at (trk_hooks_begin_pass before the run) */
static long g_pass_start = 0;
/* the first element of the line and whether it has been seen this run: a
 * pass begins each time do_tracking reaches it again */
static const void *g_first_elem = NULL;
static int g_first_seen = 0;
static int g_fast = -1;
static double *g_buf = NULL;
static long *g_loss_pass = NULL;
static int32_t *g_loss_elem32 = NULL;
static long *g_loss_elem = NULL;

typedef struct {
  const void *key;
  trk_element_state st;
} hook_state;
static hook_state *g_states = NULL;
static long g_n_states = 0;

static void check(int rc, const char *what) {
  if (rc < 0) {
    char buf[1024];
    snprintf(buf, sizeof(buf), "%s: %s", what, trk_last_error());
    bombElegant(buf, NULL);
  }
}

static trk_element_state *state_of(const void *key) {
  for (long i = 0; i < g_n_states; i++)
    if (g_states[i].key == key)
      return &g_states[i].st;
  g_states = (hook_state *)realloc(g_states, sizeof(*g_states) * (g_n_states + 1));
  memset(&g_states[g_n_states], 0, sizeof(*g_states));
  g_states[g_n_states].key = key;
  return &g_states[g_n_states++].st;
}

static int fast_math(void) {
  if (g_fast < 0) {
    const char *e = getenv("TRK_HOOKS_FAST");
    g_fast = e && atoi(e) ? 1 : 0;
  }
  return g_fast;
}

static void run_for(trk_run *run, double Po) {
  trk_run_defaults(run);
  run->p_central = Po;
  run->n_passes = 1;
  run->fast_math = fast_math();
}

static int library_type(long T) {
  switch (T) {
  case T_DRIF:
    return trk_type_code("DRIF");
  case T_EDRIFT:
    return trk_type_code("EDRIFT");
  case T_KQUAD:
    return trk_type_code("KQUAD");
  case T_KSEXT:
    return trk_type_code("KSEXT");
  case T_KOCT:
    return trk_type_code("KOCT");
  case T_CSBEND:
    return trk_type_code("CSBEND");
  case T_RFCA:
    return trk_type_code("RFCA");
  case T_WAKE:
    return trk_type_code("WAKE");
  case T_TRWAKE:
    return trk_type_code("TRWAKE");
  case T_MAXAMP:
    return trk_type_code("MAXAMP");
  case T_CHARGE:
    return trk_type_code("CHARGE");
  case T_MARK:
    return trk_type_code("MARK");
  default:
    return -1;
  }
}

/* a one-element library lattice with the values of elegant's structure */
static trk_lattice *element_lattice(long T, const char *p_elem, const char *name) {
  int type = library_type(T), idx;
  if (type < 0)
    bombElegant("element type not on the GPU path", NULL);
  trk_lattice *L;
  check(trk_lattice_create(&L), "trk_lattice_create");
  check(trk_lattice_add(L, type, name ? name : "E", &idx), "trk_lattice_add");
  ELEMENT_DESCRIPTION *ed = &entity_description[T];
  int n = trk_param_count(type);
  for (int i = 0; i < n; i++) {
    const char *pname = trk_param_name(type, i);
    for (long k = 0; k < ed->n_params; k++) {
      PARAMETER *pp = ed->parameter + k;
      if (strcmp(pp->name, pname))
        continue;
      double v;
      switch (pp->type) {
      case IS_DOUBLE:
        v = *(const double *)(p_elem + pp->offset);
        break;
      case IS_LONG:
        v = (double)*(const long *)(p_elem + pp->offset);
        break;
      case IS_SHORT:
        v = (double)*(const short *)(p_elem + pp->offset);
        break;
      default:
        continue;
      }
      check(trk_lattice_set(L, idx, pname, v), pname);
      break;
    }
  }
  return L;
}

static void maxamp_of(const MAXAMP *m, trk_maxamp *out) {
  memset(out, 0, sizeof(*out));
  out->x_max = m->x_max;
  out->y_max = m->y_max;
  out->elliptical = (int32_t)m->elliptical;
  out->exponent = (int32_t)m->exponent;
  out->y_exponent = (int32_t)m->yExponent;
}

static long element_on_device(trk_lattice *L, long pass, double z_start, const MAXAMP *maxamp,
                              trk_element_state *st, double Po) {
  trk_run run;
  trk_maxamp ma;
  long n_left = 0;
  run_for(&run, Po);
  if (maxamp && (maxamp->x_max || maxamp->y_max))
    maxamp_of(maxamp, &ma);
  check(trk_track_element(g_ctx, L, 0, pass, (int)g_elem, z_start,
                          maxamp && (maxamp->x_max || maxamp->y_max) ? &ma : NULL, st, &run, &n_left),
        "trk_track_element");
  trk_lattice_destroy(L);
  g_base.nLeft = n_left;
  return n_left;
}

/* ------------------------------------------------------------- beam */
void gpuBaseInit(double **coord, long nOriginal, double **accepted, double **lostParticles, long isMaster) {
  (void)accepted;
  (void)lostParticles;
  (void)isMaster;
  if (!g_ctx) {
    const char *dev = getenv("TRK_HOOKS_DEVICE");
    check(trk_context_create(&g_ctx, dev ? atoi(dev) : 0), "trk_context_create");
  }
  g_np = nOriginal;
  free(g_buf);
  free(g_loss_pass);
  free(g_loss_elem32);
  free(g_loss_elem);
  g_buf = (double *)malloc(sizeof(double) * 7 * (nOriginal > 0 ? nOriginal : 1));
  g_loss_pass = (long *)malloc(sizeof(long) * (nOriginal > 0 ? nOriginal : 1));
  g_loss_elem32 = (int32_t *)malloc(sizeof(int32_t) * (nOriginal > 0 ? nOriginal : 1));
  g_loss_elem = (long *)malloc(sizeof(long) * (nOriginal > 0 ? nOriginal : 1));
  for (long i = 0; i < nOriginal; i++)
    memcpy(g_buf + 7 * i, coord[i], 7 * sizeof(double));
  check(trk_beam_load(g_ctx, g_buf, nOriginal, 7), "trk_beam_load");
  memset(&g_base, 0, sizeof(g_base));
  g_base.coord = coord;
  g_base.nOriginal = nOriginal;
  g_base.nLeft = nOriginal;
  /* the beam is on the device from here on: do_tracking's first filter
   * (src/do_tracking.c:478-484) runs before any element sets the flag */
  g_base.elementOnGpu = 1;
  g_pass = g_pass_start;
  g_elem = -1;
  g_first_elem = NULL;
  g_first_seen = 0;
}

double **forceParticlesToCpu(const char *reason) {
  (void)reason;
  long n_left = 0;
  if (!g_ctx || !g_base.coord)
    return g_base.coord;
  check(trk_beam_store(g_ctx, g_buf, 7, &n_left, g_loss_pass, g_loss_elem32), "trk_beam_store");
  for (long i = 0; i < g_np; i++) {
    memcpy(g_base.coord[i], g_buf + 7 * i, 7 * sizeof(double));
    if (totalPropertiesPerParticle > lossPassIndex)
      g_base.coord[i][lossPassIndex] = (double)g_loss_pass[i];
    g_loss_elem[i] = g_loss_elem32[i];
  }
  g_base.nLeft = n_left;
  return g_base.coord;
}

const long *trk_hooks_loss_elements(void) { return g_loss_elem; }

/* do_tracking reads the particles from its coordinate array after this
 * call (src/do_tracking.c:3172-3178), so the device beam comes back first */
void gpuBaseDealloc(void) {
  if (g_ctx && g_base.coord)
    forceParticlesToCpu("gpuBaseDealloc");
  g_base.coord = NULL;
  g_first_elem = NULL;
  g_first_seen = 0;
  if (g_ctx)
    trk_context_destroy(g_ctx);
  g_ctx = NULL;
  free(g_states);
  g_states = NULL;
  g_n_states = 0;
}

void trk_hooks_begin_pass(long i_pass) {
  g_pass = g_pass_start = i_pass;
  g_elem = -1;
  g_first_elem = NULL;
  g_first_seen = 0;
}

/* do_tracking calls this for every element of every pass
 * (src/do_tracking.c:1113): the element index counts up within a pass, and
 * reaching the line's first element again starts the next pass (a caller
 * that drives its own loop calls trk_hooks_begin_pass instead) */
void setElementGpuData(void *eptr) {
  const ELEMENT_LIST *e = (const ELEMENT_LIST *)eptr;
  if (!g_first_seen) {
    g_first_elem = e;
    g_first_seen = 1;
  } else if (e && e == g_first_elem && g_elem >= 0) {
    g_pass++;
    g_elem = -1;
  }
  g_elem++;
  g_base.elementOnGpu = e && library_type(e->type) >= 0;
}

long getElementOnGpu(void) { return g_base.elementOnGpu; }
GPUBASE *getGpuBase(void) { return &g_base; }
void startGpuTimer(void) {}
void startCpuTimer(void) {}
void compareGpuCpu(long n_part, const char *name) {
  (void)n_part;
  (void)name;
}

/* ---------------------------------------------------------- elements */
long gpu_multipole_tracking2(long n_part, ELEMENT_LIST *elem, double p_error, double Po, double **accepted,
                             double z_start, MAXAMP *maxamp, APCONTOUR *apContour, APERTURE_DATA *apFileData,
                             double *sigmaDelta2, long iSlice) {
  (void)n_part;
  (void)accepted;
  if (p_error != 0 || apContour || (apFileData && apFileData->initialized) || iSlice >= 0)
    bombElegant("multipole feature outside the GPU path (p_error, APCONTOUR, aperture file, slicing)", NULL);
  if (sigmaDelta2)
    *sigmaDelta2 = 0;
  trk_lattice *L = element_lattice(elem->type, elem->p_elem, elem->name);
  return element_on_device(L, g_pass, z_start, maxamp, NULL, Po);
}

long gpu_track_through_csbend(long n_part, CSBEND *csbend, double p_error, double Po, double **accepted,
                              double z_start, double *sigmaDelta2, char *rootname, MAXAMP *maxamp,
                              APCONTOUR *apContour, APERTURE_DATA *apFileData, long iSlice, ELEMENT_LIST *eptr) {
  (void)n_part;
  (void)accepted;
  (void)rootname;
  if (p_error != 0 || apContour || (apFileData && apFileData->initialized) || iSlice >= 0)
    bombElegant("CSBEND feature outside the GPU path (p_error, APCONTOUR, aperture file, slicing)", NULL);
  if (sigmaDelta2)
    *sigmaDelta2 = 0;
  trk_lattice *L = element_lattice(T_CSBEND, (const char *)csbend, eptr ? eptr->name : "B");
  /* edges that do_tracking's determine_bend_flags turned off (split bends:
   * src/do_tracking.c:1963-1965) */
  if (csbend->edgeFlags & BEND_EDGE_DETERMINED) {
    if (!(csbend->edgeFlags & BEND_EDGE1_EFFECTS))
      check(trk_lattice_set(L, 0, "EDGE1_EFFECTS", 0), "EDGE1_EFFECTS");
    if (!(csbend->edgeFlags & BEND_EDGE2_EFFECTS))
      check(trk_lattice_set(L, 0, "EDGE2_EFFECTS", 0), "EDGE2_EFFECTS");
  }
  return element_on_device(L, g_pass, z_start, maxamp, NULL, Po);
}

void gpu_exactDrift(long np, double length) {
  (void)np;
  trk_lattice *L;
  int idx;
  check(trk_lattice_create(&L), "trk_lattice_create");
  check(trk_lattice_add(L, trk_type_code("EDRIFT"), "ED", &idx), "trk_lattice_add");
  check(trk_lattice_set(L, idx, "L", length), "L");
  element_on_device(L, g_pass, 0.0, NULL, NULL, 1.0);
}

void gpu_track_particles(VMATRIX *M, long n_part) {
  (void)n_part;
  double R[36], T[126];
  long n_left;
  memset(T, 0, sizeof(T));
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++)
      R[6 * i + j] = M->R[i][j];
  if (M->order >= 2)
    for (int i = 0; i < 6; i++)
      for (int j = 0; j < 6; j++)
        for (int k = 0; k <= j; k++)
          T[21 * i + j * (j + 1) / 2 + k] = M->T[i][j][k];
  if (M->order > 2)
    bombElegant("third-order matrices are outside the GPU path", NULL);
  check(trk_track_matrix(g_ctx, (int)M->order, M->C, R, T, fast_math(), &n_left), "trk_track_matrix");
  g_base.nLeft = n_left;
}

long gpu_trackRfCavityWithWakes(long np, RFCA *rfca, double **accepted, double *P_central, double zEnd, long iPass,
                                RUN *run, CHARGE *charge, WAKE *wake, TRWAKE *trwake, LSCKICK *LSCKick,
                                long wakesAtEnd) {
  (void)np;
  (void)accepted;
  (void)iPass;
  (void)run;
  (void)charge;
  (void)wakesAtEnd;
  if (wake || trwake || LSCKick)
    bombElegant("RFCA with attached wakes is outside the GPU path", NULL);
  trk_lattice *L = element_lattice(T_RFCA, (const char *)rfca, "RF");
  const long n = element_on_device(L, g_pass, zEnd - rfca->length, NULL, state_of(rfca), *P_central);
  if (rfca->change_p0) /* src/simple_rfca.c:977-978 */
    check(trk_match_energy(g_ctx, P_central, 0), "trk_match_energy");
  return n;
}

void gpu_track_through_wake(long np0, WAKE *wakeData, double *PoInput, RUN *run, long i_pass, CHARGE *charge) {
  /* the reference's own set-up: Green function from its file, macroparticle
   * charge (src/wake.c:340-372) */
  set_up_wake(wakeData, run, i_pass, np0, charge);
  trk_lattice *L = element_lattice(T_WAKE, (const char *)wakeData, "W");
  check(trk_lattice_set_wake(L, 0, wakeData->t, wakeData->W, NULL, wakeData->wakePoints), "trk_lattice_set_wake");
  trk_element_state *st = state_of(wakeData);
  st->macro_charge = wakeData->macroParticleCharge;
  element_on_device(L, i_pass, 0.0, NULL, st, *PoInput);
  if (wakeData->change_p0) /* src/wake.c:289-290 */
    check(trk_match_energy(g_ctx, PoInput, 0), "trk_match_energy");
}

void gpu_track_through_trwake(long np0, TRWAKE *wakeData, double Po, RUN *run, long i_pass, CHARGE *charge) {
  set_up_trwake(wakeData, run, i_pass, np0, charge);
  trk_lattice *L = element_lattice(T_TRWAKE, (const char *)wakeData, "TW");
  check(trk_lattice_set_wake(L, 0, wakeData->t, wakeData->W[0], wakeData->W[1], wakeData->wakePoints),
        "trk_lattice_set_wake");
  trk_element_state *st = state_of(wakeData);
  st->macro_charge = wakeData->macroParticleCharge;
  element_on_device(L, i_pass, 0.0, NULL, st, Po);
}

/* ------------------------------------------------------- apertures */
long gpu_limit_amplitudes(double xmax, double ymax, long np, double **accepted, double z, double Po,
                          long extrapolate_z, long openCode) {
  (void)np;
  (void)accepted;
  long n_left;
  if (openCode)
    bombElegant("open-sided apertures are outside the GPU path", NULL);
  check(trk_limit_amplitudes(g_ctx, xmax, ymax, 0, 2, 0, (int)extrapolate_z, z, Po, g_pass, (int)g_elem, &n_left),
        "trk_limit_amplitudes");
  g_base.nLeft = n_left;
  return n_left;
}

long gpu_elimit_amplitudes(double xmax, double ymax, long np, double **accepted, double z, double Po,
                           long extrapolate_z, long openCode, long exponent, long yexponent, ELEMENT_LIST *eptr) {
  (void)np;
  (void)accepted;
  (void)eptr;
  long n_left;
  if (openCode)
    bombElegant("open-sided apertures are outside the GPU path", NULL);
  check(trk_limit_amplitudes(g_ctx, xmax, ymax, 1, (int)exponent, (int)yexponent, (int)extrapolate_z, z, Po, g_pass,
                             (int)g_elem, &n_left),
        "trk_limit_amplitudes");
  g_base.nLeft = n_left;
  return n_left;
}

long gpu_removeInvalidParticles(long np, double **accepted, double z, double Po) {
  (void)np;
  (void)accepted;
  long n_left;
  check(trk_remove_invalid(g_ctx, z, Po, g_pass, (int)g_elem, &n_left), "trk_remove_invalid");
  g_base.nLeft = n_left;
  return n_left;
}

/* ------------------------------------- hooks outside the GPU path
 * setElementGpuData never puts these element types on the device, so
 * elegant does not call them; if it does, the run stops as on any elegant
 * error. */
static long outside(const char *what) {
  char buf[256];
  snprintf(buf, sizeof(buf), "%s is outside the GPU tracking path", what);
  bombElegant(buf, NULL);
  return 0;
}

long gpu_track_through_csbendCSR(long n_part, CSRCSBEND *csbend, double p_error, double Po, double **accepted,
                                 double z_start, double z_end, CHARGE *charge, char *rootname, MAXAMP *maxamp,
                                 APCONTOUR *apContour, APERTURE_DATA *apFileData, ELEMENT_LIST *eptr) {
  return outside("CSRCSBEND");
}
long gpu_track_through_driftCSR(long np, CSRDRIFT *csrDrift, double Po, double **accepted, double zStart,
                                double revolutionLength, CHARGE *charge, char *rootname) {
  return outside("CSRDRIFT");
}
void gpu_addCorrectorRadiationKick(long np, ELEMENT_LIST *elem, long type, double Po, double *sigmaDelta2,
                                   long disableISR) {
  outside("corrector radiation");
}
long gpu_track_through_rfcw(long np, RFCW *rfcw, double **accepted, double *P_central, double zEnd, RUN *run,
                            long i_pass, CHARGE *charge) {
  return outside("RFCW");
}
double gpu_findFiducialTime(long np, double s0, double sOffset, double p0, unsigned long mode) {
  return (double)outside("findFiducialTime");
}
long gpu_imposeApertureData(long np, double **accepted, double z, double Po, APERTURE_DATA *apData) {
  return outside("aperture files");
}
long gpu_rectangular_collimator(RCOL *rcol, long np, double **accepted, double z, double Po) {
  return outside("RCOL");
}
long gpu_elliptical_collimator(ECOL *ecol, long np, double **accepted, double z, double Po) {
  return outside("ECOL");
}
long gpu_beam_scraper(SCRAPER *scraper, long np, double **accepted, double z, double Po) {
  return outside("SCRAPER");
}

/* ------------------------------------------------- whole-beam observers */
void gpu_compute_centroids(double *centroid, long n_part) {
  long n = 0;
  (void)n_part;
  check(trk_beam_centroids(g_ctx, centroid, &n), "trk_beam_centroids");
}

void gpu_accumulate_beam_sums(BEAM_SUMS *sums, long n_part, double p_central, double mp_charge, double *timeValue,
                              double tMin, double tMax, long startPID, long endPID, unsigned long flags) {
  (void)n_part;
  if (timeValue)
    bombElegant("gpu_accumulate_beam_sums: caller-supplied time coordinates are not supported on the GPU path", NULL);
  trk_beam_sums s;
  memset(&s, 0, sizeof(s));
  memcpy(s.centroid, sums->centroid, sizeof(s.centroid));
  unsigned int f = 0;
  if (flags & BEAM_SUMS_SPARSE)
    f |= TRK_SUMS_SPARSE;
  if (flags & BEAM_SUMS_NOMINMAX)
    f |= TRK_SUMS_NOMINMAX;
  if (exactNormalizedEmittance)
    f |= TRK_SUMS_EXACT_NORMEMIT;
  if (sums->beamSums2) {
    f |= TRK_SUMS_SECOND_ORDER;
    memcpy(s.sigma, sums->beamSums2->sigma, sizeof(s.sigma));
    memcpy(s.sigman, sums->beamSums2->sigman, sizeof(s.sigman));
    memcpy(s.maxabs, sums->beamSums2->maxabs, sizeof(s.maxabs));
    memcpy(s.min, sums->beamSums2->min, sizeof(s.min));
    memcpy(s.max, sums->beamSums2->max, sizeof(s.max));
  }
  s.n_part = sums->n_part;
  s.p0 = sums->p0;
  s.charge = sums->charge;
  check(trk_accumulate_beam_sums(g_ctx, &s, p_central, mp_charge, NULL, tMin, tMax, startPID, endPID, f),
        "trk_accumulate_beam_sums");
  memcpy(sums->centroid, s.centroid, sizeof(s.centroid));
  if (sums->beamSums2) {
    memcpy(sums->beamSums2->sigma, s.sigma, sizeof(s.sigma));
    memcpy(sums->beamSums2->sigman, s.sigman, sizeof(s.sigman));
    memcpy(sums->beamSums2->maxabs, s.maxabs, sizeof(s.maxabs));
    memcpy(sums->beamSums2->min, s.min, sizeof(s.min));
    memcpy(sums->beamSums2->max, s.max, sizeof(s.max));
  }
  sums->n_part = s.n_part;
  sums->p0 = s.p0;
  sums->charge = s.charge;
}

void gpu_do_match_energy(long np, double *P_central, long change_beam) {
  (void)np;
  check(trk_match_energy(g_ctx, P_central, (int)change_beam), "trk_match_energy");
}

void gpu_collect_trajectory_data(double *centroid, long n) {
  long m = 0;
  (void)n;
  check(trk_beam_centroids(g_ctx, centroid, &m), "trk_beam_centroids");
}

void sortByPID(long n) {
  (void)n;
  check(trk_sort_by_id(g_ctx), "trk_sort_by_id");
}
