/*
 * TEST INFRASTRUCTURE (oracle/ref): drives elegant's own element functions,
 * compiled unmodified from the reference sources into oracle/_ref/libref.so,
 * through the pass/element loop of do_tracking() (src/do_tracking.c:144), for
 * the elements of the tracking path.  It pins the oracle restatement
 * (oracle/trk_oracle.c) and the CUDA library against the reference code.
 *
 * What this driver does itself, as do_tracking does it:
 *  - element structures filled from elegant's parameter tables
 *    (entity_description[] in src/track_data.c: defaults, then the lattice's
 *    values by parameter name), CSBEND edge indices as the parser sets them
 *    (src/mad_parse.c:1374-1379), WAKE/TRWAKE Green functions injected in
 *    place of set_up_wake's file read (src/wake.c:374-476);
 *  - the initial NaN screen (src/do_tracking.c:478-484), the element calls of
 *    the switch (:1355-1390 CHARGE, :1606 RFCA, :1883 MAXAMP, :1962 CSBEND,
 *    :2031 EDRIFT, :2039-2071 KQUAD/KSEXT/KOCT, :2242-2248 WAKE/TRWAKE; DRIF
 *    through its matrix), the after-element aperture (:2506-2524) and NaN
 *    filter (:2675), z per pass (:1101-1108) and the effort count;
 *  - the loss record: pass and element index per lost particle.
 * Rows in and out are those of the oracle (trk_oracle.h): x, xp, y, yp, s,
 * delta, id, loss pass, loss element.
 */
#include "mdb.h"
#include "track.h"

#include "trk_lattice.h"
#include "trk_oracle.h"
#ifdef REF_GPU_HOOKS
/* built a second time with elegant's HAVE_GPU hooks on (oracle/_ref/libref_gpu.so):
 * the same loop, with the beam on the device through the hooks of
 * elegant_b200/hooks/trk_elegant_hooks.c, as do_tracking drives them
 * (src/do_tracking.c:413, :925-931, :3177-3178) */
#include "gpu_base.h"
#include "gpu_compute_centroids.h"
#define REF_ENTRY refgpu_track
#define REF_DT_ENTRY refgpu_do_tracking
#define REF_OBSERVE refgpu_observe
#else
#define REF_ENTRY ref_track
#define REF_DT_ENTRY ref_do_tracking
#define REF_OBSERVE ref_observe
#endif

VMATRIX *drift_matrix(double length, long order);
void track_particles(double **final, VMATRIX *M, double **initial, long n_part);
void free_matrices(VMATRIX *M);
void compute_offsets();

#define REF_ROW 10 /* COORDINATES_PER_PARTICLE + BASIC_PROPERTIES_PER_PARTICLE */
#define REF_ORIG 9 /* weightIndex column: holds the original row (unused by the element code) */

static long ref_type(int t) {
  switch (t) {
  case TRK_MARK:
    return T_MARK;
  case TRK_DRIF:
    return T_DRIF;
  case TRK_EDRIFT:
    return T_EDRIFT;
  case TRK_KQUAD:
    return T_KQUAD;
  case TRK_KSEXT:
    return T_KSEXT;
  case TRK_KOCT:
    return T_KOCT;
  case TRK_CSBEND:
    return T_CSBEND;
  case TRK_RFCA:
    return T_RFCA;
  case TRK_WAKE:
    return T_WAKE;
  case TRK_TRWAKE:
    return T_TRWAKE;
  case TRK_MAXAMP:
    return T_MAXAMP;
  case TRK_CHARGE:
    return T_CHARGE;
  default:
    return -1;
  }
}

static int set_param(long T, char *p, const char *name, double value) {
  ELEMENT_DESCRIPTION *ed = &entity_description[T];
  for (long k = 0; k < ed->n_params; k++) {
    PARAMETER *pp = ed->parameter + k;
    if (strcmp(pp->name, name))
      continue;
    switch (pp->type) {
    case IS_DOUBLE:
      *(double *)(p + pp->offset) = value;
      return 0;
    case IS_LONG:
      *(long *)(p + pp->offset) = (long)value;
      return 0;
    case IS_SHORT:
      *(short *)(p + pp->offset) = (short)value;
      return 0;
    default:
      return -1;
    }
  }
  return -1;
}

/* elegant's parser: table defaults, then the user's values */
static char *make_element(const trk_elem *e, long T) {
  ELEMENT_DESCRIPTION *ed = &entity_description[T];
  char *p = (char *)calloc(1, ed->structure_size);
  for (long k = 0; k < ed->n_params; k++) {
    PARAMETER *pp = ed->parameter + k;
    switch (pp->type) {
    case IS_DOUBLE:
      *(double *)(p + pp->offset) = pp->number;
      break;
    case IS_LONG:
      *(long *)(p + pp->offset) = pp->integer;
      break;
    case IS_SHORT:
      *(short *)(p + pp->offset) = (short)pp->integer;
      break;
    case IS_STRING:
      *(char **)(p + pp->offset) = pp->string ? strdup(pp->string) : NULL;
      break;
    }
  }
  int n = trk_param_count(e->type);
  for (int i = 0; i < n; i++) {
    const char *name = trk_param_name(e->type, i);
    if (set_param(T, p, name, e->p[i])) {
      trk_set_error(TRK_ERR_UNSUPPORTED, "reference table of %s has no numeric parameter %s", entity_name[T], name);
      free(p);
      return NULL;
    }
  }
  if (T == T_CSBEND) {
    ((CSBEND *)p)->e1Index = 0;
    ((CSBEND *)p)->e2Index = 1;
    ((CSBEND *)p)->edgeFlip = 0;
  }
  return p;
}

/* the part of set_up_wake / set_up_trwake after the file read
 * (src/wake.c:470-476, src/trwake.c:490-510) */
static int wake_geometry(const trk_elem *e, long *points, double **t, double *dt, long *i0, long acausal) {
  if (!e->wake_t || e->wake_points < 2)
    return trk_set_error(TRK_ERR_ARG, "wake element %s has no Green function", e->name);
  *points = e->wake_points;
  *t = e->wake_t;
  double tmin, tmax;
  find_min_max(&tmin, &tmax, e->wake_t, e->wake_points);
  *dt = (tmax - tmin) / (e->wake_points - 1);
  *i0 = 0;
  if (tmin != 0) {
    if (!acausal)
      return trk_set_error(TRK_ERR_ARG, "acausal wake without ACAUSAL_ALLOWED");
    *i0 = -1;
    for (long iw = 0; iw < e->wake_points; iw++)
      if (fabs(e->wake_t[iw]) < 1e-6 * *dt) {
        *i0 = iw;
        break;
      }
    if (*i0 == -1)
      return trk_set_error(TRK_ERR_ARG, "acausal wake without t=0 sample");
  }
  return 0;
}

typedef struct {
  ELEMENT_LIST *el;
  long n;
  VMATRIX **drift;
} ref_beamline;

static void free_beamline(ref_beamline *b) {
  for (long i = 0; i < b->n; i++) {
    if (b->drift[i])
      free_matrices(b->drift[i]);
    free(b->el[i].p_elem);
  }
  free(b->el);
  free(b->drift);
}

static int build_beamline(const trk_lattice *l, ref_beamline *b) {
  /* elegant turns the parameter tables' member addresses into offsets once
   * at start-up (src/elegant.c:560) */
  static int offsets_done = 0;
  if (!offsets_done) {
    compute_offsets();
    offsets_done = 1;
  }
  b->n = l->n;
  b->el = (ELEMENT_LIST *)calloc(l->n > 0 ? l->n : 1, sizeof(ELEMENT_LIST));
  b->drift = (VMATRIX **)calloc(l->n > 0 ? l->n : 1, sizeof(VMATRIX *));
  double z = 0;
  for (int i = 0; i < l->n; i++) {
    const trk_elem *e = &l->e[i];
    long T = ref_type(e->type);
    if (T < 0)
      return trk_set_error(TRK_ERR_UNSUPPORTED, "element type %d", e->type);
    ELEMENT_LIST *el = &b->el[i];
    el->type = T;
    el->name = (char *)e->name;
    el->occurence = 1;
    el->pred = i ? &b->el[i - 1] : NULL;
    el->succ = i + 1 < l->n ? &b->el[i + 1] : NULL;
    if (!(el->p_elem = make_element(e, T)))
      return TRK_ERR_UNSUPPORTED;
    el->beg_pos = z;
    if (entity_description[T].flags & HAS_LENGTH)
      z += ((DRIFT *)el->p_elem)->length;
    el->end_pos = z;
    if (T == T_DRIF) {
      long order = ((DRIFT *)el->p_elem)->order;
      b->drift[i] = drift_matrix(((DRIFT *)el->p_elem)->length, order ? order : 2);
    } else if (T == T_WAKE) {
      WAKE *w = (WAKE *)el->p_elem;
      int rc = wake_geometry(e, &w->wakePoints, &w->t, &w->dt, &w->i0, w->acausalAllowed);
      if (rc)
        return rc;
      w->W = e->wake_w0;
      w->initialized = 1;
      w->isCopy = 1;
    } else if (T == T_TRWAKE) {
      TRWAKE *w = (TRWAKE *)el->p_elem;
      int rc = wake_geometry(e, &w->wakePoints, &w->t, &w->dt, &w->i0, w->acausalAllowed);
      if (rc)
        return rc;
      w->W[0] = e->wake_w0;
      w->W[1] = e->wake_w1;
      w->initialized = 1;
      w->isCopy = 1;
    }
  }
  return 0;
}

static void record_losses(double **coord, long nLeft, long nToTrack, long pass, long element, long *lp, long *le) {
#ifdef REF_GPU_HOOKS
  /* the device keeps the loss record; rows are not on the host here */
  return;
#endif
  for (long k = nLeft; k < nToTrack; k++) {
    long o = (long)coord[k][REF_ORIG];
    lp[o] = pass;
    le[o] = element;
  }
}

int REF_ENTRY(const trk_lattice *l, double *rows, long np, long n_passes, long pass_offset, double *P_central,
              orc_result *result) {
  if (!l || (!rows && np) || !P_central)
    return TRK_ERR_ARG;
  ref_beamline bl;
  memset(&bl, 0, sizeof(bl));
  int rc = build_beamline(l, &bl);
  if (rc) {
    free_beamline(&bl);
    return rc;
  }
  totalPropertiesPerParticle = REF_ROW;
  sizeOfParticle = REF_ROW * sizeof(double);
  double *buf = (double *)calloc((size_t)(np > 0 ? np : 1) * REF_ROW, sizeof(double));
  double **coord = (double **)calloc(np > 0 ? np : 1, sizeof(double *));
  long *lp = (long *)malloc(sizeof(long) * (np > 0 ? np : 1));
  long *le = (long *)malloc(sizeof(long) * (np > 0 ? np : 1));
  for (long i = 0; i < np; i++) {
    coord[i] = buf + (size_t)i * REF_ROW;
    memcpy(coord[i], rows + (size_t)i * ORC_STRIDE, 7 * sizeof(double));
    coord[i][7] = -1;
    coord[i][8] = 0;
    coord[i][REF_ORIG] = i;
    lp[i] = le[i] = -1;
  }
  RUN run;
  memset(&run, 0, sizeof(run));
  run.default_order = 2;
  run.wrap_around = 1;
  run.rootname = "oracle_ref";
  run.p_central = *P_central;

  long nToTrack = np, nLeft, effort = 0, nOriginal = np;
  MAXAMP *maxamp = NULL;
  double x_max = 0, y_max = 0;
  long elliptical = 0, maxampOpenCode = 0, maxampExponent = 2, maxampYExponent = 2;
  CHARGE *charge = NULL;

#ifdef REF_GPU_HOOKS
  gpuBaseInit(coord, np, NULL, NULL, 1);
  trk_hooks_begin_pass(pass_offset);
  getGpuBase()->elementOnGpu = 1;
#endif
  nLeft = limit_amplitudes(coord, DBL_MAX, DBL_MAX, nToTrack, NULL, 0.0, *P_central, 0, 0, bl.n ? bl.el : NULL);
  record_losses(coord, nLeft, nToTrack, pass_offset, -1, lp, le);
  nToTrack = nLeft;

  for (long i_pass = pass_offset; i_pass < pass_offset + n_passes; i_pass++) {
    double z = 0, last_z = 0;
#ifdef REF_GPU_HOOKS
    trk_hooks_begin_pass(i_pass);
#endif
    for (long ie = 0; ie < bl.n; ie++) {
      ELEMENT_LIST *eptr = &bl.el[ie];
#ifdef REF_GPU_HOOKS
      setElementGpuData(eptr);
#endif
      last_z = z;
      if (entity_description[eptr->type].flags & HAS_LENGTH)
        z += ((DRIFT *)eptr->p_elem)->length;
      else
        z += eptr->end_pos - eptr->beg_pos;
      nLeft = nToTrack;
      if (nToTrack) {
        switch (eptr->type) {
        case T_CHARGE:
          if (i_pass == pass_offset) {
            charge = (CHARGE *)eptr->p_elem;
            charge->idSlotsPerBunch = 0;
            charge->macroParticleCharge = 0;
            if (nOriginal)
              charge->macroParticleCharge = charge->charge / nOriginal;
            if (charge->chargePerParticle)
              charge->macroParticleCharge = charge->chargePerParticle;
          }
          break;
        case T_MARK:
          break;
        case T_DRIF:
          track_particles(coord, bl.drift[ie], coord, nToTrack);
          break;
        case T_EDRIFT:
          exactDrift(coord, nToTrack, ((EDRIFT *)eptr->p_elem)->length);
          break;
        case T_KQUAD:
        case T_KSEXT:
        case T_KOCT:
          nLeft = multipole_tracking2(coord, nToTrack, eptr, 0.0, *P_central, NULL, last_z, maxamp, NULL,
                                      &run.apertureData, NULL, -1);
          break;
        case T_CSBEND: {
          CSBEND *cs = (CSBEND *)eptr->p_elem;
          cs->edgeFlags = determine_bend_flags(eptr, cs->edge_effects[cs->e1Index], cs->edge_effects[cs->e2Index]);
          nLeft = track_through_csbend(coord, nToTrack, cs, 0.0, *P_central, NULL, last_z, NULL, run.rootname, maxamp,
                                       NULL, &run.apertureData, -1, eptr);
          break;
        }
        case T_RFCA:
          nLeft = simple_rf_cavity(coord, nToTrack, (RFCA *)eptr->p_elem, NULL, P_central, z);
          break;
        case T_WAKE:
          track_through_wake(coord, nToTrack, (WAKE *)eptr->p_elem, P_central, &run, i_pass, charge);
          break;
        case T_TRWAKE:
          track_through_trwake(coord, nToTrack, (TRWAKE *)eptr->p_elem, *P_central, &run, i_pass, charge);
          break;
        case T_MAXAMP:
          maxamp = (MAXAMP *)eptr->p_elem;
          x_max = maxamp->x_max;
          y_max = maxamp->y_max;
          elliptical = maxamp->elliptical;
          maxampOpenCode = 0;
          maxampExponent = maxamp->exponent;
          maxampYExponent = maxamp->yExponent;
          break;
        }
        if (!(entity_description[eptr->type].flags & NO_APERTURE) && (x_max || y_max)) {
          if (!elliptical)
            nLeft = limit_amplitudes(coord, x_max, y_max, nLeft, NULL, z, *P_central, eptr->type == T_DRIF,
                                     maxampOpenCode, eptr);
          else
            nLeft = elimit_amplitudes(coord, x_max, y_max, nLeft, NULL, z, *P_central, eptr->type == T_DRIF,
                                      maxampOpenCode, maxampExponent, maxampYExponent, eptr);
        }
        nLeft = limit_amplitudes(coord, DBL_MAX, DBL_MAX, nLeft, NULL, z, *P_central, 0, 0, eptr);
      }
      record_losses(coord, nLeft, nToTrack, i_pass, ie, lp, le);
      nToTrack = nLeft;
    }
    effort += nToTrack;
  }
#ifdef REF_GPU_HOOKS
  coord = forceParticlesToCpu("end of tracking");
  const long *hook_le = trk_hooks_loss_elements();
  for (long i = 0; i < np; i++) {
    double *r = rows + (size_t)i * ORC_STRIDE;
    memcpy(r, coord[i], 7 * sizeof(double));
    r[7] = coord[i][lossPassIndex];
    r[8] = hook_le[i];
  }
  gpuBaseDealloc();
#else
  for (long i = 0; i < np; i++) {
    double *r = rows + (size_t)i * ORC_STRIDE;
    long o = (long)coord[i][REF_ORIG];
    memcpy(r, coord[i], 7 * sizeof(double));
    r[7] = lp[o];
    r[8] = le[o];
  }
#endif
  if (result) {
    result->n_left = nToTrack;
    result->particle_passes = effort;
    result->p_central = *P_central;
  }
  free(buf);
  free(coord);
  free(lp);
  free(le);
  free_beamline(&bl);
  return TRK_OK;
}

/* The same run through elegant's own do_tracking() (src/do_tracking.c:144),
 * compiled unmodified: the pass loop, the element switch, the MAXAMP state,
 * the after-element filters, CHARGE and the loss record are the reference's
 * own, on the same element structures as ref_track builds.  Flags:
 * SILENT_RUNNING | INHIBIT_FILE_OUTPUT, no fiducial passes (n_passes_fiducial
 * = 0).  Rows come back in do_tracking's order, survivors first; a lost row
 * keeps the loss pass do_tracking records (recordLostParticles,
 * src/do_tracking.c:4669-4690); do_tracking records no loss element, so
 * column 8 is -2.  In the hook build the beam goes to the device in
 * do_tracking's gpuBaseInit and comes back in its gpuBaseDealloc
 * (src/do_tracking.c:413, :3172-3178); the pass the hooks record losses
 * with starts at pass_offset. */
int REF_DT_ENTRY(const trk_lattice *l, double *rows, long np, long n_passes, long pass_offset, double *P_central,
                 orc_result *result) {
  if (!l || (!rows && np) || !P_central || l->n < 1)
    return TRK_ERR_ARG;
  ref_beamline bl;
  memset(&bl, 0, sizeof(bl));
  int rc = build_beamline(l, &bl);
  if (rc) {
    free_beamline(&bl);
    return rc;
  }
  /* drifts track through their matrices (do_tracking's MATRIX_TRACKING branch) */
  for (long i = 0; i < bl.n; i++)
    bl.el[i].matrix = bl.drift[i];
  totalPropertiesPerParticle = REF_ROW;
  sizeOfParticle = REF_ROW * sizeof(double);
  double *buf = (double *)calloc((size_t)(np > 0 ? np : 1) * REF_ROW, sizeof(double));
  double **coord = (double **)calloc(np > 0 ? np : 1, sizeof(double *));
  for (long i = 0; i < np; i++) {
    coord[i] = buf + (size_t)i * REF_ROW;
    memcpy(coord[i], rows + (size_t)i * ORC_STRIDE, 7 * sizeof(double));
    coord[i][lossPassIndex] = -1;
    coord[i][8] = 0;
    coord[i][REF_ORIG] = i;
  }
  LINE_LIST line;
  memset(&line, 0, sizeof(line));
  line.name = "oracle_ref";
  line.elem = bl.el;
  line.n_elems = bl.n;
  line.elast = &bl.el[bl.n - 1];
  RUN run;
  memset(&run, 0, sizeof(run));
  run.default_order = 2;
  run.wrap_around = 1;
  run.rootname = "oracle_ref";
  run.p_central = *P_central;
  long effort = 0;
  double final_charge = 0;
#ifdef REF_GPU_HOOKS
  trk_hooks_begin_pass(pass_offset);
#endif
  const long n_left = do_tracking(NULL, coord, np, &effort, &line, P_central, NULL, NULL, NULL, NULL, &run, 0,
                                  SILENT_RUNNING | INHIBIT_FILE_OUTPUT, n_passes, pass_offset, NULL, NULL,
                                  &final_charge, NULL, NULL);
  for (long i = 0; i < np; i++) {
    double *r = rows + (size_t)i * ORC_STRIDE;
    memcpy(r, coord[i], 7 * sizeof(double));
    r[7] = i < n_left ? -1 : coord[i][lossPassIndex];
    r[8] = i < n_left ? -1 : -2;
  }
  if (result) {
    result->n_left = n_left;
    result->particle_passes = effort;
    result->p_central = *P_central;
  }
  for (long i = 0; i < bl.n; i++)
    bl.el[i].matrix = NULL;
  free(buf);
  free(coord);
  free_beamline(&bl);
  return TRK_OK;
}

/* elegant's compute_centroids and accumulate_beam_sums (src/compute_centroids.c)
 * on np surviving rows (ORC_STRIDE layout), the sums starting from
 * zero_beam_sums and accumulated `repeats` times; flags: bits 0..2 are the
 * reference's BEAM_SUMS_SPARSE/NOMINMAX/EXACTEMIT (EXACTEMIT sets
 * exactNormalizedEmittance), bit 3 keeps the BEAM_SUMS2 part.  In the hook
 * build the beam is handed to the device first (gpuBaseInit) and the calls
 * go through the GPU hooks, as do_tracking's observers do on the GPU path. */
int REF_OBSERVE(const double *rows, long np, double Po, double mp_charge, unsigned flags, long startPID, long endPID,
                double tMin, double tMax, int repeats, double *centroid, orc_beam_sums *out) {
  totalPropertiesPerParticle = REF_ROW;
  sizeOfParticle = REF_ROW * sizeof(double);
  double *buf = (double *)calloc((size_t)(np > 0 ? np : 1) * REF_ROW, sizeof(double));
  double **coord = (double **)calloc(np > 0 ? np : 1, sizeof(double *));
  for (long i = 0; i < np; i++) {
    coord[i] = buf + (size_t)i * REF_ROW;
    memcpy(coord[i], rows + (size_t)i * ORC_STRIDE, 7 * sizeof(double));
    coord[i][7] = -1;
  }
  BEAM_SUMS sums;
  BEAM_SUMS2 sums2;
  memset(&sums, 0, sizeof(sums));
  memset(&sums2, 0, sizeof(sums2));
  sums.beamSums2 = (flags & 8u) ? &sums2 : NULL;
  zero_beam_sums(&sums, 1);
  exactNormalizedEmittance = (flags & 4u) ? 1 : 0;
#ifdef REF_GPU_HOOKS
  gpuBaseInit(coord, np, NULL, NULL, 1);
  getGpuBase()->elementOnGpu = 1;
#endif
  compute_centroids(centroid, coord, np);
  for (int r = 0; r < repeats; r++)
    accumulate_beam_sums(&sums, coord, np, Po, mp_charge, NULL, tMin, tMax, startPID, endPID, flags & 7u);
#ifdef REF_GPU_HOOKS
  gpuBaseDealloc();
#endif
  exactNormalizedEmittance = 0;
  memset(out, 0, sizeof(*out));
  memcpy(out->centroid, sums.centroid, sizeof(out->centroid));
  if (sums.beamSums2) {
    memcpy(out->sigma, sums2.sigma, sizeof(out->sigma));
    memcpy(out->sigman, sums2.sigman, sizeof(out->sigman));
    memcpy(out->maxabs, sums2.maxabs, sizeof(out->maxabs));
    memcpy(out->min, sums2.min, sizeof(out->min));
    memcpy(out->max, sums2.max, sizeof(out->max));
  }
  out->n_part = sums.n_part;
  out->p0 = sums.p0;
  out->charge = sums.charge;
  free(buf);
  free(coord);
  return TRK_OK;
}

#ifndef REF_GPU_HOOKS
/* The reference's default of every parameter the lattice tables know, for
 * a test that the two tables agree: defaults[i] for parameter i of `type`
 * (trk_param_name order); returns the count or a negative error. */
int ref_param_defaults(int type, double *defaults, int max) {
  long T = ref_type(type);
  if (T < 0)
    return TRK_ERR_ARG;
  int n = trk_param_count(type);
  if (n > max)
    return TRK_ERR_ARG;
  ELEMENT_DESCRIPTION *ed = &entity_description[T];
  for (int i = 0; i < n; i++) {
    const char *name = trk_param_name(type, i);
    defaults[i] = NAN;
    for (long k = 0; k < ed->n_params; k++) {
      PARAMETER *pp = ed->parameter + k;
      if (strcmp(pp->name, name))
        continue;
      defaults[i] = pp->type == IS_DOUBLE ? pp->number : (double)pp->integer;
      break;
    }
  }
  return n;
}
#endif
