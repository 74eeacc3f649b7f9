/*
 * TEST INFRASTRUCTURE (oracle/ref): definitions behind the shim headers, for
 * linking elegant's own tracking sources (compiled unmodified from the
 * reference tree) into oracle/_ref/libref.so.
 *
 * Three groups:
 *  - SDDS toolkit helpers elegant calls but does not ship (mdbmth, mdblib):
 *    restated from their published definitions (integer powers by
 *    multiplication, Kahan's compensated sum, the arithmetic mean, zeroing
 *    allocators).  Same definitions as the oracle restatement uses.
 *  - Stand-ins for elegant functions that live in translation units this
 *    build does not compile (elegant.c, do_tracking.c, warnings.c,
 *    obstructionData.c): the serial, no-output, no-obstruction behaviour.
 *  - Mode switches so the same reference code can run with correctly
 *    rounded sin/cos/asin/tan and double-double beam sums (what the CUDA
 *    parity build computes); off by default, i.e. glibc and Kahan sums as
 *    in an elegant binary.
 */
#include <stdarg.h>

#include "mdb.h"
#include "track.h"
#include "trk_crmath.h"

/* ------------------------------------------------------------ mode switches */
static int ref_cr_math = 0;
static int ref_exact_sums = 0;
void ref_set_cr_math(int on) { ref_cr_math = on; }
void ref_set_exact_sums(int on) { ref_exact_sums = on; }

/* the reference sources are compiled with sin/cos/asin/tan renamed to these */
double ref_sin(double x) { return ref_cr_math ? trkcr_sin(x) : sin(x); }
double ref_cos(double x) { return ref_cr_math ? trkcr_cos(x) : cos(x); }
double ref_asin(double x) { return ref_cr_math ? trkcr_asin(x) : asin(x); }
double ref_tan(double x) { return ref_cr_math ? trkcr_tan(x) : tan(x); }
double ref_exp(double x) { return ref_cr_math ? trkcr_exp(x) : exp(x); }
double ref_sinh(double x) { return ref_cr_math ? trkcr_sinh(x) : sinh(x); }
double ref_cosh(double x) { return ref_cr_math ? trkcr_cosh(x) : cosh(x); }

/* ----------------------------------------------------- SDDS mdbmth helpers */
double ipow(double x, long p) {
  if (p == 0)
    return 1.0;
  if (p == 1)
    return x;
  if (p == 2)
    return x * x;
  if (p < 0)
    return 1.0 / ipow(x, -p);
  double h = ipow(x, p / 2);
  return (p & 1) ? h * h * x : h * h;
}
double ipow1(double x) { return x; }
double ipow2(double x) { return x * x; }
double ipow3(double x) { return x * x * x; }
double ipow4(double x) { return ipow(x, 4); }
double ipow5(double x) { return ipow(x, 5); }
double ipow6(double x) { return ipow(x, 6); }
double ipow7(double x) { return ipow(x, 7); }
double pow2(double x) { return x * x; }
double pow3(double x) { return x * x * x; }
double pow4(double x) { return ipow(x, 4); }
double pow5(double x) { return ipow(x, 5); }

double dfactorial(long n) {
  double f = 1;
  for (long i = 2; i <= n; i++)
    f *= i;
  return f;
}

static void dd_acc(double *hi, double *lo, double v) {
  double s = *hi + v, bb = s - *hi, e = (*hi - (s - bb)) + (v - bb);
  e += *lo;
  double h = s + e;
  *lo = e - (h - s);
  *hi = h;
}

/* Kahan, 1965.  In exact-sums mode *error carries the low word of a
 * double-double accumulator instead, so the running sum is the correctly
 * rounded value of the exact sum. */
double KahanPlus(double sum, double b, double *error) {
  if (ref_exact_sums) {
    dd_acc(&sum, error, b);
    return sum;
  }
  double y = b - *error;
  double t = sum + y;
  *error = (t - sum) - y;
  return t;
}

/* arithmetic mean, summed in index order */
long compute_average(double *value, double *x, long n) {
  if (n <= 0)
    return 0;
  double sum = 0, lo = 0;
  for (long i = 0; i < n; i++) {
    if (ref_exact_sums)
      dd_acc(&sum, &lo, x[i]);
    else
      sum += x[i];
  }
  if (ref_exact_sums)
    sum = sum + lo;
  *value = sum / n;
  return 1;
}

long find_min_max(double *min, double *max, double *list, long n) {
  if (n <= 0)
    return 0;
  double lo = DBL_MAX, hi = -DBL_MAX;
  for (long i = 0; i < n; i++) {
    if (list[i] < lo)
      lo = list[i];
    if (list[i] > hi)
      hi = list[i];
  }
  if (min)
    *min = lo;
  if (max)
    *max = hi;
  return 1;
}

int double_cmpasc(const void *a, const void *b) {
  double x = *(const double *)a, y = *(const double *)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

/* ----------------------------------------------------- SDDS mdblib helpers */
void *tmalloc(uint64_t size) {
  void *p = calloc(1, size ? size : 4);
  if (!p) {
    fprintf(stderr, "oracle/ref: allocation of %lu bytes failed\n", (unsigned long)size);
    abort();
  }
  return p;
}

void *trealloc(void *ptr, uint64_t size) {
  if (!ptr)
    return tmalloc(size);
  void *p = realloc(ptr, size ? size : 4);
  if (!p)
    abort();
  return p;
}

int tfree(void *ptr) {
  free(ptr);
  return 1;
}

void **czarray_2d(uint64_t size, uint64_t n1, uint64_t n2) {
  void **rows = (void **)tmalloc(sizeof(void *) * n1);
  char *block = (char *)tmalloc(size * n1 * n2);
  for (uint64_t i = 0; i < n1; i++)
    rows[i] = block + i * size * n2;
  return rows;
}

int free_czarray_2d(void **array, uint64_t n1, uint64_t n2) {
  (void)n1;
  (void)n2;
  if (array) {
    free(array[0]);
    free(array);
  }
  return 1;
}

void **zarray_2d(uint64_t size, uint64_t n1, uint64_t n2) {
  void **rows = (void **)tmalloc(sizeof(void *) * n1);
  for (uint64_t i = 0; i < n1; i++)
    rows[i] = tmalloc(size * n2);
  return rows;
}

int free_zarray_2d(void **array, uint64_t n1, uint64_t n2) {
  (void)n2;
  if (array) {
    for (uint64_t i = 0; i < n1; i++)
      free(array[i]);
    free(array);
  }
  return 1;
}

char *cp_str(char **s, char *t) {
  *s = t ? strdup(t) : NULL;
  return *s;
}

long match_string(char *string, char **option, long n_options, long mode) {
  (void)mode;
  if (!string)
    return -1;
  size_t l = strlen(string);
  for (long i = 0; i < n_options; i++)
    if (option[i] && strncmp(option[i], string, l) == 0)
      return i;
  return -1;
}

void bomb(char *error, char *usage) {
  fprintf(stderr, "oracle/ref: %s %s\n", error ? error : "", usage ? usage : "");
  abort();
}
void log_entry(const char *routine) { (void)routine; }
void log_exit(const char *routine) { (void)routine; }
void push_log() {}
void pop_log() {}

/* ---------------------------------- elegant functions from other files */
/* rows are exchanged by content, sizeOfParticle bytes each */
void swapParticles(double *p1, double *p2) {
  double buffer[MAX_PROPERTIES_PER_PARTICLE];
  if (p1 == p2)
    return;
  memcpy(buffer, p1, sizeOfParticle);
  memcpy(p1, p2, sizeOfParticle);
  memcpy(p2, buffer, sizeOfParticle);
}

void bombElegant(const char *error, const char *usage) {
  fprintf(stderr, "oracle/ref: elegant aborted: %s %s\n", error ? error : "", usage ? usage : "");
  abort();
}

void bombElegantVA(char *template, ...) {
  va_list ap;
  va_start(ap, template);
  fprintf(stderr, "oracle/ref: elegant aborted: ");
  vfprintf(stderr, template, ap);
  va_end(ap);
  abort();
}

void bombTracking(const char *error) { bombElegant(error, NULL); }

void exitElegant(long status) {
  fprintf(stderr, "oracle/ref: elegant exited with status %ld\n", status);
  abort();
}

/* warnings (src/warnings.c, which keeps them in the SDDS toolkit's hash
 * tables) print nothing here */
void printWarningForTracking(char *text, char *detail) {
  (void)text;
  (void)detail;
}
void printWarning(char *text, char *detail) {
  (void)text;
  (void)detail;
}

/* no obstruction data is ever defined */
long insideObstruction(double *part, short mode, double dz, long segment, long nSegments) {
  (void)part;
  (void)mode;
  (void)dz;
  (void)segment;
  (void)nSegments;
  return 0;
}
long insideObstruction_xyz(double x, double xp, double y, double yp, long particleID, double *lossCoordinates,
                           double tilt, short mode, double dz, long segment, long nSegments) {
  (void)x;
  (void)xp;
  (void)y;
  (void)yp;
  (void)particleID;
  (void)lossCoordinates;
  (void)tilt;
  (void)mode;
  (void)dz;
  (void)segment;
  (void)nSegments;
  return 0;
}

/* serial elegant (elegant.c:366-370): one process that is both master and
 * worker, all processors doing the same thing */
long isMaster = 1;
long isSlave = 1;
long notSinglePart = 0;

/* SDDS mdblib: set n doubles to value */
long fill_double_array(double *array, long n, double value) {
  for (long i = 0; i < n; i++)
    array[i] = value;
  return 1;
}

/* ------------------------- do_tracking's calls outside the tracking path
 * do_tracking() (src/do_tracking.c) calls these on every run; for the
 * elements of the tracking path they have nothing to do: there are no
 * obstructions and no RPN expressions read the stored values. */
void setObstructionsMode(long state) { (void)state; }
long rpn_create_mem(char *name, int is_string) {
  (void)name;
  (void)is_string;
  return 0;
}
long rpn_store(double value, char *str_value, long memory) {
  (void)value;
  (void)str_value;
  (void)memory;
  return 0;
}

/* src/modulate.c and src/ramp.c are built from namelist files this tree
 * does not generate; their first step returns when no modulation or ramp is
 * defined (src/modulate.c:26-27), which is the only case here */
long applyElementModulations(MODULATION_DATA *modData, LINE_LIST *beamline, double pCentral, double **coord, long np,
                             RUN *run, long iPass) {
  (void)beamline;
  (void)pCentral;
  (void)coord;
  (void)np;
  (void)run;
  (void)iPass;
  if (modData->nItems > 0)
    bombElegant("element modulations are outside the tracking path", NULL);
  return 0;
}
long applyElementRamps(RAMP_DATA *rampData, LINE_LIST *beamline, double pCentral, RUN *run, long iPass) {
  (void)beamline;
  (void)pCentral;
  (void)run;
  (void)iPass;
  if (rampData->nItems > 0)
    bombElegant("element ramps are outside the tracking path", NULL);
  return 0;
}

/* src/insertSCeffects.cc (C++, built from a namelist file this tree does
 * not generate): the count of space-charge insertion specifications, none
 * on the tracking path */
long getSCMULTSpecCount(void) { return 0; }

/* src/obstructionData.c (built from a namelist file this tree does not
 * generate): with no obstruction defined no particle is inside one, so the
 * filter keeps every row */
long filterParticlesWithObstructions(double **coord, long np, double **accepted, double z, double P_central) {
  (void)coord;
  (void)accepted;
  (void)z;
  (void)P_central;
  return np;
}
