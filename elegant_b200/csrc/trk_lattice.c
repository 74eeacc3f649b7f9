/*
 * trk_lattice.c -- element parameter tables, lattice builder and a small
 * elegant lattice-file parser.  Plain C; linked into both libtrkgpu.so and
 * the CPU oracle so both read the same lattice.
 */
#include <ctype.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "trk_lattice.h"

/* ------------------------------------------------------------ errors */
static __thread char trk_errbuf[512];

int trk_set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(trk_errbuf, sizeof(trk_errbuf), fmt, ap);
  va_end(ap);
  return code;
}

const char *trk_last_error(void) { return trk_errbuf; }
int trk_abi_version(void) { return TRK_ABI_VERSION; }

/* ------------------------------------------------------ parameter tables */
typedef struct {
  const char *name;
  double dflt;
} trk_param_def;

#define TRK_DEF_ENTRY(e, n, d) {n, d},
static const trk_param_def defs_drif[] = {TRK_PARAMS_DRIF(TRK_DEF_ENTRY)};
static const trk_param_def defs_edrift[] = {TRK_PARAMS_EDRIFT(TRK_DEF_ENTRY)};
static const trk_param_def defs_kquad[] = {TRK_PARAMS_KQUAD(TRK_DEF_ENTRY)};
static const trk_param_def defs_ksext[] = {TRK_PARAMS_KSEXT(TRK_DEF_ENTRY)};
static const trk_param_def defs_koct[] = {TRK_PARAMS_KOCT(TRK_DEF_ENTRY)};
static const trk_param_def defs_csbend[] = {TRK_PARAMS_CSBEND(TRK_DEF_ENTRY)};
static const trk_param_def defs_rfca[] = {TRK_PARAMS_RFCA(TRK_DEF_ENTRY)};
static const trk_param_def defs_wake[] = {TRK_PARAMS_WAKE(TRK_DEF_ENTRY)};
static const trk_param_def defs_trwake[] = {TRK_PARAMS_TRWAKE(TRK_DEF_ENTRY)};
static const trk_param_def defs_maxamp[] = {TRK_PARAMS_MAXAMP(TRK_DEF_ENTRY)};
static const trk_param_def defs_charge[] = {TRK_PARAMS_CHARGE(TRK_DEF_ENTRY)};
static const trk_param_def defs_mark[] = {TRK_PARAMS_MARK(TRK_DEF_ENTRY)};
#undef TRK_DEF_ENTRY

typedef struct {
  const char *name;
  const trk_param_def *defs;
  int n;
} trk_type_def;

static const trk_type_def type_defs[TRK_N_TYPES] = {
  {"MARK", defs_mark, P_MARK_COUNT_},
  {"DRIF", defs_drif, P_DRIF_COUNT_},
  {"EDRIFT", defs_edrift, P_EDRIFT_COUNT_},
  {"KQUAD", defs_kquad, P_KQUAD_COUNT_},
  {"KSEXT", defs_ksext, P_KSEXT_COUNT_},
  {"KOCT", defs_koct, P_KOCT_COUNT_},
  {"CSBEND", defs_csbend, P_CSBEND_COUNT_},
  {"RFCA", defs_rfca, P_RFCA_COUNT_},
  {"WAKE", defs_wake, P_WAKE_COUNT_},
  {"TRWAKE", defs_trwake, P_TRWAKE_COUNT_},
  {"MAXAMP", defs_maxamp, P_MAXAMP_COUNT_},
  {"CHARGE", defs_charge, P_CHARGE_COUNT_},
};

static int str_ieq(const char *a, const char *b) {
  for (; *a && *b; a++, b++)
    if (toupper((unsigned char)*a) != toupper((unsigned char)*b))
      return 0;
  return *a == *b;
}

int trk_type_code(const char *name) {
  if (!name)
    return -1;
  for (int t = 0; t < TRK_N_TYPES; t++)
    if (str_ieq(name, type_defs[t].name))
      return t;
  /* accepted spellings of the same elements in elegant lattice files */
  if (str_ieq(name, "DRIFT"))
    return TRK_DRIF;
  if (str_ieq(name, "MARKER"))
    return TRK_MARK;
  return -1;
}

const char *trk_type_name(int type) {
  if (type < 0 || type >= TRK_N_TYPES)
    return NULL;
  return type_defs[type].name;
}

int trk_param_count(int type) {
  if (type < 0 || type >= TRK_N_TYPES)
    return TRK_ERR_UNKNOWN_TYPE;
  return type_defs[type].n;
}

const char *trk_param_name(int type, int index) {
  if (type < 0 || type >= TRK_N_TYPES || index < 0 || index >= type_defs[type].n)
    return NULL;
  return type_defs[type].defs[index].name;
}

double trk_param_default(int type, int index) {
  if (type < 0 || type >= TRK_N_TYPES || index < 0 || index >= type_defs[type].n)
    return NAN;
  return type_defs[type].defs[index].dflt;
}

int trk_param_index(int type, const char *name) {
  if (type < 0 || type >= TRK_N_TYPES)
    return trk_set_error(TRK_ERR_UNKNOWN_TYPE, "unknown element type %d", type);
  if (!name)
    return trk_set_error(TRK_ERR_ARG, "null parameter name");
  /* N_KICKS is an alias of N_SLICES for CSBEND (src/track_data.c:1943-1944) */
  if (type == TRK_CSBEND && str_ieq(name, "N_KICKS"))
    return P_CSBEND_N_SLICES;
  for (int i = 0; i < type_defs[type].n; i++)
    if (str_ieq(name, type_defs[type].defs[i].name))
      return i;
  return trk_set_error(TRK_ERR_UNKNOWN_PARAM, "element type %s has no parameter %s",
                       type_defs[type].name, name);
}

/* --------------------------------------------------------------- lattice */
int trk_lattice_create(trk_lattice **lattice) {
  if (!lattice)
    return trk_set_error(TRK_ERR_ARG, "null lattice pointer");
  trk_lattice *l = (trk_lattice *)calloc(1, sizeof(*l));
  if (!l)
    return trk_set_error(TRK_ERR_NOMEM, "lattice allocation failed");
  *lattice = l;
  return TRK_OK;
}

static void elem_free_wake(trk_elem *e) {
  free(e->wake_t);
  free(e->wake_w0);
  free(e->wake_w1);
  e->wake_t = e->wake_w0 = e->wake_w1 = NULL;
  e->wake_points = 0;
}

void trk_lattice_destroy(trk_lattice *l) {
  if (!l)
    return;
  for (int i = 0; i < l->n; i++)
    elem_free_wake(&l->e[i]);
  free(l->e);
  free(l);
}

int trk_lattice_add(trk_lattice *l, int type, const char *name, int *index) {
  if (!l)
    return trk_set_error(TRK_ERR_ARG, "null lattice");
  if (type < 0 || type >= TRK_N_TYPES)
    return trk_set_error(TRK_ERR_UNKNOWN_TYPE, "unknown element type %d", type);
  if (l->n == l->cap) {
    int cap = l->cap ? 2 * l->cap : 64;
    trk_elem *e = (trk_elem *)realloc(l->e, sizeof(*e) * cap);
    if (!e)
      return trk_set_error(TRK_ERR_NOMEM, "lattice growth failed");
    l->e = e;
    l->cap = cap;
  }
  trk_elem *e = &l->e[l->n];
  memset(e, 0, sizeof(*e));
  e->type = type;
  snprintf(e->name, sizeof(e->name), "%s", name ? name : type_defs[type].name);
  for (int i = 0; i < type_defs[type].n; i++)
    e->p[i] = type_defs[type].defs[i].dflt;
  if (index)
    *index = l->n;
  l->n++;
  return TRK_OK;
}

static int check_index(const trk_lattice *l, int index) {
  if (!l)
    return trk_set_error(TRK_ERR_ARG, "null lattice");
  if (index < 0 || index >= l->n)
    return trk_set_error(TRK_ERR_ARG, "element index %d out of range [0,%d)", index, l->n);
  return TRK_OK;
}

int trk_lattice_set(trk_lattice *l, int index, const char *param, double value) {
  int rc = check_index(l, index);
  if (rc)
    return rc;
  int pi = trk_param_index(l->e[index].type, param);
  if (pi < 0)
    return pi;
  l->e[index].p[pi] = value;
  return TRK_OK;
}

int trk_lattice_get(const trk_lattice *l, int index, const char *param, double *value) {
  int rc = check_index(l, index);
  if (rc)
    return rc;
  if (!value)
    return trk_set_error(TRK_ERR_ARG, "null value pointer");
  int pi = trk_param_index(l->e[index].type, param);
  if (pi < 0)
    return pi;
  *value = l->e[index].p[pi];
  return TRK_OK;
}

int trk_lattice_length(const trk_lattice *l) { return l ? l->n : 0; }

int trk_lattice_type(const trk_lattice *l, int index) {
  if (check_index(l, index))
    return TRK_ERR_ARG;
  return l->e[index].type;
}

int trk_lattice_set_wake(trk_lattice *l, int index, const double *t, const double *W,
                         const double *Wy, long points) {
  int rc = check_index(l, index);
  if (rc)
    return rc;
  trk_elem *e = &l->e[index];
  if (e->type != TRK_WAKE && e->type != TRK_TRWAKE)
    return trk_set_error(TRK_ERR_ARG, "element %s is not a WAKE or TRWAKE", e->name);
  if (!t || !W || (e->type == TRK_TRWAKE && !Wy))
    return trk_set_error(TRK_ERR_ARG, "null wake table");
  /* set_up_wake: "too little data in WAKE file" (src/wake.c:400-403) */
  if (points < 2)
    return trk_set_error(TRK_ERR_PHYSICS, "too little data in wake table for %s (%ld points)",
                         e->name, points);
  elem_free_wake(e);
  size_t sz = sizeof(double) * (size_t)points;
  e->wake_t = (double *)malloc(sz);
  e->wake_w0 = (double *)malloc(sz);
  if (e->type == TRK_TRWAKE)
    e->wake_w1 = (double *)malloc(sz);
  if (!e->wake_t || !e->wake_w0 || (e->type == TRK_TRWAKE && !e->wake_w1)) {
    elem_free_wake(e);
    return trk_set_error(TRK_ERR_NOMEM, "wake table allocation failed");
  }
  memcpy(e->wake_t, t, sz);
  memcpy(e->wake_w0, W, sz);
  if (e->type == TRK_TRWAKE)
    memcpy(e->wake_w1, Wy, sz);
  e->wake_points = points;
  return TRK_OK;
}

double trk_elem_length(const trk_elem *e) {
  switch (e->type) {
  case TRK_DRIF:
    return TRK_P(e, DRIF_L);
  case TRK_EDRIFT:
    return TRK_P(e, EDRIFT_L);
  case TRK_KQUAD:
    return TRK_P(e, KQUAD_L);
  case TRK_KSEXT:
    return TRK_P(e, KSEXT_L);
  case TRK_KOCT:
    return TRK_P(e, KOCT_L);
  case TRK_CSBEND:
    return TRK_P(e, CSBEND_L);
  case TRK_RFCA:
    return TRK_P(e, RFCA_L);
  default:
    return 0.0;
  }
}

double trk_lattice_total_length(const trk_lattice *l) {
  double z = 0;
  if (!l)
    return 0;
  for (int i = 0; i < l->n; i++)
    z += trk_elem_length(&l->e[i]);
  return z;
}

/* ------------------------------------------------------ lattice parser */
/* Definitions of the form
 *     NAME: TYPE, PARAM=value, ...
 *     NAME: LINE=(E1, E2, n*E3, -E4, ...)
 * with '&' continuation and '!' comments, as in elegant lattice files
 * (parsed by src/get_beamline.c / src/mad_parse.c in the reference).
 * Values are numbers; RPN expressions in quotes are not evaluated.        */

typedef struct {
  char name[48];
  int is_line;
  int type;           /* element */
  double p[TRK_MAX_PARAMS];
  char *line_items;   /* line: comma separated item text */
} parse_def;

typedef struct {
  parse_def *d;
  int n, cap;
} parse_defs;

static void upcase(char *s) {
  for (; *s; s++)
    *s = (char)toupper((unsigned char)*s);
}

static char *trim(char *s) {
  while (isspace((unsigned char)*s))
    s++;
  char *e = s + strlen(s);
  while (e > s && isspace((unsigned char)e[-1]))
    *--e = 0;
  if (*s == '"' && e > s + 1 && e[-1] == '"') {
    e[-1] = 0;
    s++;
  }
  return s;
}

static parse_def *find_def(parse_defs *defs, const char *name) {
  for (int i = defs->n - 1; i >= 0; i--)
    if (str_ieq(defs->d[i].name, name))
      return &defs->d[i];
  return NULL;
}

static int expand_line(trk_lattice *l, parse_defs *defs, const char *name, int reverse, int depth) {
  if (depth > 64)
    return trk_set_error(TRK_ERR_ARG, "line nesting too deep at %s", name);
  parse_def *d = find_def(defs, name);
  if (!d)
    return trk_set_error(TRK_ERR_ARG, "undefined element or line %s", name);
  if (!d->is_line) {
    int idx, rc = trk_lattice_add(l, d->type, d->name, &idx);
    if (rc)
      return rc;
    memcpy(l->e[idx].p, d->p, sizeof(d->p));
    return TRK_OK;
  }
  /* split items */
  char *items = strdup(d->line_items);
  if (!items)
    return trk_set_error(TRK_ERR_NOMEM, "parser allocation failed");
  char *tok[4096];
  int nt = 0;
  for (char *s = strtok(items, ","); s && nt < 4096; s = strtok(NULL, ","))
    tok[nt++] = s;
  int rc = TRK_OK;
  for (int k = 0; k < nt && rc == TRK_OK; k++) {
    int i = reverse ? nt - 1 - k : k;
    char *it = trim(tok[i]);
    long count = 1;
    int rev = 0;
    char *star = strchr(it, '*');
    if (star) {
      *star = 0;
      count = strtol(trim(it), NULL, 10);
      it = trim(star + 1);
    }
    if (*it == '-') {
      rev = 1;
      it = trim(it + 1);
    }
    for (long c = 0; c < count && rc == TRK_OK; c++)
      rc = expand_line(l, defs, it, reverse ^ rev, depth + 1);
  }
  free(items);
  return rc;
}

int trk_lattice_parse(trk_lattice *l, const char *text, const char *line) {
  if (!l || !text || !line)
    return trk_set_error(TRK_ERR_ARG, "null argument to trk_lattice_parse");
  /* join continuation lines and strip comments */
  size_t n = strlen(text);
  char *buf = (char *)malloc(n + 2);
  if (!buf)
    return trk_set_error(TRK_ERR_NOMEM, "parser allocation failed");
  size_t o = 0;
  int in_quote = 0;
  for (size_t i = 0; i < n; i++) {
    char c = text[i];
    if (c == '"')
      in_quote = !in_quote;
    if (!in_quote && c == '!') {
      while (i < n && text[i] != '\n')
        i++;
      c = '\n';
    }
    if (!in_quote && c == '&') {
      while (i < n && text[i] != '\n')
        i++;
      continue;
    }
    buf[o++] = c;
  }
  buf[o] = 0;

  parse_defs defs = {NULL, 0, 0};
  int rc = TRK_OK;
  char *save = NULL;
  for (char *stmt = strtok_r(buf, "\n;", &save); stmt && rc == TRK_OK; stmt = strtok_r(NULL, "\n;", &save)) {
    char *s = trim(stmt);
    if (!*s)
      continue;
    char *colon = strchr(s, ':');
    if (!colon) {
      rc = trk_set_error(TRK_ERR_ARG, "cannot parse lattice statement: %s", s);
      break;
    }
    *colon = 0;
    char *name = trim(s);
    char *rest = trim(colon + 1);
    if (defs.n == defs.cap) {
      defs.cap = defs.cap ? 2 * defs.cap : 64;
      defs.d = (parse_def *)realloc(defs.d, sizeof(parse_def) * defs.cap);
      if (!defs.d) {
        rc = trk_set_error(TRK_ERR_NOMEM, "parser allocation failed");
        break;
      }
    }
    parse_def *d = &defs.d[defs.n];
    memset(d, 0, sizeof(*d));
    snprintf(d->name, sizeof(d->name), "%s", name);
    upcase(d->name);
    /* LINE=( ... ) */
    char head[32];
    size_t hl = strcspn(rest, ",=( \t");
    if (hl >= sizeof(head))
      hl = sizeof(head) - 1;
    memcpy(head, rest, hl);
    head[hl] = 0;
    upcase(head);
    if (strcmp(head, "LINE") == 0) {
      char *lp = strchr(rest, '('), *rp = strrchr(rest, ')');
      if (!lp || !rp || rp < lp) {
        rc = trk_set_error(TRK_ERR_ARG, "bad LINE definition for %s", d->name);
        break;
      }
      *rp = 0;
      d->is_line = 1;
      d->line_items = strdup(lp + 1);
      defs.n++;
      continue;
    }
    /* element: TYPE or previously defined element name */
    char *comma = strchr(rest, ',');
    if (comma)
      *comma = 0;
    char *tname = trim(rest);
    int type = trk_type_code(tname);
    parse_def *base = NULL;
    if (type < 0) {
      base = find_def(&defs, tname);
      if (!base || base->is_line) {
        rc = trk_set_error(TRK_ERR_UNKNOWN_TYPE, "element type %s (for %s) is not on this path", tname, d->name);
        break;
      }
      type = base->type;
    }
    d->type = type;
    for (int i = 0; i < type_defs[type].n; i++)
      d->p[i] = base ? base->p[i] : type_defs[type].defs[i].dflt;
    char *assignments = comma ? comma + 1 : NULL;
    if (assignments) {
      char *save2 = NULL;
      for (char *a = strtok_r(assignments, ",", &save2); a; a = strtok_r(NULL, ",", &save2)) {
        char *eq = strchr(a, '=');
        if (!eq)
          continue;
        *eq = 0;
        char *pname = trim(a);
        char *val = trim(eq + 1);
        int pi = trk_param_index(type, pname);
        if (pi < 0) {
          rc = pi;
          break;
        }
        char *end = NULL;
        double v = strtod(val, &end);
        if (end == val) {
          rc = trk_set_error(TRK_ERR_UNSUPPORTED, "value \"%s\" of %s.%s is not a number", val, d->name, pname);
          break;
        }
        d->p[pi] = v;
      }
    }
    if (rc == TRK_OK)
      defs.n++;
  }
  if (rc == TRK_OK)
    rc = expand_line(l, &defs, line, 0, 0);
  for (int i = 0; i < defs.n; i++)
    free(defs.d[i].line_items);
  free(defs.d);
  free(buf);
  return rc;
}
