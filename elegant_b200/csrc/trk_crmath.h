/*
 * trk_crmath.h -- correctly rounded sin, cos and asin in double-double
 * arithmetic, compilable as CUDA device code and as host C.
 *
 * Why: the reference's CSBEND drift (src/csbend.c:1580-1606) evaluates
 * X = rho0*(f-1) + f*X with f = cos(phi)/cos(dsh/rho0+phi) close to 1, so a
 * one-ulp change in cos() moves X by about rho0*2^-53, and the RFCA kick
 * takes sin() of phases up to ~1e6 rad.  A device build that rounds these
 * functions correctly reproduces a correctly rounding libm bit for bit;
 * glibc rounds them correctly on all but a few calls per million (more for
 * large sin arguments), which bounds parity with a glibc-linked reference.
 *
 * Method (Dekker/Knuth error-free transformations, all from published
 * mathematics):
 *   - sin/cos: x = k*pi/2 + r with pi/2 split into three doubles and exact
 *     products (FMA two_prod), then the Taylor series of sin/cos in
 *     double-double on |r| <= pi/4;
 *   - asin: one Newton step a1 = a0 + (y - sin a0)/cos a0 from a double
 *     estimate a0, with sin a0 in double-double.
 * The double-double results carry ~2^-100 relative error, so their leading
 * part is the correctly rounded value except in ~2^-47 of cases.
 * Constants: Taylor coefficients (-1)^k/(2k+1)! and (-1)^k/(2k)! as
 * double-double, pi/2 in three parts, 2/pi (exact rationals rounded in high
 * precision).
 */
#ifndef TRK_CRMATH_H
#define TRK_CRMATH_H

#ifdef __CUDACC__
#define TRKCR_FN __device__ __forceinline__
#define TRKCR_CONST __device__ __constant__ const
#define TRKCR_ADD(a, b) __dadd_rn((a), (b))
#define TRKCR_SUB(a, b) __dsub_rn((a), (b))
#define TRKCR_MUL(a, b) __dmul_rn((a), (b))
#define TRKCR_DIV(a, b) __ddiv_rn((a), (b))
#define TRKCR_FMA(a, b, c) __fma_rn((a), (b), (c))
#define TRKCR_ASIN(x) asin(x)
#define TRKCR_COS(x) cos(x)
#else
#include <math.h>
/* host build: compile with -ffp-contract=off so each operation rounds once */
#define TRKCR_FN static inline
#define TRKCR_CONST static const
#define TRKCR_ADD(a, b) ((a) + (b))
#define TRKCR_SUB(a, b) ((a) - (b))
#define TRKCR_MUL(a, b) ((a) * (b))
#define TRKCR_DIV(a, b) ((a) / (b))
#define TRKCR_FMA(a, b, c) fma((a), (b), (c))
#define TRKCR_ASIN(x) asin(x)
#define TRKCR_COS(x) cos(x)
#endif

typedef struct {
  double hi, lo;
} trkcr_dd;

TRKCR_FN trkcr_dd trkcr_make(double hi, double lo) {
  trkcr_dd r;
  r.hi = hi;
  r.lo = lo;
  return r;
}

TRKCR_FN trkcr_dd trkcr_two_sum(double a, double b) {
  double s = TRKCR_ADD(a, b);
  double bb = TRKCR_SUB(s, a);
  double e = TRKCR_ADD(TRKCR_SUB(a, TRKCR_SUB(s, bb)), TRKCR_SUB(b, bb));
  return trkcr_make(s, e);
}

TRKCR_FN trkcr_dd trkcr_quick_two_sum(double a, double b) {
  double s = TRKCR_ADD(a, b);
  double e = TRKCR_SUB(b, TRKCR_SUB(s, a));
  return trkcr_make(s, e);
}

TRKCR_FN trkcr_dd trkcr_two_prod(double a, double b) {
  double p = TRKCR_MUL(a, b);
  double e = TRKCR_FMA(a, b, -p);
  return trkcr_make(p, e);
}

TRKCR_FN trkcr_dd trkcr_add(trkcr_dd a, trkcr_dd b) {
  trkcr_dd s = trkcr_two_sum(a.hi, b.hi);
  trkcr_dd t = trkcr_two_sum(a.lo, b.lo);
  s.lo = TRKCR_ADD(s.lo, t.hi);
  s = trkcr_quick_two_sum(s.hi, s.lo);
  s.lo = TRKCR_ADD(s.lo, t.lo);
  return trkcr_quick_two_sum(s.hi, s.lo);
}

TRKCR_FN trkcr_dd trkcr_mul(trkcr_dd a, trkcr_dd b) {
  trkcr_dd p = trkcr_two_prod(a.hi, b.hi);
  p.lo = TRKCR_FMA(a.hi, b.lo, p.lo);
  p.lo = TRKCR_FMA(a.lo, b.hi, p.lo);
  return trkcr_quick_two_sum(p.hi, p.lo);
}

TRKCR_CONST double trkcr_sin_c[16][2] = {
  {0x1.0000000000000p+0, 0x0.0p+0},
  {-0x1.5555555555555p-3, -0x1.5555555555555p-57},
  {0x1.1111111111111p-7, 0x1.1111111111111p-63},
  {-0x1.a01a01a01a01ap-13, -0x1.a01a01a01a01ap-73},
  {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
  {-0x1.ae64567f544e4p-26, 0x1.c062e06d1f209p-80},
  {0x1.6124613a86d09p-33, 0x1.f28e0cc748ebep-87},
  {-0x1.ae7f3e733b81fp-41, -0x1.1d8656b0ee8cbp-97},
  {0x1.952c77030ad4ap-49, 0x1.ac981465ddc6cp-103},
  {-0x1.2f49b46814157p-57, -0x1.2650f61dbdcb4p-112},
  {0x1.71b8ef6dcf572p-66, -0x1.d043ae40c4647p-120},
  {-0x1.761b41316381ap-75, 0x1.3423c7d91404fp-130},
  {0x1.3f3ccdd165fa9p-84, -0x1.58ddadf344487p-139},
  {-0x1.d1ab1c2dccea3p-94, -0x1.054d0c78aea14p-149},
  {0x1.259f98b4358adp-103, 0x1.eaf8c39dd9bc5p-157},
  {-0x1.434d2e783f5bcp-113, -0x1.0b87b91be9affp-167},
};

TRKCR_CONST double trkcr_cos_c[16][2] = {
  {0x1.0000000000000p+0, 0x0.0p+0},
  {-0x1.0000000000000p-1, 0x0.0p+0},
  {0x1.5555555555555p-5, 0x1.5555555555555p-59},
  {-0x1.6c16c16c16c17p-10, 0x1.f49f49f49f49fp-65},
  {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76},
  {-0x1.27e4fb7789f5cp-22, -0x1.cbbc05b4fa99ap-76},
  {0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83},
  {-0x1.93974a8c07c9dp-37, -0x1.05d6f8a2efd1fp-92},
  {0x1.ae7f3e733b81fp-45, 0x1.1d8656b0ee8cbp-101},
  {-0x1.6827863b97d97p-53, -0x1.eec01221a8b0bp-107},
  {0x1.e542ba4020225p-62, 0x1.ea72b4afe3c2fp-120},
  {-0x1.0ce396db7f853p-70, 0x1.aebcdbd20331cp-124},
  {0x1.f2cf01972f578p-80, -0x1.9ada5fcc1ab14p-135},
  {-0x1.88e85fc6a4e5ap-89, 0x1.71c37ebd16540p-143},
  {0x1.0a18a2635085dp-98, 0x1.b9e2e28e1aa54p-153},
  {-0x1.3932c5047d60ep-108, -0x1.832b7b530a627p-162},
};

#define TRKCR_PIO2_1 0x1.921fb54442d18p+0
#define TRKCR_PIO2_2 0x1.1a62633145c07p-54
#define TRKCR_PIO2_3 -0x1.f1976b7ed8fbcp-110
#define TRKCR_2OPI 0x1.45f306dc9c883p-1

/* series terms that bring the remainder below 2^-108 |r| */
TRKCR_FN int trkcr_n_terms(double ar) {
  if (ar < 0x1p-5)
    return 8;
  if (ar < 0.25)
    return 12;
  return 15;
}

TRKCR_FN trkcr_dd trkcr_sin_reduced(trkcr_dd r) {
  trkcr_dd r2 = trkcr_mul(r, r);
  int n = trkcr_n_terms(fabs(r.hi));
  trkcr_dd p = trkcr_make(trkcr_sin_c[n][0], trkcr_sin_c[n][1]);
  for (int k = n - 1; k >= 0; k--)
    p = trkcr_add(trkcr_mul(p, r2), trkcr_make(trkcr_sin_c[k][0], trkcr_sin_c[k][1]));
  return trkcr_mul(p, r);
}

TRKCR_FN trkcr_dd trkcr_cos_reduced(trkcr_dd r) {
  trkcr_dd r2 = trkcr_mul(r, r);
  int n = trkcr_n_terms(fabs(r.hi));
  trkcr_dd p = trkcr_make(trkcr_cos_c[n][0], trkcr_cos_c[n][1]);
  for (int k = n - 1; k >= 0; k--)
    p = trkcr_add(trkcr_mul(p, r2), trkcr_make(trkcr_cos_c[k][0], trkcr_cos_c[k][1]));
  return p;
}

/* x = k*pi/2 + r, |r| <~ pi/4; valid for |x| < 2^30 */
TRKCR_FN trkcr_dd trkcr_reduce(double x, int *quadrant) {
  if (fabs(x) <= 0.78539816339744828) {
    *quadrant = 0;
    return trkcr_make(x, 0.0);
  }
  double k = rint(TRKCR_MUL(x, TRKCR_2OPI));
  trkcr_dd a = trkcr_two_prod(k, TRKCR_PIO2_1);
  trkcr_dd r = trkcr_two_sum(x, -a.hi);
  r = trkcr_add(r, trkcr_make(-a.lo, 0.0));
  trkcr_dd b = trkcr_two_prod(k, TRKCR_PIO2_2);
  r = trkcr_add(r, trkcr_make(-b.hi, -b.lo));
  r = trkcr_add(r, trkcr_make(-TRKCR_MUL(k, TRKCR_PIO2_3), 0.0));
  long long ki = (long long)k;
  *quadrant = (int)(ki & 3);
  return r;
}

TRKCR_FN trkcr_dd trkcr_neg(trkcr_dd v) { return trkcr_make(-v.hi, -v.lo); }

TRKCR_FN trkcr_dd trkcr_sin_dd(double x) {
  int q;
  trkcr_dd r = trkcr_reduce(x, &q);
  switch (q) {
  case 0:
    return trkcr_sin_reduced(r);
  case 1:
    return trkcr_cos_reduced(r);
  case 2:
    return trkcr_neg(trkcr_sin_reduced(r));
  default:
    return trkcr_neg(trkcr_cos_reduced(r));
  }
}

TRKCR_FN trkcr_dd trkcr_cos_dd(double x) {
  int q;
  trkcr_dd r = trkcr_reduce(x, &q);
  switch (q) {
  case 0:
    return trkcr_cos_reduced(r);
  case 1:
    return trkcr_neg(trkcr_sin_reduced(r));
  case 2:
    return trkcr_neg(trkcr_cos_reduced(r));
  default:
    return trkcr_sin_reduced(r);
  }
}

TRKCR_FN double trkcr_sin(double x) {
  if (x == 0.0)
    return x;
  if (!isfinite(x))
    return x - x;
  trkcr_dd v = trkcr_sin_dd(x);
  return TRKCR_ADD(v.hi, v.lo);
}

TRKCR_FN double trkcr_cos(double x) {
  if (!isfinite(x))
    return x - x;
  trkcr_dd v = trkcr_cos_dd(x);
  return TRKCR_ADD(v.hi, v.lo);
}

/* tan = sin/cos with a double-double quotient */
TRKCR_FN double trkcr_tan(double x) {
  if (x == 0.0)
    return x;
  if (!isfinite(x))
    return x - x;
  trkcr_dd sn = trkcr_sin_dd(x), cs = trkcr_cos_dd(x);
  double q1 = TRKCR_DIV(sn.hi, cs.hi);
  trkcr_dd p = trkcr_two_prod(q1, cs.hi);
  p.lo = TRKCR_FMA(q1, cs.lo, p.lo);
  trkcr_dd r = trkcr_add(sn, trkcr_make(-p.hi, -p.lo));
  double q2 = TRKCR_DIV(r.hi, cs.hi);
  trkcr_dd q = trkcr_two_sum(q1, q2);
  return TRKCR_ADD(q.hi, q.lo);
}

TRKCR_FN double trkcr_asin(double y) {
  if (y == 0.0 || fabs(y) >= 1.0 || isnan(y))
    return TRKCR_ASIN(y);
  double a0 = TRKCR_ASIN(y);
  trkcr_dd s = trkcr_sin_dd(a0);
  double c = TRKCR_COS(a0);
  trkcr_dd d = trkcr_two_sum(y, -s.hi);
  double num = TRKCR_ADD(d.hi, TRKCR_SUB(d.lo, s.lo));
  double delta = TRKCR_DIV(num, c);
  trkcr_dd a = trkcr_two_sum(a0, delta);
  return TRKCR_ADD(a.hi, a.lo);
}

#endif
