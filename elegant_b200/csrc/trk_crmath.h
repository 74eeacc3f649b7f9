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
#define TRKCR_SLOW static __device__ __noinline__
#define TRKCR_CONST __device__ __constant__ const
#define TRKCR_ADD(a, b) __dadd_rn((a), (b))
#define TRKCR_SUB(a, b) __dsub_rn((a), (b))
#define TRKCR_MUL(a, b) __dmul_rn((a), (b))
#define TRKCR_DIV(a, b) __ddiv_rn((a), (b))
#define TRKCR_FMA(a, b, c) __fma_rn((a), (b), (c))
#define TRKCR_ASIN(x) asin(x)
#define TRKCR_COS(x) cos(x)
#define TRKCR_EXP(x) exp(x)
#define TRKCR_SINH(x) sinh(x)
#define TRKCR_COSH(x) cosh(x)
#define TRKCR_LDEXP(x, k) ldexp((x), (k))
#define TRKCR_HIWORD(x) ((unsigned)__double2hiint(x))
#else
#include <math.h>
/* host build: compile with -ffp-contract=off so each operation rounds once */
#define TRKCR_FN static inline
#define TRKCR_SLOW static
#define TRKCR_CONST static const
#define TRKCR_ADD(a, b) ((a) + (b))
#define TRKCR_SUB(a, b) ((a) - (b))
#define TRKCR_MUL(a, b) ((a) * (b))
#define TRKCR_DIV(a, b) ((a) / (b))
#define TRKCR_FMA(a, b, c) fma((a), (b), (c))
#define TRKCR_ASIN(x) asin(x)
#define TRKCR_COS(x) cos(x)
#define TRKCR_EXP(x) exp(x)
#define TRKCR_SINH(x) sinh(x)
#define TRKCR_COSH(x) cosh(x)
#define TRKCR_LDEXP(x, k) ldexp((x), (k))
#include <stdint.h>
#include <string.h>
static inline unsigned trkcr_hiword(double x) {
  uint64_t b;
  memcpy(&b, &x, sizeof b);
  return (unsigned)(b >> 32);
}
#define TRKCR_HIWORD(x) trkcr_hiword(x)
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

TRKCR_SLOW double trkcr_sin_slow(double x) {
  if (x == 0.0)
    return x;
  if (!isfinite(x))
    return x - x;
  trkcr_dd v = trkcr_sin_dd(x);
  return TRKCR_ADD(v.hi, v.lo);
}

TRKCR_SLOW double trkcr_cos_slow(double x) {
  if (!isfinite(x))
    return x - x;
  trkcr_dd v = trkcr_cos_dd(x);
  return TRKCR_ADD(v.hi, v.lo);
}

/*
 * Fast paths for small arguments (|x| <= 2^-5, the CSBEND substep angles and
 * slopes), after Ziv's strategy: evaluate the function as hi + L with a
 * rigorous bound e on |f(x) - (hi + L)|, and return RN(hi + L) when
 * RN(hi + L + e) == RN(hi + L - e), i.e. when every value the true result
 * can take rounds the same way.  Otherwise the caller takes the
 * double-double path above.  The bound is a few times 2^-100 |x|, so the
 * test fails only for arguments whose result lies within that distance of
 * a rounding boundary (about one call in 2^20 or fewer).
 *
 * The leading correction (x^3/6 for sin and asin, x^2/2 for cos) is formed
 * exactly or to ~2^-104 relative with error-free products; the rest of the
 * series, c2 (at most 2^-27 |x| for sin and asin, 2^-22 for cos), in plain
 * double.  Error budget, written into e:
 *   2^-49 |c2|        the plain-double tail (at most 7 roundings, 2^-50.2
 *                     relative, from the rounded powers, coefficients and
 *                     Horner steps) and its truncation (below 2^-62 |c2|);
 *   2^-100 |x|        the leading correction's low part (below 2^-103 |x^3|);
 *   2^-51 |L|         the roundings of L and of L +- e in the test itself.
 * Each term carries a factor of two or more over the error it covers, which
 * also absorbs the roundings of e's own sum.
 * Arguments below 2^-26 (2^-27 for cos) return x (1) directly: the first
 * correction is then under half an ulp.
 */
#define TRKCR_SMALL 0x1p-5

TRKCR_FN int trkcr_round_test(double hi, double L, double e, double *out) {
  const double u = TRKCR_ADD(hi, TRKCR_ADD(L, e));
  const double v = TRKCR_ADD(hi, TRKCR_SUB(L, e));
  *out = u;
  return u == v;
}

/* x + sgn*x^3/6 + x^5 P(x^2) split as hi + L, with the error bound; sgn is
 * -1 for sin, +1 for asin */
TRKCR_FN double trkcr_odd_small(double x, double sgn, double c2, double zh, double zl, double th, double tl,
                                double *L, double *e) {
  const double S1h = 0x1.5555555555555p-3, S1l = 0x1.5555555555555p-57; /* 1/6 */
  /* x^3 = th + tl + zl x, |zl x| rounding below 2^-106 |x^3| */
  const double t_lo = TRKCR_ADD(tl, TRKCR_MUL(zl, x));
  const double c1h = TRKCR_MUL(sgn, TRKCR_MUL(th, S1h));
  const double e1 = TRKCR_FMA(sgn * th, S1h, -c1h);
  const double c1l = TRKCR_ADD(e1, TRKCR_MUL(sgn, TRKCR_ADD(TRKCR_MUL(th, S1l), TRKCR_MUL(t_lo, S1h))));
  const double lo = TRKCR_ADD(c1l, c2);
  const double sh = TRKCR_ADD(x, c1h);
  const double sl = TRKCR_SUB(c1h, TRKCR_SUB(sh, x));
  *L = TRKCR_ADD(sl, lo);
  *e = TRKCR_ADD(TRKCR_ADD(TRKCR_MUL(0x1p-49, fabs(c2)), TRKCR_MUL(0x1p-100, fabs(x))),
                 TRKCR_MUL(0x1p-51, fabs(*L)));
  return sh;
}

/* sin x as hi + L within e, for 2^-26 <= |x| <= 2^-5, from zh + zl = x^2 */
TRKCR_FN double trkcr_sin_parts(double x, double zh, double zl, double *L, double *e) {
  const double th = TRKCR_MUL(zh, x);
  const double tl = TRKCR_FMA(zh, x, -th);
  /* x^5 (1/120 - z/5040 + z^2/362880 - z^3/39916800) */
  double P = TRKCR_FMA(zh, -0x1.ae64567f544e4p-26, 0x1.71de3a556c734p-19);
  P = TRKCR_FMA(zh, P, -0x1.a01a01a01a01ap-13);
  P = TRKCR_FMA(zh, P, 0x1.1111111111111p-7);
  const double c2 = TRKCR_MUL(TRKCR_MUL(th, zh), P);
  return trkcr_odd_small(x, -1.0, c2, zh, zl, th, tl, L, e);
}

/* cos x as hi + L within e, for 2^-27 <= |x| <= 2^-5, from zh + zl = x^2:
 * cos = (1 - zh/2) + (-zl/2 + zh^2 Q(zh)),
 * Q = 1/24 - z/720 + z^2/40320 - z^3/3628800 + z^4/479001600 (first omitted
 * term z^7/14! below 2^-106); the tail's error (the rounded zh^2, the
 * dropped 2 zh zl, Q's roundings) stays under 2^-50.5 |zh^2 Q|, covered by
 * 2^-48 (|t| + |zl|) */
TRKCR_FN double trkcr_cos_parts(double zh, double zl, double *L, double *e) {
  const double ah = TRKCR_SUB(1.0, TRKCR_MUL(0.5, zh));
  const double al = TRKCR_SUB(TRKCR_SUB(1.0, ah), TRKCR_MUL(0.5, zh));
  double Q = TRKCR_FMA(zh, 0x1.1eed8eff8d898p-29, -0x1.27e4fb7789f5cp-22);
  Q = TRKCR_FMA(zh, Q, 0x1.a01a01a01a01ap-16);
  Q = TRKCR_FMA(zh, Q, -0x1.6c16c16c16c17p-10);
  Q = TRKCR_FMA(zh, Q, 0x1.5555555555555p-5);
  const double t = TRKCR_FMA(TRKCR_MUL(zh, zh), Q, TRKCR_MUL(-0.5, zl));
  *L = TRKCR_ADD(al, t);
  *e = TRKCR_ADD(TRKCR_ADD(TRKCR_MUL(0x1p-48, TRKCR_ADD(fabs(t), fabs(zl))), TRKCR_MUL(0x1p-51, fabs(*L))),
                 0x1p-110);
  return ah;
}

/* correctly rounded sin of |x| <= 2^-5, or 0 when the rounding test fails */
TRKCR_FN int trkcr_sin_small(double x, double *s) {
  if (fabs(x) < 0x1p-26) {
    *s = x;
    return 1;
  }
  double L, e;
  const double zh = TRKCR_MUL(x, x);
  const double hi = trkcr_sin_parts(x, zh, TRKCR_FMA(x, x, -zh), &L, &e);
  return trkcr_round_test(hi, L, e, s);
}

/* correctly rounded cos of |x| <= 2^-5, or 0 when the rounding test fails */
TRKCR_FN int trkcr_cos_small(double x, double *c) {
  if (fabs(x) < 0x1p-27) {
    *c = 1.0;
    return 1;
  }
  double L, e;
  const double zh = TRKCR_MUL(x, x);
  const double hi = trkcr_cos_parts(zh, TRKCR_FMA(x, x, -zh), &L, &e);
  return trkcr_round_test(hi, L, e, c);
}

/*
 * Tiny arguments (2^-27 <= |x| <= 2^-7, the CSBEND substep angles and most
 * slopes): the correction to the leading term (x for sin and asin, 1 for
 * cos) is formed in plain double, with a rigorous relative error bound, and
 * the same rounding test decides.  With |x| <= 2^-7 the correction is at
 * most 2^-15.4 |x| (sin, asin) or 2^-15 (cos), so a relative error of
 * 2^-50 in it is a few 2^-66 of the result: the test then fails for about
 * one call in 2^13 (cos near |x| = 2^-7) to far fewer (smaller |x|), and
 * the caller takes the next path.
 *
 * Error budget of the correction c (sin, asin: c = x^3 P(x^2); cos:
 * c = x^2 Q(x^2), result 1 - c): x^2 rounded (2^-53), x^3 or the final
 * product rounded (2^-53 each), P or Q rounded (2^-53 from its last FMA and
 * 2^-53.4 from its leading coefficient; the other terms are scaled by
 * x^2 <= 2^-14), truncation of the series (below 2^-56 relative): in all
 * below 2^-50.7 |c|.  The test widens c by e = 2^-49 |c|, which covers that
 * error and the rounding of c +- e.
 * Series: sin  P = -1/6 + z/120 - z^2/5040          (next: z^3/9!, 2^-58 rel.)
 *         asin P = 1/6 + 3z/40 + 5z^2/112 + 35z^3/1152 + 63z^4/2816
 *                                                    (next: 231 z^5/13312)
 *         cos  Q = 1/2 - z/24 + z^2/720              (next: z^3/8!, 2^-56 rel.)
 */
#define TRKCR_TINY 0x1p-7

TRKCR_FN int trkcr_tiny_test(double lead, double c, double *out) {
  const double ac = fabs(c);
  const double u = TRKCR_ADD(lead, TRKCR_FMA(ac, 0x1p-49, c));
  const double v = TRKCR_ADD(lead, TRKCR_FMA(-ac, 0x1p-49, c));
  *out = u;
  return u == v;
}

/* the corrections: sin x = x + c, cos x = 1 + c, asin y = y + c */
TRKCR_FN double trkcr_sin_tiny_c(double x, double z) {
  double P = TRKCR_FMA(z, -0x1.a01a01a01a01ap-13, 0x1.1111111111111p-7);
  P = TRKCR_FMA(z, P, -0x1.5555555555555p-3);
  return TRKCR_MUL(TRKCR_MUL(x, z), P);
}

TRKCR_FN double trkcr_cos_tiny_c(double z) {
  double Q = TRKCR_FMA(z, 0x1.6c16c16c16c17p-10, -0x1.5555555555555p-5);
  Q = TRKCR_FMA(z, Q, 0.5);
  return -TRKCR_MUL(z, Q);
}

TRKCR_FN double trkcr_asin_tiny_c(double y, double z) {
  double P = TRKCR_FMA(z, 63.0 / 2816.0, 35.0 / 1152.0);
  P = TRKCR_FMA(z, P, 5.0 / 112.0);
  P = TRKCR_FMA(z, P, 3.0 / 40.0);
  P = TRKCR_FMA(z, P, 0x1.5555555555555p-3);
  return TRKCR_MUL(TRKCR_MUL(y, z), P);
}

/* sin x, 2^-26 <= |x| <= 2^-7, z = RN(x^2) */
TRKCR_FN int trkcr_sin_tiny(double x, double z, double *s) { return trkcr_tiny_test(x, trkcr_sin_tiny_c(x, z), s); }

/* cos x, 2^-27 <= |x| <= 2^-7, z = RN(x^2) */
TRKCR_FN int trkcr_cos_tiny(double z, double *c) { return trkcr_tiny_test(1.0, trkcr_cos_tiny_c(z), c); }

/* asin y, 2^-26 <= |y| <= 2^-7, z = RN(y^2) */
TRKCR_FN int trkcr_asin_tiny(double y, double z, double *a) {
  return trkcr_tiny_test(y, trkcr_asin_tiny_c(y, z), a);
}

/* the paths of |x| <= 2^-5 after the tiny one: double-double correction,
 * then the full double-double evaluation */
TRKCR_SLOW double trkcr_sin_mid(double x) {
  double s;
  if (fabs(x) <= TRKCR_SMALL && trkcr_sin_small(x, &s))
    return s;
  return trkcr_sin_slow(x);
}

TRKCR_SLOW double trkcr_cos_mid(double x) {
  double c;
  if (fabs(x) <= TRKCR_SMALL && trkcr_cos_small(x, &c))
    return c;
  return trkcr_cos_slow(x);
}

TRKCR_FN double trkcr_sin(double x) {
  const double ax = fabs(x);
  if (ax < 0x1p-26)
    return x;
  double s;
  if (ax <= TRKCR_TINY && trkcr_sin_tiny(x, TRKCR_MUL(x, x), &s))
    return s;
  return trkcr_sin_mid(x);
}

TRKCR_FN double trkcr_cos(double x) {
  const double ax = fabs(x);
  if (ax < 0x1p-27)
    return 1.0;
  double c;
  if (ax <= TRKCR_TINY && trkcr_cos_tiny(TRKCR_MUL(x, x), &c))
    return c;
  return trkcr_cos_mid(x);
}

/* sin and cos of one argument (the CSBEND drift needs both): x^2 formed once */
TRKCR_FN void trkcr_sincos(double x, double *s, double *c) {
  const double ax = fabs(x);
  if (ax < 0x1p-27) {
    *s = x;
    *c = 1.0;
    return;
  }
  if (ax <= TRKCR_TINY) {
    const double z = TRKCR_MUL(x, x);
    if (ax < 0x1p-26)
      *s = x;
    else if (!trkcr_sin_tiny(x, z, s))
      *s = trkcr_sin_mid(x);
    if (!trkcr_cos_tiny(z, c))
      *c = trkcr_cos_mid(x);
    return;
  }
  *s = trkcr_sin_mid(x);
  *c = trkcr_cos_mid(x);
}

/* tan = sin/cos with a double-double quotient (bend edges only: not inlined) */
TRKCR_SLOW double trkcr_tan(double x) {
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

TRKCR_SLOW double trkcr_asin_slow(double y) {
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

/* asin(y) = y + y^3/6 + y^5 R(y^2), R = sum_{n>=2} (2n)!/(4^n (n!)^2 (2n+1)) z^(n-2):
 * 3/40, 5/112, 35/1152, 63/2816, 231/13312, 143/10240; the first omitted
 * term (6435/557056 y^17) is below 2^-62 |y^5 R| for |y| <= 2^-5 */
TRKCR_FN double trkcr_asin_parts(double y, double zh, double zl, double *L, double *e) {
  const double th = TRKCR_MUL(zh, y);
  const double tl = TRKCR_FMA(zh, y, -th);
  double R = TRKCR_FMA(zh, 143.0 / 10240.0, 231.0 / 13312.0);
  R = TRKCR_FMA(zh, R, 63.0 / 2816.0);
  R = TRKCR_FMA(zh, R, 35.0 / 1152.0);
  R = TRKCR_FMA(zh, R, 5.0 / 112.0);
  R = TRKCR_FMA(zh, R, 3.0 / 40.0);
  const double c2 = TRKCR_MUL(TRKCR_MUL(th, zh), R);
  return trkcr_odd_small(y, 1.0, c2, zh, zl, th, tl, L, e);
}

TRKCR_SLOW double trkcr_asin_mid(double y) {
  const double ay = fabs(y);
  if (ay <= TRKCR_SMALL) {
    double L, e, out;
    const double zh = TRKCR_MUL(y, y);
    const double hi = trkcr_asin_parts(y, zh, TRKCR_FMA(y, y, -zh), &L, &e);
    if (trkcr_round_test(hi, L, e, &out))
      return out;
  }
  return trkcr_asin_slow(y);
}

TRKCR_FN double trkcr_asin(double y) {
  const double ay = fabs(y);
  if (ay < 0x1p-26)
    return y;
  double a;
  if (ay <= TRKCR_TINY && trkcr_asin_tiny(y, TRKCR_MUL(y, y), &a))
    return a;
  return trkcr_asin_mid(y);
}

/*
 * exp, correctly rounded for |x| <= 700 (the CSBEND Hwang-Lindberg fringe
 * takes exp of a small product per particle, src/csbend.c:4466, :4506).
 * Tiny |x| <= 2^-7: exp x = (1 + x) + x^2 P(x), P = 1/2 + x/6 + ... +
 * x^6/8! (next term x^9/9!, below 2^-66 of x^2/2); 1 + x is
 * split exactly (sh + sl), the rest L = sl + x^2 P in plain double with
 * error below 2^-51.4 |x^2 P| + 2^-53 |L|, and the rounding test widens L
 * by 2^-49 |x^2 P| + 2^-52 |L|.  Otherwise: x = k ln2 + r with ln2 in three
 * parts, exp(r/256) by its Taylor series in double-double, squared eight
 * times, times 2^k (~2^-92 relative); beyond |x| > 700 the library's exp.
 */
TRKCR_CONST double trkcr_exp_c[13][2] = {
  {0x1.0000000000000p+0, 0x0.0p+0},           {0x1.0000000000000p+0, 0x0.0p+0},
  {0x1.0000000000000p-1, 0x0.0p+0},           {0x1.5555555555555p-3, 0x1.5555555555555p-57},
  {0x1.5555555555555p-5, 0x1.5555555555555p-59}, {0x1.1111111111111p-7, 0x1.1111111111111p-63},
  {0x1.6c16c16c16c17p-10, -0x1.f49f49f49f49fp-65}, {0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-73},
  {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76}, {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
  {0x1.27e4fb7789f5cp-22, 0x1.cbbc05b4fa99ap-76}, {0x1.ae64567f544e4p-26, -0x1.c062e06d1f209p-80},
  {0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83},
};
#define TRKCR_LN2_1 0x1.62e42fefa39efp-1
#define TRKCR_LN2_2 0x1.abc9e3b39803fp-56
#define TRKCR_LN2_3 0x1.7b57a079a1934p-111
#define TRKCR_INVLN2 0x1.71547652b82fep+0

/* exp x as a double-double, |x| <= 700 */
TRKCR_FN trkcr_dd trkcr_exp_dd(double x) {
  const double k = rint(TRKCR_MUL(x, TRKCR_INVLN2));
  trkcr_dd a = trkcr_two_prod(k, TRKCR_LN2_1);
  trkcr_dd r = trkcr_two_sum(x, -a.hi);
  r = trkcr_add(r, trkcr_make(-a.lo, 0.0));
  trkcr_dd b = trkcr_two_prod(k, TRKCR_LN2_2);
  r = trkcr_add(r, trkcr_make(-b.hi, -b.lo));
  r = trkcr_add(r, trkcr_make(-TRKCR_MUL(k, TRKCR_LN2_3), 0.0));
  r.hi = TRKCR_MUL(r.hi, 0x1p-8);
  r.lo = TRKCR_MUL(r.lo, 0x1p-8);
  trkcr_dd p = trkcr_make(trkcr_exp_c[12][0], trkcr_exp_c[12][1]);
  for (int i = 11; i >= 0; i--)
    p = trkcr_add(trkcr_mul(p, r), trkcr_make(trkcr_exp_c[i][0], trkcr_exp_c[i][1]));
  for (int i = 0; i < 8; i++)
    p = trkcr_mul(p, p);
  return trkcr_make(TRKCR_LDEXP(p.hi, (int)k), TRKCR_LDEXP(p.lo, (int)k));
}

/* the x^2 P(x) of the tiny path */
TRKCR_FN double trkcr_exp_tiny_t(double x) {
  double P = TRKCR_FMA(x, 0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-13);
  P = TRKCR_FMA(x, P, 0x1.6c16c16c16c17p-10);
  P = TRKCR_FMA(x, P, 0x1.1111111111111p-7);
  P = TRKCR_FMA(x, P, 0x1.5555555555555p-5);
  P = TRKCR_FMA(x, P, 0x1.5555555555555p-3);
  P = TRKCR_FMA(x, P, 0.5);
  return TRKCR_MUL(TRKCR_MUL(x, x), P);
}

TRKCR_SLOW double trkcr_exp_slow(double x) {
  if (!(fabs(x) <= 700.0))
    return TRKCR_EXP(x);
  const trkcr_dd v = trkcr_exp_dd(x);
  return TRKCR_ADD(v.hi, v.lo);
}

TRKCR_FN double trkcr_exp(double x) {
  if (fabs(x) <= TRKCR_TINY) {
    if (x == 0.0)
      return 1.0;
    const double sh = TRKCR_ADD(1.0, x);
    const double sl = TRKCR_ADD(TRKCR_SUB(1.0, sh), x);
    const double t = trkcr_exp_tiny_t(x);
    const double L = TRKCR_ADD(sl, t);
    const double e = TRKCR_FMA(fabs(t), 0x1p-49, TRKCR_MUL(fabs(L), 0x1p-52));
    const double u = TRKCR_ADD(sh, TRKCR_ADD(L, e)), v = TRKCR_ADD(sh, TRKCR_SUB(L, e));
    if (u == v)
      return u;
  }
  return trkcr_exp_slow(x);
}

/* a / b for a double-double a and a double b: the quotient of the high
 * parts and one correction from the exact remainder */
TRKCR_FN trkcr_dd trkcr_div_d(trkcr_dd a, double b) {
  const double q1 = TRKCR_DIV(a.hi, b);
  const trkcr_dd p = trkcr_two_prod(q1, b);
  const double r = TRKCR_ADD(TRKCR_SUB(TRKCR_SUB(a.hi, p.hi), p.lo), a.lo);
  return trkcr_two_sum(q1, TRKCR_DIV(r, b));
}

/* 1 / b for a double-double b, in the same way */
TRKCR_FN trkcr_dd trkcr_recip_dd(trkcr_dd b) {
  const double q1 = TRKCR_DIV(1.0, b.hi);
  trkcr_dd p = trkcr_two_prod(q1, b.hi);
  p.lo = TRKCR_FMA(q1, b.lo, p.lo);
  const trkcr_dd r = trkcr_add(trkcr_make(1.0, 0.0), trkcr_make(-p.hi, -p.lo));
  return trkcr_two_sum(q1, TRKCR_DIV(r.hi, b.hi));
}

/* sinh and cosh of |x| in double-double: the Taylor series below 1/8 (its
 * terms fall by (1/8)^2 / 6 at least, so ten reach 2^-110 of the sum and
 * nothing cancels), (e^|x| -/+ e^-|x|)/2 above */
TRKCR_FN trkcr_dd trkcr_sinh_dd(double ax) {
  if (ax < 0.125) {
    const trkcr_dd x2 = trkcr_two_prod(ax, ax);
    trkcr_dd term = trkcr_make(ax, 0.0), sum = term;
    for (int k = 1; k <= 10; k++) {
      term = trkcr_div_d(trkcr_mul(term, x2), (double)((2 * k) * (2 * k + 1)));
      sum = trkcr_add(sum, term);
    }
    return sum;
  }
  const trkcr_dd E = trkcr_exp_dd(ax), iE = trkcr_recip_dd(E);
  const trkcr_dd d = trkcr_add(E, trkcr_neg(iE));
  return trkcr_make(TRKCR_MUL(d.hi, 0.5), TRKCR_MUL(d.lo, 0.5));
}

TRKCR_FN trkcr_dd trkcr_cosh_dd(double ax) {
  if (ax < 0.125) {
    const trkcr_dd x2 = trkcr_two_prod(ax, ax);
    trkcr_dd term = trkcr_make(1.0, 0.0), sum = term;
    for (int k = 1; k <= 10; k++) {
      term = trkcr_div_d(trkcr_mul(term, x2), (double)((2 * k - 1) * (2 * k)));
      sum = trkcr_add(sum, term);
    }
    return sum;
  }
  const trkcr_dd E = trkcr_exp_dd(ax), iE = trkcr_recip_dd(E);
  const trkcr_dd d = trkcr_add(E, iE);
  return trkcr_make(TRKCR_MUL(d.hi, 0.5), TRKCR_MUL(d.lo, 0.5));
}

/* sinh, cosh rounded once from the double-double values (bend fringes
 * only: not inlined); beyond |x| = 700 and for non-finite x, the library's */
TRKCR_SLOW double trkcr_sinh(double x) {
  if (x == 0.0 || !(fabs(x) <= 700.0))
    return TRKCR_SINH(x);
  const trkcr_dd v = trkcr_sinh_dd(fabs(x));
  const double r = TRKCR_ADD(v.hi, v.lo);
  return x < 0 ? -r : r;
}

TRKCR_SLOW double trkcr_cosh(double x) {
  if (x == 0.0)
    return 1.0;
  if (!(fabs(x) <= 700.0))
    return TRKCR_COSH(x);
  const trkcr_dd v = trkcr_cosh_dd(fabs(x));
  return TRKCR_ADD(v.hi, v.lo);
}

/*
 * RN(a/b) from y = RN(1/b), the correctly rounded reciprocal of b (formed
 * once for a divisor used many times): q0 = RN(a y) is within 1.5 ulp of
 * a/b; one FMA correction q1 = RN(q0 + (a - b q0) y) leaves it within an
 * ulp (its error is ~(2u)^2 relative plus the final rounding); a second,
 * q2 = RN(q1 + (a - b q1) y), with the residual exact because q1 is
 * faithful, is RN(a/b) by Markstein's theorem (P. Markstein, IBM J. Res.
 * Dev. 34 (1990) 111; the basis of FMA division on IA-64).  The theorem
 * assumes no underflow or overflow in the intermediates: quotients outside
 * [2^-958, 2^960) in magnitude (and zeros, infinities, NaNs) take the IEEE
 * division, so signed zeros and special values are the IEEE ones.
 */
TRKCR_FN double trkcr_div_rcp(double a, double b, double y) {
  const double q0 = TRKCR_MUL(a, y);
  const double q1 = TRKCR_FMA(TRKCR_FMA(-b, q0, a), y, q0);
  const double q2 = TRKCR_FMA(TRKCR_FMA(-b, q1, a), y, q1);
  const unsigned e = (TRKCR_HIWORD(q0) >> 20) & 0x7ffu;
  return (e - 65u < 1918u) ? q2 : TRKCR_DIV(a, b);
}

#endif
