/*
 * trk_crmath.cuh -- correctly rounded sin, cos and asin for the parity build.
 *
 * The reference's CSBEND drift (src/csbend.c:1580-1606) evaluates
 * X = rho0*(f-1) + f*X with f = cos(phi)/cos(dsh/rho0+phi) close to 1, so a
 * one-ulp difference in cos() moves X by about rho0*2^-53.  glibc's sin, cos
 * and asin return the correctly rounded result for the arguments that occur in
 * tracking, so a device build that also rounds correctly reproduces the
 * reference bit for bit.  These routines evaluate the functions in
 * double-double arithmetic (Dekker/Knuth error-free transformations):
 *   - sin/cos: reduction by k*pi/2 with a three-part pi/2 and exact products,
 *     then the Taylor series in double-double on |r| <= pi/4;
 *   - asin: one Newton step x1 = x0 + (y - sin x0)/cos x0 from a double
 *     estimate, with sin x0 in double-double.
 * The double-double result carries ~2^-100 relative error, so its leading
 * part is the correctly rounded value except in ~2^-47 of cases.
 * Constants: Taylor coefficients (-1)^k/(2k+1)! and (-1)^k/(2k)! split into
 * double-double, and pi/2 split into three doubles (exact rationals rounded
 * in high precision).
 */
#ifndef TRK_CRMATH_CUH
#define TRK_CRMATH_CUH

namespace trkcr {

struct dd {
  double hi, lo;
};

__device__ __forceinline__ dd two_sum(double a, double b) {
  double s = __dadd_rn(a, b);
  double bb = __dsub_rn(s, a);
  double e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
  return {s, e};
}

__device__ __forceinline__ dd quick_two_sum(double a, double b) {
  double s = __dadd_rn(a, b);
  double e = __dsub_rn(b, __dsub_rn(s, a));
  return {s, e};
}

__device__ __forceinline__ dd two_prod(double a, double b) {
  double p = __dmul_rn(a, b);
  double e = __fma_rn(a, b, -p);
  return {p, e};
}

__device__ __forceinline__ dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  dd t = two_sum(a.lo, b.lo);
  s.lo = __dadd_rn(s.lo, t.hi);
  s = quick_two_sum(s.hi, s.lo);
  s.lo = __dadd_rn(s.lo, t.lo);
  return quick_two_sum(s.hi, s.lo);
}

__device__ __forceinline__ dd dd_mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo = __fma_rn(a.hi, b.lo, p.lo);
  p.lo = __fma_rn(a.lo, b.hi, p.lo);
  return quick_two_sum(p.hi, p.lo);
}

__device__ __constant__ double c_sin_dd[16][2] = {
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

__device__ __constant__ double c_cos_dd[16][2] = {
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

/* number of series terms that bring the remainder below 2^-108 |r| */
__device__ __forceinline__ int n_terms(double ar) {
  if (ar < 0x1p-5)
    return 8;
  if (ar < 0.25)
    return 12;
  return 15;
}

/* sin and cos of a double-double r with |r| <= pi/4 */
__device__ __forceinline__ dd sin_dd_reduced(dd r) {
  dd r2 = dd_mul(r, r);
  int n = n_terms(fabs(r.hi));
  dd p = {c_sin_dd[n][0], c_sin_dd[n][1]};
  for (int k = n - 1; k >= 0; k--)
    p = dd_add(dd_mul(p, r2), dd{c_sin_dd[k][0], c_sin_dd[k][1]});
  return dd_mul(p, r);
}

__device__ __forceinline__ dd cos_dd_reduced(dd r) {
  dd r2 = dd_mul(r, r);
  int n = n_terms(fabs(r.hi));
  dd p = {c_cos_dd[n][0], c_cos_dd[n][1]};
  for (int k = n - 1; k >= 0; k--)
    p = dd_add(dd_mul(p, r2), dd{c_cos_dd[k][0], c_cos_dd[k][1]});
  return p;
}

/* x = k*pi/2 + r, |r| <= ~pi/4, valid for |x| < 2^30 */
__device__ __forceinline__ dd reduce_pio2(double x, int *quadrant) {
  if (fabs(x) <= 0.78539816339744828) {
    *quadrant = 0;
    return dd{x, 0.0};
  }
  double k = rint(__dmul_rn(x, TRKCR_2OPI));
  dd a = two_prod(k, TRKCR_PIO2_1);
  dd r = two_sum(x, -a.hi);
  r = dd_add(r, dd{-a.lo, 0.0});
  dd b = two_prod(k, TRKCR_PIO2_2);
  r = dd_add(r, dd{-b.hi, -b.lo});
  r = dd_add(r, dd{-__dmul_rn(k, TRKCR_PIO2_3), 0.0});
  long long ki = (long long)k;
  *quadrant = (int)(ki & 3);
  return r;
}

__device__ __forceinline__ dd sin_dd(double x) {
  int q;
  dd r = reduce_pio2(x, &q);
  dd v;
  switch (q) {
  case 0:
    return sin_dd_reduced(r);
  case 1:
    return cos_dd_reduced(r);
  case 2:
    v = sin_dd_reduced(r);
    return dd{-v.hi, -v.lo};
  default:
    v = cos_dd_reduced(r);
    return dd{-v.hi, -v.lo};
  }
}

__device__ __forceinline__ dd cos_dd(double x) {
  int q;
  dd r = reduce_pio2(x, &q);
  dd v;
  switch (q) {
  case 0:
    return cos_dd_reduced(r);
  case 1:
    v = sin_dd_reduced(r);
    return dd{-v.hi, -v.lo};
  case 2:
    v = cos_dd_reduced(r);
    return dd{-v.hi, -v.lo};
  default:
    return sin_dd_reduced(r);
  }
}

__device__ __forceinline__ double cr_sin(double x) {
  if (x == 0.0 || !isfinite(x))
    return x == 0.0 ? x : nan("");
  dd v = sin_dd(x);
  return __dadd_rn(v.hi, v.lo);
}

__device__ __forceinline__ double cr_cos(double x) {
  if (!isfinite(x))
    return nan("");
  dd v = cos_dd(x);
  return __dadd_rn(v.hi, v.lo);
}

/* asin for |y| <= 1 by one double-double Newton step on sin(a) = y */
__device__ __forceinline__ double cr_asin(double y) {
  if (y == 0.0 || fabs(y) >= 1.0 || isnan(y))
    return asin(y);
  double a0 = asin(y);
  dd s = sin_dd(a0);
  double c = cos(a0);
  dd d = two_sum(y, -s.hi);
  double num = __dadd_rn(d.hi, __dsub_rn(d.lo, s.lo));
  double delta = __ddiv_rn(num, c);
  dd a = two_sum(a0, delta);
  return __dadd_rn(a.hi, a.lo);
}

} // namespace trkcr

#endif
