/*
 * trk_kernels.cu -- particle-tracking kernels for sm_100a.
 *
 * Compiled twice into libtrkgpu.so:
 *   TRK_FAST=0 (namespace trk_exact, -fmad=false): the reference's operation
 *     order, no FMA contraction, correctly rounded sin/cos/asin; reproduces
 *     elegant's CPU results bit for bit on the tracking path.
 *   TRK_FAST=1 (namespace trk_fast): FMA contraction, reciprocal multiplies
 *     and a transcendental-free CSBEND drift; same physics, error comparable
 *     to the reference's own FP64 rounding.
 *
 * Layout: the beam is a structure of arrays (x, x', y, y', s, delta) in FP64
 * plus int32 loss pass / loss element; one thread owns one particle and keeps
 * its six coordinates in registers across a whole fused segment of elements
 * (and across passes when no collective element intervenes).  Element
 * records (trk_op) are read with warp-uniform loads through the read-only
 * path.  FP64 throughout: long-term symplectic tracking and the loss
 * boundaries need it, and no dense contraction exists for the tensor cores.
 */
#include <cuda_runtime.h>
#include <stddef.h>

#include <algorithm>
#include <stdint.h>

#include "trk_constants.h"
#include "trk_crmath.h"
#include "trk_philox.h"

#include <cfloat>

#include "trk_kernels.h"
#include "trk_ops.h"

#ifndef TRK_FAST
#error "TRK_FAST must be defined to 0 or 1"
#endif

#if TRK_FAST
#define TRK_NS trk_fast
#define M_SIN(x) sin(x)
#define M_COS(x) cos(x)
#define M_ASIN(x) asin(x)
#define M_TAN(x) tan(x)
#define M_SINCOS(x, s, c) sincos((x), (s), (c))
#define M_EXP(x) exp(x)
#define M_SINH(x) sinh(x)
#define M_COSH(x) cosh(x)
#else
#define TRK_NS trk_exact
#define M_SIN(x) trkcr_sin(x)
#define M_COS(x) trkcr_cos(x)
#define M_ASIN(x) trkcr_asin(x)
#define M_TAN(x) trkcr_tan(x)
#define M_SINCOS(x, s, c) trkcr_sincos((x), (s), (c))
#define M_EXP(x) trkcr_exp(x)
#define M_SINH(x) trkcr_sinh(x)
#define M_COSH(x) trkcr_cosh(x)
#endif

namespace TRK_NS {

struct Part {
  double x, xp, y, yp, s, dp;
};

__device__ __forceinline__ double sqr(double v) { return v * v; }

#if TRK_FAST
/* Reciprocal and square root for the fast build: the hardware approximation
 * y0 (about 20 correct bits) and one third-order correction from the series
 *   1/x       = y0 / (1 - e)       = y0 (1 + e + e^2 + ...),   e = 1 - x y0
 *   1/sqrt(x) = y0 (1 + r)^(-1/2)  = y0 (1 - r/2 + 3 r^2/8 - ...),  r = x y0^2 - 1
 * truncated after the quadratic term (remainder ~e^3, r^3 ~ 2^-60), and
 * sqrt(x) = (x y0)(1 + r)^(-1/2) with r formed from the rounded product
 * x y0, so its rounding cancels to first order.  Results agree with IEEE
 * 1/x and sqrt(x) to within an ulp.  There are no special-value paths:
 * callers pass positive normal arguments, except that sqrt_fast returns 0
 * for x <= 0 (as the reference's conditions need) and sqrt_nan returns NaN
 * for x <= 0. */
__device__ __forceinline__ double rcp_fast(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x, y, 1.0);
  return fma(y, fma(e, e, e), y);
}

__device__ __forceinline__ double rsqrt_fast(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double r = fma(x * y, y, -1.0);
  return fma(y * r, fma(0.375, r, -0.5), y);
}

__device__ __forceinline__ double sqrt_nan(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double s = x * y;
  const double r = fma(s, y, -1.0);
  return fma(s * r, fma(0.375, r, -0.5), s);
}

/* a / x with the reciprocal's correction applied to the quotient:
 * a y0 (1 + e + e^2), e = 1 - x y0 (one dependent step shorter than
 * a * rcp_fast(x)); NaN for x = 0. */
__device__ __forceinline__ double div_fast(double a, double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double q = a * y;
  const double e = fma(-x, y, 1.0);
  return fma(q, fma(e, e, e), q);
}

__device__ __forceinline__ double sqrt_fast(double x) { return x > 0 ? sqrt_nan(x) : 0.0; }

#endif

__device__ __forceinline__ double ipow_d(double x, int p) {
  if (p == 2)
    return x * x;
  if (p == 0)
    return 1.0;
  if (p == 1)
    return x;
  /* repeated squaring; exponent 2 is the only one on the tracking path */
  double h = 1.0, b = x;
  for (int e = p < 0 ? -p : p; e; e >>= 1) {
    if (e & 1)
      h = h * b;
    b = b * b;
  }
  return p < 0 ? 1.0 / h : h;
}

__device__ __forceinline__ void exact_drift(Part &p, double L) {
  p.x += p.xp * L;
  p.y += p.yp * L;
  p.s += L * sqrt(1 + sqr(p.xp) + sqr(p.yp));
}

/* rotateBeamCoordinatesForMisalignment with precomputed cos/sin
 * (src/tilt_matrices.c:156-190) */
__device__ __forceinline__ void rotate(Part &p, double ca, double sa) {
  double x = p.x, xp = p.xp, y = p.y, yp = p.yp;
  p.x = x * ca + y * sa;
  p.y = -x * sa + y * ca;
  p.xp = xp * ca + yp * sa;
  p.yp = -xp * sa + yp * ca;
}

/* offsetBeamCoordinatesForMisalignment (src/malign_mat.c:257-267) */
__device__ __forceinline__ void offset(Part &p, double dx, double dy, double dz) {
  p.s += dz * sqrt(1 + sqr(p.xp) + sqr(p.yp));
  p.x = p.x - dx + dz * p.xp;
  p.y = p.y - dy + dz * p.yp;
}

/* checkMultAperture (src/multipole.c:1751-1798) without aperture files */
__device__ __forceinline__ bool check_aperture(double x, double y, const trk_aperture *ap, bool tilt, double rc,
                                               double rs) {
  if (!ap)
    return true;
  x = x - 0.0;
  y = y - 0.0;
  if (tilt) {
    double x0 = x, y0 = y;
    x = x0 * rc + y0 * rs;
    y = -x0 * rs + y0 * rc;
  }
  double xMax = ap->x_max, yMax = ap->y_max;
  if (ap->elliptical == 0 || xMax <= 0 || yMax <= 0) {
    if ((xMax > 0 && fabs(x) > xMax) || (yMax > 0 && fabs(y) > yMax))
      return false;
  } else {
    double xa = x / xMax, yb = y / yMax;
    if (ipow_d(xa, ap->xexp) + ipow_d(yb, ap->yexp) >= 1)
      return false;
  }
  return true;
}

/* ------------------------------------------------------------- multipoles */
__device__ __forceinline__ bool momenta_to_slopes(double &xp, double &yp, double qx, double qy, double delta,
                                                  int expand) {
  if (expand) {
    xp = qx / (1 + delta);
    yp = qy / (1 + delta);
    return true;
  }
  double denom = sqr(1 + delta) - sqr(qx) - sqr(qy);
  if (denom <= 0)
    return false;
#if TRK_FAST
  const double inv = rsqrt_fast(denom);
  xp = qx * inv;
  yp = qy * inv;
#else
  denom = sqrt(denom);
  xp = qx / denom;
  yp = qy / denom;
#endif
  return true;
}

/* apply_canonical_multipole_kicks_ret (src/multipole.h:391-421) for the
 * orders on this path, with the reference's term order and coefficients
 * (src/multipole.h:76-146). */
__device__ __forceinline__ void mkick(double &qx, double &qy, double x, double y, int order, double K, int skew,
                                      const double *coef, double *dqx = nullptr, double *dqy = nullptr) {
  double sFx, sFy;
  switch (order) {
  case 0:
    sFy = 1.0;
    sFx = 0.0;
    break;
  case 1:
    sFy = x;
    sFx = y;
    break;
  case 2: {
    double x2 = x * x, y2 = y * y;
    sFy = 0.5 * x2 + (-0.5) * y2;
    sFx = x * y;
    break;
  }
  case 3: {
    double x2 = x * x, y2 = y * y;
    double x3 = x2 * x, y3 = y2 * y;
    double f0 = coef[6] * x3;
    double f1 = (coef[7] * x2) * y;
    double f2 = (coef[8] * x) * y2;
    double f3 = coef[9] * y3;
    sFy = f0 + f2;
    sFx = f1 + f3;
    break;
  }
  default:
    sFy = sFx = 0.0;
  }
  if (skew) {
    double t = sFx;
    sFx = -sFy;
    sFy = t;
  }
  qx -= K * sFy;
  qy += K * sFx;
  if (dqx) { /* the kick returned for the radiation field (src/multipole.h:416-419) */
    *dqx -= K * sFy;
    *dqy += K * sFx;
  }
}

__device__ __constant__ double c_coef[10]; /* expansion coefficients, orders 0..3 at n(n+1)/2 */

#if TRK_FAST
/* Fast-build body of integrate_kick_multipole_ordn for one normal multipole
 * of order ORDER with the 4th-order integrator and no steering kicks: the
 * four substeps are unrolled, (1+delta)^2 is hoisted and the slope
 * conversion uses one reciprocal square root.  Returns 0 if the particle
 * survives the body, 1 for an aperture loss (x, y at the loss point are
 * reported), 2 for undefined slopes; `done` counts completed drift substeps. */
template <int ORDER>
__device__ __forceinline__ int mult_body_fast(const double *__restrict__ d, int n_parts, const trk_aperture *ap,
                                              bool aptilt, double apc, double aps, double mdx, double mdy, double &x,
                                              double &xp, double &y, double &yp, double &s, double &qx, double &qy,
                                              const double dp, int &done) {
  const double opd2 = (1 + dp) * (1 + dp);
  /* path-length factor sqrt(1 + xp^2 + yp^2): once from the entry slopes,
   * then (1+delta) / sqrt((1+delta)^2 - qx^2 - qy^2) from each slope update,
   * which is the same quantity without another square root */
  double sf = sqrt_fast(fma(yp, yp, fma(xp, xp, 1.0)));
  done = 0;
  for (int i_kick = 0; i_kick < n_parts; i_kick++) {
    if (ap && !check_aperture(x + mdx, y + mdy, ap, aptilt, apc, aps))
      return 1;
#pragma unroll
    for (int step = 0; step < 4; step++) {
      const double dsh = __ldg(&d[MD_DSH + step]);
      x = fma(xp, dsh, x);
      y = fma(yp, dsh, y);
      s = fma(dsh, sf, s);
      done++;
      if (step == 3)
        break;
      const double K = __ldg(&d[MD_KQ + step * 3]);
      if (ORDER == 1) {
        qx = fma(-K, x, qx);
        qy = fma(K, y, qy);
      } else if (ORDER == 2) {
        qx = fma(-K, 0.5 * (x * x - y * y), qx);
        qy = fma(K, x * y, qy);
      } else {
        const double x2 = x * x, y2 = y * y;
        qx = fma(-K, (x2 * x - 3 * x * y2) * (1.0 / 6), qx);
        qy = fma(K, (3 * x2 * y - y2 * y) * (1.0 / 6), qy);
      }
      const double den = opd2 - qx * qx - qy * qy;
      if (!(den > 0))
        return 2;
      const double r = rsqrt_fast(den);
      xp = qx * r;
      yp = qy * r;
      sf = (1 + dp) * r;
    }
  }
  if (ap && !check_aperture(x + mdx, y + mdy, ap, aptilt, apc, aps))
    return 1;
  return 0;
}
#endif

/* what an incoherent-radiation deviate is keyed by: the run's seed, the
 * particle ID, the pass and the element (op index); `single`: one particle
 * is tracked (ISR1PART=0 then turns ISR off, src/multipole.c:758) */
struct IsrKey {
  unsigned long long seed;
  unsigned int id, pass, elem;
  double limit;
  bool single;
};

/* quadFringe (src/fringe.c:25-219) on one particle: slopes to momenta, the
 * first linear part, the nonlinear generator of order |higherOrder| (2:
 * leading, 3: higher), the second linear part, the path-length change,
 * momenta back to slopes; `fr` holds the edge's M1, M2, nonlinear factor,
 * higherOrder and linear flag (compile_mult), each expression in the
 * reference's operation order. */
__device__ __noinline__ void quad_fringe(Part &p, const double *__restrict__ fr, double K1, int inFringe) {
  const double nonlinearFactor = __ldg(&fr[16]);
  const int higherOrder = (int)__ldg(&fr[17]);
  const bool linear = __ldg(&fr[18]) != 0;
  const double delta = p.dp;
  double x, px, y, py, v1, v3, a, dx = 0, dpx = 0, dy = 0, dpy = 0, ds = 0;
  {
    const double xp = p.xp, yp = p.yp;
    const double denom = sqrt(1 + sqr(xp) + sqr(yp));
    v1 = (1 + delta) * xp / denom;
    v3 = (1 + delta) * yp / denom;
  }
  if (linear) {
    x = __ldg(&fr[0]) * p.x + __ldg(&fr[1]) * v1;
    px = __ldg(&fr[2]) * p.x + __ldg(&fr[3]) * v1;
    y = __ldg(&fr[4]) * p.y + __ldg(&fr[5]) * v3;
    py = __ldg(&fr[6]) * p.y + __ldg(&fr[7]) * v3;
  } else {
    x = p.x;
    px = v1;
    y = p.y;
    py = v3;
  }
  a = -inFringe * K1 / (12 * (1 + delta));
  const int ho = higherOrder < 0 ? -higherOrder : higherOrder;
  if (ho > 1) {
    double xpow[9], ypow[9];
    xpow[0] = ypow[0] = 1;
    if (ho > 2) {
      double apow[4];
      apow[0] = 1;
#pragma unroll
      for (int i = 1; i < 9; i++) {
        xpow[i] = xpow[i - 1] * x;
        ypow[i] = ypow[i - 1] * y;
      }
#pragma unroll
      for (int i = 1; i < 4; i++)
        apow[i] = apow[i - 1] * a;
      dpx = (a * (12 * a * (-4 * py * x * y + px * (xpow[2] - 5 * ypow[2])) * (xpow[2] - ypow[2]) -
                  24 * (-2 * py * x * y + px * (xpow[2] + ypow[2])) +
                  4 * apow[2] *
                    (-2 * py * x * y * (3 * xpow[4] + 50 * xpow[2] * ypow[2] - 21 * ypow[4]) +
                     px * (xpow[6] + 75 * xpow[4] * ypow[2] - 105 * xpow[2] * ypow[4] - 35 * ypow[6])) +
                  3 * apow[3] *
                    (-8 * py * x * y * (xpow[6] - 27 * xpow[4] * ypow[2] + 83 * xpow[2] * ypow[4] + 7 * ypow[6]) +
                     px * (xpow[8] - 108 * xpow[6] * ypow[2] + 830 * xpow[4] * ypow[4] + 196 * xpow[2] * ypow[6] +
                           105 * ypow[8])))) /
            8;
      dpy = (a * (-8 * px * x * y *
                    (6 - 6 * a * (xpow[2] - ypow[2]) + apow[2] * (21 * xpow[4] - 50 * xpow[2] * ypow[2] - 3 * ypow[4]) +
                     3 * apow[3] * (7 * xpow[6] + 83 * xpow[4] * ypow[2] - 27 * xpow[2] * ypow[4] + ypow[6])) +
                  py * (315 * apow[3] * xpow[8] + 28 * apow[2] * xpow[6] * (5 + 21 * a * ypow[2]) +
                        30 * a * xpow[4] * (2 + 14 * a * ypow[2] + 83 * apow[2] * ypow[4]) +
                        ypow[2] * (24 + 12 * a * ypow[2] - 4 * apow[2] * ypow[4] + 3 * apow[3] * ypow[6]) -
                        12 * xpow[2] * (-2 + 6 * a * ypow[2] + 25 * apow[2] * ypow[4] + 27 * apow[3] * ypow[6])))) /
            8;
      if (higherOrder > 0) {
        dx = (a * x *
              (8 * (xpow[2] + 3 * ypow[2]) +
               4 * apow[2] * (5 * xpow[6] + 21 * xpow[4] * ypow[2] - 25 * xpow[2] * ypow[4] - ypow[6]) +
               apow[3] * (35 * xpow[8] + 84 * xpow[6] * ypow[2] + 498 * xpow[4] * ypow[4] - 108 * xpow[2] * ypow[6] +
                          3 * ypow[8]) +
               12 * a * sqr(xpow[2] - ypow[2]))) /
             8;
        dy = (a * y *
              (-8 * (3 * xpow[2] + ypow[2]) +
               4 * apow[2] * (xpow[6] + 25 * xpow[4] * ypow[2] - 21 * xpow[2] * ypow[4] - 5 * ypow[6]) +
               apow[3] * (3 * xpow[8] - 108 * xpow[6] * ypow[2] + 498 * xpow[4] * ypow[4] + 84 * xpow[2] * ypow[6] +
                          35 * ypow[8]) +
               12 * a * sqr(xpow[2] - ypow[2]))) /
             8;
      }
    } else {
#pragma unroll
      for (int i = 1; i < 4; i++) {
        xpow[i] = xpow[i - 1] * x;
        ypow[i] = ypow[i - 1] * y;
      }
      dpx = 3 * a * (-px * xpow[2] + 2 * py * x * y - px * ypow[2]);
      dpy = 3 * a * (py * xpow[2] - 2 * px * x * y + py * ypow[2]);
      if (higherOrder > 0) {
        dx = a * (xpow[3] + 3 * x * ypow[2]);
        dy = a * (-3 * xpow[2] * y - ypow[3]);
      }
    }
    ds = (a / (1 + delta)) * (3 * py * y * xpow[2] - px * xpow[3] - 3 * px * x * ypow[2] + py * ypow[3]);
  }
  x += nonlinearFactor * dx;
  px += nonlinearFactor * dpx;
  y += nonlinearFactor * dy;
  py += nonlinearFactor * dpy;
  if (linear) {
    p.x = __ldg(&fr[8]) * x + __ldg(&fr[9]) * px;
    v1 = __ldg(&fr[10]) * x + __ldg(&fr[11]) * px;
    p.y = __ldg(&fr[12]) * y + __ldg(&fr[13]) * py;
    v3 = __ldg(&fr[14]) * y + __ldg(&fr[15]) * py;
  } else {
    p.x = x;
    v1 = px;
    p.y = y;
    v3 = py;
  }
  p.s -= nonlinearFactor * ds;
  double denom = sqr(1 + delta) - sqr(v1) - sqr(v3);
  if (denom > 0) {
    denom = sqrt(denom);
    p.xp = v1 / denom;
    p.yp = v3 / denom;
  } else
    p.xp = p.yp = DBL_MAX;
}

/* multipole_tracking2 + integrate_kick_multipole_ordn (src/multipole.c:660-1456) */
__device__ __forceinline__ bool op_mult(const trk_op *__restrict__ op, Part &p, double Po, double z_start,
                                        const trk_aperture *ap, const IsrKey *isr = nullptr) {
  const int n_parts = __ldg(&op->i[0]);
  const int nSub = __ldg(&op->i[1]);
  const int expand = __ldg(&op->i[2]);
  const int orders = __ldg(&op->i[4]);
  const int skews = __ldg(&op->i[5]);
  const int flags = __ldg(&op->i[6]);
  const double *d = op->d;
  const double mdx = __ldg(&d[MD_DX]), mdy = __ldg(&d[MD_DY]), mdz = __ldg(&d[MD_DZ]);

  if (flags & MF_OFFSET)
    offset(p, mdx, mdy, mdz);
  if (flags & MF_TILT)
    rotate(p, __ldg(&d[MD_TC]), __ldg(&d[MD_TS]));
  if (flags & MF_ENDDRIFT)
    exact_drift(p, __ldg(&d[MD_LEND]));
  if (flags & MF_FRINGE1) /* KQUAD entrance fringe (src/multipole.c:999-1006) */
    quad_fringe(p, d + MD_FR1, __ldg(&d[MD_FRK1]), -1);

  bool ok = true;
  double dzLoss = 0;
  {
    double x = p.x, xp = p.xp, y = p.y, yp = p.yp, s = 0, dp = p.dp, qx, qy;
    const bool aptilt = (flags & MF_APTILT) != 0;
    const double apc = __ldg(&d[MD_APC]), aps = __ldg(&d[MD_APS]);
    const double drift = __ldg(&d[MD_DRIFT]);
    if (isnan(x) || isnan(xp) || isnan(y) || isnan(yp) || fabs(x) > TRK_COORD_LIMIT || fabs(y) > TRK_COORD_LIMIT ||
        fabs(xp) > TRK_SLOPE_LIMIT || fabs(yp) > TRK_SLOPE_LIMIT) {
      /* the reference records the previous particle's dzLoss here; taken
       * as that of a particle that went through (MD_DZFULL) */
      dzLoss = __ldg(&d[MD_DZFULL]);
      ok = false;
      goto done;
    }
    if (expand) {
      qx = (1 + dp) * xp;
      qy = (1 + dp) * yp;
    } else {
#if TRK_FAST
      const double r = (1 + dp) * rsqrt_fast(1 + sqr(xp) + sqr(yp));
      qx = xp * r;
      qy = yp * r;
#else
      double denom = sqrt(1 + sqr(xp) + sqr(yp));
      qx = (1 + dp) * xp / denom;
      qy = (1 + dp) * yp / denom;
#endif
    }
    if (!momenta_to_slopes(xp, yp, qx, qy, dp, expand)) {
      ok = false;
      goto done;
    }
#if TRK_FAST
    if (nSub == 4 && !expand && drift != 0 && (orders & 0xff) >= 1 && (orders & 0xff) <= 3 && !(skews & 1) &&
        !(flags & (MF_KNL1 | MF_KNL2 | MF_XKICK | MF_YKICK | MF_RAD))) {
      int done = 0, rc;
      const int o = orders & 0xff;
      if (o == 1)
        rc = mult_body_fast<1>(d, n_parts, ap, aptilt, apc, aps, mdx, mdy, x, xp, y, yp, s, qx, qy, dp, done);
      else if (o == 2)
        rc = mult_body_fast<2>(d, n_parts, ap, aptilt, apc, aps, mdx, mdy, x, xp, y, yp, s, qx, qy, dp, done);
      else
        rc = mult_body_fast<3>(d, n_parts, ap, aptilt, apc, aps, mdx, mdy, x, xp, y, yp, s, qx, qy, dp, done);
      for (int k = 0; k < done; k++)
        dzLoss += __ldg(&d[MD_DSH + (k & 3)]);
      if (rc) {
        if (rc == 1) {
          p.x = x;
          p.y = y;
        }
        ok = false;
        goto done;
      }
      goto body_done;
    }
#endif
    for (int i_kick = 0; i_kick < n_parts; i_kick++) {
      if (!check_aperture(x + mdx, y + mdy, ap, aptilt, apc, aps)) {
        p.x = x;
        p.y = y;
        ok = false;
        goto done;
      }
      for (int step = 0; step < nSub; step++) {
        if (drift != 0) {
          double dsh = __ldg(&d[MD_DSH + step]);
          x += xp * dsh;
          y += yp * dsh;
          if (expand)
            s += dsh * (1 + (sqr(xp) + sqr(yp)) / 2);
          else
#if TRK_FAST
            s += dsh * sqrt_fast(1 + sqr(xp) + sqr(yp));
#else
            s += dsh * sqrt(1 + sqr(xp) + sqr(yp));
#endif
          dzLoss += dsh;
        }
        if (step == nSub - 1)
          break; /* kickFrac of the last substep is 0 for orders 2, 4, 6 */
        double dqx = 0, dqy = 0;
        const bool rad = (flags & MF_RAD) != 0;
        if (flags & MF_KNL0)
          mkick(qx, qy, x, y, orders & 0xff, __ldg(&d[MD_KQ + step * 3 + 0]), skews & 1, c_coef, rad ? &dqx : nullptr,
                &dqy);
        if (flags & MF_KNL1)
          mkick(qx, qy, x, y, (orders >> 8) & 0xff, __ldg(&d[MD_KQ + step * 3 + 1]), (skews >> 1) & 1, c_coef,
                rad ? &dqx : nullptr, &dqy);
        if (flags & MF_KNL2)
          mkick(qx, qy, x, y, (orders >> 16) & 0xff, __ldg(&d[MD_KQ + step * 3 + 2]), (skews >> 2) & 1, c_coef,
                rad ? &dqx : nullptr, &dqy);
        if (flags & MF_XKICK)
          mkick(qx, qy, x, y, 0, __ldg(&d[MD_KX + step]), 0, c_coef);
        if (flags & MF_YKICK)
          mkick(qx, qy, x, y, 0, __ldg(&d[MD_KY + step]), 1, c_coef);
        if (!momenta_to_slopes(xp, yp, qx, qy, dp, expand)) {
          ok = false;
          goto done;
        }
        if (rad && drift != 0) {
          /* classical radiation after the kick (src/multipole.c:1359-1389):
           * the field from the returned kick, dp -= rad_coef (1+dp)^2 F^2 ds */
          qx /= (1 + dp);
          qy /= (1 + dp);
          const double deltaFactor = sqr(1 + dp);
          const double kfs = __ldg(&d[MD_KFRAC + step]);
          dqx /= kfs;
          dqy /= kfs;
          const double xkr = __ldg(&d[MD_XKR]), ykr = __ldg(&d[MD_YKR]);
          const double F2 = sqr(dqx / drift - xkr / drift) + sqr(dqy / drift + ykr / drift);
          double dsFactor = sqrt(1 + sqr(xp) + sqr(yp));
          const double dsISRFactor = dsFactor * drift / (nSub - 1);
          dsFactor *= drift * kfs;
          const double rad_coef = __ldg(&d[MD_RAD]);
          if (rad_coef != 0)
            dp -= rad_coef * deltaFactor * F2 * dsFactor;
          if ((flags & MF_ISR) && isr && !(isr->single && (flags & MF_ISR1OFF))) {
            /* quantum excitation (src/multipole.c:1380-1381) */
            const double g = trk_isr_gauss(isr->seed, isr->id, isr->pass, isr->elem, (unsigned)(i_kick * 8 + step),
                                           isr->limit);
            dp -= __ldg(&d[MD_ISR]) * deltaFactor * pow(F2, 0.75) * sqrt(dsISRFactor) * g;
          }
          qx *= (1 + dp);
          qy *= (1 + dp);
          if (!momenta_to_slopes(xp, yp, qx, qy, dp, expand)) {
            ok = false;
            goto done;
          }
          continue;
        }
#if !TRK_FAST
        /* the radiation block's (1 + dp) divide/multiply round trip, entered
         * for every kick with drift since isr_coef != 0 for Po > 0
         * (src/multipole.c:1359-1389, :757-760); it can move qx, qy by an
         * ulp.  The fast build leaves it out. */
        if (drift != 0) {
          qx /= (1 + dp);
          qy /= (1 + dp);
          qx *= (1 + dp);
          qy *= (1 + dp);
          if (!momenta_to_slopes(xp, yp, qx, qy, dp, expand)) {
            ok = false;
            goto done;
          }
        }
#endif
      }
    }
    if (!check_aperture(x + mdx, y + mdy, ap, aptilt, apc, aps)) {
      p.x = x;
      p.y = y;
      ok = false;
      goto done;
    }
#if TRK_FAST
  body_done:
#endif
    if (!momenta_to_slopes(xp, yp, qx, qy, dp, expand)) {
      ok = false;
      goto done;
    }
    p.x = x;
    p.xp = xp;
    p.y = y;
    p.yp = yp;
    if (__ldg(&d[MD_RAD]) != 0) {
      /* the path length rescaled to the new velocity (src/multipole.c:1437-1441) */
      const double p0 = Po * (1 + p.dp), p1 = Po * (1 + dp);
      const double beta0 = p0 / sqrt(sqr(p0) + 1), beta1 = p1 / sqrt(sqr(p1) + 1);
      p.s = beta1 * (p.s / beta0 + 2 * s / (beta0 + beta1));
    } else
      p.s += s;
    p.dp = dp;
    if (isnan(x) || isnan(xp) || isnan(y) || isnan(yp) || fabs(x) > TRK_COORD_LIMIT || fabs(y) > TRK_COORD_LIMIT ||
        fabs(xp) > TRK_SLOPE_LIMIT || fabs(yp) > TRK_SLOPE_LIMIT)
      ok = false;
  }
done:
  if (!ok) {
    p.s = z_start + dzLoss;
    p.dp = Po * (1 + p.dp);
  }
  /* KQUAD exit fringe, lost particles included as in the reference
   * (src/multipole.c:1054-1061 runs it over all n_part rows) */
  if (flags & MF_FRINGE2)
    quad_fringe(p, d + MD_FR2, __ldg(&d[MD_FRK1]), 1);
  if (flags & MF_ENDDRIFT)
    exact_drift(p, __ldg(&d[MD_LEND]));
  if (flags & MF_TILT)
    rotate(p, __ldg(&d[MD_XC]), __ldg(&d[MD_XS]));
  if (flags & MF_OFFSET)
    offset(p, -mdx, -mdy, -mdz);
  return ok;
}

/* ---------------------------------------------------------------- CSBEND */
#if !TRK_FAST
/* Body of a pure-dipole CSBEND in the parity build: integrate_csbend_ordn
 * (src/csbend.c:1561-1660) with Fx = 0, Fy = 1 and no radiation, every
 * operation rounded as the reference rounds it, with these shortcuts that
 * change no result:
 *  - 1 + delta is constant through the body, and so is f = sqrt((1+delta)^2
 *    - QY^2) while QY^2 rounds to the same double (QY moves only by the
 *    (1+delta) divide/multiply round trip, by an ulp at most): f and its
 *    reciprocal are re-formed only when QY^2 changes;
 *  - divisions by f, rho0, rho_actual and 1 + delta use their correctly
 *    rounded reciprocals, formed once (trkcr_div_rcp: Markstein's two FMA
 *    corrections give the IEEE quotient for five FP64 operations, about a
 *    third of an IEEE division's cost on B200);
 *  - the kick's Fx term, ((ds (1 + X/rho0)) 0)/rho_actual, is a signed zero
 *    (or NaN), formed by multiplying by 1/rho_actual instead of dividing;
 *  - dz_lost is summed only for a lost particle, from the substeps done.
 * Loss conditions, their order and the state left at a loss are the
 * reference's: aperture at the start of each slice, f <= 0, |QX/f| > 1 and
 * cos(dsh/rho0 + phi) == 0 before any coordinate of the substep changes. */
__device__ __forceinline__ bool bend_dipole_exact(const double *__restrict__ d, int nSlices, int nSub, double rho0,
                                                  bool roundtrip, const trk_aperture *ap, bool aptilt, double apc,
                                                  double aps, double &X, double &QX, double &Y, double &QY,
                                                  const double D, double &dist, int &done) {
  const double opd = __dadd_rn(1.0, D);
  const double opd2 = __dmul_rn(opd, opd);
  const double yopd = __drcp_rn(opd);
  const double yrho0 = __ldg(&d[BD_RHOINV]);
  const double rho_a = __ldg(&d[BD_RHOA]), yrho_a = __ldg(&d[BD_INVRHOA]);
  double qy2 = __dmul_rn(QY, QY);
  double f2 = __dsub_rn(opd2, qy2);
  double f = __dsqrt_rn(f2);
  double yf = __drcp_rn(f);
  done = 0;
  for (int i = 0; i < nSlices; i++) {
    if (!check_aperture(X, Y, ap, aptilt, apc, aps))
      return false;
    for (int j = 0; j < nSub; j++) {
      if (f2 <= 0)
        return false;
      const double sin_phi = trkcr_div_rcp(QX, f, yf);
      if (fabs(sin_phi) > 1)
        return false;
      const double phi = trkcr_asin(sin_phi);
      double sine, cosi;
      trkcr_sincos(__dadd_rn(__ldg(&d[BD_ARG + j]), phi), &sine, &cosi);
      if (cosi == 0)
        return false;
      const double tang = __ddiv_rn(sine, cosi);
      const double cos_phi = trkcr_cos(phi);
      QX = __dmul_rn(f, sine);
      const double a3 = trkcr_div_rcp(__dmul_rn(__dadd_rn(rho0, X), cos_phi), f, yf);
      const double factor = __dmul_rn(a3, __dsub_rn(tang, __ddiv_rn(sin_phi, cos_phi)));
      Y = __dadd_rn(Y, __dmul_rn(QY, factor));
      dist = __dadd_rn(dist, __dmul_rn(factor, opd));
      done++;
      const double fr = __ddiv_rn(cos_phi, cosi);
      X = __dadd_rn(__dmul_rn(rho0, __dsub_rn(fr, 1.0)), __dmul_rn(fr, X));
      if (j == nSub - 1)
        break;
      /* kick: QX += -ds (1 + X/rho0) Fy / rho_a, QY += ds (1 + X/rho0) Fx / rho_a */
      const double ds = __ldg(&d[BD_DS + j]);
      const double w = __dmul_rn(ds, __dadd_rn(1.0, trkcr_div_rcp(X, rho0, yrho0)));
      QX = __dadd_rn(QX, trkcr_div_rcp(-w, rho_a, yrho_a));
      QY = __dadd_rn(QY, __dmul_rn(__dmul_rn(w, 0.0), yrho_a));
      if (roundtrip) {
        /* QX /= (1 + delta); QY /= ...; QX *= (1 + delta); QY *= ... */
        QX = __dmul_rn(trkcr_div_rcp(QX, opd, yopd), opd);
        QY = __dmul_rn(trkcr_div_rcp(QY, opd, yopd), opd);
      }
      const double q2 = __dmul_rn(QY, QY);
      if (q2 != qy2) {
        qy2 = q2;
        f2 = __dsub_rn(opd2, qy2);
        f = __dsqrt_rn(f2);
        yf = __drcp_rn(f);
      }
    }
  }
  return true;
}
#endif

/* computeCSBENDFields (src/csbend.c:99-172): y powers are formed on the fly
 * (the same products as the reference's yp[] table) so nothing is indexed
 * in local memory. */
__device__ __forceinline__ void bend_fields(int mode, int eo1, const double *__restrict__ Fx_xy,
                                            const double *__restrict__ Fy_xy, double x, double y, double &Fx,
                                            double &Fy) {
  double sumFx = 0, sumFy = 0;
  double xt = 1;
  for (int i = 0; i < eo1; i++) {
    double ypj = 1;
    for (int j = 0; j < eo1 - i; j++) {
      if (mode == 2) {
        sumFx += __ldg(&Fx_xy[i * 11 + j]) * xt * ypj;
        sumFy += __ldg(&Fy_xy[i * 11 + j]) * xt * ypj;
      } else if (j & 1)
        sumFx += __ldg(&Fx_xy[i * 11 + j]) * xt * ypj;
      else
        sumFy += __ldg(&Fy_xy[i * 11 + j]) * xt * ypj;
      ypj = ypj * y;
    }
    xt *= x;
  }
  Fx = sumFx;
  Fy = sumFy;
}

#if TRK_FAST
/* Body of a pure-dipole CSBEND in the fast build.  With no field gradient
 * QY and delta are constant through the body, so f^2 = (1+delta)^2 - QY^2 is
 * formed once per bend, and Y and the path length grow by QY and (1+delta)
 * times the same factor each substep, so one running sum F of the factors
 * gives both.  The drift is written in f cos(phi) = sqrt(f^2 - QX^2) and
 * f sin(phi) = QX, so no division by f is needed, with tabulated sin/cos of
 * the substep angle a = dsh/rho0 and 1 - cos(a) = 2 sin^2(a/2) (no
 * cancellation):
 *   f cos(a+phi) = cos(a) f cos(phi) - sin(a) QX
 *   QX'          = f sin(a+phi) = sin(a) f cos(phi) + cos(a) QX
 *   u            = (rho0 + X) / (f cos(a+phi))
 *   factor       = u sin(a)                          (= tan(a+phi)-tan(phi), times (rho0+X)cos(phi)/f)
 *   X'           = X + u ((1-cos a) f cos(phi) + sin(a) QX)
 * the last from cos(phi)/cos(a+phi) - 1 = 2 sin(a/2) sin(a/2+phi)/cos(a+phi).
 * The kick is QX -= ds (1 + X/rho0)/rho_actual.  Loss conditions are the
 * reference's (f<=0, |QX/f|>1, cos(a+phi)=0, aperture per slice); `done`
 * counts the completed drift substeps for the loss position. */

/* One slice of the dipole body; `checked` evaluates the reference's loss
 * conditions at every substep, otherwise non-finite values are left to
 * propagate and the caller re-runs the slice checked. */
template <int NSUB, bool CHECKED>
__device__ __forceinline__ bool dipole_slice(const double *__restrict__ d, int nSub, double rho0, double f2,
                                             double &X, double &QX, double &F, int &done) {
#pragma unroll
  for (int j = 0; j < (NSUB > 0 ? NSUB : 8); j++) {
    if (NSUB == 0 && j >= nSub)
      break;
    const double u2 = fma(-QX, QX, f2);
    if (CHECKED && !(u2 >= 0)) /* |sin(phi)| = |QX/f| > 1 */
      return false;
    const double fc = CHECKED ? sqrt_fast(u2) : sqrt_nan(u2);
    const double sa = __ldg(&d[BD_SA + j]), ca = __ldg(&d[BD_CA + j]);
    const double saq = sa * QX;
    const double fcosi = fma(ca, fc, -saq);
    if (CHECKED && fcosi == 0)
      return false;
    const double u = div_fast(rho0 + X, fcosi);
    QX = fma(sa, fc, ca * QX);
    F = fma(u, sa, F);
    X = fma(u, fma(__ldg(&d[BD_OMC + j]), fc, saq), X);
    if (CHECKED)
      done++;
    if (j == nSub - 1)
      break;
    QX = fma(-__ldg(&d[BD_C2 + j]), X, QX - __ldg(&d[BD_C1 + j]));
  }
  return true;
}

struct SliceState {
  double X, QX, F;
  int done;
  bool ok;
};

/* The checked re-run of one slice, out of line so that the common path does
 * not hold registers for it. */
__device__ __noinline__ SliceState dipole_slice_redo(const double *__restrict__ d, int nSub, double rho0, double f2,
                                                     double X, double QX, double F, int done) {
  SliceState r;
  if (nSub == 4)
    r.ok = dipole_slice<4, true>(d, nSub, rho0, f2, X, QX, F, done);
  else
    r.ok = dipole_slice<0, true>(d, nSub, rho0, f2, X, QX, F, done);
  r.X = X;
  r.QX = QX;
  r.F = F;
  r.done = done;
  return r;
}

template <int NSUB>
__device__ __forceinline__ bool bend_dipole_fast(const double *__restrict__ d, int nSlices, int nSub_rt, double rho0,
                                                 const trk_aperture *ap, bool aptilt, double apc, double aps,
                                                 double &X, double &QX, double &Y, const double QY, const double D,
                                                 double &dist, int &done) {
  const int nSub = NSUB > 0 ? NSUB : nSub_rt;
  const double opd = 1 + D;
  const double f2 = opd * opd - QY * QY;
  const double Y0 = Y;
  double F = 0;
  bool ok = true;
  done = 0;
  for (int i = 0; i < nSlices; i++) {
    if (ap && !check_aperture(X, Y0 + QY * F, ap, aptilt, apc, aps)) {
      ok = false;
      break;
    }
    if (!(f2 > 0)) {
      ok = false;
      break;
    }
    /* re-read the substep constants every slice (L1 hits) rather than
     * holding 20 doubles in registers across the slice loop */
    const double *dd = d;
    asm volatile("" : "+l"(dd));
    const double X0 = X, QX0 = QX, F0 = F;
    dipole_slice<NSUB, false>(dd, nSub, rho0, f2, X, QX, F, done);
    if (!isfinite(X + QX + F)) {
      /* a loss condition may have fired: redo the slice with the checks */
      const SliceState r = dipole_slice_redo(dd, nSub, rho0, f2, X0, QX0, F0, done);
      X = r.X;
      QX = r.QX;
      F = r.F;
      done = r.done;
      if (!r.ok) {
        ok = false;
        break;
      }
      done -= nSub;
    }
    done += nSub;
  }
  Y = Y0 + QY * F;
  dist = opd * F;
  return ok;
}

/* Body of a combined-function CSBEND in the fast build: a normal-only field
 * expansion of order 4 (K1 and/or K2; expansionOrder1 = 5).  The drift is
 * the pure dipole's, with f^2 = (1+delta)^2 - QY^2 re-formed every substep
 * because the kicks now change QY, and Y and the path length advanced by
 * their own terms.  The field is computeCSBENDFields (src/csbend.c:99-172)
 * regrouped by powers of y and evaluated in Horner form in x:
 *   Fy = P0(x) + y^2 (P2(x) + y^2 P4),   Fx = y (Q1(x) + y^2 Q3(x)),
 * with Pj, Qj the table columns j (terms i + j <= 4). */
#define CF_T(T, i, j) __ldg(&(T)[(i) * 11 + (j)])
__device__ __forceinline__ void cf_fields(const double *__restrict__ Fx_xy, const double *__restrict__ Fy_xy,
                                          double x, double y, double &Fx, double &Fy) {
  const double y2 = y * y;
  const double p0 = fma(fma(fma(fma(CF_T(Fy_xy, 4, 0), x, CF_T(Fy_xy, 3, 0)), x, CF_T(Fy_xy, 2, 0)), x,
                            CF_T(Fy_xy, 1, 0)),
                        x, CF_T(Fy_xy, 0, 0));
  const double p2 = fma(fma(CF_T(Fy_xy, 2, 2), x, CF_T(Fy_xy, 1, 2)), x, CF_T(Fy_xy, 0, 2));
  Fy = fma(y2, fma(y2, CF_T(Fy_xy, 0, 4), p2), p0);
  const double q1 = fma(fma(fma(CF_T(Fx_xy, 3, 1), x, CF_T(Fx_xy, 2, 1)), x, CF_T(Fx_xy, 1, 1)), x,
                        CF_T(Fx_xy, 0, 1));
  const double q3 = fma(CF_T(Fx_xy, 1, 3), x, CF_T(Fx_xy, 0, 3));
  Fx = y * fma(y2, q3, q1);
}
#undef CF_T

/* One slice (4 drift substeps, 3 kicks); `checked` as in dipole_slice. */
template <bool CHECKED>
__device__ __forceinline__ bool cf_slice(const double *__restrict__ d, const double *__restrict__ fxy, double rho0,
                                         double opd, double &X, double &QX, double &Y, double &QY, double &dist,
                                         int &done) {
  const double opd2 = opd * opd;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const double f2 = fma(-QY, QY, opd2);
    if (CHECKED && !(f2 > 0))
      return false;
    const double u2 = fma(-QX, QX, f2);
    if (CHECKED && !(u2 >= 0)) /* |sin(phi)| = |QX/f| > 1 */
      return false;
    const double fc = CHECKED ? sqrt_fast(u2) : sqrt_nan(u2);
    const double sa = __ldg(&d[BD_SA + j]), ca = __ldg(&d[BD_CA + j]);
    const double saq = sa * QX;
    const double fcosi = fma(ca, fc, -saq);
    if (CHECKED && fcosi == 0)
      return false;
    const double u = div_fast(rho0 + X, fcosi);
    const double fac = u * sa;
    QX = fma(sa, fc, ca * QX);
    Y = fma(QY, fac, Y);
    dist = fma(fac, opd, dist);
    X = fma(u, fma(__ldg(&d[BD_OMC + j]), fc, saq), X);
    if (CHECKED)
      done++;
    if (j == 3)
      break;
    double Fx, Fy;
    cf_fields(fxy, fxy + 121, X, Y, Fx, Fy);
    const double w = fma(__ldg(&d[BD_C2 + j]), X, __ldg(&d[BD_C1 + j]));
    QX = fma(-w, Fy, QX);
    QY = fma(w, Fx, QY);
  }
  return true;
}

struct CfState {
  double X, QX, Y, QY, dist;
  int done;
  bool ok;
};

__device__ __noinline__ CfState cf_slice_redo(const double *__restrict__ d, const double *__restrict__ fxy,
                                              double rho0, double opd, double X, double QX, double Y, double QY,
                                              double dist, int done) {
  CfState r;
  r.ok = cf_slice<true>(d, fxy, rho0, opd, X, QX, Y, QY, dist, done);
  r.X = X;
  r.QX = QX;
  r.Y = Y;
  r.QY = QY;
  r.dist = dist;
  r.done = done;
  return r;
}

__device__ __forceinline__ bool bend_cf_fast(const double *__restrict__ d, const double *__restrict__ fxy,
                                             int nSlices, double rho0, const trk_aperture *ap, double &X, double &QX,
                                             double &Y, double &QY, const double D, double &dist, int &done) {
  const double opd = 1 + D;
  bool ok = true;
  dist = 0;
  done = 0;
  for (int i = 0; i < nSlices; i++) {
    if (ap && !check_aperture(X, Y, ap, false, 1.0, 0.0)) {
      ok = false;
      break;
    }
    const double *dd = d;
    asm volatile("" : "+l"(dd));
    const double X0 = X, QX0 = QX, Y0 = Y, QY0 = QY, S0 = dist;
    cf_slice<false>(dd, fxy, rho0, opd, X, QX, Y, QY, dist, done);
    if (!isfinite(X + QX + Y + QY + dist)) {
      const CfState r = cf_slice_redo(dd, fxy, rho0, opd, X0, QX0, Y0, QY0, S0, done);
      X = r.X;
      QX = r.QX;
      Y = r.Y;
      QY = r.QY;
      dist = r.dist;
      done = r.done;
      if (!r.ok) {
        ok = false;
        break;
      }
      done -= 4;
    }
    done += 4;
  }
  return ok;
}
#endif

/* apply_edge_effects (src/csbend.c:4291-4333) */
__device__ void edge_order2(double &x, double &xp, double &y, double &yp, double rho, double n, double beta,
                            double tanb, double secb, double he, double psi, int which_edge) {
  double h, tan_beta, tan2_beta, sec_beta, sec2_beta, h2;
  double R21, R43, T111, T133, T211, T441, T331, T221, T233, T243, T431, T432;
  h = 1 / rho;
  R21 = h * (tan_beta = tanb);
  R43 = -h * M_TAN(beta - psi);
  h2 = sqr(h);
  T111 = which_edge * h / 2 * (tan2_beta = sqr(tan_beta));
  sec_beta = secb;
  sec2_beta = sqr(sec_beta);
  T133 = -which_edge * h / 2 * sec2_beta;
  T211 = which_edge == -1 ? -n * h2 * tan_beta : -h2 * (n + tan2_beta / 2) * tan_beta;
  T441 = -(T331 = T221 = -which_edge * h * tan2_beta);
  T233 = which_edge == -1 ? h2 * (n + .5 + tan2_beta) * tan_beta : h2 * (n - tan2_beta / 2) * tan_beta;
  T243 = which_edge * h * tan2_beta;
  T431 = h2 * (2 * n + (which_edge == 1 ? sec2_beta : 0)) * tan_beta;
  T432 = which_edge * h * sec2_beta;
  if (he != 0) {
    double term = h / 2 * he * sec2_beta * sec_beta;
    T211 += term;
    T233 -= term;
    T431 -= 2 * term;
  }
  double x0 = x, xp0 = xp, y0 = y, yp0 = yp;
  x = x0 + T111 * sqr(x0) + T133 * sqr(y0);
  xp = xp0 + R21 * x0 + T211 * sqr(x0) + T221 * x0 * xp0 + T233 * sqr(y0) + T243 * y0 * yp0;
  y = y0 + T331 * x0 * y0;
  yp = yp0 + R43 * y0 + T441 * yp0 * x0 + T431 * x0 * y0 + T432 * xp0 * y0;
}

/* edge kick of track_through_csbend (src/csbend.c:1126-1204, 1306-1382) */
/* K. Hwang's dipole fringe (dipoleFringeKHwang, src/csbend.c:4336-4408) in
 * dipole canonical coordinates, each expression in the reference's operation
 * order; sec, tan, sin, cos of the edge angle come from the element record */
#define FR_P2(v) ((v) * (v))
#define FR_P3(v) ((v) * (v) * (v))
__device__ __noinline__ void fringe_hwang(double &x, double &px, double &y, double &py, double dp, double rho,
                                          double inFringe, bool second_order, double sec_edge, double tan_edge,
                                          double sin_edge, double cos_edge, double gap, double fint, double Rhe) {
  const double k0 = FR_P2(TRK_PI) / 6., k2 = fint, k3 = 1.0 * 1. / 6., k4 = -1.0 * FR_P2(TRK_PI) / 3., k5 = 0.0,
               k6 = -1.0;
  const double x0 = x, px0 = px, y0 = y, py0 = py, dp0 = dp;
  double dx = 0, dpx = 0, dy = 0, dpy = 0;
  if (second_order) {
    dx = inFringe * FR_P2(sec_edge) * FR_P2(gap) * k0 / rho / (1 + dp0) +
         inFringe * FR_P2(x0) * FR_P2(tan_edge) / 2 / rho / (1 + dp0) -
         inFringe * FR_P2(y0) * FR_P2(sec_edge) / 2 / rho / (1 + dp0);
    dy = -inFringe * x0 * y0 * FR_P2(tan_edge) / rho / (1 + dp0);
    if (inFringe == -1.) {
      dpx = -1. * FR_P3(sec_edge) * sin_edge * FR_P2(gap) * k0 / rho / rho / (1 + dp0) + tan_edge * x0 / rho +
            FR_P2(y0) / 2 * (2 * FR_P3(tan_edge)) / FR_P2(rho) / (1 + dp0) +
            FR_P2(y0) / 2 * (tan_edge) / FR_P2(rho) / (1 + dp0) -
            inFringe * (x0 * px0 - y0 * py0) * FR_P2(tan_edge) / rho / (1 + dp0) +
            k4 * FR_P2(sin_edge) * FR_P2(gap) / 2 / FR_P3(cos_edge) / rho * Rhe -
            k5 * x0 * sin_edge * gap / FR_P3(cos_edge) / rho * Rhe +
            k6 * (y0 * y0 - x0 * x0) / 2 / FR_P3(cos_edge) / rho * Rhe;
      dpy = -1. * tan_edge * y0 / rho + k2 * y0 * (1 + FR_P2(sin_edge)) * gap / (1 + dp0) / FR_P2(rho) / FR_P3(cos_edge) +
            inFringe * (x0 * py0 + y0 * px0) * FR_P2(tan_edge) / rho / (1 + dp0) +
            inFringe * y0 * px0 / rho / (1 + dp0) +
            k3 * FR_P3(y0) * (2. / 3. / cos_edge - 4. / 3. / FR_P3(cos_edge)) / (1 + dp0) / rho / rho / gap +
            k6 * x0 * y0 / FR_P3(cos_edge) / rho * Rhe;
    } else {
      dpx = tan_edge * x0 / rho - FR_P2(y0) / 2 * (1 * FR_P3(tan_edge)) / FR_P2(rho) / (1 + dp0) -
            FR_P2(x0) / 2 * (1 * FR_P3(tan_edge)) / FR_P2(rho) / (1 + dp0) -
            inFringe * (x0 * px0 - y0 * py0) * FR_P2(tan_edge) / rho / (1 + dp0) +
            k4 * FR_P2(sin_edge) * FR_P2(gap) / 2 / FR_P3(cos_edge) / rho * Rhe -
            k5 * x0 * sin_edge * gap / FR_P3(cos_edge) / rho * Rhe +
            k6 * (y0 * y0 - x0 * x0) / 2 / FR_P3(cos_edge) / rho * Rhe;
      dpy = -1. * tan_edge * y0 / rho + k2 * y0 * (1 + FR_P2(sin_edge)) * gap / (1 + dp0) / FR_P2(rho) / FR_P3(cos_edge) +
            inFringe * (x0 * py0 + y0 * px0) * FR_P2(tan_edge) / rho / (1 + dp0) +
            inFringe * y0 * px0 / rho / (1 + dp0) + x0 * y0 * FR_P2(sec_edge) * tan_edge / FR_P2(rho) / (1 + dp0) +
            k3 * FR_P3(y0) * (2. / 3. / cos_edge - 4. / 3. / FR_P3(cos_edge)) / (1 + dp0) / rho / rho / gap -
            k5 * y0 * sin_edge * gap / FR_P3(cos_edge) / rho * Rhe + k6 * x0 * y0 / FR_P3(cos_edge) / rho * Rhe;
    }
  } else {
    dx = inFringe * FR_P2(sec_edge) * FR_P2(gap) * k0 / rho / (1 + dp0);
    if (inFringe == -1.) {
      dpx = -1. * FR_P3(sec_edge) * sin_edge * FR_P2(gap) * k0 / rho / rho / (1 + dp0) + tan_edge * x0 / rho +
            k4 * FR_P2(sin_edge) * FR_P2(gap) / 2 / FR_P3(cos_edge) / rho * Rhe -
            k5 * x0 * sin_edge * gap / FR_P3(cos_edge) / rho * Rhe;
      dpy = -1. * tan_edge * y0 / rho + k2 * y0 * (1 + FR_P2(sin_edge)) * gap / (1 + dp0) / FR_P2(rho) / FR_P3(cos_edge);
    } else {
      dpx = tan_edge * x0 / rho + k4 * FR_P2(sin_edge) * FR_P2(gap) / 2 / FR_P3(cos_edge) / rho * Rhe -
            k5 * x0 * sin_edge * gap / FR_P3(cos_edge) / rho * Rhe;
      dpy = -1. * tan_edge * y0 / rho + k2 * y0 * (1 + FR_P2(sin_edge)) * gap / (1 + dp0) / FR_P2(rho) / FR_P3(cos_edge) -
            k5 * y0 * sin_edge * gap / FR_P3(cos_edge) / rho * Rhe;
    }
  }
  x = x0 + dx;
  px = px0 + dpx;
  y = y0 + dy;
  py = py0 + dpy;
}

/* the same symplectified by R. Lindberg (dipoleFringeKHwangRLindberg,
 * src/csbend.c:4413-4520): five maps in sequence */
__device__ __noinline__ void fringe_hwang_lindberg(double &x, double &px, double &y, double &py, double dp, double rho,
                                                   double inFringe, double sec_edge, double tan_edge, double sin_edge,
                                                   double cos_edge, double gap, double fint, double Rhe) {
  const double k0 = FR_P2(TRK_PI) / 6., k2 = fint, k3 = 1.0 * 1. / 6., k4 = -1.0 * FR_P2(TRK_PI) / 3., k5 = 0.0,
               k6 = -1.0;
  const double rho2 = FR_P2(rho);
  const double x0 = x, px0 = px, y0 = y, py0 = py, dp0 = dp;
  const double sec2_edge = FR_P2(sec_edge), cos3_edge = FR_P3(cos_edge), tan2_edge = FR_P2(tan_edge),
               tan3_edge = FR_P3(tan_edge);
  double x1, px1, y1, py1, x2, px2, x3, py3, px4, y4, py4, t1, t2;
  if (inFringe == -1) {
    x1 = x0;
    px1 = px0 + tan_edge / rho * x0 + tan_edge / (2 * rho2 * (1 + dp0)) * FR_P2(y0) -
          tan3_edge / (rho2 * (1 + dp0)) * FR_P2(x0) - gap * k5 * sin_edge * Rhe / (rho * cos3_edge) * x0 +
          k6 * sec2_edge * Rhe / (2 * rho) * (FR_P2(y0) - FR_P2(x0));
    y1 = y0;
    py1 = py0 - tan_edge / rho * y0 + tan_edge / (rho2 * (1 + dp0)) * x0 * y0 +
          gap * k2 * (1 + FR_P2(sin_edge)) / (rho2 * (1 + dp0) * cos3_edge) * y0 +
          2 * k3 * (FR_P2(cos_edge) - 2) / (3 * gap * rho2 * cos3_edge) * FR_P3(y0) +
          gap * k5 * sin_edge * Rhe / (rho * cos3_edge) * y0 + k6 * FR_P3(sec_edge) * Rhe / rho * x0 * y0;
    t1 = (1 + tan2_edge / (2 * rho * (1 + dp0)) * x1);
    x2 = x1 / t1;
    px2 = px1 * FR_P2(t1);
    t1 = sec2_edge / (rho * (1 + dp0));
    x3 = x2 + t1 / 2 * FR_P2(y1);
    py3 = py1 - t1 * y1 * px2;
    t1 = tan2_edge / (rho * (1 + dp0));
    t2 = M_EXP(t1 * x3);
    px4 = px2 - t1 * y1 * py3;
    y4 = y1 * t2;
    py4 = py3 / t2;
    t1 = FR_P2(gap) * k0 * sec2_edge / (rho * (1 + dp0));
    x = x3 - t1;
    px = px4 - t1 * tan_edge / rho + FR_P2(gap) * k4 * FR_P2(sin_edge) * Rhe / (2 * rho * cos3_edge);
  } else {
    x1 = x0;
    px1 = px0 + tan_edge / rho * x0 + tan3_edge / (2 * rho2 * (1 + dp0)) * FR_P2(y0) +
          tan3_edge / (2 * rho2 * (1 + dp0)) * FR_P2(x0) - gap * k5 * sin_edge * Rhe / (rho * cos3_edge) * x0 +
          k6 * sec2_edge * Rhe / (2 * rho) * (FR_P2(y0) - FR_P2(x0));
    y1 = y0;
    py1 = py0 - tan_edge / rho * y0 + tan3_edge / (rho2 * (1 + dp0)) * x0 * y0 +
          gap * k2 * (1 + FR_P2(sin_edge)) / (rho2 * (1 + dp0) * cos3_edge) * y0 +
          2 * k3 * (FR_P2(cos_edge) - 2) / (3 * gap * rho2 * cos3_edge) * FR_P3(y0) +
          gap * k5 * sin_edge * Rhe / (rho * cos3_edge) * y0 + k6 * FR_P3(sec_edge) * Rhe / rho * x0 * y0;
    t1 = (1 - tan2_edge / (2 * rho * (1 + dp0)) * x1);
    x2 = x1 / t1;
    px2 = px1 * FR_P2(t1);
    t1 = sec2_edge / (rho * (1 + dp0));
    x3 = x2 - t1 / 2 * FR_P2(y1);
    py3 = py1 + t1 * y1 * px2;
    t1 = -tan2_edge / (rho * (1 + dp0));
    t2 = M_EXP(t1 * x3);
    px4 = px2 - t1 * y1 * py3;
    y4 = y1 * t2;
    py4 = py3 / t2;
    x = x3 + FR_P2(gap) * k0 * sec2_edge / (rho * (1 + dp0));
    px = px4 + FR_P2(gap) * k4 * FR_P2(sin_edge) * Rhe / (2 * rho * cos3_edge);
  }
  y = y4;
  py = py4;
}
#undef FR_P2
#undef FR_P3

/* R. Lindberg's curved-dipole fringe (curvedDipoleFringe, src/csbend.c:
 * 5693-5969) in dipole canonical coordinates: the linear map through the
 * fringe field from the edge integrals K0..K6 (fr[0..6]), the same at both
 * ends, then for EDGE_ORDER > 1 the edge's second-order terms, which differ
 * in sign between entrance (inFringe -1) and exit.  fr[7], fr[8]: tan and sec
 * of the edge angle.  Each expression in the reference's operation order;
 * returns the path-length change dtau (the reference adds -dtau to s). */
__device__ __noinline__ double fringe_curved(double &x, double &px, double &y, double &py, double dp, double rho,
                                             int inFringe, bool second_order, double K1,
                                             const double *__restrict__ fr) {
  const double x0 = x, px0 = px, y0 = y, py0 = py, dp0 = dp;
  const double intK0 = __ldg(&fr[0]), intK1 = __ldg(&fr[1]), intK2 = __ldg(&fr[2]), intK3 = __ldg(&fr[3]),
               intK4 = __ldg(&fr[4]), intK5 = __ldg(&fr[5]), intK6 = __ldg(&fr[6]);
  const double tan_edge = __ldg(&fr[7]), sec_edge = __ldg(&fr[8]);
  double x1, px1, y1, py1, dtau;
  const double mx = (intK3 + intK4) / (1.0 + dp0);
  const double my = intK3 / (1.0 + dp0);
  const double delX = intK0 / (1.0 + dp0);
  const double focX = intK1 + tan_edge / rho;
  const double focY = intK2 / (1.0 + dp0);
  if (fabs(mx) < 1.0e-5) {
    x1 = x0 * M_EXP(-mx) + dp0 * delX * (1.0 - 0.5 * mx * (1.0 - mx / 3.0 + mx * mx / 12.0));
    px1 = px0 * M_EXP(mx) + focX * (x0 * (1.0 + mx * mx / 6.0) + dp0 * delX * (0.5 + mx * mx / 24.0));
    dtau = px0 * (mx * x0 + delX) / (1.0 + dp0) + delX * px0 * 0.5 * mx * (1.0 + mx / 3.0 + mx * mx / 12.0) +
           focX * x0 * x0 * mx * (0.5 - (mx - 0.5 * mx * mx) / 3.0) / (1.0 + dp0) +
           dp0 * focX * delX * (delX + mx * x0 / (1.0 + dp0)) * (1.0 + 0.05 * mx * mx) / 6.0 +
           focX * delX * x0 * 0.5 * (1.0 + mx * mx / 12.0) / (1.0 + dp0) +
           dp0 * focX * delX * (2.0 * mx * x0 - dp0 * delX) * (1.0 - mx * (0.75 - mx * (0.35 - 0.125 * mx))) /
             (6.0 * (1.0 + dp0));
  } else {
    const double emx = M_EXP(-mx), epx = M_EXP(mx), e2mx = M_EXP(-2.0 * mx);
    const double shx = M_SINH(mx), chx = M_COSH(mx);
    x1 = x0 * emx + dp0 * delX * (1.0 - emx) / mx;
    px1 = px0 * epx + focX * (x0 * shx / mx + dp0 * delX * (chx - 1.0) / (mx * mx));
    dtau = px0 * (mx * x0 + delX) / (1.0 + dp0) + delX * px0 * (epx - 1.0 - mx) / mx +
           focX * x0 * x0 * 0.25 * ((e2mx - 1.0) / mx + 2.0) / (1.0 + dp0) +
           dp0 * focX * delX * (delX + mx * x0 / (1.0 + dp0)) * (shx - mx) / (mx * mx * mx) +
           focX * delX * x0 * (chx - 1.0) / (mx * mx * (1.0 + dp0)) +
           dp0 * focX * delX * (2.0 * mx * x0 - dp0 * delX) * 0.25 * (2.0 - (3.0 + e2mx - 4.0 * emx) / mx) /
             (mx * mx * (1.0 + dp0));
  }
  if (fabs(my) < 1.0e-5) {
    y1 = y0 * M_EXP(my);
    py1 = py0 * M_EXP(-my) + y0 * (focY - focX) * (1.0 + my * my / 6.0);
    dtau += (-my * py0 * y0 + 0.5 * (focY + focX * (my + my * my * (2.0 + my) / 3.0) * y0 * y0)) / (1.0 + dp0);
  } else {
    y1 = y0 * M_EXP(my);
    py1 = py0 * M_EXP(-my) + y0 * (focY - focX) * M_SINH(my) / my;
    dtau += (-my * py0 * y0 + 0.5 * (focY + 0.5 * focX * ((M_EXP(2.0 * my) - 1.0) / my - 2.0)) * y0 * y0) /
            (1.0 + dp0);
  }
  if (second_order) {
    const double sect2_rho = sec_edge * sec_edge / (rho * (1.0 + dp0));
    const double tant_rho = tan_edge / (rho * (1.0 + dp0));
    double x2, y2, px2, py2;
    if (inFringe == -1) {
      x2 = x1;
      y2 = y1 * M_EXP(tan_edge * tant_rho * x1);
      px2 = px1 - tan_edge * tant_rho * y1 * py1 - (tan_edge * (tan_edge * tant_rho / rho - K1) - 0.5 * intK6) * x1 * x1;
      py2 = py1 * M_EXP(-tan_edge * tant_rho * x1);
      dtau += -tan_edge * tant_rho * tant_rho * x1 * x1 * x1 / 3.0 - tant_rho * tant_rho * rho * x1 * y1 * py1;
      x1 = x2 + 0.5 * sect2_rho * y2 * y2;
      y1 = y2;
      px1 = px2 + (0.5 * tant_rho / rho - 0.5 * intK5 - K1 * tan_edge + 0.25 * intK1 * sect2_rho) * y2 * y2;
      py1 = py2 + (tant_rho / rho - intK5 - 2.0 * K1 * tan_edge + 0.5 * intK1 * sect2_rho) * x2 * y2 -
            sect2_rho * y2 * px2;
      dtau += (0.5 * sect2_rho * (0.25 * (2.0 * tan_edge * K1 + intK5) * y2 * y2 - px2) +
               (0.5 * tant_rho / rho + 0.25 * intK1 * sect2_rho) * x2) *
              y2 * y2 / (1.0 + dp0);
      x2 = x1 / (1.0 + 0.5 * tan_edge * tant_rho * x1);
      y2 = y1;
      px2 = px1 * (1.0 + 0.5 * tan_edge * tant_rho * x1) * (1.0 + 0.5 * tan_edge * tant_rho * x1);
      py2 = py1;
      dtau += 0.5 * tant_rho * tant_rho * rho * x1 * x1 * px1;
    } else {
      x2 = x1;
      y2 = y1 * M_EXP(-tan_edge * tant_rho * x1);
      px2 = px1 + tan_edge * tant_rho * y1 * py1 +
            (tan_edge * (0.5 * tan_edge * tant_rho / rho + K1) + 0.5 * intK6) * x1 * x1;
      py2 = py1 * M_EXP(tan_edge * tant_rho * x1);
      dtau += tan_edge * tant_rho * tant_rho * x1 * x1 * x1 / 6.0 + tant_rho * tant_rho * rho * x1 * y1 * py1;
      x1 = x2 - 0.5 * sect2_rho * y2 * y2;
      y1 = y2;
      px1 = px2 + (0.5 * tan_edge * tan_edge * tant_rho / rho - 0.5 * intK5 - K1 * tan_edge - 0.25 * intK1 * sect2_rho) *
                    y2 * y2;
      py1 = py2 +
            (tan_edge * tan_edge * tant_rho / rho - intK5 - 2.0 * K1 * tan_edge - 0.5 * intK1 * sect2_rho) * x2 * y2 +
            sect2_rho * y2 * px2;
      dtau += (-0.5 * sect2_rho * (0.25 * (2.0 * tan_edge * K1 + intK5) * y2 * y2 - px2) +
               (0.5 * tan_edge * tan_edge * tant_rho / rho - 0.25 * intK1 * sect2_rho) * x2) *
              y2 * y2 / (1.0 + dp0);
      x2 = x1 / (1.0 - 0.5 * tan_edge * tant_rho * x1);
      y2 = y1;
      px2 = px1 * (1.0 - 0.5 * tan_edge * tant_rho * x1) * (1.0 + 0.5 * tan_edge * tant_rho * x1);
      py2 = py1;
      dtau += -0.5 * tant_rho * tant_rho * rho * x1 * x1 * px1;
    }
    x1 = x2;
    px1 = px2;
    y1 = y2;
    py1 = py2;
  }
  /* the reference adds the changes to the initial values */
  x = x0 + (x1 - x0);
  px = px0 + (px1 - px0);
  y = y0 + (y1 - y0);
  py = py0 + (py1 - py0);
  return dtau;
}

/* linear edge kick, EDGE_EFFECTS=1 with EDGE_ORDER <= 1 (src/csbend.c:1127-1134) */
__device__ __forceinline__ void edge_lin1(const double *__restrict__ d, int base, double rho_a, double x, double &xp,
                                          double y, double &yp, double dp) {
  const double e = __ldg(&d[base + 0]), te = __ldg(&d[base + 1]), psi = __ldg(&d[base + 2]);
  const double lim = __ldg(&d[base + 3]);
  double rho = (1 + dp) * rho_a;
  double delta_xp = te / rho * x;
  if (lim > 0 && fabs(delta_xp) > lim)
    delta_xp = (delta_xp < 0 ? -1 : 1) * lim;
  xp += delta_xp;
  double t2 = psi == 0 ? te : M_TAN(e - psi / (1 + dp));
  yp -= t2 / rho * y;
}

__device__ __forceinline__ void bend_edge(int mode, const double *__restrict__ d, int base, int which, double rho_a,
                                          double nidx, const double *__restrict__ fr, bool expanded, double &x,
                                          double &xp, double &y, double &yp, double &s, double dp) {
  const double e = __ldg(&d[base + 0]), te = __ldg(&d[base + 1]), psi = __ldg(&d[base + 2]);
  const double lim = __ldg(&d[base + 3]), he = __ldg(&d[base + 4]), secb = __ldg(&d[base + 5]);
  if (mode == EDGE_LIN1) {
    edge_lin1(d, base, rho_a, x, xp, y, yp, dp);
  } else if (mode == EDGE_LIN2) {
    double rho = (1 + dp) * rho_a;
    edge_order2(x, xp, y, yp, rho, nidx, e, te, secb, he, psi * (1 + dp), which);
  } else if (mode == EDGE_SYMP) {
    /* applySimpleDipoleEdgeKick (src/csbend.c:5664-5690) */
    double Q1 = xp, Q3 = yp;
    double f = expanded ? (1 + dp) : (1 + dp) / sqrt(1 + sqr(Q1) + sqr(Q3));
    Q1 *= f;
    Q3 *= f;
    double dqx = te / rho_a * x;
    if (lim > 0 && fabs(dqx) > lim)
      dqx = (dqx < 0 ? -1 : 1) * lim;
    double t2 = psi == 0 ? te : M_TAN(e - psi / (1 + dp));
    double dqy = -t2 / rho_a * y;
    Q1 += dqx;
    Q3 += dqy;
    f = expanded ? 1 / (1 + dp) : 1 / sqrt(sqr(1 + dp) - sqr(Q1) - sqr(Q3));
    xp = Q1 * f;
    yp = Q3 * f;
  } else if (mode == EDGE_HWANG1 || mode == EDGE_HWANG2 || mode == EDGE_HWANGL) {
    /* in dipole canonical coordinates (src/csbend.c:1139-1182, :1319-1359;
     * convert{To,From}DipoleCanonicalCoordinates, :1436-1457) */
    double f = expanded ? (1 + dp) : (1 + dp) / sqrt(1 + sqr(xp) + sqr(yp));
    double px = xp * f, py = yp * f;
    const int k = which < 0 ? 0 : 1;
    const double sn = __ldg(&d[BD_FS1 + 3 * k]), cs = __ldg(&d[BD_FC1 + 3 * k]), fint = __ldg(&d[BD_FF1 + 3 * k]);
    const double gap = __ldg(&d[BD_GAP]);
    if (mode == EDGE_HWANGL)
      fringe_hwang_lindberg(x, px, y, py, dp, rho_a, (double)which, secb, te, sn, cs, gap, fint, he);
    else
      fringe_hwang(x, px, y, py, dp, rho_a, (double)which, mode == EDGE_HWANG2, secb, te, sn, cs, gap, fint, he);
    f = expanded ? 1 / (1 + dp) : 1 / sqrt(sqr(1 + dp) - sqr(px) - sqr(py));
    xp = px * f;
    yp = py * f;
  } else if (mode == EDGE_CURV1 || mode == EDGE_CURV2) {
    /* src/csbend.c:1183-1203, :1360-1377: the same coordinates, and s takes
     * the fringe's path-length change */
    double f = expanded ? (1 + dp) : (1 + dp) / sqrt(1 + sqr(xp) + sqr(yp));
    double px = xp * f, py = yp * f;
    const double dtau = fringe_curved(x, px, y, py, dp, rho_a, which, mode == EDGE_CURV2, __ldg(&d[BD_K1F]), fr);
    f = expanded ? 1 / (1 + dp) : 1 / sqrt(sqr(1 + dp) - sqr(px) - sqr(py));
    xp = px * f;
    yp = py * f;
    s += -dtau;
  }
}

/* the radiation correction of delta at a bend edge of nonzero angle,
 * dp' x tan(e) with dp' = -rad_coef F^2 (1+delta)^2 sqrt((1+x/rho0)^2 + x'^2
 * + y'^2) (src/csbend.c:1215-1222, :1270-1281) */
__device__ __noinline__ double rad_edge_dp(const double *__restrict__ d, int te_index, int fmode, int eo1,
                                           const double *__restrict__ Fx_xy, const double *__restrict__ Fy_xy,
                                           double rho0, double x, double xp, double y, double yp, double dp) {
  double Fx, Fy;
  if (fmode == 0) {
    Fx = 0;
    Fy = 1;
  } else
    bend_fields(fmode, eo1, Fx_xy, Fy_xy, x, y, Fx, Fy);
  const double dp_prime =
    -__ldg(&d[BD_RAD]) * (sqr(Fx) + sqr(Fy)) * sqr(1 + dp) * sqrt(sqr(1 + x / rho0) + sqr(xp) + sqr(yp));
  return dp_prime * x * __ldg(&d[te_index]);
}

/* integrate_csbend_ordn_expanded (src/csbend.c:1722-1900): leading-order
 * drift, aperture after every drift substep as well as per slice; out of
 * line so that the exact body's register allocation does not carry it */
__device__ __noinline__ bool bend_body_expanded(const trk_op *__restrict__ op, const double *__restrict__ Fx_xy,
                                                const double *__restrict__ Fy_xy, int fmode, int eo1, int nSlices,
                                                int nSub, int flags, double rho0, double rho_a, const trk_aperture *ap,
                                                bool aptilt, double apc, double aps, const IsrKey *isr, double &X,
                                                double &QX, double &Y, double &QY, double &D, double &dist,
                                                double &dz_lost) {
  const double *d = op->d;
  const double sl = __ldg(&d[BD_SLICE]);
  bool ok = true;
  for (int i = 0; i < nSlices && ok; i++) {
    if (!check_aperture(X, Y, ap, aptilt, apc, aps)) {
      ok = false;
      break;
    }
    for (int j = 0; j < nSub; j++) {
      const double dsh = __ldg(&d[BD_DSH + j]);
      QX += dsh * (1 + D) / (2 * rho0);
      dist += dsh * (1 + (sqr(QX) + sqr(QY)) / 2);
      dz_lost += dsh;
      X += QX * dsh / (1 + D);
      Y += QY * dsh / (1 + D);
      QX += dsh * (1 + D) / (2 * rho0);
      if (!check_aperture(X, Y, ap, aptilt, apc, aps)) {
        ok = false;
        break;
      }
      if (j == nSub - 1)
        break;
      const double ds = __ldg(&d[BD_DS + j]);
      double Fx, Fy;
      if (fmode == 0) {
        Fx = 0;
        Fy = 1;
      } else
        bend_fields(fmode, eo1, Fx_xy, Fy_xy, X, Y, Fx, Fy);
      QX += -ds * (1 + X / rho0) * Fy / rho_a;
      QY += ds * (1 + X / rho0) * Fx / rho_a;
      if (flags & BF_RAD) {
        /* src/csbend.c:1833-1863 (dsISR = s/3 in this integrator) */
        const double hX = 1 + X * __ldg(&d[BD_RHOINV]);
        const double f = hX / sqrt(sqr(1 + D) - sqr(QX) - sqr(QY));
        const double xpr = QX * f, ypr = QY * f;
        const double dsFactor = sqrt(sqr(hX) + sqr(xpr) + sqr(ypr));
        const double F2 = sqr(Fx) + sqr(Fy);
        const double deltaFactor = sqr(1 + D);
        const double dsISR = sl / 3;
        QX /= (1 + D);
        QY /= (1 + D);
        const double rad_coef = __ldg(&d[BD_RAD]);
        if (rad_coef != 0)
          D -= rad_coef * deltaFactor * F2 * ds * dsFactor;
        if ((flags & BF_ISR) && isr && !(isr->single && (flags & BF_ISR1OFF))) {
          const double g =
            trk_isr_gauss(isr->seed, isr->id, isr->pass, isr->elem, (unsigned)(i * 8 + j), isr->limit);
          D -= __ldg(&d[BD_ISR]) * deltaFactor * pow(F2, 0.75) * sqrt(dsISR * dsFactor) * g;
        }
        QX *= (1 + D);
        QY *= (1 + D);
      } else if (flags & BF_ISR_ROUNDTRIP) {
        QX /= (1 + D);
        QY /= (1 + D);
        QX *= (1 + D);
        QY *= (1 + D);
      }
    }
  }
  return ok;
}

/* track_through_csbend (src/csbend.c:654-1434) with integrate_csbend_ordn
 * (src/csbend.c:1459-1720); no radiation, MALIGN_METHOD=0. */
__device__ __forceinline__ bool op_bend(const trk_op *__restrict__ op, Part &p, double Po, double z_start,
                                        const trk_aperture *ap, const double *__restrict__ field,
                                        const IsrKey *isr = nullptr) {
  const double *d = op->d;
  const int nSlices = __ldg(&op->i[0]);
  const int nSub = __ldg(&op->i[1]);
  const int fmode = __ldg(&op->i[2]);
  const int eo1 = __ldg(&op->i[3]);
  const double *Fx_xy = field + __ldg(&op->i[4]);
  const double *Fy_xy = Fx_xy + 121;
  const double *Fr = Fx_xy + (fmode ? 242 : 0); /* curved-fringe records */
  const int edge1 = __ldg(&op->i[5]), edge2 = __ldg(&op->i[6]);
  const int flags = __ldg(&op->i[7]);
  const bool expanded = (flags & BF_EXPAND) != 0;
  const double rho0 = __ldg(&d[BD_RHO0]), rho_a = __ldg(&d[BD_RHOA]);
  const double ct = __ldg(&d[BD_CT]), st = __ldg(&d[BD_ST]);
  const bool aptilt = (flags & BF_APTILT) != 0;
  const double apc = __ldg(&d[BD_APC]), aps = __ldg(&d[BD_APS]);

  double x, xp, y, yp, s, dp;
  double dp0;
  if (flags & BF_MISALIGN) {
    const double dxi = __ldg(&d[BD_DXI]), dyi = __ldg(&d[BD_DYI]), dzi = __ldg(&d[BD_DZI]);
    p.s += dzi * sqrt(1 + sqr(p.xp) + sqr(p.yp));
    p.x = p.x + dxi + dzi * p.xp;
    p.y = p.y + dyi + dzi * p.yp;
    x = p.x * ct + p.y * st;
    y = -p.x * st + p.y * ct;
    xp = p.xp * ct + p.yp * st;
    yp = -p.xp * st + p.yp * ct;
  } else {
    x = p.x;
    y = p.y;
    xp = p.xp;
    yp = p.yp;
  }
  s = p.s;
  dp = p.dp;
  dp0 = p.dp;
  const double nidx = __ldg(&d[BD_N]);
  if (edge1)
    bend_edge(edge1, d, BD_E1, -1, rho_a, nidx, Fr, expanded, x, xp, y, yp, s, dp);

  double X = x, QX, Y = y, QY, S = 0, D = dp;
  if (flags & BF_RADE1) /* radiation: delta pre-adjusted for the sector integration (src/csbend.c:1215-1222) */
    D -= rad_edge_dp(d, BD_TE1, fmode, eo1, Fx_xy, Fy_xy, rho0, x, xp, y, yp, dp);
  /* convertToDipoleCanonicalCoordinates */
  {
    double f = expanded ? (1 + D) : (1 + D) / sqrt(1 + sqr(xp) + sqr(yp));
    QX = xp * f;
    QY = yp * f;
  }
  /* integrate_csbend_ordn */
  bool ok = true;
  double dist = 0, dz_lost = 0;
  const double sl = __ldg(&d[BD_SLICE]);
  if (expanded) {
    ok = bend_body_expanded(op, Fx_xy, Fy_xy, fmode, eo1, nSlices, nSub, flags, rho0, rho_a, ap, aptilt, apc, aps, isr,
                            X, QX, Y, QY, D, dist, dz_lost);
  } else if (fmode == 0 && !(flags & BF_RAD)) { /* the radiating dipole takes the general body */
    int done = 0;
#if TRK_FAST
    if (nSub == 4)
      ok = bend_dipole_fast<4>(d, nSlices, nSub, rho0, ap, aptilt, apc, aps, X, QX, Y, QY, D, dist, done);
    else
      ok = bend_dipole_fast<0>(d, nSlices, nSub, rho0, ap, aptilt, apc, aps, X, QX, Y, QY, D, dist, done);
#else
    ok = bend_dipole_exact(d, nSlices, nSub, rho0, (flags & BF_ISR_ROUNDTRIP) != 0, ap, aptilt, apc, aps, X, QX, Y,
                           QY, D, dist, done);
#endif
    if (!ok) /* loss position: the drift substeps completed so far */
      for (int k = 0; k < done; k++)
        dz_lost += __ldg(&d[BD_DSH + k % nSub]);
  } else
  for (int i = 0; i < nSlices && ok; i++) {
    if (!check_aperture(X, Y, ap, aptilt, apc, aps)) {
      ok = false;
      break;
    }
    for (int j = 0; j < nSub; j++) {
      const double dsh = __ldg(&d[BD_DSH + j]);
#if TRK_FAST
      /* sin/cos(dsh/rho0 + phi) by the angle-addition formulas with
       * tabulated sin/cos(dsh/rho0); tan(a+phi)-tan(phi) = sin a/(cos(a+phi) cos phi)
       * and cos(phi)/cos(a+phi) - 1 = 2 sin(a/2+phi) sin(a/2)/cos(a+phi) avoid
       * the cancellations of the reference expressions. */
      double f2 = sqr(1 + D) - sqr(QY);
      if (f2 <= 0) {
        ok = false;
        break;
      }
      double f = sqrt(f2);
      double finv = 1.0 / f;
      double sin_phi = QX * finv;
      if (fabs(sin_phi) > 1) {
        ok = false;
        break;
      }
      double cos_phi = sqrt(fma(-sin_phi, sin_phi, 1.0));
      const double sa = __ldg(&d[BD_SA + j]), ca = __ldg(&d[BD_CA + j]);
      const double sh = __ldg(&d[BD_SH + j]), ch = __ldg(&d[BD_CH + j]);
      double sine = sa * cos_phi + ca * sin_phi;
      double cosi = ca * cos_phi - sa * sin_phi;
      if (cosi == 0) {
        ok = false;
        break;
      }
      double cinv = 1.0 / cosi;
      QX = f * sine;
      double factor = (rho0 + X) * sa * finv * cinv;
      Y += QY * factor;
      dist += factor * (1 + D);
      dz_lost += dsh;
      double fm1 = 2 * (sh * cos_phi + ch * sin_phi) * sh * cinv; /* cos_phi/cosi - 1 */
      X = rho0 * fm1 + (1 + fm1) * X;
#else
      double f = sqr(1 + D) - sqr(QY);
      if (f <= 0) {
        ok = false;
        break;
      }
      f = sqrt(f);
      if (fabs(QX / f) > 1) {
        ok = false;
        break;
      }
      double sin_phi = QX / f;
      double phi = M_ASIN(sin_phi);
      const double arg = __ldg(&d[BD_ARG + j]);
      double sine, cosi;
      M_SINCOS(arg + phi, &sine, &cosi);
      if (cosi == 0) {
        ok = false;
        break;
      }
      double tang = sine / cosi;
      double cos_phi = M_COS(phi);
      QX = f * sine;
      double factor = (rho0 + X) * cos_phi / f * (tang - sin_phi / cos_phi);
      Y += QY * factor;
      dist += factor * (1 + D);
      dz_lost += dsh;
      f = cos_phi / cosi;
      X = rho0 * (f - 1) + f * X;
#endif
      if (j == nSub - 1)
        break;
      const double ds = __ldg(&d[BD_DS + j]);
      double Fx, Fy;
      if (fmode == 0) {
        Fx = 0;
        Fy = 1;
      } else
        bend_fields(fmode, eo1, Fx_xy, Fy_xy, X, Y, Fx, Fy);
#if TRK_FAST
      const double w = ds * (1 + X * __ldg(&d[BD_RHOINV])) * __ldg(&d[BD_INVRHOA]);
      QX += -w * Fy;
      QY += w * Fx;
#else
      QX += -ds * (1 + X / rho0) * Fy / rho_a;
      QY += ds * (1 + X / rho0) * Fx / rho_a;
#endif
      if (flags & BF_RAD) {
        /* classical radiation after the kick (src/csbend.c:1627-1656) */
        const double hX = 1 + X * __ldg(&d[BD_RHOINV]);
        const double f = hX / sqrt(sqr(1 + D) - sqr(QX) - sqr(QY));
        const double xpr = QX * f, ypr = QY * f;
        const double dsFactor = sqrt(sqr(hX) + sqr(xpr) + sqr(ypr));
        const double F2 = sqr(Fx) + sqr(Fy);
        const double deltaFactor = sqr(1 + D);
        const double dsISR = sl / (nSub - 1);
        QX /= (1 + D);
        QY /= (1 + D);
        const double rad_coef = __ldg(&d[BD_RAD]);
        if (rad_coef != 0)
          D -= rad_coef * deltaFactor * F2 * ds * dsFactor;
        if ((flags & BF_ISR) && isr && !(isr->single && (flags & BF_ISR1OFF))) {
          /* quantum excitation (src/csbend.c:1649-1651) */
          const double g =
            trk_isr_gauss(isr->seed, isr->id, isr->pass, isr->elem, (unsigned)(i * 8 + j), isr->limit);
          D -= __ldg(&d[BD_ISR]) * deltaFactor * pow(F2, 0.75) * sqrt(dsISR * dsFactor) * g;
        }
        QX *= (1 + D);
        QY *= (1 + D);
        continue;
      }
#if !TRK_FAST
      if (flags & BF_ISR_ROUNDTRIP) {
        QX /= (1 + D);
        QY /= (1 + D);
        QX *= (1 + D);
        QY *= (1 + D);
      }
#endif
    }
  }
  if (ok) {
    dz_lost = nSlices * sl;
    if (!check_aperture(X, Y, ap, aptilt, apc, aps))
      ok = false;
    else
      S += dist;
  }
  /* convertFromDipoleCanonicalCoordinates */
  {
    double f = expanded ? 1 / (1 + D) : 1 / sqrt(sqr(1 + D) - sqr(QX) - sqr(QY));
    QX *= f;
    QY *= f;
  }
  if (!ok) {
    /* convertFromCSBendCoords (src/csbend.c:4527-4548) then loss record */
    p.x = X * ct - Y * st;
    p.y = X * st + Y * ct;
    p.xp = QX * ct - QY * st;
    p.yp = QX * st + QY * ct;
    p.s = z_start + dz_lost;
    p.dp = Po * (1 + D);
    return false;
  }
  if (flags & BF_RADE2) /* radiation: delta post-adjusted (src/csbend.c:1270-1281) */
    D -= rad_edge_dp(d, BD_TE2, fmode, eo1, Fx_xy, Fy_xy, rho0, X, QX, Y, QY, D);
#if TRK_FAST
  if (flags & BF_RAD) {
    const double p0 = Po * (1 + dp0), p1 = Po * (1 + D);
    s = p1 / sqrt(sqr(p1) + 1) * s / (p0 / sqrt(sqr(p0) + 1)) + S;
  } else
    s += S;
#else
  if (flags & BF_ISR_ROUNDTRIP) {
    double p0 = Po * (1 + dp0);
    double beta0 = p0 / sqrt(sqr(p0) + 1);
    double p1 = Po * (1 + D);
    double beta1 = p1 / sqrt(sqr(p1) + 1);
    s = beta1 * s / beta0 + S;
  } else
    s += S;
#endif
  x = X;
  xp = QX;
  y = Y;
  yp = QY;
  dp = D;
  if (edge2)
    bend_edge(edge2, d, BD_E2, 1, rho_a, nidx, Fr + FR_CURV_LEN, expanded, x, xp, y, yp, s, dp);
  if (flags & BF_MISALIGN) {
    p.x = x * ct - y * st + __ldg(&d[BD_ET + 0]);
    p.y = x * st + y * ct + __ldg(&d[BD_ET + 2]);
    p.xp = xp * ct - yp * st + __ldg(&d[BD_ET + 1]);
    p.yp = xp * st + yp * ct + __ldg(&d[BD_ET + 3]);
    p.s = s + __ldg(&d[BD_ET + 4]);
    p.dp = dp;
    const double dxf = __ldg(&d[BD_DXF]), dyf = __ldg(&d[BD_DYF]), dzf = __ldg(&d[BD_DZF]);
    p.x += dxf + dzf * p.xp;
    p.y += dyf + dzf * p.yp;
    p.s += dzf * sqrt(1 + sqr(p.xp) + sqr(p.yp));
  } else {
    p.x = x;
    p.xp = xp;
    p.y = y;
    p.yp = yp;
    p.s = s;
    p.dp = dp;
  }
  return true;
}

#if !TRK_FAST
/* op_bend restricted to what a plain pure dipole reaches (OPK_DIPOLE: no
 * misalignment, tilt, radiation, field expansion or expanded Hamiltonian;
 * edges at most the linear kick), with the same operations in the same
 * order, the signed-zero-preserving tilt products of a loss included.  The
 * lean parity kernels take it so that the general body's other branches do
 * not weigh on their register allocation. */
__device__ __forceinline__ bool op_dipole_exact(const trk_op *__restrict__ op, Part &p, double Po, double z_start,
                                                const trk_aperture *ap) {
  const double *d = op->d;
  const int nSlices = __ldg(&op->i[0]);
  const int nSub = __ldg(&op->i[1]);
  const int edge1 = __ldg(&op->i[5]), edge2 = __ldg(&op->i[6]);
  const int flags = __ldg(&op->i[7]);
  const double rho0 = __ldg(&d[BD_RHO0]), rho_a = __ldg(&d[BD_RHOA]);
  double x = p.x, y = p.y, xp = p.xp, yp = p.yp, s = p.s, dp = p.dp;
  const double dp0 = p.dp;
  if (edge1 == EDGE_LIN1)
    edge_lin1(d, BD_E1, rho_a, x, xp, y, yp, dp);
  double X = x, QX, Y = y, QY, S = 0, D = dp;
  {
    double f = (1 + D) / sqrt(1 + sqr(xp) + sqr(yp));
    QX = xp * f;
    QY = yp * f;
  }
  double dist = 0, dz_lost = 0;
  int done = 0;
  bool ok = bend_dipole_exact(d, nSlices, nSub, rho0, (flags & BF_ISR_ROUNDTRIP) != 0, ap, false, 1.0, 0.0, X, QX,
                              Y, QY, D, dist, done);
  if (!ok)
    for (int k = 0; k < done; k++)
      dz_lost += __ldg(&d[BD_DSH + k % nSub]);
  if (ok) {
    dz_lost = nSlices * __ldg(&d[BD_SLICE]);
    if (!check_aperture(X, Y, ap, false, 1.0, 0.0))
      ok = false;
    else
      S += dist;
  }
  {
    double f = 1 / sqrt(sqr(1 + D) - sqr(QX) - sqr(QY));
    QX *= f;
    QY *= f;
  }
  if (!ok) {
    const double ct = __ldg(&d[BD_CT]), st = __ldg(&d[BD_ST]);
    p.x = X * ct - Y * st;
    p.y = X * st + Y * ct;
    p.xp = QX * ct - QY * st;
    p.yp = QX * st + QY * ct;
    p.s = z_start + dz_lost;
    p.dp = Po * (1 + D);
    return false;
  }
  if (flags & BF_ISR_ROUNDTRIP) {
    double p0 = Po * (1 + dp0);
    double beta0 = p0 / sqrt(sqr(p0) + 1);
    double p1 = Po * (1 + D);
    double beta1 = p1 / sqrt(sqr(p1) + 1);
    s = beta1 * s / beta0 + S;
  } else
    s += S;
  x = X;
  xp = QX;
  y = Y;
  yp = QY;
  dp = D;
  if (edge2 == EDGE_LIN1)
    edge_lin1(d, BD_E2, rho_a, x, xp, y, yp, dp);
  p.x = x;
  p.xp = xp;
  p.y = y;
  p.yp = yp;
  p.s = s;
  p.dp = dp;
  return true;
}
#endif

/* ----------------------------------------------------------------- RFCA */
/* add_to_particle_energy (src/simple_rfca.c:987-1006) */
__device__ __forceinline__ void add_energy(Part &p, double t, double Po, double dgamma) {
  double P = Po * (1 + p.dp);
  double gamma = sqrt(P * P + 1);
  double gamma1 = gamma + dgamma;
  if (gamma1 <= 1)
    gamma1 = 1 + 1e-7;
  double P1 = sqrt(gamma1 * gamma1 - 1);
  p.dp = (P1 - Po) / Po;
  p.s = t * TRK_C_MKS * P1 / gamma1;
  double Pz = P / sqrt(1 + sqr(p.xp) + sqr(p.yp));
  double Pz1 = sqrt(Pz * Pz + gamma1 * gamma1 - gamma * gamma);
  double PRatio = Pz / Pz1;
  p.xp *= PRatio;
  p.yp *= PRatio;
}

/* trackRfCavityWithWakes (src/simple_rfca.c:295-985), kick method,
 * traveling wave, per particle; ends with removeInvalidParticles. */
/* LOCK_PHASE / LINEARIZE set-up (src/simple_rfca.c:550-556): the locked
 * phase replaces the fiducial one; returns dgammaAve.  Out of line, as is
 * the linearized kick, so the common cavity carries neither. */
__device__ __noinline__ double rf_locked_phase(const double *__restrict__ d, int flags, double volt, double omega,
                                               double tAve, double &phase) {
  if (flags & RF_LOCK) {
    phase = __ldg(&d[RD_PHASE_LOCK]);
    return volt * M_SIN(phase);
  }
  return volt * M_SIN(omega * (tAve - 0.0) + phase);
}

/* the linearized kick (src/simple_rfca.c:603-604) */
__device__ __noinline__ double rf_linear_dgamma(double dgammaAve, double volt, double omega, double t, double tAve,
                                                double phase) {
  return dgammaAve + volt * omega * (t - tAve) * M_COS(omega * (tAve - 0.0) + phase);
}

__device__ __forceinline__ bool op_rf(const trk_op *__restrict__ op, Part &p, double Po, double z_end,
                                      const double *__restrict__ rf_phase, const double *__restrict__ rf_tave) {
  const double *d = op->d;
  const int nKicks = __ldg(&op->i[0]);
  const int slot = __ldg(&op->i[1]);
  const int flags = __ldg(&op->i[3]);
  const double omega = __ldg(&d[RD_OMEGA]), volt = __ldg(&d[RD_VOLT]), length = __ldg(&d[RD_LEN]);
  const double dtLight = __ldg(&d[RD_DTL]), tau = __ldg(&d[RD_TAU]);
  const double phase_fid = rf_phase[slot];
  double t0 = omega ? -phase_fid / omega : 0;
  double phase = phase_fid + __ldg(&d[RD_PHASE_ADD]);
  double dgamma = 0;
  if (flags & RF_SAME_DGAMMA)
    dgamma = volt * M_SIN(phase);
  /* LOCK_PHASE / LINEARIZE: the pass's mean arrival time (src/simple_rfca.c:500-556) */
  double tAve = 0, dgammaAve = 0;
  if (flags & (RF_LOCK | RF_LINEAR)) {
    tAve = rf_tave[slot];
    dgammaAve = rf_locked_phase(d, flags, volt, omega, tAve, phase);
  }
  if (flags & RF_OFFSET) {
    p.x -= __ldg(&d[RD_DX]);
    p.y -= __ldg(&d[RD_DY]);
  }
  double inverseF = 0;
  for (int ik = 0; ik < nKicks; ik++) {
    if (p.dp != -1) {
      double dc4 = length ? length / 2 * sqrt(1 + sqr(p.xp) + sqr(p.yp)) : 0;
      double P = Po * (1 + p.dp);
      double gamma = sqrt(sqr(P) + 1);
      double beta_i = P / gamma;
      double t = (p.s + dc4) / (TRK_C_MKS * beta_i) - 0.0;
      double dt = t - t0;
      if (dt < 0)
        dt = 0;
      if (!(flags & RF_SAME_DGAMMA)) {
        if (!(flags & RF_LINEAR)) {
          double phi = omega * (t - ((flags & RF_LOCK) ? tAve : 0) - ik * dtLight) + phase;
          double dfactor = tau ? sqrt(1 - exp(-dt / tau)) : 1;
          dgamma = volt * M_SIN(phi) * dfactor;
        } else
          dgamma = rf_linear_dgamma(dgammaAve, volt, omega, t, tAve, phase);
      }
      if (length) {
        if ((flags & RF_END1) && ik == 0) {
          inverseF = dgamma / (2 * gamma * length);
          p.xp -= p.x * inverseF;
          p.yp -= p.y * inverseF;
        }
        p.x += p.xp * length / 2;
        p.y += p.yp * length / 2;
        p.s += length / 2 * sqrt(1 + sqr(p.xp) + sqr(p.yp));
      }
      add_energy(p, t, Po, dgamma);
      double gamma1 = gamma + dgamma;
      if (gamma1 <= 1)
        p.dp = -1;
      else
        inverseF = -dgamma / (2 * gamma1 * length);
    }
    if (length) {
      p.x += p.xp * length / 2;
      p.y += p.yp * length / 2;
      p.s += length / 2 * sqrt(1 + sqr(p.xp) + sqr(p.yp));
      if ((flags & RF_END2) && ik == nKicks - 1) {
        p.xp -= p.x * inverseF;
        p.yp -= p.y * inverseF;
      }
    }
  }
  if (flags & RF_OFFSET) {
    p.x += __ldg(&d[RD_DX]);
    p.y += __ldg(&d[RD_DY]);
  }
  /* removeInvalidParticles (src/limit_amplitudes.c:~290-345) */
  if (isnan(p.x) || isnan(p.xp) || isnan(p.y) || isnan(p.yp) || isnan(p.s) || isnan(p.dp) || p.dp <= -1) {
    p.s = z_end;
    p.dp = Po * (1 + p.dp);
    return false;
  }
  return true;
}

#if TRK_FAST
/* OPK_MULT1 in the fast build: multipole_tracking2 for one normal multipole
 * with no misalignment, steering or end drifts (src/multipole.c:660-1084),
 * body unrolled by mult_body_fast.  The slope->momentum->slope round trip of
 * the reference before the body (src/multipole.c:1190-1228) is an identity
 * in exact arithmetic and is skipped. */
__device__ __forceinline__ bool op_mult1_fast(const trk_op *__restrict__ op, Part &p, double Po, double z_start,
                                              const trk_aperture *ap) {
  const int n_parts = __ldg(&op->i[0]);
  const int order = __ldg(&op->i[4]) & 0xff;
  const int flags = __ldg(&op->i[6]);
  const double *d = op->d;
  const bool aptilt = (flags & MF_APTILT) != 0;
  const double apc = __ldg(&d[MD_APC]), aps = __ldg(&d[MD_APS]);
  double x = p.x, xp = p.xp, y = p.y, yp = p.yp, s = 0;
  const double dp = p.dp;
  double dzLoss = 0;
  bool ok = !(isnan(x) || isnan(xp) || isnan(y) || isnan(yp) || fabs(x) > TRK_COORD_LIMIT ||
              fabs(y) > TRK_COORD_LIMIT || fabs(xp) > TRK_SLOPE_LIMIT || fabs(yp) > TRK_SLOPE_LIMIT);
  if (!ok)
    dzLoss = __ldg(&d[MD_DZFULL]); /* as in op_mult */
  if (ok) {
    const double r = (1 + dp) * rsqrt_fast(fma(yp, yp, fma(xp, xp, 1.0)));
    double qx = xp * r, qy = yp * r;
    int done = 0, rc;
    if (order == 1)
      rc = mult_body_fast<1>(d, n_parts, ap, aptilt, apc, aps, 0.0, 0.0, x, xp, y, yp, s, qx, qy, dp, done);
    else if (order == 2)
      rc = mult_body_fast<2>(d, n_parts, ap, aptilt, apc, aps, 0.0, 0.0, x, xp, y, yp, s, qx, qy, dp, done);
    else
      rc = mult_body_fast<3>(d, n_parts, ap, aptilt, apc, aps, 0.0, 0.0, x, xp, y, yp, s, qx, qy, dp, done);
    if (rc) {
      for (int k = 0; k < done; k++)
        dzLoss += __ldg(&d[MD_DSH + (k & 3)]);
      if (rc == 1) {
        p.x = x;
        p.y = y;
      }
      ok = false;
    } else {
      const double den = (1 + dp) * (1 + dp) - qx * qx - qy * qy;
      if (!(den > 0)) {
        for (int k = 0; k < done; k++)
          dzLoss += __ldg(&d[MD_DSH + (k & 3)]);
        ok = false;
      } else {
        const double ri = rsqrt_fast(den);
        xp = qx * ri;
        yp = qy * ri;
        p.x = x;
        p.xp = xp;
        p.y = y;
        p.yp = yp;
        p.s += s;
        p.dp = dp;
        if (isnan(x) || isnan(xp) || isnan(y) || isnan(yp) || fabs(x) > TRK_COORD_LIMIT ||
            fabs(y) > TRK_COORD_LIMIT || fabs(xp) > TRK_SLOPE_LIMIT || fabs(yp) > TRK_SLOPE_LIMIT) {
          for (int k = 0; k < done; k++)
            dzLoss += __ldg(&d[MD_DSH + (k & 3)]);
          ok = false;
        }
      }
    }
  }
  if (!ok) {
    p.s = z_start + dzLoss;
    p.dp = Po * (1 + p.dp);
  }
  return ok;
}

/* OPK_DIPOLE in the fast build: track_through_csbend for a pure dipole with
 * no misalignment and no edge kick (src/csbend.c:654-1434), body by
 * bend_dipole_fast. */
__device__ __forceinline__ bool op_dipole_fast(const trk_op *__restrict__ op, Part &p, double Po, double z_start,
                                               const trk_aperture *ap) {
  const double *d = op->d;
  const int nSlices = __ldg(&op->i[0]);
  const double rho0 = __ldg(&d[BD_RHO0]);
  const double D = p.dp;
  const double r = (1 + D) * rsqrt_fast(fma(p.yp, p.yp, fma(p.xp, p.xp, 1.0)));
  double X = p.x, Y = p.y, QX = p.xp * r;
  const double QY = p.yp * r;
  double dist = 0;
  int done = 0;
  bool ok = bend_dipole_fast<4>(d, nSlices, 4, rho0, ap, false, 1.0, 0.0, X, QX, Y, QY, D, dist, done);
  double dz_lost = 0;
  if (ok) {
    dz_lost = nSlices * __ldg(&d[BD_SLICE]);
    if (ap && !check_aperture(X, Y, ap, false, 1.0, 0.0))
      ok = false;
  } else
    for (int k = 0; k < done; k++)
      dz_lost += __ldg(&d[BD_DSH + (k & 3)]);
  const double f = rsqrt_fast((1 + D) * (1 + D) - QX * QX - QY * QY);
  p.x = X;
  p.y = Y;
  p.xp = QX * f;
  p.yp = QY * f;
  if (!ok) {
    p.s = z_start + dz_lost;
    p.dp = Po * (1 + D);
    return false;
  }
  p.s += dist;
  p.dp = D;
  return true;
}

/* OPK_CFBEND in the fast build: track_through_csbend for a combined-function
 * dipole (normal field expansion of order 4) with no misalignment and no edge
 * kick (src/csbend.c:654-1434), body by bend_cf_fast. */
__device__ __forceinline__ bool op_cfbend_fast(const trk_op *__restrict__ op, Part &p, double Po, double z_start,
                                               const trk_aperture *ap, const double *__restrict__ field) {
  const double *d = op->d;
  const int nSlices = __ldg(&op->i[0]);
  const double *fxy = field + __ldg(&op->i[4]);
  const double rho0 = __ldg(&d[BD_RHO0]);
  const double D = p.dp;
  const double r = (1 + D) * rsqrt_fast(fma(p.yp, p.yp, fma(p.xp, p.xp, 1.0)));
  double X = p.x, Y = p.y, QX = p.xp * r, QY = p.yp * r;
  double dist = 0;
  int done = 0;
  bool ok = bend_cf_fast(d, fxy, nSlices, rho0, ap, X, QX, Y, QY, D, dist, done);
  double dz_lost = 0;
  if (ok) {
    dz_lost = nSlices * __ldg(&d[BD_SLICE]);
    if (ap && !check_aperture(X, Y, ap, false, 1.0, 0.0))
      ok = false;
  } else
    for (int k = 0; k < done; k++)
      dz_lost += __ldg(&d[BD_DSH + (k & 3)]);
  const double f = rsqrt_fast((1 + D) * (1 + D) - QX * QX - QY * QY);
  p.x = X;
  p.y = Y;
  p.xp = QX * f;
  p.yp = QY * f;
  if (!ok) {
    p.s = z_start + dz_lost;
    p.dp = Po * (1 + D);
    return false;
  }
  p.s += dist;
  p.dp = D;
  return true;
}

/* Two particles through one pure dipole with their substep chains
 * interleaved: the body of each particle is a serial dependency chain
 * (sqrt -> reciprocal -> update), so a thread that carries two independent
 * chains keeps the FP64 pipe busier at the same occupancy.  Same arithmetic
 * per particle as op_dipole_fast; a slice that produced a non-finite value is
 * re-run for that particle with the reference's per-substep loss checks. */
struct DipoleState {
  double X, QX, F, QY, Y0, opd, f2;
  int done;
  bool ok;
};

__device__ __forceinline__ void dipole_begin(DipoleState &q, const Part &p) {
  q.opd = 1 + p.dp;
  const double r = q.opd * rsqrt_fast(fma(p.yp, p.yp, fma(p.xp, p.xp, 1.0)));
  q.X = p.x;
  q.Y0 = p.y;
  q.QX = p.xp * r;
  q.QY = p.yp * r;
  q.F = 0;
  q.f2 = q.opd * q.opd - q.QY * q.QY;
  q.done = 0;
}

__device__ __forceinline__ void dipole_step(DipoleState &q, double rho0, double sa, double ca, double omc) {
  const double fc = sqrt_nan(fma(-q.QX, q.QX, q.f2));
  const double saq = sa * q.QX;
  const double u = div_fast(rho0 + q.X, fma(ca, fc, -saq));
  q.QX = fma(sa, fc, ca * q.QX);
  q.F = fma(u, sa, q.F);
  q.X = fma(u, fma(omc, fc, saq), q.X);
}

__device__ __forceinline__ bool dipole_finish(DipoleState &q, Part &p, const double *__restrict__ d, int nSlices,
                                              double Po, double z_start, const trk_aperture *ap) {
  double dz_lost = 0;
  const double Y = q.Y0 + q.QY * q.F;
  bool ok = q.ok;
  if (ok) {
    dz_lost = nSlices * __ldg(&d[BD_SLICE]);
    if (ap && !check_aperture(q.X, Y, ap, false, 1.0, 0.0))
      ok = false;
  } else
    for (int k = 0; k < q.done; k++)
      dz_lost += __ldg(&d[BD_DSH + (k & 3)]);
  const double f = rsqrt_fast(q.opd * q.opd - q.QX * q.QX - q.QY * q.QY);
  p.x = q.X;
  p.y = Y;
  p.xp = q.QX * f;
  p.yp = q.QY * f;
  if (!ok) {
    p.s = z_start + dz_lost;
    p.dp = Po * q.opd; /* Po * (1 + delta) */
    return false;
  }
  p.s += q.opd * q.F;
  return true;
}

/* one slice for one particle with the reference's loss checks (rare path) */
__device__ __forceinline__ void dipole_slice_checked(DipoleState &q, const double *__restrict__ d, double rho0) {
  const SliceState r = dipole_slice_redo(d, 4, rho0, q.f2, q.X, q.QX, q.F, q.done);
  q.ok = r.ok;
  q.X = r.X;
  q.QX = r.QX;
  q.F = r.F;
  q.done = r.done;
}

__device__ __forceinline__ void op_dipole_fast2(const trk_op *__restrict__ op, Part &p0, Part &p1, bool &ok0,
                                                bool &ok1, double Po, double z_start, const trk_aperture *ap) {
  const double *d = op->d;
  const int nSlices = __ldg(&op->i[0]);
  const double rho0 = __ldg(&d[BD_RHO0]);
  DipoleState q0, q1;
  dipole_begin(q0, p0);
  dipole_begin(q1, p1);
  q0.ok = ok0;
  q1.ok = ok1;
  for (int i = 0; i < nSlices; i++) {
    if (ap) {
      if (q0.ok && !check_aperture(q0.X, q0.Y0 + q0.QY * q0.F, ap, false, 1.0, 0.0))
        q0.ok = false;
      if (q1.ok && !check_aperture(q1.X, q1.Y0 + q1.QY * q1.F, ap, false, 1.0, 0.0))
        q1.ok = false;
    }
    if (!(q0.f2 > 0))
      q0.ok = false;
    if (!(q1.f2 > 0))
      q1.ok = false;
    if (!q0.ok && !q1.ok)
      break;
    const double X0a = q0.X, QX0a = q0.QX, F0a = q0.F;
    const double X0b = q1.X, QX0b = q1.QX, F0b = q1.F;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const double sa = __ldg(&d[BD_SA + j]), ca = __ldg(&d[BD_CA + j]);
      const double omc = __ldg(&d[BD_OMC + j]);
      dipole_step(q0, rho0, sa, ca, omc);
      dipole_step(q1, rho0, sa, ca, omc);
      if (j == 3)
        break;
      const double c1 = __ldg(&d[BD_C1 + j]), c2 = __ldg(&d[BD_C2 + j]);
      q0.QX = fma(-c2, q0.X, q0.QX - c1);
      q1.QX = fma(-c2, q1.X, q1.QX - c1);
    }
    if (q0.ok) {
      if (isfinite(q0.X + q0.QX + q0.F))
        q0.done += 4;
      else {
        q0.X = X0a;
        q0.QX = QX0a;
        q0.F = F0a;
        dipole_slice_checked(q0, d, rho0);
      }
    } else {
      /* lost: keep the coordinates where the loss was found */
      q0.X = X0a;
      q0.QX = QX0a;
      q0.F = F0a;
    }
    if (q1.ok) {
      if (isfinite(q1.X + q1.QX + q1.F))
        q1.done += 4;
      else {
        q1.X = X0b;
        q1.QX = QX0b;
        q1.F = F0b;
        dipole_slice_checked(q1, d, rho0);
      }
    } else {
      /* lost: keep the coordinates where the loss was found */
      q1.X = X0b;
      q1.QX = QX0b;
      q1.F = F0b;
    }
  }
  if (ok0)
    ok0 = dipole_finish(q0, p0, d, nSlices, Po, z_start, ap);
  if (ok1)
    ok1 = dipole_finish(q1, p1, d, nSlices, Po, z_start, ap);
}
#endif

/* ------------------------------------------------------ after-element */
/* limit_amplitudes / elimit_amplitudes (src/limit_amplitudes.c:197-288,
 * 487-~620) for one particle; returns true if lost. */
__device__ __forceinline__ bool post_aperture_body(Part &p, const trk_aperture *__restrict__ ap, int extrapolate,
                                                   double z, double Po) {
  double xmax = ap->x_max, ymax = ap->y_max;
  if (ap->elliptical && xmax > 0 && ymax > 0) {
    if (isinf(p.x) || isinf(p.y) || isnan(p.x) || isnan(p.y)) {
      p.s = z;
      p.dp = sqrt(sqr(Po * (1 + p.dp)) + 1);
      return true;
    }
    const int xe = ap->xexp, ye = ap->yexp;
    const double a2 = ap->a2, b2 = ap->b2;
    if ((ipow_d(p.x, xe) / a2 + ipow_d(p.y, ye) / b2) > 1) {
      double dz = 0;
      if (extrapolate && xe == 2 && ye == 2) {
        double c0 = sqr(p.x) / a2 + sqr(p.y) / b2 - 1;
        double c1 = 2 * (p.x * p.xp / a2 + p.y * p.yp / b2);
        double c2 = sqr(p.xp) / a2 + sqr(p.yp) / b2;
        double det = sqr(c1) - 4 * c0 * c2;
        if (z > 0 && c2 && det >= 0) {
          if ((dz = (-c1 + sqrt(det)) / (2 * c2)) > 0)
            dz = (-c1 - sqrt(det)) / (2 * c2);
          if ((z + dz) < 0)
            dz = -z;
          p.x += dz * p.xp;
          p.y += dz * p.yp;
        }
      }
      p.s = z + dz;
      p.dp = sqrt(sqr(Po * (1 + p.dp)) + 1);
      return true;
    }
    return false;
  }
  if (xmax < 0 && ymax < 0)
    return false;
  int is_out = 0;
  if (xmax > 0 && fabs(p.x) > xmax)
    is_out += 1;
  if (ymax > 0 && fabs(p.y) > ymax)
    is_out += 2;
  if (isinf(p.x) || isinf(p.y) || isnan(p.x) || isnan(p.y))
    is_out += 4;
  if (!is_out)
    return false;
  double dz = 0;
  if (!(is_out & 4) && extrapolate) {
    double dzx = -1.7976931348623157e308, dzy = -1.7976931348623157e308;
    if ((is_out & 1) && p.xp != 0)
      dzx = (p.x - (p.xp < 0 ? -1 : 1) * xmax) / p.xp;
    if ((is_out & 2) && p.yp != 0)
      dzy = (p.y - (p.yp < 0 ? -1 : 1) * ymax) / p.yp;
    if (dzx > dzy)
      dz = -dzx;
    else
      dz = -dzy;
    if (dz == -1.7976931348623157e308)
      dz = 0;
  }
  p.x += dz * p.xp;
  p.y += dz * p.yp;
  p.s = z + dz;
  p.dp = Po * (1 + p.dp);
  return true;
}

/* True when the reference's after-element aperture test certainly keeps the
 * particle (finite x, y inside the rectangle or ellipse, evaluated with the
 * reference's arithmetic); anything else goes to post_aperture_full. */
__device__ __forceinline__ bool post_aperture_inside(const Part &p, const trk_aperture *__restrict__ ap) {
  const double xmax = __ldg(&ap->x_max), ymax = __ldg(&ap->y_max);
  if (!(isfinite(p.x) && isfinite(p.y)))
    return false;
  if (__ldg(&ap->elliptical) && xmax > 0 && ymax > 0)
    return (ipow_d(p.x, __ldg(&ap->xexp)) / __ldg(&ap->a2) + ipow_d(p.y, __ldg(&ap->yexp)) / __ldg(&ap->b2)) <= 1;
  return (!(xmax > 0) || fabs(p.x) <= xmax) && (!(ymax > 0) || fabs(p.y) <= ymax);
}

struct PartLoss {
  Part p;
  int lost;
};

/* Out of line, with the particle passed and returned by value (a reference
 * would pin the caller's coordinates in local memory): it only runs for
 * particles that post_aperture_inside could not clear. */
__device__ __noinline__ PartLoss post_aperture_full(Part p, const trk_aperture *__restrict__ ap, int extrapolate,
                                                    double z, double Po) {
  PartLoss r;
  r.lost = post_aperture_body(p, ap, extrapolate, z, Po);
  r.p = p;
  return r;
}

__device__ __forceinline__ bool post_aperture(Part &p, const trk_aperture *__restrict__ ap, int extrapolate, double z,
                                              double Po) {
  if (post_aperture_inside(p, ap))
    return false;
  const PartLoss r = post_aperture_full(p, ap, extrapolate, z, Po);
  p = r.p;
  return r.lost != 0;
}

/* DRIF through its order-1/2 matrix (src/compute_matrices.c:391-413,
 * src/matrix.c:310-422): the structural zeros contribute only signed zeros
 * for finite input and NaN when any coordinate is not finite. */
__device__ __forceinline__ void op_drift(const trk_op *__restrict__ op, Part &p) {
  const double L = __ldg(&op->d[DD_L]);
  const int order = __ldg(&op->i[0]);
#if TRK_FAST
  /* any non-finite coordinate makes x and y NaN, so the after-element filter
   * records the loss here as the reference does */
  const double nan_if = (p.s + p.dp) * 0.0;
  p.x += nan_if;
  p.y += nan_if;
#else
  if (!(isfinite(p.x) && isfinite(p.xp) && isfinite(p.y) && isfinite(p.yp) && isfinite(p.s) && isfinite(p.dp))) {
    const double qnan = __longlong_as_double(0x7ff8000000000000ULL);
    p.x = p.xp = p.y = p.yp = p.s = p.dp = qnan;
    return;
  }
#endif
  double xp = p.xp, yp = p.yp;
  double x1 = L * xp + p.x;
  double y1 = L * yp + p.y;
  double s1;
  if (order >= 2) {
    const double T = __ldg(&op->d[DD_T]);
    double a = L + p.s;
    double b = (T * yp) * yp;
#if TRK_FAST
    s1 = (a + b) + (T * xp) * xp;
#else
    s1 = __dadd_rn(__dadd_rn(a, b), __dmul_rn(__dmul_rn(T, xp), xp));
#endif
  } else
    s1 = L + p.s;
  p.x = x1;
  p.y = y1;
  p.s = s1;
}

/* ------------------------------------------------------------- kernels */
__device__ __forceinline__ void load_part(const TrackArgs &a, long i, Part &p) {
  p.x = a.x[i];
  p.xp = a.xp[i];
  p.y = a.y[i];
  p.yp = a.yp[i];
  p.s = a.s[i];
  p.dp = a.dp[i];
}

__device__ __forceinline__ void store_part(const TrackArgs &a, long i, const Part &p) {
  a.x[i] = p.x;
  a.xp[i] = p.xp;
  a.y[i] = p.y;
  a.yp[i] = p.yp;
  a.s[i] = p.s;
  a.dp[i] = p.dp;
}

/* Track one particle through ops [ob, oe) for passes [pb, pe).  Returns
 * false if it was lost (loss recorded). */
/* The per-element header fields every particle reads, fetched with three
 * 16-byte loads (trk_op starts with 8 int32 fields; z_start and z_end follow
 * at byte 64). */
struct OpHead {
  int kind, elem, ap_post, ap_in, extrapolate, no_aperture;
  double z_start, z_end;
};
static_assert(offsetof(trk_op, z_start) == 64 && sizeof(trk_op) % 16 == 0, "trk_op header layout");

__device__ __forceinline__ OpHead load_head(const trk_op *__restrict__ op, int var) {
  const int4 h0 = __ldg(reinterpret_cast<const int4 *>(op));
  const int4 h1 = __ldg(reinterpret_cast<const int4 *>(op) + 1);
  const double2 z = __ldg(reinterpret_cast<const double2 *>(&op->z_start));
  OpHead h;
  h.kind = h0.x;
  h.elem = h0.y;
  h.ap_post = var ? h0.w : h0.z;
  h.ap_in = var ? h1.y : h1.x;
  h.extrapolate = h1.z;
  h.no_aperture = h1.w;
  h.z_start = z.x;
  h.z_end = z.y;
  return h;
}

/* After-element filters of do_tracking (src/do_tracking.c:2506-2524 MAXAMP
 * aperture, :2675-2684 NaN/inf filter) and the loss record of one particle. */
__device__ __forceinline__ bool after_element(const TrackArgs &a, const OpHead &h, Part &p, bool ok, long i,
                                              long pass) {
  if (ok && !h.no_aperture && h.ap_post >= 0 && !a.element_only)
    ok = !post_aperture(p, a.aps + h.ap_post, h.extrapolate, h.z_end, a.Po);
  if (ok && !a.element_only && (isinf(p.x) || isinf(p.y) || isnan(p.x) || isnan(p.y))) {
    p.s = h.z_end;
    p.dp = a.Po * (1 + p.dp);
    ok = false;
  }
  if (!ok) {
    a.lost_pass[i] = (int32_t)pass;
    a.lost_elem[i] = h.elem;
  }
  return ok;
}

/* LEAN: 0 every element kind; 1 the kinds of lean lattices (no general
 * multipole or bend bodies); 2 as 1 plus combined-function bends, a flavour
 * of its own because their body, inlined into the loop, costs lattices
 * without them 3 % (register allocation of the whole loop) */
template <int LEAN>
__device__ __forceinline__ bool track_particle(const TrackArgs &a, const trk_op *__restrict__ ops, Part &p, long i) {
  for (long pass = a.pass_begin; pass < a.pass_end; pass++) {
    const int var = (pass == a.fresh_pass) ? 0 : 1;
    for (int k = a.op_begin; k < a.op_end; k++) {
      const trk_op *op = ops + k;
      const OpHead h = load_head(op, var);
      const trk_aperture *ap_in = h.ap_in >= 0 ? a.aps + h.ap_in : nullptr;
      bool ok = true;
      switch (h.kind) {
      case OPK_DRIFT:
        op_drift(op, p);
        break;
      case OPK_EDRIFT:
      case OPK_RFDRIFT:
        exact_drift(p, __ldg(&op->d[DD_L]));
        break;
      case OPK_MULT1:
#if TRK_FAST
        ok = op_mult1_fast(op, p, a.Po, h.z_start, ap_in);
#else
        ok = op_mult(op, p, a.Po, h.z_start, ap_in);
#endif
        break;
      case OPK_DIPOLE:
#if TRK_FAST
        ok = op_dipole_fast(op, p, a.Po, h.z_start, ap_in);
#else
        ok = op_dipole_exact(op, p, a.Po, h.z_start, ap_in);
#endif
        break;
      case OPK_CFBEND:
#if TRK_FAST
        if (LEAN != 1)
          ok = op_cfbend_fast(op, p, a.Po, h.z_start, ap_in, a.field);
#else
        if (LEAN != 1) /* flavour 1 lattices hold no combined-function bend */
          ok = op_bend(op, p, a.Po, h.z_start, ap_in, a.field);
#endif
        break;
      case OPK_RF:
        ok = op_rf(op, p, a.Po, h.z_end, a.rf_phase, a.rf_tave);
        break;
      case OPK_MULT:
      case OPK_BEND:
        if (!LEAN) {
          IsrKey key;
          key.seed = a.isr_seed;
          key.id = (unsigned int)(long long)__ldg(&a.id[i]);
          key.pass = (unsigned int)pass;
          key.elem = (unsigned int)k;
          key.limit = a.isr_limit;
          key.single = a.n == 1;
          if (h.kind == OPK_MULT)
            ok = op_mult(op, p, a.Po, h.z_start, ap_in, &key);
          else
            ok = op_bend(op, p, a.Po, h.z_start, ap_in, a.field, &key);
        }
        break;
      default:
        break;
      }
      if (!after_element(a, h, p, ok, i, pass))
        return false;
    }
  }
  return true;
}

/* Ensemble variant v of particle i: offsets[v] <= i < offsets[v+1] (the
 * variants hold the same element structure with other values). */
__device__ __forceinline__ int ens_variant(const long *__restrict__ offsets, int n_variants, long i) {
  int lo = 0, hi = n_variants;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&offsets[mid]) <= i)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

/* Kernel variants (block size, minimum resident blocks per SM) trade
 * registers against occupancy; trk_run.variant or the autotuner picks one. */
template <int BLOCK, int MINB, int LEAN>
__global__ void __launch_bounds__(BLOCK, MINB) track_kernel(TrackArgs a) {
  const long stride = (long)gridDim.x * blockDim.x;
  const long n = a.live ? __ldg(a.live_n) : a.n;
  for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
    const long i = a.live ? __ldg(&a.live[k]) : k;
    if (a.lost_pass[i] >= 0)
      continue;
    const trk_op *ops = a.ops;
    if (a.ens_offsets) /* ensemble: the records of this particle's variant */
      ops += (long)ens_variant(a.ens_offsets, a.ens_variants, i) * a.ens_ops;
    Part p;
    load_part(a, i, p);
    track_particle<LEAN>(a, ops, p, i);
    store_part(a, i, p);
  }
}

#if TRK_FAST
__device__ __forceinline__ bool lean_op(const TrackArgs &a, const trk_op *__restrict__ op, const OpHead &h, Part &p,
                                        const trk_aperture *ap_in) {
  const double z_start = h.z_start;
  switch (h.kind) {
  case OPK_DRIFT:
    op_drift(op, p);
    return true;
  case OPK_EDRIFT:
  case OPK_RFDRIFT:
    exact_drift(p, __ldg(&op->d[DD_L]));
    return true;
  case OPK_MULT1:
    return op_mult1_fast(op, p, a.Po, z_start, ap_in);
  case OPK_DIPOLE:
    return op_dipole_fast(op, p, a.Po, z_start, ap_in);
  case OPK_CFBEND:
    return op_cfbend_fast(op, p, a.Po, z_start, ap_in, a.field);
  case OPK_RF:
    return op_rf(op, p, a.Po, h.z_end, a.rf_phase, a.rf_tave);
  default:
    return true;
  }
}

/* Two particles per thread (lean lattices, fast build): particles i and
 * i + BLOCK of the block's tile. */
template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) track_kernel2(TrackArgs a) {
  const long tile = 2L * BLOCK;
  const long n = a.live ? __ldg(a.live_n) : a.n;
  for (long base = (long)blockIdx.x * tile; base < n; base += (long)gridDim.x * tile) {
    const long k0 = base + threadIdx.x, k1 = k0 + BLOCK;
    const long i0 = k0 < n && a.live ? __ldg(&a.live[k0]) : k0;
    const long i1 = k1 < n && a.live ? __ldg(&a.live[k1]) : k1;
    bool al0 = k0 < n && a.lost_pass[i0] < 0;
    bool al1 = k1 < n && a.lost_pass[i1] < 0;
    if (!al0 && !al1)
      continue;
    Part p0, p1;
    if (al0)
      load_part(a, i0, p0);
    else
      p0 = Part{0, 0, 0, 0, 0, 0};
    if (al1)
      load_part(a, i1, p1);
    else
      p1 = Part{0, 0, 0, 0, 0, 0};
    const bool was0 = al0, was1 = al1;
    for (long pass = a.pass_begin; pass < a.pass_end && (al0 || al1); pass++) {
      const int var = (pass == a.fresh_pass) ? 0 : 1;
      for (int k = a.op_begin; k < a.op_end && (al0 || al1); k++) {
        const trk_op *op = a.ops + k;
        const OpHead h = load_head(op, var);
        const trk_aperture *ap_in = h.ap_in >= 0 ? a.aps + h.ap_in : nullptr;
        bool ok0 = al0, ok1 = al1;
        if (h.kind == OPK_DIPOLE) {
          op_dipole_fast2(op, p0, p1, ok0, ok1, a.Po, h.z_start, ap_in);
        } else {
          if (al0)
            ok0 = lean_op(a, op, h, p0, ap_in);
          if (al1)
            ok1 = lean_op(a, op, h, p1, ap_in);
        }
        if (al0)
          al0 = after_element(a, h, p0, ok0, i0, pass);
        if (al1)
          al1 = after_element(a, h, p1, ok1, i1, pass);
      }
    }
    if (was0)
      store_part(a, i0, p0);
    if (was1)
      store_part(a, i1, p1);
  }
}
#endif

/* computeTimeCoordinatesOnly (src/trwake.c:519-527), rounded step by step
 * in both builds so the statistics, binning and kick kernels agree. */
__device__ __forceinline__ double wake_time(double Po, double dp, double s) {
  double P = __dmul_rn(Po, __dadd_rn(dp, 1.0));
  double num = __dmul_rn(s, __dsqrt_rn(__dadd_rn(__dmul_rn(P, P), 1.0)));
  return __ddiv_rn(num, __dmul_rn(TRK_C_MKS, P));
}

/* bin index (long)((t - tmin)/dt + 0.5) of binTimeDistribution (src/wake.c:509) */
__device__ __forceinline__ long wake_bin(double t, double tmin, double dt) {
  return (long)__dadd_rn(__ddiv_rn(__dsub_rn(t, tmin), dt), 0.5);
}

/* --------------------------------------------------------- reductions */
/* Sum of per-particle times for WAKE (computeTimeCoordinatesOnly,
 * src/trwake.c:519-527) or the RFCA "tmean" fiducial (findFiducialTime,
 * src/simple_rfca.c:191-230), in double-double so the block partials do not
 * depend on the launch shape; min/max and the survivor count alongside. */
__global__ void __launch_bounds__(TRK_BLOCK) time_stats_kernel(TimeStatsArgs a) {
  __shared__ double sh_hi[TRK_BLOCK], sh_lo[TRK_BLOCK], sh_min[TRK_BLOCK], sh_max[TRK_BLOCK];
  __shared__ long long sh_n[TRK_BLOCK];
  trkcr_dd acc = trkcr_make(0.0, 0.0);
  double tmin = 1.7976931348623157e308, tmax = -1.7976931348623157e308;
  long long cnt = 0;
  /* particles are assigned to blocks in fixed chunks so the result does
   * not depend on the grid size */
  const long chunk = a.chunk;
  for (long c = blockIdx.x; c * chunk < a.n; c += gridDim.x) {
    const long lo = c * chunk, hi = min(a.n, lo + chunk);
    trkcr_dd cacc = trkcr_make(0.0, 0.0);
    for (long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
      if (a.lost_pass[i] >= 0)
        continue;
      double t;
      if (a.mode == 0) {
        t = wake_time(a.Po, a.dp[i], a.s[i]);
      } else {
        double p = a.Po * (1 + a.dp[i]);
        double beta = p / sqrt(p * p + 1);
        t = (a.s[i] + a.sOffset) / (TRK_C_MKS * beta);
      }
      cacc = trkcr_add(cacc, trkcr_make(t, 0.0));
      tmin = fmin(tmin, t);
      tmax = fmax(tmax, t);
      cnt++;
    }
    acc = trkcr_add(acc, cacc);
  }
  const int tid = threadIdx.x;
  sh_hi[tid] = acc.hi;
  sh_lo[tid] = acc.lo;
  sh_min[tid] = tmin;
  sh_max[tid] = tmax;
  sh_n[tid] = cnt;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (tid < w) {
      trkcr_dd u = trkcr_add(trkcr_make(sh_hi[tid], sh_lo[tid]), trkcr_make(sh_hi[tid + w], sh_lo[tid + w]));
      sh_hi[tid] = u.hi;
      sh_lo[tid] = u.lo;
      sh_min[tid] = fmin(sh_min[tid], sh_min[tid + w]);
      sh_max[tid] = fmax(sh_max[tid], sh_max[tid + w]);
      sh_n[tid] += sh_n[tid + w];
    }
    __syncthreads();
  }
  if (tid == 0) {
    a.part_hi[blockIdx.x] = sh_hi[0];
    a.part_lo[blockIdx.x] = sh_lo[0];
    a.part_min[blockIdx.x] = sh_min[0];
    a.part_max[blockIdx.x] = sh_max[0];
    a.part_n[blockIdx.x] = sh_n[0];
  }
}

/* Combine block partials in index order; write {sum, n, min, max}. */
/* Sum of the block partials: 256 threads each add a strided subset in order,
 * then a fixed-order tree; out = {sum, count, min, max, sum_hi, sum_lo} with
 * sum the double-double total rounded once. */
#define TRK_FINISH_THREADS 256
__global__ void __launch_bounds__(TRK_FINISH_THREADS) time_stats_finish_kernel(TimeStatsArgs a, int nblocks) {
  __shared__ double s_hi[TRK_FINISH_THREADS], s_lo[TRK_FINISH_THREADS], s_min[TRK_FINISH_THREADS],
    s_max[TRK_FINISH_THREADS];
  __shared__ long long s_n[TRK_FINISH_THREADS];
  const int t = threadIdx.x;
  trkcr_dd acc = trkcr_make(0.0, 0.0);
  double tmin = 1.7976931348623157e308, tmax = -1.7976931348623157e308;
  long long n = 0;
  for (int b = t; b < nblocks; b += TRK_FINISH_THREADS) {
    acc = trkcr_add(acc, trkcr_make(a.part_hi[b], a.part_lo[b]));
    tmin = fmin(tmin, a.part_min[b]);
    tmax = fmax(tmax, a.part_max[b]);
    n += a.part_n[b];
  }
  s_hi[t] = acc.hi;
  s_lo[t] = acc.lo;
  s_min[t] = tmin;
  s_max[t] = tmax;
  s_n[t] = n;
  __syncthreads();
  for (int w = TRK_FINISH_THREADS / 2; w > 0; w >>= 1) {
    if (t < w) {
      const trkcr_dd r = trkcr_add(trkcr_make(s_hi[t], s_lo[t]), trkcr_make(s_hi[t + w], s_lo[t + w]));
      s_hi[t] = r.hi;
      s_lo[t] = r.lo;
      s_min[t] = fmin(s_min[t], s_min[t + w]);
      s_max[t] = fmax(s_max[t], s_max[t + w]);
      s_n[t] += s_n[t + w];
    }
    __syncthreads();
  }
  if (t == 0) {
    a.out[0] = __dadd_rn(s_hi[0], s_lo[0]);
    a.out[1] = (double)s_n[0];
    a.out[2] = s_min[0];
    a.out[3] = s_max[0];
    a.out[4] = s_hi[0];
    a.out[5] = s_lo[0];
  }
}

/* Combine the statistics all-gathered from `ranks` ranks (6 doubles each, as
 * written by time_stats_finish_kernel) in rank order. */
__global__ void stats_combine_kernel(const double *gathered, int ranks, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0)
    return;
  trkcr_dd acc = trkcr_make(0.0, 0.0);
  double n = 0, tmin = 1.7976931348623157e308, tmax = -1.7976931348623157e308;
  for (int r = 0; r < ranks; r++) {
    const double *g = gathered + 6 * r;
    acc = trkcr_add(acc, trkcr_make(g[4], g[5]));
    n += g[1];
    tmin = fmin(tmin, g[2]);
    tmax = fmax(tmax, g[3]);
  }
  out[0] = __dadd_rn(acc.hi, acc.lo);
  out[1] = n;
  out[2] = tmin;
  out[3] = tmax;
  out[4] = acc.hi;
  out[5] = acc.lo;
}

/* RFCA fiducial: phase_fiducial = -omega * tmean (src/simple_rfca.c:412-445) */
__global__ void rf_fiducial_kernel(const double *stats, double omega, double t_reference, double *rf_phase, int slot,
                                   int *status) {
  if (threadIdx.x != 0 || blockIdx.x != 0)
    return;
  double t0;
  if (t_reference != -1)
    t0 = t_reference;
  else {
    if (stats[1] <= 0) {
      atomicOr(status, TRK_STATUS_NO_PARTICLES);
      t0 = 0;
    } else
      t0 = stats[0] / stats[1];
  }
  rf_phase[slot] = -omega * t0;
}

/* the mean arrival time of the pass for LOCK_PHASE / LINEARIZE: the same
 * sum as the "tmean" fiducial's, divided by the particle count */
__global__ void rf_tave_kernel(const double *stats, double *rf_tave, int slot) {
  if (threadIdx.x != 0 || blockIdx.x != 0)
    return;
  rf_tave[slot] = stats[0] / stats[1];
}

/* ------------------------------------------------------------ wakes */

/* Wake geometry of one pass (src/wake.c:118-190, src/trwake.c:105-150) */
__global__ void wake_setup_kernel(WakeArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0)
    return;
  const double *st = a.stats;
  double n = st[1];
  WakeState *w = a.state;
  w->nb = 0;
  if (n <= 0)
    return;
  double tmean = a.transverse ? 0.0 : st[0] / n;
  double tmin = st[2], tmax = st[3];
  if ((tmax - tmin) > a.wake_span && !a.allow_long_beam) {
    atomicOr(a.status, TRK_STATUS_LONG_BEAM);
    return;
  }
  long nb;
  if (a.n_bins) {
    nb = a.n_bins;
    tmin = tmean - a.dt * nb / 2.0;
  } else {
    nb = (long)((tmax - tmin) / a.dt + 3);
    tmin -= a.dt;
  }
  if (nb > a.max_bins) {
    atomicOr(a.status, TRK_STATUS_TOO_MANY_BINS);
    return;
  }
  w->nb = nb;
  w->tmin = tmin;
  w->ramp = (a.pass >= a.ramp_passes - 1) ? 1.0 : (a.pass + 1.0) / a.ramp_passes;
  if (a.macro_mode == 0)
    w->macro = a.macro_charge;
  else if (a.macro_mode == 1)
    w->macro = a.charge / n; /* set_up_wake: charge / particles on pass 0 (src/wake.c:350-358) */
}

/* Bin particle times (binTimeDistribution, src/wake.c:498-518): integer
 * counts through a shared-memory histogram, then one global atomic per
 * non-empty bin per block.  Transverse wakes also sum x-dx and y-dy per bin
 * (binTransverseTimeDistribution, src/trwake.c:610-641). */
__global__ void __launch_bounds__(TRK_BLOCK) wake_bin_kernel(WakeArgs a) {
  extern __shared__ unsigned int sh_cnt[];
  const WakeState *w = a.state;
  const long nb = w->nb;
  if (nb <= 0)
    return;
  const bool use_smem = nb <= a.smem_bins && !a.transverse;
  if (use_smem) {
    for (long b = threadIdx.x; b < nb; b += blockDim.x)
      sh_cnt[b] = 0;
    __syncthreads();
  }
  const double tmin = w->tmin, dt = a.dt;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    if (a.lost_pass[i] >= 0)
      continue;
    double t = wake_time(a.Po, a.dp[i], a.s[i]);
    long ib = wake_bin(t, tmin, dt);
    if (ib < 0 || ib > nb - 1)
      continue;
    if (a.transverse) {
      double vx, vy;
      if (a.x_power == 1)
        vx = a.x[i] - a.tdx;
      else if (a.x_power < 1)
        vx = 1;
      else
        vx = ipow_d(a.x[i] - a.tdx, a.x_power);
      if (a.y_power == 1)
        vy = a.y[i] - a.tdy;
      else if (a.y_power < 1)
        vy = 1;
      else
        vy = ipow_d(a.y[i] - a.tdy, a.y_power);
      atomicAdd(&a.hist_x[ib], vx);
      atomicAdd(&a.hist_y[ib], vy);
    } else if (use_smem) {
      atomicAdd(&sh_cnt[ib], 1u);
    } else {
      atomicAdd(&a.counts[ib], 1ull);
    }
  }
  if (use_smem) {
    __syncthreads();
    for (long b = threadIdx.x; b < nb; b += blockDim.x)
      if (sh_cnt[b])
        atomicAdd(&a.counts[b], (unsigned long long)sh_cnt[b]);
  }
}

/* convolveArrays (src/wake.c:480-496) in the reference's summation order,
 * one output bin per thread; scaled by Q_macro * sign * FACTOR * ramp
 * (src/wake.c:254-261). */
__global__ void wake_convolve_kernel(WakeArgs a, int plane) {
  const WakeState *w = a.state;
  const long nb = w->nb;
  const long ib = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (ib > nb)
    return;
  double *V = plane ? a.V_y : a.V;
  if (ib == nb) {
    V[nb] = 0;
    return;
  }
  const double *W = plane ? a.W_y : a.W;
  const long n2 = a.wake_points;
  long ib2 = ib + a.i0, ib1 = 0;
  if (ib2 >= n2) {
    long di = ib2 - n2 + 1;
    ib1 += di;
    ib2 -= di;
  }
  double out = 0;
  if (a.transverse) {
    const double *I = plane ? a.hist_y : a.hist_x;
    for (; ib1 < nb && ib2 >= 0; ib1++, ib2--)
      out += I[ib1] * W[ib2];
  } else {
    for (; ib1 < nb && ib2 >= 0; ib1++, ib2--)
      out += (double)a.counts[ib1] * W[ib2];
  }
  double factor = w->macro * TRK_PARTICLE_REL_SIGN * a.factor;
  if (a.transverse)
    factor *= (plane ? a.yfactor : a.xfactor) * w->ramp;
  else
    factor *= w->ramp;
  V[ib] = out * factor;
}

/* applyLongitudinalWakeKicks (src/wake.c:306-330) / applyTransverseWakeKicks
 * (src/trwake.c:289-314), then the element's after-element filters. */
__global__ void __launch_bounds__(TRK_BLOCK) wake_kick_kernel(WakeArgs a) {
  const WakeState *w = a.state;
  const long nb = w->nb;
  const double tmin = w->tmin, dt = a.dt;
  const long stride = (long)gridDim.x * blockDim.x;
  const double mass = 1e6 * TRK_ME_MEV * TRK_PARTICLE_REL_SIGN;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    if (a.lost_pass[i] >= 0)
      continue;
    Part p;
    p.x = a.x[i];
    p.xp = a.xp[i];
    p.y = a.y[i];
    p.yp = a.yp[i];
    p.s = a.s[i];
    p.dp = a.dp[i];
    if (nb > 0) {
      double t = wake_time(a.Po, p.dp, p.s);
      long ib = wake_bin(t, tmin, dt);
      if (ib >= 0 && ib <= nb - 1) {
        if (!a.transverse) {
          double dgam;
          if (a.interpolate) {
            double dt1 = t - (tmin + dt * ib);
            if ((dt1 < 0 && ib) || ib == nb - 1) {
              ib--;
              dt1 += dt;
            }
            dgam = (a.V[ib] + (a.V[ib + 1] - a.V[ib]) / dt * dt1) / mass;
          } else
            dgam = a.V[ib] / mass;
          if (dgam)
            add_energy(p, t, a.Po, -dgam);
        } else {
          double pz = a.Po * (1 + p.dp) / sqrt(1 + sqr(p.xp) + sqr(p.yp));
          for (int plane = 0; plane < 2; plane++) {
            if (!(a.active_planes & (1 << plane)))
              continue;
            const double *V = plane ? a.V_y : a.V;
            long jb = ib;
            double Vi;
            if (a.interpolate) {
              double dt1 = t - (tmin + dt * jb);
              if ((dt1 < 0 && jb) || jb == nb - 1) {
                jb--;
                dt1 += dt;
              }
              Vi = V[jb] + (V[jb + 1] - V[jb]) / dt * dt1;
            } else
              Vi = V[jb];
            int exponent = plane ? a.y_probe : a.x_probe;
            if (exponent)
              Vi *= ipow_d(plane ? p.y : p.x, exponent);
            if (Vi) {
              if (plane)
                p.yp += Vi / mass / pz;
              else
                p.xp += Vi / mass / pz;
            }
          }
        }
      }
    }
    if (a.untilt)
      rotate(p, a.tilt_c, a.tilt_s);
    /* after-element filters of the wake element */
    bool lost = false;
    if (a.ap_post >= 0)
      lost = post_aperture(p, a.aps + a.ap_post, 0, a.z_end, a.Po);
    if (!lost && !a.element_only && (isinf(p.x) || isinf(p.y) || isnan(p.x) || isnan(p.y))) {
      p.s = a.z_end;
      p.dp = a.Po * (1 + p.dp);
      lost = true;
    }
    if (lost) {
      a.lost_pass[i] = (int32_t)a.pass;
      a.lost_elem[i] = a.elem;
    }
    a.x[i] = p.x;
    a.xp[i] = p.xp;
    a.y[i] = p.y;
    a.yp[i] = p.yp;
    a.s[i] = p.s;
    a.dp[i] = p.dp;
  }
}

/* rotateBeamCoordinatesForMisalignment over the surviving beam (TRWAKE TILT) */
__global__ void rotate_kernel(TrackArgs a, double ca, double sa) {
  const long stride = (long)gridDim.x * blockDim.x;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    if (a.lost_pass[i] >= 0)
      continue;
    Part p;
    load_part(a, i, p);
    rotate(p, ca, sa);
    store_part(a, i, p);
  }
}

/* After-element filter on its own (limit_amplitudes / elimit_amplitudes,
 * src/limit_amplitudes.c:197-288, 487-620): `ap` with x_max = y_max =
 * DBL_MAX is the NaN filter.  mode 1: removeInvalidParticles
 * (:289-331): a NaN coordinate or delta <= -1 loses the particle at z. */
__global__ void limit_kernel(TrackArgs a, trk_aperture ap, int mode, int extrapolate, double z, long pass, int elem) {
  const long stride = (long)gridDim.x * blockDim.x;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    if (a.lost_pass[i] >= 0)
      continue;
    Part p;
    load_part(a, i, p);
    bool lost;
    if (mode == 1) {
      lost = isnan(p.x) || isnan(p.xp) || isnan(p.y) || isnan(p.yp) || isnan(p.s) || isnan(p.dp) || p.dp <= -1;
      if (lost) {
        p.s = z;
        p.dp = a.Po * (1 + p.dp);
      }
    } else
      lost = post_aperture_body(p, &ap, extrapolate, z, a.Po);
    if (lost) {
      store_part(a, i, p);
      a.lost_pass[i] = (int32_t)pass;
      a.lost_elem[i] = elem;
    }
  }
}

/* track_particles for a first- or second-order transport matrix
 * (src/matrix.c:212-469 with TURBO_FASTMATTRACK=3): C[6], R[6][6] and the
 * lower triangle T[i][j][k], k <= j, packed as 21 values per i, summed in the
 * reference's order (i, j, k descending). */
__global__ void matrix_kernel(TrackArgs a, const double *__restrict__ m, int order) {
  const double *C = m, *R = m + 6, *T = m + 42;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    if (a.lost_pass[i] >= 0)
      continue;
    Part p;
    load_part(a, i, p);
    const double ini[6] = {p.x, p.xp, p.y, p.yp, p.s, p.dp};
    double fin[6];
    for (int r = 5; r >= 0; r--) {
      double sum = __ldg(&C[r]);
      for (int j = 5; j >= 0; j--) {
        if (order >= 2) {
          double sum1 = __ldg(&R[6 * r + j]);
          for (int k = j; k >= 0; k--)
            sum1 += __ldg(&T[21 * r + j * (j + 1) / 2 + k]) * ini[k];
          sum += sum1 * ini[j];
        } else
          sum += __ldg(&R[6 * r + j]) * ini[j];
      }
      fin[r] = sum;
    }
    p.x = fin[0];
    p.xp = fin[1];
    p.y = fin[2];
    p.yp = fin[3];
    p.s = fin[4];
    p.dp = fin[5];
    store_part(a, i, p);
  }
}

#if TRK_FAST
/* ------------------------------------------------------------- adjoint
 * Reverse mode through the fast build's element maps.  The forward values
 * inside an element are recomputed from its entry state (recorded per pass
 * by adj_record_kernel) and the chain rule is applied backwards, operation
 * by operation, to the adjoint (lambda) of x, x', y, y', delta.  Parameter
 * sensitivities of the kick strengths are summed per warp and added to the
 * gradient with one atomic per warp and element. */
#define TRK_ADJ_MAX_KICKS 48  /* multipole: slices * 3 kicks */
#define TRK_ADJ_MAX_STEPS 128 /* dipole: slices * 4 substeps */

/* (sx, sy) = (qx, qy) / sqrt((1+delta)^2 - qx^2 - qy^2): adds the adjoint of
 * qx, qy, delta given that of sx, sy */
__device__ __forceinline__ void adj_m2s(double qx, double qy, double opd, double lsx, double lsy, double &lqx,
                                        double &lqy, double &ldp) {
  const double g = rsqrt_fast(opd * opd - qx * qx - qy * qy);
  const double g3 = g * g * g;
  lqx += lsx * (g + qx * qx * g3) + lsy * (qx * qy * g3);
  lqy += lsx * (qx * qy * g3) + lsy * (g + qy * qy * g3);
  ldp -= (lsx * qx + lsy * qy) * opd * g3;
}

/* (qx, qy) = (1+delta) (xp, yp) / sqrt(1 + xp^2 + yp^2): adjoint of xp, yp,
 * delta given that of qx, qy */
__device__ __forceinline__ void adj_s2m(double xp, double yp, double opd, double lqx, double lqy, double &lxp,
                                        double &lyp, double &ldp) {
  const double rs = rsqrt_fast(fma(yp, yp, fma(xp, xp, 1.0)));
  const double rs3 = rs * rs * rs;
  lxp += lqx * opd * (rs - xp * xp * rs3) - lqy * opd * xp * yp * rs3;
  lyp += lqy * opd * (rs - yp * yp * rs3) - lqx * opd * xp * yp * rs3;
  ldp += (lqx * xp + lqy * yp) * rs;
}

/* normal multipole field of order 1..3 with the fast build's coefficients:
 * kick qx -= K Fy, qy += K Fx, and the partial derivatives */
__device__ __forceinline__ void mult_field(int order, double x, double y, double &Fy, double &Fx, double &Fyx,
                                           double &Fyy, double &Fxx, double &Fxy) {
  if (order == 1) {
    Fy = x;
    Fx = y;
    Fyx = 1;
    Fyy = 0;
    Fxx = 0;
    Fxy = 1;
  } else if (order == 2) {
    Fy = 0.5 * (x * x - y * y);
    Fx = x * y;
    Fyx = x;
    Fyy = -y;
    Fxx = y;
    Fxy = x;
  } else {
    const double x2 = x * x, y2 = y * y;
    Fy = (x2 * x - 3 * x * y2) * (1.0 / 6);
    Fx = (3 * x2 * y - y2 * y) * (1.0 / 6);
    Fyx = 0.5 * (x2 - y2);
    Fyy = -x * y;
    Fxx = x * y;
    Fxy = 0.5 * (x2 - y2);
  }
}

/* adjoint of op_mult1_fast (the body of mult_body_fast); returns the
 * sensitivity of the particle's contribution to the element's parameter */
__device__ double adj_mult1(const trk_op *__restrict__ op, const double *__restrict__ dk, double x, double xp,
                            double y, double yp, double dp, double &lx, double &lxp, double &ly, double &lyp,
                            double &ldp) {
  const double *d = op->d;
  const int n_parts = __ldg(&op->i[0]);
  const int order = __ldg(&op->i[4]) & 0xff;
  const double opd = 1 + dp, opd2 = opd * opd;
  double KX[TRK_ADJ_MAX_KICKS], KY[TRK_ADJ_MAX_KICKS], QX[TRK_ADJ_MAX_KICKS], QY[TRK_ADJ_MAX_KICKS];
  const double r = opd * rsqrt_fast(fma(yp, yp, fma(xp, xp, 1.0)));
  double qx = xp * r, qy = yp * r, sx = xp, sy = yp;
  int nk = 0;
  for (int i_kick = 0; i_kick < n_parts; i_kick++)
    for (int step = 0; step < 4; step++) {
      const double dsh = __ldg(&d[MD_DSH + step]);
      x = fma(sx, dsh, x);
      y = fma(sy, dsh, y);
      if (step == 3)
        break;
      const double K = __ldg(&d[MD_KQ + step * 3]);
      double Fy, Fx, a, b, c, e;
      mult_field(order, x, y, Fy, Fx, a, b, c, e);
      qx = fma(-K, Fy, qx);
      qy = fma(K, Fx, qy);
      const double rr = rsqrt_fast(opd2 - qx * qx - qy * qy);
      sx = qx * rr;
      sy = qy * rr;
      KX[nk] = x;
      KY[nk] = y;
      QX[nk] = qx;
      QY[nk] = qy;
      nk++;
    }
  /* exit slopes from the final momenta */
  double lqx = 0, lqy = 0, lsx = 0, lsy = 0, sens = 0;
  adj_m2s(qx, qy, opd, lxp, lyp, lqx, lqy, ldp);
  for (int i_kick = n_parts - 1; i_kick >= 0; i_kick--)
    for (int step = 3; step >= 0; step--) {
      if (step < 3) {
        nk--;
        adj_m2s(QX[nk], QY[nk], opd, lsx, lsy, lqx, lqy, ldp);
        lsx = lsy = 0;
        const double K = __ldg(&d[MD_KQ + step * 3]);
        double Fy, Fx, Fyx, Fyy, Fxx, Fxy;
        mult_field(order, KX[nk], KY[nk], Fy, Fx, Fyx, Fyy, Fxx, Fxy);
        lx += K * (-Fyx * lqx + Fxx * lqy);
        ly += K * (-Fyy * lqx + Fxy * lqy);
        sens += (-Fy * lqx + Fx * lqy) * __ldg(&dk[step]);
      }
      const double dsh = __ldg(&d[MD_DSH + step]);
      lsx += dsh * lx;
      lsy += dsh * ly;
    }
  /* entry: the first drift used the incoming slopes; the momenta came from them */
  double lxp_in = lsx, lyp_in = lsy;
  adj_s2m(xp, yp, opd, lqx, lqy, lxp_in, lyp_in, ldp);
  lxp = lxp_in;
  lyp = lyp_in;
  return sens;
}

/* adjoint of op_dipole_fast (bend_dipole_fast / dipole_slice) */
/* The adjoint of the pure-dipole body; with dk (the bend's field
 * derivative tables, dF/dK1 at dk and dF/dK2 at dk + 242) it also returns
 * the sensitivities to the bend's K1 and K2 at K1 = K2 = 0: each kick
 * QX -= w Fy, QY += w Fx changes by -w dFy, +w dFx per unit K, weighted by
 * the adjoints of QX and QY after the kick (QY's running adjoint collects
 * the later drifts' shares as the sweep goes back). */
__device__ void adj_dipole(const trk_op *__restrict__ op, double x, double xp, double y, double yp, double dp,
                           double &lx, double &lxp, double &ly, double &lyp, double &ldp,
                           const double *__restrict__ dk = nullptr, double *sk = nullptr) {
  const double *d = op->d;
  const int nSlices = __ldg(&op->i[0]);
  const double rho0 = __ldg(&d[BD_RHO0]);
  const double opd = 1 + dp;
  const double rs = rsqrt_fast(fma(yp, yp, fma(xp, xp, 1.0)));
  const double QY = yp * opd * rs;
  const double f2 = opd * opd - QY * QY;
  double X = x, Q = xp * opd * rs, F = 0;
  double SX[TRK_ADJ_MAX_STEPS], SQ[TRK_ADJ_MAX_STEPS], SF[TRK_ADJ_MAX_STEPS];
  int m = 0;
  for (int i = 0; i < nSlices; i++)
    for (int j = 0; j < 4; j++) {
      SX[m] = X;
      SQ[m] = Q;
      SF[m] = F;
      m++;
      const double sa = __ldg(&d[BD_SA + j]), ca = __ldg(&d[BD_CA + j]), omc = __ldg(&d[BD_OMC + j]);
      const double fc = sqrt_nan(fma(-Q, Q, f2));
      const double saq = sa * Q;
      const double u = div_fast(rho0 + X, fma(ca, fc, -saq));
      Q = fma(sa, fc, ca * Q);
      F = fma(u, sa, F);
      X = fma(u, fma(omc, fc, saq), X);
      if (j < 3)
        Q = fma(-__ldg(&d[BD_C2 + j]), X, Q - __ldg(&d[BD_C1 + j]));
    }
  const int nsteps = m;
  /* exit: x = X, y = y0 + QY F, (xp, yp) = (Q, QY) / sqrt(opd^2 - Q^2 - QY^2) */
  double lX = lx, lQ = 0, lQY = 0, lopd = 0, lF = QY * ly, lf2 = 0;
  {
    const double g = rsqrt_fast(opd * opd - Q * Q - QY * QY);
    const double g3 = g * g * g;
    lQ += lxp * (g + Q * Q * g3) + lyp * Q * QY * g3;
    lQY += lyp * (g + QY * QY * g3) + lxp * Q * QY * g3;
    lopd -= (lxp * Q + lyp * QY) * opd * g3;
  }
  double sk1 = 0, sk2 = 0;
  for (int i = nSlices - 1; i >= 0; i--)
    for (int j = 3; j >= 0; j--) {
      if (j < 3) {
        const double c2 = __ldg(&d[BD_C2 + j]);
        if (dk) {
          /* the kick at the end of drift j: position X1, Y1 = y + QY F1 */
          const double X1 = m < nsteps ? SX[m] : X, Y1 = fma(QY, m < nsteps ? SF[m] : F, y);
          const double w = fma(c2, X1, __ldg(&d[BD_C1 + j]));
          double dFx, dFy;
          cf_fields(dk, dk + 121, X1, Y1, dFx, dFy);
          sk1 += w * (lQY * dFx - lQ * dFy);
          cf_fields(dk + 242, dk + 363, X1, Y1, dFx, dFy);
          sk2 += w * (lQY * dFx - lQ * dFy);
        }
        lX -= c2 * lQ;
      }
      m--;
      const double Xs = SX[m], Qs = SQ[m];
      const double sa = __ldg(&d[BD_SA + j]), ca = __ldg(&d[BD_CA + j]), omc = __ldg(&d[BD_OMC + j]);
      const double fc = sqrt_nan(fma(-Qs, Qs, f2));
      const double saq = sa * Qs;
      const double fcosi = fma(ca, fc, -saq);
      const double u = div_fast(rho0 + Xs, fcosi);
      const double lu = lF * sa + lX * fma(omc, fc, saq);
      double lfc = lQ * sa + lX * u * omc;
      double lsaq = lX * u;
      double lQs = lQ * ca;
      double lXs = lX;
      const double lfcosi = -lu * u / fcosi;
      lXs += lu / fcosi;
      lfc += ca * lfcosi;
      lsaq -= lfcosi;
      lQs += sa * lsaq;
      const double lu2 = lfc / (2 * fc);
      lf2 += lu2;
      /* this drift's share of QY's adjoint: Y grows by QY u sa, f2 holds -QY^2 */
      lQY += ly * u * sa - 2 * QY * lu2;
      lQs -= 2 * Qs * lu2;
      lX = lXs;
      lQ = lQs;
    }
  lopd += 2 * opd * lf2;
  if (sk) {
    sk[0] = sk1;
    sk[1] = sk2;
  }
  /* entry: X = x, (Q, QY) = opd (xp, yp) / sqrt(1 + xp^2 + yp^2) */
  const double rs3 = rs * rs * rs;
  lx = lX;
  lxp = lQ * opd * (rs - xp * xp * rs3) - lQY * opd * xp * yp * rs3;
  lyp = lQY * opd * (rs - yp * yp * rs3) - lQ * opd * xp * yp * rs3;
  lopd += (lQ * xp + lQY * yp) * rs;
  ldp += lopd;
}

#define TRK_ADJ_MAX_SLICES 32 /* combined-function bend: slices */

/* partial derivatives of the cf_fields expansion at (x, y) */
#define CF_T(T, i, j) __ldg(&(T)[(i) * 11 + (j)])
__device__ __forceinline__ void cf_fields_d(const double *__restrict__ Fx_xy, const double *__restrict__ Fy_xy,
                                            double x, double y, double &Fyx, double &Fyy, double &Fxx,
                                            double &Fxy) {
  const double y2 = y * y;
  const double dp0 = fma(fma(fma(4 * CF_T(Fy_xy, 4, 0), x, 3 * CF_T(Fy_xy, 3, 0)), x, 2 * CF_T(Fy_xy, 2, 0)), x,
                         CF_T(Fy_xy, 1, 0));
  const double p2 = fma(fma(CF_T(Fy_xy, 2, 2), x, CF_T(Fy_xy, 1, 2)), x, CF_T(Fy_xy, 0, 2));
  const double dp2 = fma(2 * CF_T(Fy_xy, 2, 2), x, CF_T(Fy_xy, 1, 2));
  Fyx = fma(y2, dp2, dp0);
  Fyy = 2 * y * fma(2 * y2, CF_T(Fy_xy, 0, 4), p2);
  const double q1 = fma(fma(fma(CF_T(Fx_xy, 3, 1), x, CF_T(Fx_xy, 2, 1)), x, CF_T(Fx_xy, 1, 1)), x,
                        CF_T(Fx_xy, 0, 1));
  const double dq1 = fma(fma(3 * CF_T(Fx_xy, 3, 1), x, 2 * CF_T(Fx_xy, 2, 1)), x, CF_T(Fx_xy, 1, 1));
  const double q3 = fma(CF_T(Fx_xy, 1, 3), x, CF_T(Fx_xy, 0, 3));
  Fxx = y * fma(y2, CF_T(Fx_xy, 1, 3), dq1);
  Fxy = fma(3 * y2, q3, q1);
}
#undef CF_T

/* one drift substep j of cf_slice (no path length) */
__device__ __forceinline__ void cf_drift(const double *__restrict__ d, int j, double rho0, double opd2, double &X,
                                         double &QX, double &Y, const double QY) {
  const double fc = sqrt_nan(fma(-QX, QX, fma(-QY, QY, opd2)));
  const double sa = __ldg(&d[BD_SA + j]), ca = __ldg(&d[BD_CA + j]);
  const double saq = sa * QX;
  const double u = div_fast(rho0 + X, fma(ca, fc, -saq));
  QX = fma(sa, fc, ca * QX);
  Y = fma(QY, u * sa, Y);
  X = fma(u, fma(__ldg(&d[BD_OMC + j]), fc, saq), X);
}

/* adjoint of op_cfbend_fast (bend_cf_fast / cf_slice): the entry state of
 * every slice is kept, and each slice's four substeps are recomputed from it
 * while the slices are reversed */
__device__ void adj_cfbend(const trk_op *__restrict__ op, const double *__restrict__ field, double x, double xp,
                           double y, double yp, double dp, double &lx, double &lxp, double &ly, double &lyp,
                           double &ldp, const double *__restrict__ dk = nullptr, double *sk = nullptr) {
  const double *d = op->d;
  const double *fx = field + __ldg(&op->i[4]);
  const double *fy = fx + 121;
  const int nSlices = __ldg(&op->i[0]);
  const double rho0 = __ldg(&d[BD_RHO0]);
  const double opd = 1 + dp, opd2 = opd * opd;
  const double r = opd * rsqrt_fast(fma(yp, yp, fma(xp, xp, 1.0)));
  double X = x, QX = xp * r, Y = y, QY = yp * r;
  double CX[TRK_ADJ_MAX_SLICES], CQX[TRK_ADJ_MAX_SLICES], CY[TRK_ADJ_MAX_SLICES], CQY[TRK_ADJ_MAX_SLICES];
  for (int i = 0; i < nSlices; i++) {
    CX[i] = X;
    CQX[i] = QX;
    CY[i] = Y;
    CQY[i] = QY;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      cf_drift(d, j, rho0, opd2, X, QX, Y, QY);
      if (j == 3)
        break;
      double Fx, Fy;
      cf_fields(fx, fy, X, Y, Fx, Fy);
      const double w = fma(__ldg(&d[BD_C2 + j]), X, __ldg(&d[BD_C1 + j]));
      QX = fma(-w, Fy, QX);
      QY = fma(w, Fx, QY);
    }
  }
  /* exit: x = X, y = Y, (xp, yp) = (QX, QY) / sqrt(opd^2 - QX^2 - QY^2) */
  double lX = lx, lY = ly, lQX = 0, lQY = 0, lopd = 0, sk1 = 0, sk2 = 0;
  adj_m2s(QX, QY, opd, lxp, lyp, lQX, lQY, lopd);
  for (int i = nSlices - 1; i >= 0; i--) {
    /* substep entry states of slice i (and the kick positions) */
    double sX[5], sQX[4], sY[5], sQY[4];
    X = CX[i];
    QX = CQX[i];
    Y = CY[i];
    QY = CQY[i];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      sX[j] = X;
      sQX[j] = QX;
      sY[j] = Y;
      sQY[j] = QY;
      cf_drift(d, j, rho0, opd2, X, QX, Y, QY);
      sX[j + 1] = X;
      sY[j + 1] = Y;
      if (j == 3)
        break;
      double Fx, Fy;
      cf_fields(fx, fy, X, Y, Fx, Fy);
      const double w = fma(__ldg(&d[BD_C2 + j]), X, __ldg(&d[BD_C1 + j]));
      QX = fma(-w, Fy, QX);
      QY = fma(w, Fx, QY);
    }
#pragma unroll
    for (int j = 3; j >= 0; j--) {
      if (j < 3) {
        /* kick at (X1, Y1) = (sX[j+1], sY[j+1]): QX -= w Fy, QY += w Fx */
        const double X1 = sX[j + 1], Y1 = sY[j + 1];
        const double c2 = __ldg(&d[BD_C2 + j]);
        const double w = fma(c2, X1, __ldg(&d[BD_C1 + j]));
        double Fx, Fy, Fyx, Fyy, Fxx, Fxy;
        cf_fields(fx, fy, X1, Y1, Fx, Fy);
        cf_fields_d(fx, fy, X1, Y1, Fyx, Fyy, Fxx, Fxy);
        const double lw = fma(-lQX, Fy, lQY * Fx);
        lX += lw * c2 + w * fma(-lQX, Fyx, lQY * Fxx);
        lY += w * fma(-lQX, Fyy, lQY * Fxy);
        if (dk) { /* d(kick)/dK1, d(kick)/dK2 with the adjoints after the kick */
          double dFx, dFy;
          cf_fields(dk, dk + 121, X1, Y1, dFx, dFy);
          sk1 += w * (lQY * dFx - lQX * dFy);
          cf_fields(dk + 242, dk + 363, X1, Y1, dFx, dFy);
          sk2 += w * (lQY * dFx - lQX * dFy);
        }
      }
      /* drift from (Xs, QXs, Ys, QYs): X' = Xs + u (omc fc + sa QXs),
       * QX' = sa fc + ca QXs, Y' = Ys + QYs u sa, with
       * fc = sqrt(opd^2 - QYs^2 - QXs^2), u = (rho0 + Xs) / (ca fc - sa QXs) */
      const double Xs = sX[j], QXs = sQX[j], QYs = sQY[j];
      const double sa = __ldg(&d[BD_SA + j]), ca = __ldg(&d[BD_CA + j]), omc = __ldg(&d[BD_OMC + j]);
      const double fc = sqrt_nan(fma(-QXs, QXs, fma(-QYs, QYs, opd2)));
      const double saq = sa * QXs;
      const double fcosi = fma(ca, fc, -saq);
      const double u = div_fast(rho0 + Xs, fcosi);
      lQY += lY * u * sa;
      const double lu = lY * QYs * sa + lX * fma(omc, fc, saq);
      double lfc = lX * u * omc + lQX * sa;
      double lsaq = lX * u;
      double lQXs = lQX * ca;
      double lXs = lX;
      const double lfcosi = -lu * u / fcosi;
      lXs += lu / fcosi;
      lfc += ca * lfcosi;
      lsaq -= lfcosi;
      lQXs += sa * lsaq;
      const double lu2 = lfc / (2 * fc);
      lQXs -= 2 * QXs * lu2;
      lopd += 2 * opd * lu2;
      lQY -= 2 * QYs * lu2;
      lX = lXs;
      lQX = lQXs;
    }
  }
  if (sk) {
    sk[0] = sk1;
    sk[1] = sk2;
  }
  /* entry: X = x, Y = y, (QX, QY) = opd (xp, yp) / sqrt(1 + xp^2 + yp^2) */
  lx = lX;
  ly = lY;
  double lxp_in = 0, lyp_in = 0;
  adj_s2m(xp, yp, opd, lQX, lQY, lxp_in, lyp_in, ldp);
  lxp = lxp_in;
  lyp = lyp_in;
  ldp += lopd;
}

/* forward pass from a checkpoint, recording every element's entry state */
__global__ void adj_record_kernel(TrackArgs a, AdjArgs g) {
  const long n = a.n, stride = (long)gridDim.x * blockDim.x;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    if (a.lost_pass[i] >= 0)
      continue;
    Part p;
    p.x = g.ck[i];
    p.xp = g.ck[n + i];
    p.y = g.ck[2 * n + i];
    p.yp = g.ck[3 * n + i];
    p.s = 0;
    p.dp = a.dp[i];
    const trk_op *ops = a.ops;
    if (a.ens_offsets)
      ops += (long)ens_variant(a.ens_offsets, a.ens_variants, i) * a.ens_ops;
    for (int k = 0; k < g.n_ops; k++) {
      const trk_op *op = ops + k;
      double *e = g.entry + (size_t)k * 4 * n;
      e[i] = p.x;
      e[n + i] = p.xp;
      e[2 * n + i] = p.y;
      e[3 * n + i] = p.yp;
      switch (__ldg(&op->kind)) {
      case OPK_DRIFT:
        op_drift(op, p);
        break;
      case OPK_EDRIFT:
      case OPK_RFDRIFT:
        exact_drift(p, __ldg(&op->d[DD_L]));
        break;
      case OPK_MULT1:
        op_mult1_fast(op, p, a.Po, 0.0, nullptr);
        break;
      case OPK_DIPOLE:
        op_dipole_fast(op, p, a.Po, 0.0, nullptr);
        break;
      case OPK_CFBEND:
        op_cfbend_fast(op, p, a.Po, 0.0, nullptr, a.field);
        break;
      default:
        break;
      }
    }
  }
}

/* one pass backwards: lambda at the end of the pass -> at its start */
__global__ void __launch_bounds__(128) adj_reverse_kernel(TrackArgs a, AdjArgs g) {
  const long n = a.n;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < n && a.lost_pass[i] < 0;
  double lx = 0, lxp = 0, ly = 0, lyp = 0, ldp = 0, dp = 0;
  /* variant of this particle (ensembles); lanes past the end take the last
   * particle's, so a warp of one variant stays uniform */
  int v = 0;
  if (a.ens_offsets && n > 0)
    v = ens_variant(a.ens_offsets, a.ens_variants, i < n ? i : n - 1);
  const trk_op *ops = a.ops + (long)v * a.ens_ops;
  const bool warp_uniform = __all_sync(0xffffffffu, v == __shfl_sync(0xffffffffu, v, 0));
  if (act) {
    lx = g.lam[i];
    lxp = g.lam[n + i];
    ly = g.lam[2 * n + i];
    lyp = g.lam[3 * n + i];
    ldp = g.lam[4 * n + i];
    dp = a.dp[i];
  }
  for (int k = g.n_ops - 1; k >= 0; k--) {
    const trk_op *op = ops + k;
    double x = 0, xp = 0, y = 0, yp = 0;
    if (act) {
      const double *e = g.entry + (size_t)k * 4 * n;
      x = e[i];
      xp = e[n + i];
      y = e[2 * n + i];
      yp = e[3 * n + i];
    }
    double sens = 0, sk[2] = {0, 0};
    const int prm = __ldg(&g.op_param[k]);
    const int dfo = g.op_dfield ? __ldg(&g.op_dfield[k]) : -1;
    const double *dk = (prm >= 0 && dfo >= 0) ? g.dfield + dfo : nullptr;
    bool two = false;
    switch (__ldg(&op->kind)) {
    case OPK_DRIFT:
    case OPK_EDRIFT:
    case OPK_RFDRIFT: {
      const double L = __ldg(&op->d[DD_L]);
      lxp += L * lx;
      lyp += L * ly;
      break;
    }
    case OPK_MULT1:
      sens = adj_mult1(op, g.op_dk + 3 * ((long)v * g.n_ops + k), x, xp, y, yp, dp, lx, lxp, ly, lyp, ldp);
      break;
    case OPK_DIPOLE:
      adj_dipole(op, x, xp, y, yp, dp, lx, lxp, ly, lyp, ldp, dk, sk);
      two = dk != nullptr;
      break;
    case OPK_CFBEND:
      adj_cfbend(op, a.field, x, xp, y, yp, dp, lx, lxp, ly, lyp, ldp, dk, sk);
      two = dk != nullptr;
      break;
    default:
      break;
    }
    if (prm >= 0) {
      /* one parameter (multipole K) or two (CSBEND K1, K2 at prm, prm + 1) */
      for (int q = 0; q < (two ? 2 : 1); q++) {
        double sv = two ? sk[q] : sens;
        if (!act)
          sv = 0;
        if (warp_uniform) {
          for (int off = 16; off > 0; off >>= 1)
            sv += __shfl_xor_sync(0xffffffffu, sv, off);
          if ((threadIdx.x & 31) == 0 && sv != 0)
            atomicAdd(&g.grad[(long)v * g.n_params + prm + q], sv);
        } else if (sv != 0) {
          atomicAdd(&g.grad[(long)v * g.n_params + prm + q], sv);
        }
      }
    }
  }
  if (act) {
    g.lam[i] = lx;
    g.lam[n + i] = lxp;
    g.lam[2 * n + i] = ly;
    g.lam[3 * n + i] = lyp;
    g.lam[4 * n + i] = ldp;
  }
}
#endif

/* ------------------------------------------------------------- launchers */
int track_variant_block(int variant) {
  switch (variant) {
  case 2:
  case 8:
    return 256;
  case 3:
    return 64;
  default:
    return 128;
  }
}

template <int LEAN>
static void launch_track_t(const TrackArgs &a, int variant, int grid, int block, cudaStream_t st) {
  switch (variant) {
  case 1:
    track_kernel<128, 4, LEAN><<<grid, block, 0, st>>>(a);
    break;
  case 2:
    track_kernel<256, 2, LEAN><<<grid, block, 0, st>>>(a);
    break;
  case 3:
    track_kernel<64, 8, LEAN><<<grid, block, 0, st>>>(a);
    break;
  case 4:
    track_kernel<128, 5, LEAN><<<grid, block, 0, st>>>(a);
    break;
  case 7:
    track_kernel<128, 6, LEAN><<<grid, block, 0, st>>>(a);
    break;
  case 8:
    track_kernel<256, 3, LEAN><<<grid, block, 0, st>>>(a);
    break;
  default:
    track_kernel<128, 1, LEAN><<<grid, block, 0, st>>>(a);
    break;
  }
}

void launch_track(const TrackArgs &a, int variant, int lean, long n, int max_blocks, cudaStream_t st) {
#if TRK_FAST
  if (lean && (variant == 5 || variant == 6)) {
    long g = (n + 2 * 128 - 1) / (2 * 128);
    if (g < 1)
      g = 1;
    if (g > max_blocks)
      g = max_blocks;
    if (variant == 5)
      track_kernel2<128, 3><<<(int)g, 128, 0, st>>>(a);
    else
      track_kernel2<128, 2><<<(int)g, 128, 0, st>>>(a);
    return;
  }
#endif
  if (variant == 5 || variant == 6 || variant < 0 || variant >= TRK_N_VARIANTS)
    variant = 1;
  const int block = track_variant_block(variant);
  long g = (n + block - 1) / block;
  if (g < 1)
    g = 1;
  if (g > max_blocks)
    g = max_blocks;
#if TRK_FAST
  if (lean == 2)
    launch_track_t<2>(a, variant, (int)g, block, st);
  else if (lean)
#else
  /* the parity build's combined-function bends take the general body, which
   * flavour 1 leaves out: such lattices run the full flavour */
  if (lean == 1)
#endif
    launch_track_t<1>(a, variant, (int)g, block, st);
  else
    launch_track_t<0>(a, variant, (int)g, block, st);
}

void launch_time_stats(const TimeStatsArgs &a, int grid, cudaStream_t st) {
  time_stats_kernel<<<grid, TRK_BLOCK, 0, st>>>(a);
  time_stats_finish_kernel<<<1, TRK_FINISH_THREADS, 0, st>>>(a, grid);
}

void launch_rf_fiducial(const double *stats, double omega, double t_reference, double *rf_phase, int slot,
                        int *status, cudaStream_t st) {
  rf_fiducial_kernel<<<1, 1, 0, st>>>(stats, omega, t_reference, rf_phase, slot, status);
}

void launch_rf_tave(const double *stats, double *rf_tave, int slot, cudaStream_t st) {
  rf_tave_kernel<<<1, 1, 0, st>>>(stats, rf_tave, slot);
}

void launch_wake(const WakeArgs &a, int grid, cudaStream_t st) {
  launch_wake_bin(a, grid, st);
  launch_wake_apply(a, grid, st);
}

/* geometry and histogram (the part before the cross-rank histogram sum) */
void launch_wake_bin(const WakeArgs &a, int grid, cudaStream_t st) {
  wake_setup_kernel<<<1, 1, 0, st>>>(a);
  size_t smem = a.transverse ? 0 : (size_t)a.smem_bins * sizeof(unsigned int);
  wake_bin_kernel<<<grid, TRK_BLOCK, smem, st>>>(a);
}

/* convolution and kicks (after it) */
void launch_wake_apply(const WakeArgs &a, int grid, cudaStream_t st) {
  int cb = (int)((a.max_bins + 1 + 127) / 128);
  wake_convolve_kernel<<<cb, 128, 0, st>>>(a, 0);
  if (a.transverse)
    wake_convolve_kernel<<<cb, 128, 0, st>>>(a, 1);
  wake_kick_kernel<<<grid, TRK_BLOCK, 0, st>>>(a);
}

void launch_stats_combine(const double *gathered, int ranks, double *out, cudaStream_t st) {
  stats_combine_kernel<<<1, 1, 0, st>>>(gathered, ranks, out);
}

void launch_rotate(const TrackArgs &a, double ca, double sa, int grid, cudaStream_t st) {
  rotate_kernel<<<grid, TRK_BLOCK, 0, st>>>(a, ca, sa);
}

/* launch shapes an ensemble can use (the one-particle-per-thread kernels) */
int ensemble_variant_ok(int variant) { return variant >= 0 && variant < TRK_N_VARIANTS && variant != 5 && variant != 6; }

void launch_track_ensemble(const TrackArgs &a, const long *offsets, int n_variants, int ops_per_variant, int variant,
                           int lean, long n, int max_blocks, cudaStream_t st) {
  TrackArgs e = a;
  e.ens_offsets = offsets;
  e.ens_variants = n_variants;
  e.ens_ops = ops_per_variant;
  launch_track(e, ensemble_variant_ok(variant) ? variant : 1, lean, n, max_blocks, st);
}

void launch_adjoint_record(const TrackArgs &a, const AdjArgs &g, cudaStream_t st) {
#if TRK_FAST
  const long grid = std::min<long>((a.n + 127) / 128, 148L * 64);
  adj_record_kernel<<<(int)std::max<long>(grid, 1), 128, 0, st>>>(a, g);
#else
  (void)a;
  (void)g;
  (void)st;
#endif
}

void launch_adjoint_reverse(const TrackArgs &a, const AdjArgs &g, cudaStream_t st) {
#if TRK_FAST
  const long grid = (a.n + 127) / 128;
  adj_reverse_kernel<<<(int)std::max<long>(grid, 1), 128, 0, st>>>(a, g);
#else
  (void)a;
  (void)g;
  (void)st;
#endif
}

void launch_limit(const TrackArgs &a, const trk_aperture &ap, int mode, int extrapolate, double z, long pass, int elem,
                  int grid, cudaStream_t st) {
  limit_kernel<<<grid, TRK_BLOCK, 0, st>>>(a, ap, mode, extrapolate, z, pass, elem);
}

void launch_matrix(const TrackArgs &a, const double *m, int order, int grid, cudaStream_t st) {
  matrix_kernel<<<grid, TRK_BLOCK, 0, st>>>(a, m, order);
}

cudaError_t set_coefficients(const double *coef10) {
  return cudaMemcpyToSymbol(c_coef, coef10, sizeof(double) * 10);
}

} // namespace TRK_NS
