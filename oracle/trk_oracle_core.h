/*
 * trk_oracle_core.h -- TEST INFRASTRUCTURE ONLY (the CPU oracle).
 *
 * Per-particle maps of elegant's tracking path, restated in plain C with the
 * reference's operation order, so that a build without FMA contraction
 * reproduces the reference bit for bit.  Nothing in the product library
 * includes this file; only tests, smoke() and bench.py's CPU baseline use the
 * oracle, as a checker.
 *
 * The real type is the macro ORC_R (double by default) and the math functions
 * are the ORC_* macros, so the same code can be compiled with a counting
 * type to measure algorithmic flops per particle.
 */
#ifndef TRK_ORACLE_CORE_H
#define TRK_ORACLE_CORE_H

#include <math.h>
#include <stdint.h>
#include "trk_constants.h"
#include "trk_crmath.h"
#include "trk_philox.h"

/* what an incoherent-radiation deviate is keyed by (the library draws the
 * same deviates): the run's seed, the particle ID, the pass, the element
 * index; `single`: one particle tracked (ISR1PART=0 then turns ISR off) */
typedef struct {
  uint64_t seed;
  uint32_t id, pass, elem;
  int single;
} orc_isr_key;
static orc_isr_key orc_isr;

/* 0: the C library's sin/cos/asin (as the reference links them);
 * 1: correctly rounded double-double evaluations (trk_crmath.h), the values a
 *    correctly rounding libm returns and the GPU parity build computes. */
static int orc_cr_math = 0;
static inline double orc_sin_sel(double x) { return orc_cr_math ? trkcr_sin(x) : sin(x); }
static inline double orc_cos_sel(double x) { return orc_cr_math ? trkcr_cos(x) : cos(x); }
static inline double orc_asin_sel(double x) { return orc_cr_math ? trkcr_asin(x) : asin(x); }
static inline double orc_tan_sel(double x) { return orc_cr_math ? trkcr_tan(x) : tan(x); }
static inline double orc_exp_sel(double x) { return orc_cr_math ? trkcr_exp(x) : exp(x); }
static inline double orc_sinh_sel(double x) { return orc_cr_math ? trkcr_sinh(x) : sinh(x); }
static inline double orc_cosh_sel(double x) { return orc_cr_math ? trkcr_cosh(x) : cosh(x); }

#ifndef ORC_R
#define ORC_R double
#define ORC_SQRT(x) sqrt(x)
#define ORC_SIN(x) orc_sin_sel(x)
#define ORC_COS(x) orc_cos_sel(x)
#define ORC_TAN(x) tan(x)
#define ORC_ASIN(x) orc_asin_sel(x)
#define ORC_FABS(x) fabs(x)
#define ORC_ISNAN(x) isnan(x)
#define ORC_ISINF(x) isinf(x)
#define ORC_VAL(x) (x)
#endif

typedef ORC_R orc_r;

static inline orc_r orc_sqr(orc_r x) { return x * x; }

/* Integer power by repeated squaring.  The reference calls SDDS mdbmth
 * ipow(), which is not shipped with it; only exponent 2 (x*x) is exercised on
 * this path, where every evaluation order gives the same product. */
static inline orc_r orc_ipow(orc_r x, long p) {
  if (p == 0)
    return 1.0;
  if (p == 1)
    return x;
  if (p == 2)
    return x * x;
  if (p < 0)
    return 1.0 / orc_ipow(x, -p);
  orc_r h = orc_ipow(x, p / 2);
  return (p & 1) ? h * h * x : h * h;
}

/* Integrator substep tables (src/multipole.c:1118-1141, src/csbend.c:1480-1503). */
static const double orc_drift_frac2[2] = {0.5, 0.5};
static const double orc_kick_frac2[2] = {1.0, 0.0};
static const double orc_drift_frac4[4] = {0.5 / (2 - TRK_BETA), (1 - TRK_BETA) / (2 - TRK_BETA) / 2,
                                          (1 - TRK_BETA) / (2 - TRK_BETA) / 2, 0.5 / (2 - TRK_BETA)};
static const double orc_kick_frac4[4] = {1. / (2 - TRK_BETA), -TRK_BETA / (2 - TRK_BETA), 1 / (2 - TRK_BETA), 0};
static const double orc_drift_frac6[8] = {0.39225680523878,     0.5100434119184585, -0.47105338540975655,
                                          0.0687531682525181,   0.0687531682525181, -0.47105338540975655,
                                          0.5100434119184585,   0.39225680523878};
static const double orc_kick_frac6[8] = {0.784513610477560,  0.235573213359357, -1.17767998417887,
                                         1.3151863206839063, -1.17767998417887, 0.235573213359357,
                                         0.784513610477560,  0};

static inline int orc_substeps(int integration_order, const double **df, const double **kf) {
  switch (integration_order) {
  case 2:
    *df = orc_drift_frac2;
    *kf = orc_kick_frac2;
    return 2;
  case 4:
    *df = orc_drift_frac4;
    *kf = orc_kick_frac4;
    return 4;
  case 6:
    *df = orc_drift_frac6;
    *kf = orc_kick_frac6;
    return 8;
  default:
    return 0;
  }
}

/* ---------------------------------------------------------- apertures */
/* MULT_APERTURE_DATA as filled by setupMultApertureData() from the current
 * MAXAMP (src/multipole.c:1690-1749); no aperture files or contours. */
typedef struct {
  double xMax, yMax;
  int elliptical;
  long xExponent, yExponent;
  double reverseTilt, reverseTiltC, reverseTiltS;
} orc_aperture;

/* checkMultAperture (src/multipole.c:1751-1798) */
static inline int orc_check_mult_aperture(orc_r xInput, orc_r yInput, const orc_aperture *ap) {
  orc_r x, y;
  if (!ap)
    return 1;
  x = xInput - 0.0; /* xCen = 0 without aperture files */
  y = yInput - 0.0;
  if (ap->reverseTilt) {
    orc_r x0 = x, y0 = y;
    x = x0 * ap->reverseTiltC + y0 * ap->reverseTiltS;
    y = -x0 * ap->reverseTiltS + y0 * ap->reverseTiltC;
  }
  if (ap->elliptical == 0 || ap->xMax <= 0 || ap->yMax <= 0) {
    if ((ap->xMax > 0 && ORC_VAL(ORC_FABS(x)) > ap->xMax) || (ap->yMax > 0 && ORC_VAL(ORC_FABS(y)) > ap->yMax))
      return 0;
  } else {
    orc_r xa = x / ap->xMax;
    orc_r yb = y / ap->yMax;
    if (ORC_VAL(orc_ipow(xa, ap->xExponent) + orc_ipow(yb, ap->yExponent)) >= 1)
      return 0;
  }
  return 1;
}

/* ------------------------------------------------- kick multipoles */
/* convertSlopesToMomenta / convertMomentaToSlopes (src/multipole.h:448-480) */
static inline void orc_slopes_to_momenta(orc_r *qx, orc_r *qy, orc_r xp, orc_r yp, orc_r delta, int expand) {
  if (expand) {
    *qx = (1 + delta) * xp;
    *qy = (1 + delta) * yp;
  } else {
    orc_r denom = ORC_SQRT(1 + orc_sqr(xp) + orc_sqr(yp));
    *qx = (1 + delta) * xp / denom;
    *qy = (1 + delta) * yp / denom;
  }
}

static inline int orc_momenta_to_slopes(orc_r *xp, orc_r *yp, orc_r qx, orc_r qy, orc_r delta, int expand) {
  if (expand) {
    *xp = qx / (1 + delta);
    *yp = qy / (1 + delta);
  } else {
    orc_r denom = orc_sqr(1 + delta) - orc_sqr(qx) - orc_sqr(qy);
    if (ORC_VAL(denom) <= 0)
      return 0;
    denom = ORC_SQRT(denom);
    *xp = qx / denom;
    *yp = qy / denom;
  }
  return 1;
}

/* expansion_coefficients(n) (src/multipole.h:76-146): coef[i] =
 * (-1)^(i/2) / (i! (n-i)!); orders 0..2 are literal tables in the reference,
 * higher orders use the formula with the factorial product formed first. */
static inline void orc_expansion_coefficients(int n, double *coef) {
  if (n == 0) {
    coef[0] = 1.;
    return;
  }
  if (n == 1) {
    coef[0] = 1.;
    coef[1] = 1.;
    return;
  }
  if (n == 2) {
    coef[0] = 1. / 2;
    coef[1] = 1.;
    coef[2] = -1. / 2;
    return;
  }
  for (int i = 0; i <= n; i++) {
    double fi = 1, fn = 1;
    for (long k = i; k > 1; k--)
      fi *= k;
    for (long k = n - i; k > 1; k--)
      fn *= k;
    coef[i] = (((i / 2) & 1) ? -1.0 : 1.0) / (fi * fn);
  }
}

/* apply_canonical_multipole_kicks_ret / _noret (src/multipole.h:391-446) */
static inline void orc_mkick(orc_r *qx, orc_r *qy, orc_r *dqx, orc_r *dqy, const orc_r *xpow,
                             const orc_r *ypow, int order, orc_r KnL, int skew) {
  double coef[16];
  orc_r sum_Fx = 0, sum_Fy = 0;
  orc_expansion_coefficients(order, coef);
  for (int i = 0; i <= order; i++) {
    orc_r f = coef[i] * xpow[order - i] * ypow[i];
    if (i & 1)
      sum_Fx += f;
    else
      sum_Fy += f;
  }
  if (skew) {
    orc_r t = sum_Fx;
    sum_Fx = sum_Fy;
    sum_Fy = t;
    sum_Fx = -sum_Fx;
  }
  *qx -= KnL * sum_Fy;
  *qy += KnL * sum_Fx;
  if (dqx) {
    *dqx -= KnL * sum_Fy;
    *dqy += KnL * sum_Fx;
  }
}

/* Prepared per-element values of multipole_tracking2 (src/multipole.c:660-1084) */
typedef struct {
  int order[3];
  int skew[3];
  orc_r KnL[3];
  double drift;      /* lEffective (or L) */
  double dx, dy;     /* offsets seen by the aperture check */
  orc_r xkick, ykick;
  int nSlices;       /* n_parts */
  int integ_order;
  int expand;
  int maxOrder;
  double rad_coef; /* classical radiation (SYNCH_RAD), 0 without */
  double isr_coef; /* incoherent radiation (ISR), 0 without */
  int isr1off;     /* ISR1PART=0 */
} orc_mult;

/* integrate_kick_multipole_ordn (src/multipole.c:1099-1456) with
 * TURBO_APPLY_KICKS_FAST=4 (src/manual.h:77-79), no radiation, no error or
 * edge multipoles, iSlice=-1.  Returns 1 if the particle survives. */
static int orc_integrate_kick_multipole(orc_r *coord, const orc_mult *m, double Po, const orc_aperture *ap,
                                        orc_r *dzLoss) {
  orc_r p, qx, qy, dp, s;
  orc_r x, y, xp, yp, delta_qx, delta_qy;
  orc_r xpow[16], ypow[16];
  orc_r KnLp[3];
  const double *driftFrac, *kickFrac;
  int nSubsteps = orc_substeps(m->integ_order, &driftFrac, &kickFrac);
  long n_parts = m->nSlices;
  double drift = m->drift / n_parts;
  orc_r xkick = m->xkick / n_parts;
  orc_r ykick = m->ykick / n_parts;
  long i_kick;

  x = coord[0];
  xp = coord[1];
  y = coord[2];
  yp = coord[3];
  s = 0;
  dp = coord[5];
  p = Po * (1 + dp);
  orc_r beta0 = p / ORC_SQRT(orc_sqr(p) + 1);

  if (ORC_ISNAN(x) || ORC_ISNAN(xp) || ORC_ISNAN(y) || ORC_ISNAN(yp))
    return 0;
  if (ORC_VAL(ORC_FABS(x)) > TRK_COORD_LIMIT || ORC_VAL(ORC_FABS(y)) > TRK_COORD_LIMIT ||
      ORC_VAL(ORC_FABS(xp)) > TRK_SLOPE_LIMIT || ORC_VAL(ORC_FABS(yp)) > TRK_SLOPE_LIMIT)
    return 0;

  orc_slopes_to_momenta(&qx, &qy, xp, yp, dp, m->expand);
  for (int i = 0; i < 3; i++)
    KnLp[i] = m->KnL[i] / n_parts;

  if (!orc_momenta_to_slopes(&xp, &yp, qx, qy, dp, m->expand))
    return 0;

  *dzLoss = 0;
  for (i_kick = 0; i_kick < n_parts; i_kick++) {
    if (ap && !orc_check_mult_aperture(x + m->dx, y + m->dy, ap)) {
      coord[0] = x;
      coord[2] = y;
      return 0;
    }
    delta_qx = delta_qy = 0;
    for (int step = 0; step < nSubsteps; step++) {
      if (drift) {
        double dsh = drift * driftFrac[step];
        x += xp * dsh;
        y += yp * dsh;
        if (m->expand)
          s += dsh * (1 + (orc_sqr(xp) + orc_sqr(yp)) / 2);
        else
          s += dsh * ORC_SQRT(1 + orc_sqr(xp) + orc_sqr(yp));
        *dzLoss += dsh;
      }
      if (!kickFrac[step])
        break;
      xpow[0] = 1;
      ypow[0] = 1;
      for (int i = 1; i <= m->maxOrder; i++) {
        xpow[i] = xpow[i - 1] * x;
        ypow[i] = ypow[i - 1] * y;
      }
      delta_qx = delta_qy = 0;
      for (int iOrder = 0; iOrder < 3; iOrder++)
        if (ORC_VAL(m->KnL[iOrder]))
          orc_mkick(&qx, &qy, &delta_qx, &delta_qy, xpow, ypow, m->order[iOrder], KnLp[iOrder] * kickFrac[step],
                    m->skew[iOrder]);
      if (ORC_VAL(xkick))
        orc_mkick(&qx, &qy, NULL, NULL, xpow, ypow, 0, -xkick * kickFrac[step], 0);
      if (ORC_VAL(ykick))
        orc_mkick(&qx, &qy, NULL, NULL, xpow, ypow, 0, -ykick * kickFrac[step], 1);
      if (!orc_momenta_to_slopes(&xp, &yp, qx, qy, dp, m->expand))
        return 0;
      /* (rad_coef || isr_coef) && drift (src/multipole.c:1359-1389): isr_coef
       * is nonzero whenever Po > 0 (negated when ISR is off, :757-760), so
       * after every kick the momenta are divided by (1 + dp) and multiplied
       * back, which can move them by an ulp, and the slopes are recomputed. */
      if (drift && (m->rad_coef || m->isr_coef > 0)) {
        /* the radiation block with SYNCH_RAD (src/multipole.c:1359-1389):
         * field from the returned kick, dp -= rad_coef (1+dp)^2 F^2 ds */
        qx /= (1 + dp);
        qy /= (1 + dp);
        orc_r deltaFactor = orc_sqr(1 + dp);
        delta_qx /= kickFrac[step];
        delta_qy /= kickFrac[step];
        orc_r F2 = orc_sqr(delta_qx / drift - xkick / drift) + orc_sqr(delta_qy / drift + ykick / drift);
        delta_qx = 0;
        delta_qy = 0;
        orc_r dsFactor = ORC_SQRT(1 + orc_sqr(xp) + orc_sqr(yp));
        orc_r dsISRFactor = dsFactor * drift / (nSubsteps - 1);
        dsFactor *= drift * kickFrac[step];
        if (m->rad_coef)
          dp -= m->rad_coef * deltaFactor * F2 * dsFactor;
        if (m->isr_coef > 0 && !(orc_isr.single && m->isr1off)) {
          /* src/multipole.c:1380-1381, with the library's deviates */
          const double g = trk_isr_gauss(orc_isr.seed, (uint32_t)(long long)ORC_VAL(coord[6]), orc_isr.pass,
                                         orc_isr.elem, (uint32_t)(i_kick * 8 + step), 3.0);
          dp -= m->isr_coef * deltaFactor * pow(ORC_VAL(F2), 0.75) * ORC_SQRT(dsISRFactor) * g;
        }
        qx *= (1 + dp);
        qy *= (1 + dp);
        if (!orc_momenta_to_slopes(&xp, &yp, qx, qy, dp, m->expand))
          return 0;
      } else if (drift) {
        qx /= (1 + dp);
        qy /= (1 + dp);
        qx *= (1 + dp);
        qy *= (1 + dp);
        if (!orc_momenta_to_slopes(&xp, &yp, qx, qy, dp, m->expand))
          return 0;
      }
    }
  }
  (void)delta_qx;
  (void)delta_qy;
  if (ap && !orc_check_mult_aperture(x + m->dx, y + m->dy, ap)) {
    coord[0] = x;
    coord[2] = y;
    return 0;
  }
  if (!orc_momenta_to_slopes(&xp, &yp, qx, qy, dp, m->expand))
    return 0;
  coord[0] = x;
  coord[1] = xp;
  coord[2] = y;
  coord[3] = yp;
  if (m->rad_coef) {
    /* the path length rescaled to the new velocity (src/multipole.c:1437-1441) */
    p = Po * (1 + dp);
    orc_r beta1 = p / ORC_SQRT(orc_sqr(p) + 1);
    coord[4] = beta1 * (coord[4] / beta0 + 2 * s / (beta0 + beta1));
  } else
    coord[4] += s;
  coord[5] = dp;
  if (ORC_ISNAN(x) || ORC_ISNAN(xp) || ORC_ISNAN(y) || ORC_ISNAN(yp))
    return 0;
  if (ORC_VAL(ORC_FABS(x)) > TRK_COORD_LIMIT || ORC_VAL(ORC_FABS(y)) > TRK_COORD_LIMIT ||
      ORC_VAL(ORC_FABS(xp)) > TRK_SLOPE_LIMIT || ORC_VAL(ORC_FABS(yp)) > TRK_SLOPE_LIMIT)
    return 0;
  return 1;
}

/* ---------------------------------------------------------------- CSBEND */
typedef struct {
  double rho0, rho_actual;
  double length;
  int nSlices;
  int integ_order;
  int hasNormal, hasSkew;
  int expansionOrder1;
  double Fx_xy[11][11], Fy_xy[11][11];
  int isr_or_rad; /* (rad_coef || isrConstant) in the reference: true for Po>0 */
  double rad_coef; /* classical radiation (SYNCH_RAD), 0 without */
  double isr_constant; /* incoherent radiation (ISR), 0 without */
  int isr1off;         /* ISR1PART=0 */
  int expanded;        /* EXPAND_HAMILTONIAN */
} orc_bend;

/* computeCSBENDFields (src/csbend.c:99-172) */
static inline void orc_csbend_fields(const orc_bend *b, orc_r *Fx, orc_r *Fy, orc_r x, orc_r y) {
  orc_r yp[11];
  orc_r sumFx = 0, sumFy = 0;
  if (!b->hasSkew && !b->hasNormal) {
    *Fx = 0;
    *Fy = 1;
    return;
  }
  yp[0] = 1;
  for (int i = 1; i < b->expansionOrder1; i++)
    yp[i] = yp[i - 1] * y;
  orc_r xt = 1;
  if (b->hasSkew) {
    for (int i = 0; i < b->expansionOrder1; i++) {
      for (int j = 0; j < b->expansionOrder1 - i; j++) {
        sumFx += b->Fx_xy[i][j] * xt * yp[j];
        sumFy += b->Fy_xy[i][j] * xt * yp[j];
      }
      xt *= x;
    }
  } else {
    for (int i = 0; i < b->expansionOrder1; i++) {
      for (int j = 0; j < b->expansionOrder1 - i; j++) {
        if (j & 1)
          sumFx += b->Fx_xy[i][j] * xt * yp[j];
        else
          sumFy += b->Fy_xy[i][j] * xt * yp[j];
      }
      xt *= x;
    }
  }
  *Fx = sumFx;
  *Fy = sumFy;
}

/* integrate_csbend_ordn (src/csbend.c:1459-1720), non-expanded Hamiltonian,
 * no radiation, no reference-trajectory correction, iSlice=-1. */
static int orc_integrate_csbend(orc_r *Qf, const orc_r *Qi, const orc_bend *b, const orc_aperture *ap,
                                orc_r *dz_lost) {
  const double *driftFrac, *kickFrac;
  int nSubsteps = orc_substeps(b->integ_order, &driftFrac, &kickFrac);
  double rho0 = b->rho0;
  long n = b->nSlices, i;
  orc_r dist, f, phi, sine, cosi, tang, sin_phi, cos_phi, factor, Fx, Fy;
  double s = b->length;
  for (int k = 0; k < 6; k++)
    Qf[k] = Qi[k];
  dist = 0;
  s /= n;
  *dz_lost = 0;
  for (i = 0; i < n; i++) {
    if (ap && !orc_check_mult_aperture(Qf[0], Qf[2], ap))
      return 0;
    for (int j = 0; j < nSubsteps; j++) {
      double dsh = s * driftFrac[j];
      f = orc_sqr(1 + Qf[5]) - orc_sqr(Qf[3]);
      if (ORC_VAL(f) <= 0)
        return 0;
      f = ORC_SQRT(f);
      if (ORC_VAL(ORC_FABS(Qf[1] / f)) > 1)
        return 0;
      sin_phi = Qf[1] / f;
      phi = ORC_ASIN(sin_phi);
      sine = ORC_SIN(dsh / rho0 + phi);
      cosi = ORC_COS(dsh / rho0 + phi);
      if (ORC_VAL(cosi) == 0)
        return 0;
      tang = sine / cosi;
      cos_phi = ORC_COS(phi);
      Qf[1] = f * sine;
      factor = (rho0 + Qf[0]) * cos_phi / f * (tang - sin_phi / cos_phi);
      Qf[2] += Qf[3] * factor;
      dist += factor * (1 + Qf[5]);
      *dz_lost += dsh;
      f = cos_phi / cosi;
      Qf[0] = rho0 * (f - 1) + f * Qf[0];
      if (kickFrac[j] == 0)
        break;
      double ds = s * kickFrac[j];
      orc_csbend_fields(b, &Fx, &Fy, Qf[0], Qf[2]);
      Qf[1] += -ds * (1 + Qf[0] / rho0) * Fy / b->rho_actual;
      Qf[3] += ds * (1 + Qf[0] / rho0) * Fx / b->rho_actual;
      if (b->isr_or_rad && (b->rad_coef || b->isr_constant > 0)) {
        /* src/csbend.c:1627-1656 with SYNCH_RAD */
        orc_r f = (1 + Qf[0] * (1. / rho0)) / ORC_SQRT(orc_sqr(1 + Qf[5]) - orc_sqr(Qf[1]) - orc_sqr(Qf[3]));
        orc_r xp = Qf[1] * f;
        orc_r yp = Qf[3] * f;
        orc_r dsFactor = ORC_SQRT(orc_sqr(1 + Qf[0] * (1. / rho0)) + orc_sqr(xp) + orc_sqr(yp));
        orc_r F2 = orc_sqr(Fx) + orc_sqr(Fy);
        orc_r deltaFactor = orc_sqr(1 + Qf[5]);
        double dsISR = s / (nSubsteps - 1);
        Qf[1] /= (1 + Qf[5]);
        Qf[3] /= (1 + Qf[5]);
        if (b->rad_coef)
          Qf[5] -= b->rad_coef * deltaFactor * F2 * ds * dsFactor;
        if (b->isr_constant > 0 && !(orc_isr.single && b->isr1off)) {
          /* src/csbend.c:1649-1651, with the library's deviates */
          const double g =
            trk_isr_gauss(orc_isr.seed, orc_isr.id, orc_isr.pass, orc_isr.elem, (uint32_t)(i * 8 + j), 3.0);
          Qf[5] -= b->isr_constant * deltaFactor * pow(ORC_VAL(F2), 0.75) * ORC_SQRT(dsISR * dsFactor) * g;
        }
        Qf[1] *= (1 + Qf[5]);
        Qf[3] *= (1 + Qf[5]);
      } else if (b->isr_or_rad) {
        /* src/csbend.c:1628-1656: with SYNCH_RAD=0 and ISR=0 the reference
         * still divides and re-multiplies QX, QY by (1+DPoP) */
        Qf[1] /= (1 + Qf[5]);
        Qf[3] /= (1 + Qf[5]);
        Qf[1] *= (1 + Qf[5]);
        Qf[3] *= (1 + Qf[5]);
      }
    }
  }
  *dz_lost = n * s;
  if (ap && !orc_check_mult_aperture(Qf[0], Qf[2], ap))
    return 0;
  Qf[4] += dist;
  return 1;
}

/* convertToDipoleCanonicalCoordinates / convertFrom... (src/csbend.c:1436-1454);
 * with the expanded Hamiltonian the factors are (1+delta) and 1/(1+delta) */
static inline void orc_to_dipole_canonical_x(orc_r *Q, int expanded) {
  orc_r f;
  if (expanded)
    f = (1 + Q[5]);
  else
    f = (1 + Q[5]) / ORC_SQRT(1 + orc_sqr(Q[1]) + orc_sqr(Q[3]));
  Q[1] *= f;
  Q[3] *= f;
}

static inline void orc_from_dipole_canonical_x(orc_r *Q, int expanded) {
  orc_r f;
  if (expanded)
    f = 1 / (1 + Q[5]);
  else
    f = 1 / ORC_SQRT(orc_sqr(1 + Q[5]) - orc_sqr(Q[1]) - orc_sqr(Q[3]));
  Q[1] *= f;
  Q[3] *= f;
}

static inline void orc_to_dipole_canonical(orc_r *Q) { orc_to_dipole_canonical_x(Q, 0); }
static inline void orc_from_dipole_canonical(orc_r *Q) { orc_from_dipole_canonical_x(Q, 0); }

/* integrate_csbend_ordn_expanded (src/csbend.c:1722-1900): the Hamiltonian
 * expanded to leading order, drift Hd1 + Hd2 + Hd1 with
 * Hd1 = -(1+x/rho0)(1+delta)/2 and Hd2 = (qx^2+qy^2)/(2(1+delta)); the
 * aperture is checked at each slice start, after every drift substep and at
 * the end; no reference-trajectory correction, iSlice=-1. */
static int orc_integrate_csbend_expanded(orc_r *Qf, const orc_r *Qi, const orc_bend *b, const orc_aperture *ap,
                                         orc_r *dz_lost) {
  const double *driftFrac, *kickFrac;
  int nSubsteps = orc_substeps(b->integ_order, &driftFrac, &kickFrac);
  double rho0 = b->rho0;
  long n = b->nSlices, i;
  orc_r dist, Fx, Fy;
  double s = b->length;
  for (int k = 0; k < 6; k++)
    Qf[k] = Qi[k];
  dist = 0;
  s /= n;
  *dz_lost = 0;
  for (i = 0; i < n; i++) {
    if (ap && !orc_check_mult_aperture(Qf[0], Qf[2], ap))
      return 0;
    for (int j = 0; j < nSubsteps; j++) {
      double dsh = s * driftFrac[j];
      Qf[1] += dsh * (1 + Qf[5]) / (2 * rho0);
      dist += dsh * (1 + (orc_sqr(Qf[1]) + orc_sqr(Qf[3])) / 2);
      *dz_lost += dsh;
      Qf[0] += Qf[1] * dsh / (1 + Qf[5]);
      Qf[2] += Qf[3] * dsh / (1 + Qf[5]);
      Qf[1] += dsh * (1 + Qf[5]) / (2 * rho0);
      if (ap && !orc_check_mult_aperture(Qf[0], Qf[2], ap))
        return 0;
      if (kickFrac[j] == 0)
        break;
      double ds = s * kickFrac[j];
      orc_csbend_fields(b, &Fx, &Fy, Qf[0], Qf[2]);
      Qf[1] += -ds * (1 + Qf[0] / rho0) * Fy / b->rho_actual;
      Qf[3] += ds * (1 + Qf[0] / rho0) * Fx / b->rho_actual;
      if (b->isr_or_rad && (b->rad_coef || b->isr_constant > 0)) {
        /* src/csbend.c:1833-1863 */
        orc_r f = (1 + Qf[0] * (1. / rho0)) / ORC_SQRT(orc_sqr(1 + Qf[5]) - orc_sqr(Qf[1]) - orc_sqr(Qf[3]));
        orc_r xp = Qf[1] * f;
        orc_r yp = Qf[3] * f;
        orc_r dsFactor = ORC_SQRT(orc_sqr(1 + Qf[0] * (1. / rho0)) + orc_sqr(xp) + orc_sqr(yp));
        orc_r F2 = orc_sqr(Fx) + orc_sqr(Fy);
        orc_r deltaFactor = orc_sqr(1 + Qf[5]);
        double dsISR = s / 3;
        Qf[1] /= (1 + Qf[5]);
        Qf[3] /= (1 + Qf[5]);
        if (b->rad_coef)
          Qf[5] -= b->rad_coef * deltaFactor * F2 * ds * dsFactor;
        if (b->isr_constant > 0 && !(orc_isr.single && b->isr1off)) {
          const double g =
            trk_isr_gauss(orc_isr.seed, orc_isr.id, orc_isr.pass, orc_isr.elem, (uint32_t)(i * 8 + j), 3.0);
          Qf[5] -= b->isr_constant * deltaFactor * pow(ORC_VAL(F2), 0.75) * ORC_SQRT(dsISR * dsFactor) * g;
        }
        Qf[1] *= (1 + Qf[5]);
        Qf[3] *= (1 + Qf[5]);
      } else if (b->isr_or_rad) {
        Qf[1] /= (1 + Qf[5]);
        Qf[3] /= (1 + Qf[5]);
        Qf[1] *= (1 + Qf[5]);
        Qf[3] *= (1 + Qf[5]);
      }
    }
  }
  if (ap && !orc_check_mult_aperture(Qf[0], Qf[2], ap)) {
    *dz_lost = n * s;
    return 0;
  }
  Qf[4] += dist;
  return 1;
}

/* ------------------------------------------------------------ RF energy */
/* add_to_particle_energy (src/simple_rfca.c:987-1006) */
static inline void orc_add_to_particle_energy(orc_r *coord, orc_r timeOfFlight, double Po, orc_r dgamma) {
  orc_r gamma, gamma1, PRatio, P, P1, Pz1, Pz;
  P = Po * (1 + coord[5]);
  gamma = ORC_SQRT(P * P + 1);
  gamma1 = gamma + dgamma;
  if (ORC_VAL(gamma1) <= 1)
    gamma1 = 1 + 1e-7;
  P1 = ORC_SQRT(gamma1 * gamma1 - 1);
  coord[5] = (P1 - Po) / Po;
  coord[4] = timeOfFlight * TRK_C_MKS * P1 / gamma1;
  Pz = P / ORC_SQRT(1 + orc_sqr(coord[1]) + orc_sqr(coord[3]));
  Pz1 = ORC_SQRT(Pz * Pz + gamma1 * gamma1 - gamma * gamma);
  PRatio = Pz / Pz1;
  coord[1] *= PRatio;
  coord[3] *= PRatio;
}

#endif
