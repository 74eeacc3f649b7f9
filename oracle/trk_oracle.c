/*
 * trk_oracle.c -- TEST INFRASTRUCTURE ONLY: the CPU oracle.
 *
 * A plain-C restatement of the reference's element functions for this path
 * and of the do_tracking() pass/element loop, on array-of-structures rows as
 * the reference keeps them (lost particles are swapped behind the survivors).
 * It is the checker for the CUDA path: tests, smoke() and bench.py's CPU
 * baseline call it; the product library neither links nor calls it.
 *
 * Each function cites the reference code it restates (paths relative to the
 * reference project root).  Compile without FMA contraction
 * (-ffp-contract=off) so that it rounds like the reference build
 * (Makefile.rules:218 -O3 -m64, no -march).
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <stdint.h>
#include <string.h>

#include "trk_lattice.h"
#include "trk_oracle.h"
#include "trk_oracle_core.h"

#define SIGN(x) ((x) < 0 ? -1 : 1)

static void swap_rows(double *a, double *b) {
  double t[ORC_STRIDE];
  memcpy(t, a, sizeof(t));
  memcpy(a, b, sizeof(t));
  memcpy(b, t, sizeof(t));
}
#define ROW(i) (coord + (size_t)(i) * ORC_STRIDE)

/* ------------------------------------------------------------ MAXAMP state */
typedef struct {
  int seen;          /* a MAXAMP has been passed (maxamp != NULL) */
  double x_max, y_max;
  int elliptical;
  long exponent, yExponent;
} orc_maxamp;

static void maxamp_update(orc_maxamp *st, const trk_elem *e) {
  st->seen = 1;
  st->x_max = TRK_P(e, MAXAMP_X_MAX);
  st->y_max = TRK_P(e, MAXAMP_Y_MAX);
  st->elliptical = (int)TRK_P(e, MAXAMP_ELLIPTICAL);
  st->exponent = (long)TRK_P(e, MAXAMP_EXPONENT);
  st->yExponent = (long)TRK_P(e, MAXAMP_YEXPONENT);
}

/* setupMultApertureData (src/multipole.c:1690-1749) */
static void setup_aperture(orc_aperture *ap, double reverseTilt, const orc_maxamp *st) {
  memset(ap, 0, sizeof(*ap));
  ap->reverseTilt = reverseTilt;
  ap->reverseTiltC = cos(reverseTilt);
  ap->reverseTiltS = sin(reverseTilt);
  if (st->seen) {
    ap->xMax = st->x_max;
    ap->yMax = st->y_max;
    ap->elliptical = st->elliptical;
    ap->xExponent = ap->yExponent = st->exponent;
    if (st->yExponent)
      ap->yExponent = st->yExponent;
  }
}

/* ---------------------------------------------------- loss filters */
/* limit_amplitudes (src/limit_amplitudes.c:197-288), no open sides */
static long limit_amplitudes(double *coord, double xmax, double ymax, long np, double z, double Po,
                             int extrapolate_z) {
  long ip, itop, is_out;
  double *part, dz, dzx, dzy;
  if (xmax < 0 && ymax < 0)
    return np;
  itop = np - 1;
  for (ip = 0; ip < np; ip++) {
    part = ROW(ip);
    is_out = 0;
    if (xmax > 0 && fabs(part[0]) > xmax)
      is_out += 1;
    if (ymax > 0 && fabs(part[2]) > ymax)
      is_out += 2;
    if (isinf(part[0]) || isinf(part[2]) || isnan(part[0]) || isnan(part[2]))
      is_out += 4;
    dz = 0;
    if (is_out && !(is_out & 4) && extrapolate_z) {
      dzx = dzy = -DBL_MAX;
      if (is_out & 1 && part[1] != 0)
        dzx = (part[0] - SIGN(part[1]) * xmax) / part[1];
      if (is_out & 2 && part[3] != 0)
        dzy = (part[2] - SIGN(part[3]) * ymax) / part[3];
      if (dzx > dzy)
        dz = -dzx;
      else
        dz = -dzy;
      if (dz == -DBL_MAX)
        dz = 0;
    }
    if (is_out) {
      if (ip != itop)
        swap_rows(ROW(ip), ROW(itop));
      ROW(itop)[0] += dz * ROW(itop)[1];
      ROW(itop)[2] += dz * ROW(itop)[3];
      ROW(itop)[4] = z + dz;
      ROW(itop)[5] = Po * (1 + ROW(itop)[5]);
      --itop;
      --ip;
      np--;
    }
  }
  return np;
}

/* elimit_amplitudes (src/limit_amplitudes.c:487-~620), no open sides */
static long elimit_amplitudes(double *coord, double xmax, double ymax, long np, double z, double Po,
                              int extrapolate_z, long exponent, long yexponent, int *err) {
  long ip, itop, xe, ye;
  double *part, a2, b2, c0, c1, c2, dz, det;
  if ((xe = exponent) < 2 || xe % 2) {
    *err = 1;
    return np;
  }
  ye = xe;
  if (yexponent) {
    if ((ye = yexponent) < 2 || ye % 2) {
      *err = 1;
      return np;
    }
  }
  if (xmax <= 0 || ymax <= 0) {
    if (xmax > 0 || ymax > 0)
      return limit_amplitudes(coord, xmax, ymax, np, z, Po, extrapolate_z);
    return np;
  }
  a2 = orc_ipow(xmax, xe);
  b2 = orc_ipow(ymax, ye);
  itop = np - 1;
  for (ip = 0; ip < np; ip++) {
    part = ROW(ip);
    if (isinf(part[0]) || isinf(part[2]) || isnan(part[0]) || isnan(part[2])) {
      swap_rows(ROW(ip), ROW(itop));
      ROW(itop)[4] = z;
      ROW(itop)[5] = sqrt(orc_sqr(Po * (1 + ROW(itop)[5])) + 1);
      --itop;
      --ip;
      np--;
      continue;
    }
    if ((orc_ipow(part[0], xe) / a2 + orc_ipow(part[2], ye) / b2) > 1) {
      dz = 0;
      if (extrapolate_z && xe == 2 && ye == 2) {
        c0 = orc_sqr(part[0]) / a2 + orc_sqr(part[2]) / b2 - 1;
        c1 = 2 * (part[0] * part[1] / a2 + part[2] * part[3] / b2);
        c2 = orc_sqr(part[1]) / a2 + orc_sqr(part[3]) / b2;
        det = orc_sqr(c1) - 4 * c0 * c2;
        if (z > 0 && c2 && det >= 0) {
          if ((dz = (-c1 + sqrt(det)) / (2 * c2)) > 0)
            dz = (-c1 - sqrt(det)) / (2 * c2);
          if ((z + dz) < 0)
            dz = -z;
          part[0] += dz * part[1];
          part[2] += dz * part[3];
        }
      }
      swap_rows(ROW(ip), ROW(itop));
      ROW(itop)[4] = z + dz;
      ROW(itop)[5] = sqrt(orc_sqr(Po * (1 + ROW(itop)[5])) + 1);
      --itop;
      --ip;
      np--;
    }
  }
  return np;
}

/* removeInvalidParticles (src/limit_amplitudes.c:~290-345) */
static long remove_invalid(double *coord, long np, double z, double Po) {
  long ip, itop = np - 1;
  for (ip = 0; ip < np; ip++) {
    double *part = ROW(ip);
    int is_out = 0;
    for (int ic = 0; ic < 6; ic++)
      if (isnan(part[ic])) {
        is_out = 1;
        break;
      }
    if (part[5] <= -1)
      is_out = 1;
    if (is_out) {
      swap_rows(ROW(ip), ROW(itop));
      ROW(itop)[4] = z;
      ROW(itop)[5] = Po * (1 + ROW(itop)[5]);
      --itop;
      --ip;
      np--;
    }
  }
  return np;
}

/* ------------------------------------------------------- simple maps */
/* DRIF: drift_matrix (src/compute_matrices.c:391-413) tracked by
 * track_particles (src/matrix.c:212-469) with TURBO_FASTMATTRACK=3, i.e.
 * fin[i] = C[i] + sum_{j=5..0} (R[i][j] + sum_{k=j..0} T[i][j][k] ini[k]) ini[j]
 * over the full 6x6 / 6x21 arrays, zeros included. */
static void drift_matrix_track(double *coord, long np, double L, long order) {
  double C[6] = {0}, R[6][6] = {{0}}, T[6][6][6] = {{{0}}};
  if (order == 0)
    order = 2; /* run->default_order (src/elegant.nl:43) */
  if (order > 2)
    order = 2;
  C[4] = L;
  R[0][0] = R[1][1] = R[2][2] = R[3][3] = R[4][4] = R[5][5] = 1;
  R[0][1] = R[2][3] = L;
  if (order > 1)
    T[4][1][1] = T[4][3][3] = L / 2;
  for (long ip = 0; ip < np; ip++) {
    double *ini = ROW(ip), temp[6];
    for (int i = 5; i >= 0; i--) {
      double sum = C[i];
      if (order == 2) {
        for (int j = 5; j >= 0; j--) {
          double sum1 = R[i][j];
          for (int k = j; k >= 0; k--)
            sum1 += T[i][j][k] * ini[k];
          sum += sum1 * ini[j];
        }
      } else {
        for (int j = 5; j >= 0; j--)
          sum += R[i][j] * ini[j];
      }
      temp[i] = sum;
    }
    for (int i = 5; i >= 0; i--)
      ini[i] = temp[i];
  }
}

/* exactDrift (src/csbend.c:3792-3816) */
static void exact_drift(double *coord, long np, double L) {
  for (long i = 0; i < np; i++) {
    double *c = ROW(i);
    c[0] += c[1] * L;
    c[2] += c[3] * L;
    c[4] += L * sqrt(1 + orc_sqr(c[1]) + orc_sqr(c[3]));
  }
}

/* offsetBeamCoordinatesForMisalignment (src/malign_mat.c:257-267) */
static void offset_beam(double *coord, long np, double dx, double dy, double dz) {
  for (long ip = np - 1; ip >= 0; ip--) {
    double *part = ROW(ip);
    part[4] += dz * sqrt(1 + orc_sqr(part[1]) + orc_sqr(part[3]));
    part[0] = part[0] - dx + dz * part[1];
    part[2] = part[2] - dy + dz * part[3];
  }
}

/* rotateBeamCoordinatesForMisalignment (src/tilt_matrices.c:156-190) */
static void rotate_beam(double *coord, long np, double angle) {
  double sin_a, cos_a;
  if (!angle || fabs(fabs(angle) - TRK_PIx2) < 1e-12)
    return;
  if (fabs(fabs(angle) - TRK_PI) < 1e-12) {
    cos_a = -1;
    sin_a = 0;
  } else if (fabs(angle - TRK_PIo2) < 1e-12) {
    cos_a = 0;
    sin_a = 1;
  } else if (fabs(angle + TRK_PIo2) < 1e-12) {
    cos_a = 0;
    sin_a = -1;
  } else {
    cos_a = cos(angle);
    sin_a = sin(angle);
  }
  for (long i = 0; i < np; i++) {
    double *c = ROW(i);
    double x = c[0], xp = c[1], y = c[2], yp = c[3];
    c[0] = x * cos_a + y * sin_a;
    c[2] = -x * sin_a + y * cos_a;
    c[1] = xp * cos_a + yp * sin_a;
    c[3] = -xp * sin_a + yp * cos_a;
  }
}

/* ------------------------------------------------------------ multipoles */
/* multipole_tracking2 (src/multipole.c:660-1084) for KQUAD, KSEXT, KOCT,
 * MALIGN_METHOD=0, no radiation, no fringe, no error multipoles. */
/* quadPartialFringeMatrix (src/fringe.c:231-275): the 2x2 blocks of one
 * linear fringe part, R = {R00, R01, R10, R11, R22, R23, R32, R33} */
static void quad_partial_fringe_matrix(double *R, double K1, long inFringe, const double *fringeInt, long part) {
  double J1x, J2x, J3x, J1y, J2y, J3y, K1sqr, expJ1x, expJ1y;
  K1sqr = orc_sqr(K1);
  if (part == 1) {
    J1x = inFringe * (K1 * fringeInt[1] - 2 * K1sqr * fringeInt[3] / 3. - K1sqr * fringeInt[0] * fringeInt[2] / 2);
    J2x = inFringe * K1 * fringeInt[2];
    J3x = inFringe * K1sqr * (fringeInt[2] + fringeInt[4] + fringeInt[0] * fringeInt[1]);
    J1y = inFringe * (-K1 * fringeInt[1] - 2 * K1sqr * fringeInt[3] / 3. - K1sqr * fringeInt[0] * fringeInt[2] / 2);
    J2y = -J2x;
    J3y = J3x;
  } else {
    J1x = inFringe * (K1 * fringeInt[1] + K1sqr * fringeInt[0] * fringeInt[2] / 2);
    J2x = inFringe * K1 * fringeInt[2];
    J3x = inFringe * K1sqr * (fringeInt[4] - fringeInt[0] * fringeInt[1]);
    J1y = inFringe * (-K1 * fringeInt[1] + K1sqr * fringeInt[0] * fringeInt[2] / 2);
    J2y = -J2x;
    J3y = J3x;
  }
  expJ1x = R[0] = orc_exp_sel(J1x);
  R[1] = J2x / expJ1x;
  R[2] = expJ1x * J3x;
  R[3] = (1 + J2x * J3x) / expJ1x;
  expJ1y = R[4] = orc_exp_sel(J1y);
  R[5] = J2y / expJ1y;
  R[6] = expJ1y * J3y;
  R[7] = (1 + J2y * J3y) / expJ1y;
}

#define ORC_SWAP(a, b)                                                                                             \
  do {                                                                                                             \
    double t_ = (a);                                                                                               \
    (a) = (b);                                                                                                     \
    (b) = t_;                                                                                                      \
  } while (0)

/* quadFringe (src/fringe.c:25-219): KQUAD hard-edge fringe, linear parts
 * from the fringe integrals and the leading (|higherOrder| = 2) or higher
 * (3) order nonlinear generator, on every row of coord */
static void quad_fringe(double *coord, long np, double K1, const double *fringeIntM, const double *fringeIntP,
                        int backtrack, int inFringe, int higherOrder, int linearFlag, double nonlinearFactor) {
  double M1[8], M2[8];
  if (linearFlag) {
    quad_partial_fringe_matrix(M1, K1, 1, fringeIntM, 1);
    quad_partial_fringe_matrix(M2, K1, 1, fringeIntP, 2);
    if (inFringe * (backtrack ? -1 : 1) == -1) {
      ORC_SWAP(M1[0], M1[3]);
      ORC_SWAP(M1[4], M1[7]);
      ORC_SWAP(M2[0], M2[3]);
      ORC_SWAP(M2[4], M2[7]);
      for (int k = 0; k < 8; k++)
        ORC_SWAP(M1[k], M2[k]);
    }
    if (backtrack) {
      ORC_SWAP(M1[0], M1[3]);
      ORC_SWAP(M1[4], M1[7]);
      M1[1] *= -1;
      M1[2] *= -1;
      M1[5] *= -1;
      M1[6] *= -1;
      ORC_SWAP(M2[0], M2[3]);
      ORC_SWAP(M2[4], M2[7]);
      M2[1] *= -1;
      M2[2] *= -1;
      M2[5] *= -1;
      M2[6] *= -1;
    }
  }
  for (long ip = 0; ip < np; ip++) {
    double *vec = ROW(ip);
    double x, px, y, py, delta, xp, yp, denom, a, dx, dpx, dy, dpy, ds;
    delta = vec[5];
    xp = vec[1];
    yp = vec[3];
    denom = sqrt(1 + orc_sqr(xp) + orc_sqr(yp));
    vec[1] = (1 + delta) * xp / denom;
    vec[3] = (1 + delta) * yp / denom;
    if (linearFlag) {
      x = M1[0] * vec[0] + M1[1] * vec[1];
      px = M1[2] * vec[0] + M1[3] * vec[1];
      y = M1[4] * vec[2] + M1[5] * vec[3];
      py = M1[6] * vec[2] + M1[7] * vec[3];
    } else {
      x = vec[0];
      px = vec[1];
      y = vec[2];
      py = vec[3];
    }
    a = -inFringe * K1 / (12 * (1 + delta));
    dx = dpx = dy = dpy = ds = 0;
    if (abs(higherOrder) > 1) {
      double xpow[9], ypow[9], apow[4];
      xpow[0] = ypow[0] = apow[0] = 1;
      if (abs(higherOrder) > 2) {
        for (int i = 1; i < 9; i++) {
          xpow[i] = xpow[i - 1] * x;
          ypow[i] = ypow[i - 1] * y;
        }
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
                 12 * a * orc_sqr(xpow[2] - ypow[2]))) /
               8;
          dy = (a * y *
                (-8 * (3 * xpow[2] + ypow[2]) +
                 4 * apow[2] * (xpow[6] + 25 * xpow[4] * ypow[2] - 21 * xpow[2] * ypow[4] - 5 * ypow[6]) +
                 apow[3] * (3 * xpow[8] - 108 * xpow[6] * ypow[2] + 498 * xpow[4] * ypow[4] + 84 * xpow[2] * ypow[6] +
                            35 * ypow[8]) +
                 12 * a * orc_sqr(xpow[2] - ypow[2]))) /
               8;
        }
      } else {
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
    if (linearFlag) {
      vec[0] = M2[0] * x + M2[1] * px;
      vec[1] = M2[2] * x + M2[3] * px;
      vec[2] = M2[4] * y + M2[5] * py;
      vec[3] = M2[6] * y + M2[7] * py;
    } else {
      vec[0] = x;
      vec[1] = px;
      vec[2] = y;
      vec[3] = py;
    }
    vec[4] -= nonlinearFactor * ds;
    px = vec[1];
    py = vec[3];
    denom = orc_sqr(1 + delta) - orc_sqr(px) - orc_sqr(py);
    if (denom > 0) {
      denom = sqrt(denom);
      vec[1] = px / denom;
      vec[3] = py / denom;
    } else
      vec[1] = vec[3] = DBL_MAX;
  }
}

static long multipole_tracking2(double *coord, long n_part, const trk_elem *e, double Po, double z_start,
                                const orc_maxamp *st, int *err) {
  orc_mult m;
  double tilt = 0, dx = 0, dy = 0, dz = 0, lEnd = 0, lEffective;
  long n_kicks = 0, nSlices = 0;
  int doEndDrift = 0;
  double cfac = TRK_E_MKS / (TRK_ME_MKS * TRK_C_MKS * Po);
  memset(&m, 0, sizeof(m));
  switch (e->type) {
  case TRK_KQUAD:
    nSlices = (long)TRK_P(e, KQUAD_N_SLICES);
    n_kicks = (long)TRK_P(e, KQUAD_N_KICKS);
    m.expand = (int)TRK_P(e, KQUAD_EXPAND_HAMILTONIAN);
    m.order[0] = 1;
    if ((lEffective = TRK_P(e, KQUAD_LEFFECTIVE)) <= 0)
      lEffective = TRK_P(e, KQUAD_L);
    else {
      lEnd = (TRK_P(e, KQUAD_L) - lEffective) / 2;
      doEndDrift = 1;
    }
    if (TRK_P(e, KQUAD_BORE))
      m.KnL[0] = TRK_P(e, KQUAD_B) / TRK_P(e, KQUAD_BORE) * cfac * lEffective * (1 + TRK_P(e, KQUAD_FSE));
    else
      m.KnL[0] = TRK_P(e, KQUAD_K1) * lEffective * (1 + TRK_P(e, KQUAD_FSE));
    m.drift = lEffective;
    tilt = TRK_P(e, KQUAD_TILT);
    dx = TRK_P(e, KQUAD_DX);
    dy = TRK_P(e, KQUAD_DY);
    dz = TRK_P(e, KQUAD_DZ);
    m.xkick = TRK_P(e, KQUAD_HKICK) * TRK_P(e, KQUAD_HCALIBRATION);
    m.ykick = TRK_P(e, KQUAD_VKICK) * TRK_P(e, KQUAD_VCALIBRATION);
    m.integ_order = (int)TRK_P(e, KQUAD_INTEGRATION_ORDER);
    break;
  case TRK_KSEXT:
    n_kicks = (long)TRK_P(e, KSEXT_N_KICKS);
    nSlices = (long)TRK_P(e, KSEXT_N_SLICES);
    m.expand = (int)TRK_P(e, KSEXT_EXPAND_HAMILTONIAN);
    m.order[0] = 2;
    if (TRK_P(e, KSEXT_BORE))
      m.KnL[0] = 2 * TRK_P(e, KSEXT_B) / orc_sqr(TRK_P(e, KSEXT_BORE)) * cfac * TRK_P(e, KSEXT_L) *
                 (1 + TRK_P(e, KSEXT_FSE));
    else
      m.KnL[0] = TRK_P(e, KSEXT_K2) * TRK_P(e, KSEXT_L) * (1 + TRK_P(e, KSEXT_FSE));
    m.drift = lEffective = TRK_P(e, KSEXT_L);
    tilt = TRK_P(e, KSEXT_TILT);
    dx = TRK_P(e, KSEXT_DX);
    dy = TRK_P(e, KSEXT_DY);
    dz = TRK_P(e, KSEXT_DZ);
    m.xkick = TRK_P(e, KSEXT_HKICK) * TRK_P(e, KSEXT_HCALIBRATION);
    m.ykick = TRK_P(e, KSEXT_VKICK) * TRK_P(e, KSEXT_VCALIBRATION);
    m.integ_order = (int)TRK_P(e, KSEXT_INTEGRATION_ORDER);
    if (TRK_P(e, KSEXT_K1)) {
      m.KnL[1] = TRK_P(e, KSEXT_K1) * TRK_P(e, KSEXT_L);
      m.order[1] = 1;
    }
    if (TRK_P(e, KSEXT_J1)) {
      m.KnL[2] = TRK_P(e, KSEXT_J1) * TRK_P(e, KSEXT_L);
      m.order[2] = 1;
      m.skew[2] = 1;
    }
    break;
  case TRK_KOCT:
    n_kicks = (long)TRK_P(e, KOCT_N_KICKS);
    nSlices = (long)TRK_P(e, KOCT_N_SLICES);
    m.expand = (int)TRK_P(e, KOCT_EXPAND_HAMILTONIAN);
    m.order[0] = 3;
    if (TRK_P(e, KOCT_BORE))
      m.KnL[0] = 6 * TRK_P(e, KOCT_B) / orc_ipow(TRK_P(e, KOCT_BORE), 3) * cfac * TRK_P(e, KOCT_L) *
                 (1 + TRK_P(e, KOCT_FSE));
    else
      m.KnL[0] = TRK_P(e, KOCT_K3) * TRK_P(e, KOCT_L) * (1 + TRK_P(e, KOCT_FSE));
    m.drift = lEffective = TRK_P(e, KOCT_L);
    tilt = TRK_P(e, KOCT_TILT);
    dx = TRK_P(e, KOCT_DX);
    dy = TRK_P(e, KOCT_DY);
    dz = TRK_P(e, KOCT_DZ);
    m.integ_order = (int)TRK_P(e, KOCT_INTEGRATION_ORDER);
    break;
  default:
    *err = 1;
    return n_part;
  }
  (void)lEffective;
  {
    /* SYNCH_RAD: rad_coef = e^2 Po^3 / (6 pi eps0 c^2 m), dropped for
     * elements shorter than 1e-6 m (src/multipole.c:755-763) */
    int synch = 0;
    double length = 0;
    if (e->type == TRK_KQUAD) {
      synch = TRK_P(e, KQUAD_SYNCH_RAD) != 0;
      length = TRK_P(e, KQUAD_L);
    } else if (e->type == TRK_KSEXT) {
      synch = TRK_P(e, KSEXT_SYNCH_RAD) != 0;
      length = TRK_P(e, KSEXT_L);
    } else {
      synch = TRK_P(e, KOCT_SYNCH_RAD) != 0;
      length = TRK_P(e, KOCT_L);
    }
    if (synch && !(length < 1e-6))
      m.rad_coef = (TRK_E_MKS * TRK_E_MKS) * (Po * Po * Po) /
                   (6 * TRK_PI * TRK_EPSILON_O * (TRK_C_MKS * TRK_C_MKS) * TRK_ME_MKS);
    /* ISR: isr_coef = r_e sqrt(55/(24 sqrt 3) Po^5 137.0359895) (src/multipole.c:757-763) */
    int isr = 0, isr1 = 1;
    if (e->type == TRK_KQUAD) {
      isr = TRK_P(e, KQUAD_ISR) != 0;
      isr1 = TRK_P(e, KQUAD_ISR1PART) != 0;
    } else if (e->type == TRK_KSEXT) {
      isr = TRK_P(e, KSEXT_ISR) != 0;
      isr1 = TRK_P(e, KSEXT_ISR1PART) != 0;
    } else {
      isr = TRK_P(e, KOCT_ISR) != 0;
      isr1 = TRK_P(e, KOCT_ISR1PART) != 0;
    }
    if (isr && !(length < 1e-6)) {
      m.isr_coef = TRK_RE_MKS * sqrt(55.0 / (24 * sqrt(3.0)) * orc_ipow(Po, 5) * 137.0359895);
      m.isr1off = !isr1;
    }
  }
  if (m.integ_order != 2 && m.integ_order != 4 && m.integ_order != 6) {
    *err = 1;
    return n_part;
  }
  if (n_kicks <= 0) {
    if (nSlices <= 0) {
      *err = 1;
      return n_part;
    }
  } else {
    if (m.integ_order > 2) {
      if ((nSlices = (long)ceil(n_kicks / (1.0 * m.integ_order))) < 1)
        nSlices = 1;
    } else
      nSlices = n_kicks;
  }
  m.nSlices = (int)nSlices;
  m.maxOrder = m.order[0] > m.order[1] ? m.order[0] : m.order[1];
  if (m.order[2] > m.maxOrder)
    m.maxOrder = m.order[2];
  m.dx = dx;
  m.dy = dy;

  orc_aperture ap;
  setup_aperture(&ap, -tilt, st);

  /* offsetParticlesForMisalignment, mode 0 entry (src/malign_mat.c:578-584) */
  if (dx || dy || dz)
    offset_beam(coord, n_part, dx, dy, dz);
  if (tilt)
    rotate_beam(coord, n_part, tilt);
  if (doEndDrift)
    exact_drift(coord, n_part, lEnd);
  /* KQUAD entrance fringe (src/multipole.c:999-1006) */
  if (e->type == TRK_KQUAD && TRK_P(e, KQUAD_EDGE1_EFFECTS) > 0)
    quad_fringe(coord, n_part, TRK_P(e, KQUAD_K1), &TRK_P(e, KQUAD_I0M), &TRK_P(e, KQUAD_I0P), TRK_P(e, KQUAD_L) < 0,
                -1, (int)TRK_P(e, KQUAD_EDGE1_EFFECTS), (int)TRK_P(e, KQUAD_EDGE1_LINEAR),
                TRK_P(e, KQUAD_EDGE1_NONLINEAR_FACTOR));

  long i_top = n_part - 1;
  /* one dzLoss for the whole call, as in the reference (src/multipole.c:686):
   * integrate_kick_multipole_ordn resets it only after its entry checks
   * (:1179-1186, :1232), so a particle rejected there is recorded at
   * z_start plus the previous particle's dzLoss */
  double dzLoss = 0;
  for (long i_part = 0; i_part <= i_top; i_part++) {
    if (!orc_integrate_kick_multipole(ROW(i_part), &m, Po, &ap, &dzLoss)) {
      swap_rows(ROW(i_part), ROW(i_top));
      ROW(i_top)[4] = z_start + dzLoss;
      ROW(i_top)[5] = Po * (1 + ROW(i_top)[5]);
      i_top--;
      i_part--;
    }
  }
  /* KQUAD exit fringe, on every row, lost ones included (src/multipole.c:1054-1061) */
  if (e->type == TRK_KQUAD && TRK_P(e, KQUAD_EDGE2_EFFECTS) > 0)
    quad_fringe(coord, n_part, TRK_P(e, KQUAD_K1), &TRK_P(e, KQUAD_I0M), &TRK_P(e, KQUAD_I0P), TRK_P(e, KQUAD_L) < 0,
                1, (int)TRK_P(e, KQUAD_EDGE2_EFFECTS), (int)TRK_P(e, KQUAD_EDGE2_LINEAR),
                TRK_P(e, KQUAD_EDGE2_NONLINEAR_FACTOR));
  if (doEndDrift)
    exact_drift(coord, n_part, lEnd);
  if (dx || dy || dz || tilt) {
    if (tilt)
      rotate_beam(coord, n_part, -tilt);
    if (dx || dy || dz)
      offset_beam(coord, n_part, -dx, -dy, -dz);
  }
  return i_top + 1;
}

/* ------------------------------------------------------------- CSBEND */
/* Field-expansion coefficients of a curved multipole magnet.  The
 * reference evaluates closed forms (computeCSBENDFieldCoefficients,
 * src/csbend.c:175-~650); here the same coefficients come from the recursion
 * that Laplace's equation imposes in the curvilinear frame with curvature h:
 *   curl:  (i+1) a[i+1][j] = (j+1) c[i][j+1]
 *   div :  (i+1) (c[i+1][j] + h c[i][j]) + (j+1) (a[i][j+1] + h a[i-1][j+1]) = 0
 * where a[i][j], c[i][j] are the coefficients of x^i y^j in Fy and Fx, and the
 * mid-plane data are a[i][0] = b_i / i!, c[i][0] = -c_i / i! (i = 1..8).  The
 * dipole / steering terms enter only [0][0], as in the reference. */
static void csbend_field_table(orc_bend *bd, const double *b, const double *c, double h, int nonlinear,
                               long expansionOrder) {
  double a[12][12], cx[12][12];
  int i, j;
  if (expansionOrder == 0) {
    for (i = 8; i >= 0; i--)
      if (b[i] || c[i])
        break;
    if ((expansionOrder = i + 2) < 4)
      expansionOrder = 4;
  }
  bd->expansionOrder1 = (int)expansionOrder + 1;
  bd->hasNormal = bd->hasSkew = 0;
  for (i = 0; i < 9; i++) {
    if (b[i])
      bd->hasNormal = 1;
    if (c[i])
      bd->hasSkew = 1;
  }
  memset(a, 0, sizeof(a));
  memset(cx, 0, sizeof(cx));
  double fact = 1;
  for (i = 1; i <= 8; i++) {
    fact *= i;
    a[i][0] = b[i] / fact;
    cx[i][0] = -c[i] / fact;
  }
  for (j = 0; j < 10; j++) {
    for (i = 0; i + j + 1 <= 10; i++)
      cx[i][j + 1] = (i + 1) * a[i + 1][j] / (j + 1);
    for (i = 0; i + j + 1 <= 10; i++) {
      double prev = i > 0 ? a[i - 1][j + 1] : 0.0;
      a[i][j + 1] = -h * prev - (i + 1) * (cx[i + 1][j] + h * cx[i][j]) / (j + 1);
    }
  }
  memset(bd->Fx_xy, 0, sizeof(bd->Fx_xy));
  memset(bd->Fy_xy, 0, sizeof(bd->Fy_xy));
  if (nonlinear) {
    for (i = 0; i <= 10; i++)
      for (j = 0; i + j <= 10; j++) {
        bd->Fx_xy[i][j] = cx[i][j];
        bd->Fy_xy[i][j] = a[i][j];
      }
  } else {
    bd->Fx_xy[0][1] = cx[0][1];
    bd->Fy_xy[1][0] = a[1][0];
    bd->Fy_xy[0][1] = a[0][1];
    bd->Fx_xy[1][0] = cx[1][0];
  }
  bd->Fx_xy[0][0] = c[0];
  bd->Fy_xy[0][0] = 1 - b[0];
}

typedef struct {
  orc_bend bd;
  double angle, e1, e2, tilt, etilt, rho0, h, n, fse, rho_actual;
  double psi1, psi2, e1_kick_limit, e2_kick_limit, he1, he2;
  double hgap, fint1, fint2; /* fringe: HGAP and FINT1/FINT2 (FINT where negative) */
  double fringe_int[2][7];   /* EDGE_EFFECTS=5: FRINGE1K0..6, FRINGE2K0..6 */
  double k1_fringe;          /* b[1]/rho0, the body gradient the edge maps take */
  double cos_ttilt, sin_ttilt, dcoord_etilt[6];
  double dxi, dyi, dzi, dxf, dyf, dzf;
  int edge1, edge2, edge_order, edge1_effects, edge2_effects;
  int is_drift;
} orc_csbend_setup;

/* computeEtiltCentroidOffset (src/csbend.c:4748-4790) */
static void etilt_centroid_offset(double *d, double rho0, double angle, double etilt) {
  double q1a, q2a, q3a, q1b, q2b, q3b, qp1, qp2, qp3, dz, tan_alpha, k;
  if (!etilt) {
    for (int i = 0; i < 6; i++)
      d[i] = 0;
    return;
  }
  etilt *= -1;
  q1a = (1 - cos(angle)) * rho0 * (cos(etilt) - 1);
  q2a = 0;
  q3a = (1 - cos(angle)) * rho0 * sin(etilt);
  qp1 = sin(angle) * cos(etilt);
  qp2 = cos(angle);
  k = sqrt(orc_sqr(qp1) + orc_sqr(qp2));
  qp1 /= k;
  qp2 /= k;
  qp3 = sin(angle) * sin(etilt) / k;
  tan_alpha = 1. / tan(angle) / cos(etilt);
  q1b = q1a * tan_alpha / (tan(angle) + tan_alpha);
  q2b = -q1b * tan(angle);
  dz = sqrt(orc_sqr(q1b - q1a) + orc_sqr(q2b - q2a));
  q3b = q3a + qp3 * dz;
  d[0] = sqrt(orc_sqr(q1b) + orc_sqr(q2b));
  d[1] = tan(atan(tan_alpha) - (TRK_PIo2 - angle));
  d[2] = q3b;
  d[3] = qp3;
  d[4] = dz * sqrt(1 + orc_sqr(qp3));
  d[5] = 0;
}

/* determine_bend_flags (src/bend_matrix.c:1347-1394): an edge is active
 * unless a same-named CSBEND is adjacent (through MARKs). */
static void bend_edge_flags(const trk_lattice *l, int idx, int *edge1, int *edge2) {
  const trk_elem *e = &l->e[idx];
  int precedes = 0, follows = 0;
  for (int k = idx - 1; k >= 0; k--) {
    if (l->e[k].type == e->type && strcmp(l->e[k].name, e->name) == 0) {
      precedes = 1;
      break;
    }
    if (l->e[k].type != TRK_MARK)
      break;
  }
  for (int k = idx + 1; k < l->n; k++) {
    if (l->e[k].type == e->type && strcmp(l->e[k].name, e->name) == 0) {
      follows = 1;
      break;
    }
    if (l->e[k].type != TRK_MARK)
      break;
  }
  *edge1 = TRK_P(e, CSBEND_EDGE1_EFFECTS) && !precedes;
  *edge2 = TRK_P(e, CSBEND_EDGE2_EFFECTS) && !follows;
}

/* Per-call set-up of track_through_csbend (src/csbend.c:654-1078) */
static int csbend_setup(const trk_lattice *l, int idx, double Po, orc_csbend_setup *S) {
  const trk_elem *e = &l->e[idx];
  double b[9], c[9];
  memset(S, 0, sizeof(*S));
  if (TRK_P(e, CSBEND_REFERENCE_CORRECTION) || TRK_P(e, CSBEND_FSE_CORRECTION) || TRK_P(e, CSBEND_MALIGN_METHOD) ||
      TRK_P(e, CSBEND_USE_RAD_DIST))
    return 1;
  if (TRK_P(e, CSBEND_ANGLE) == 0) {
    S->is_drift = 1;
    return 0;
  }
  int io = (int)TRK_P(e, CSBEND_INTEGRATION_ORDER);
  if (io != 2 && io != 4 && io != 6)
    return 1;
  double L = TRK_P(e, CSBEND_L), ANGLE = TRK_P(e, CSBEND_ANGLE);
  double rho0 = L / ANGLE;
  b[0] = 0;
  if (TRK_P(e, CSBEND_USE_BN)) {
    for (int i = 1; i <= 8; i++)
      b[i] = e->p[P_CSBEND_B1 + i - 1];
  } else {
    for (int i = 1; i <= 8; i++)
      b[i] = e->p[P_CSBEND_K1 + i - 1] * rho0;
  }
  for (int j = 0; j < 9; j++)
    c[j] = 0;
  /* fractional field errors fn, gn at XREFERENCE (src/csbend.c:824-848) */
  if (TRK_P(e, CSBEND_XREFERENCE) > 0) {
    const double xr = TRK_P(e, CSBEND_XREFERENCE);
    double term = 1 / xr;
    for (int i = 0; i < 8; i++) {
      b[i + 1] += e->p[P_CSBEND_F1 + i] * term;
      c[i + 1] += e->p[P_CSBEND_G1 + i] * term;
      term *= (i + 2) / xr;
    }
  }
  double fse_ = TRK_P(e, CSBEND_FSE), fseD = TRK_P(e, CSBEND_FSE_DIPOLE), fseQ = TRK_P(e, CSBEND_FSE_QUADRUPOLE);
  b[1] *= (1 + fse_ + fseQ) / (1 + fse_ + fseD);
  c[1] *= (1 + fse_ + fseQ) / (1 + fse_ + fseD);
  S->k1_fringe = b[1] / rho0;
  for (int k = 0; k < 7; k++) {
    S->fringe_int[0][k] = e->p[P_CSBEND_FRINGE1K0 + k];
    S->fringe_int[1][k] = e->p[P_CSBEND_FRINGE2K0 + k];
  }
  b[2] *= (1 + fse_) / (1 + fse_ + fseD);
  c[2] *= (1 + fse_) / (1 + fse_ + fseD);
  b[0] = TRK_P(e, CSBEND_XKICK) / ANGLE;
  c[0] = TRK_P(e, CSBEND_YKICK) / ANGLE;
  S->he1 = TRK_P(e, CSBEND_H1);
  S->he2 = TRK_P(e, CSBEND_H2);
  if (ANGLE < 0) {
    S->angle = -ANGLE;
    S->e1 = -TRK_P(e, CSBEND_E1);
    S->e2 = -TRK_P(e, CSBEND_E2);
    S->etilt = TRK_P(e, CSBEND_ETILT) * TRK_P(e, CSBEND_ETILT_SIGN);
    S->tilt = TRK_P(e, CSBEND_TILT) + TRK_PI;
    rho0 = L / S->angle;
    for (int i = 1; i < 9; i += 2) {
      b[i] *= -1;
      c[i] *= -1;
    }
  } else {
    S->angle = ANGLE;
    S->e1 = TRK_P(e, CSBEND_E1);
    S->e2 = TRK_P(e, CSBEND_E2);
    S->etilt = TRK_P(e, CSBEND_ETILT) * TRK_P(e, CSBEND_ETILT_SIGN);
    S->tilt = TRK_P(e, CSBEND_TILT);
    rho0 = L / S->angle;
  }
  if (fabs(rho0) > 1e6) {
    if (TRK_P(e, CSBEND_K1) != 0 || TRK_P(e, CSBEND_K2) != 0)
      return 1; /* treated as KQUAD by the reference; not on this path */
    S->is_drift = 1;
    return 0;
  }
  S->rho0 = rho0;
  S->fse = fse_ + fseD;
  S->h = 1 / rho0;
  S->n = -b[1] / S->h;
  if (fabs(S->fse + 1) < 1e-12)
    S->fse = -1 + 1e-12;
  S->rho_actual = 1 / ((1 + S->fse) * S->h);
  S->e1_kick_limit = TRK_P(e, CSBEND_EDGE1_KICK_LIMIT);
  S->e2_kick_limit = TRK_P(e, CSBEND_EDGE2_KICK_LIMIT);
  if (TRK_P(e, CSBEND_KICK_LIMIT_SCALING)) {
    S->e1_kick_limit *= rho0 / S->rho_actual;
    S->e2_kick_limit *= rho0 / S->rho_actual;
  }
  double hgap = TRK_P(e, CSBEND_HGAP);
  double fint1 = TRK_P(e, CSBEND_FINT1) >= 0 ? TRK_P(e, CSBEND_FINT1) : TRK_P(e, CSBEND_FINT);
  double fint2 = TRK_P(e, CSBEND_FINT2) >= 0 ? TRK_P(e, CSBEND_FINT2) : TRK_P(e, CSBEND_FINT);
  S->hgap = hgap;
  S->fint1 = fint1;
  S->fint2 = fint2;
  double Kg1 = 2 * hgap * fint1 * SIGN(rho0);
  S->psi1 = Kg1 / fabs(S->rho_actual) / cos(S->e1) * (1 + orc_sqr(sin(S->e1)));
  double Kg2 = 2 * hgap * fint2 * SIGN(rho0);
  S->psi2 = Kg2 / fabs(S->rho_actual) / cos(S->e2) * (1 + orc_sqr(sin(S->e2)));
  if (L < 0) {
    S->psi1 *= -1;
    S->psi2 *= -1;
  }
  S->bd.rho0 = rho0;
  S->bd.rho_actual = S->rho_actual;
  S->bd.length = L;
  S->bd.nSlices = (int)TRK_P(e, CSBEND_N_SLICES);
  if (S->bd.nSlices < 1)
    return 1;
  S->bd.integ_order = io;
  S->bd.expanded = TRK_P(e, CSBEND_EXPAND_HAMILTONIAN) != 0;
  /* isrConstant is nonzero (negative) whenever Po>0 even with ISR=0
   * (src/csbend.c:931-934), which enables the (1+DPoP) round trip */
  S->bd.isr_or_rad = Po > 0;
  /* SYNCH_RAD (src/csbend.c:953-959) */
  if (TRK_P(e, CSBEND_ISR)) {
    /* isrConstant (src/csbend.c:961-964) */
    const double ra = fabs(S->rho_actual);
    S->bd.isr_constant = TRK_RE_MKS * sqrt(55.0 / (24 * sqrt(3.0)) * orc_ipow(Po, 5) * 137.0359895 / (ra * ra * ra));
    S->bd.isr1off = TRK_P(e, CSBEND_ISR1PART) == 0;
  }
  if (TRK_P(e, CSBEND_SYNCH_RAD))
    S->bd.rad_coef = (TRK_E_MKS * TRK_E_MKS) * (Po * Po * Po) * ((1 + S->fse) * (1 + S->fse)) /
                     (6 * TRK_PI * TRK_EPSILON_O * (TRK_C_MKS * TRK_C_MKS) * TRK_ME_MKS * (S->bd.rho0 * S->bd.rho0));
  csbend_field_table(&S->bd, b, c, S->h, (int)TRK_P(e, CSBEND_NONLINEAR), (long)TRK_P(e, CSBEND_EXPANSION_ORDER));

  double ttilt = S->tilt + S->etilt;
  if (ttilt == 0) {
    S->cos_ttilt = 1;
    S->sin_ttilt = 0;
  } else if (fabs(fabs(ttilt) - TRK_PI) < 1e-12) {
    S->cos_ttilt = -1;
    S->sin_ttilt = 0;
  } else if (fabs(ttilt - TRK_PIo2) < 1e-12) {
    S->cos_ttilt = 0;
    S->sin_ttilt = 1;
  } else if (fabs(ttilt + TRK_PIo2) < 1e-12) {
    S->cos_ttilt = 0;
    S->sin_ttilt = -1;
  } else {
    S->cos_ttilt = cos(ttilt);
    S->sin_ttilt = sin(ttilt);
  }
  etilt_centroid_offset(S->dcoord_etilt, rho0, S->angle, S->etilt);
  double dx = TRK_P(e, CSBEND_DX), dy = TRK_P(e, CSBEND_DY), dz = TRK_P(e, CSBEND_DZ);
  S->dxi = -dx;
  S->dzi = dz;
  S->dyi = -dy;
  S->dxf = dx * cos(ANGLE) + dz * sin(ANGLE);
  S->dzf = dx * sin(ANGLE) - dz * cos(ANGLE);
  S->dyf = dy;
  bend_edge_flags(l, idx, &S->edge1, &S->edge2);
  S->edge_order = (int)TRK_P(e, CSBEND_EDGE_ORDER);
  S->edge1_effects = (int)TRK_P(e, CSBEND_EDGE1_EFFECTS);
  S->edge2_effects = (int)TRK_P(e, CSBEND_EDGE2_EFFECTS);
  for (int k = 0; k < 2; k++) {
    int eff = k ? S->edge2_effects : S->edge1_effects;
    int on = k ? S->edge2 : S->edge1;
    if (on && (eff < 0 || eff > 5))
      return 1;
    /* EDGE_ORDER > 1 with Hwang's fringe needs HGAP (src/csbend.c:711-712) */
    if (eff == 2 && S->edge_order > 1 && S->hgap == 0)
      return 1;
  }
  return 0;
}

/* apply_edge_effects (src/csbend.c:4291-4333) */
static void apply_edge_effects(double *x, double *xp, double *y, double *yp, double rho, double n, double beta,
                               double he, double psi, long which_edge) {
  double h, tan_beta, tan2_beta, sec_beta, sec2_beta, h2;
  double R21, R43, T111, T133, T211, T441, T331, T221, T233, T243, T431, T432;
  double x0, xp0, y0, yp0;
  h = 1 / rho;
  R21 = h * (tan_beta = tan(beta));
  R43 = -h * orc_tan_sel(beta - psi);
  h2 = orc_sqr(h);
  T111 = which_edge * h / 2 * (tan2_beta = orc_sqr(tan_beta));
  sec_beta = 1. / cos(beta);
  sec2_beta = orc_sqr(sec_beta);
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
  x0 = *x;
  xp0 = *xp;
  y0 = *y;
  yp0 = *yp;
  *x = x0 + T111 * orc_sqr(x0) + T133 * orc_sqr(y0);
  *xp = xp0 + R21 * x0 + T211 * orc_sqr(x0) + T221 * x0 * xp0 + T233 * orc_sqr(y0) + T243 * y0 * yp0;
  *y = y0 + T331 * x0 * y0;
  *yp = yp0 + R43 * y0 + T441 * yp0 * x0 + T431 * x0 * y0 + T432 * xp0 * y0;
}

/* applySimpleDipoleEdgeKick (src/csbend.c:5664-5690) */
static void simple_dipole_edge_kick(double *xp, double *yp, double x, double y, double delta, double rho,
                                    double ea, double psi, double kickLimit, int expanded) {
  double Qi[6] = {x, *xp, y, *yp, 0, delta};
  double dqx, dqy;
  orc_to_dipole_canonical_x(Qi, expanded);
  dqx = tan(ea) / rho * x;
  if (kickLimit > 0 && fabs(dqx) > kickLimit)
    dqx = SIGN(dqx) * kickLimit;
  dqy = -orc_tan_sel(ea - psi / (1 + delta)) / rho * y;
  Qi[1] += dqx;
  Qi[3] += dqy;
  orc_from_dipole_canonical_x(Qi, expanded);
  *xp = Qi[1];
  *yp = Qi[3];
}

/* dipoleFringeKHwang (src/csbend.c:4336-4408): K. Hwang's dipole fringe in
 * dipole canonical coordinates, inFringe = -1 entrance, +1 exit */
static void fringe_hwang(double *Qf, const double *Qi, double rho, double inFringe, long edgeOrder, double edge,
                         double gap, double fint, double Rhe) {
  double dx, dpx, dy, dpy, tan_edge, sin_edge, sec_edge, cos_edge, x0, px0, y0, py0, dp0;
  const double k0 = orc_sqr(TRK_PI) / 6., k2 = fint, k3 = 1.0 * 1. / 6., k4 = -1.0 * orc_sqr(TRK_PI) / 3., k5 = 0.0,
               k6 = -1.0;
  x0 = Qi[0];
  px0 = Qi[1];
  y0 = Qi[2];
  py0 = Qi[3];
  dp0 = Qi[5];
  dx = dpx = dy = dpy = 0;
  sec_edge = 1. / cos(edge);
  tan_edge = tan(edge);
  sin_edge = sin(edge);
  cos_edge = cos(edge);
#define P2(v) ((v) * (v))
#define P3(v) ((v) * (v) * (v))
  if (edgeOrder > 1) {
    if (inFringe == -1.) {
      dx = inFringe * P2(sec_edge) * P2(gap) * k0 / rho / (1 + dp0) + inFringe * P2(x0) * P2(tan_edge) / 2 / rho / (1 + dp0) -
           inFringe * P2(y0) * P2(sec_edge) / 2 / rho / (1 + dp0);
      dy = -inFringe * x0 * y0 * P2(tan_edge) / rho / (1 + dp0);
      dpx = -1. * P3(sec_edge) * sin_edge * P2(gap) * k0 / rho / rho / (1 + dp0) + tan_edge * x0 / rho +
            P2(y0) / 2 * (2 * P3(tan_edge)) / P2(rho) / (1 + dp0) + P2(y0) / 2 * (tan_edge) / P2(rho) / (1 + dp0) -
            inFringe * (x0 * px0 - y0 * py0) * P2(tan_edge) / rho / (1 + dp0) +
            k4 * P2(sin_edge) * P2(gap) / 2 / P3(cos_edge) / rho * Rhe - k5 * x0 * sin_edge * gap / P3(cos_edge) / rho * Rhe +
            k6 * (y0 * y0 - x0 * x0) / 2 / P3(cos_edge) / rho * Rhe;
      dpy = -1. * tan_edge * y0 / rho + k2 * y0 * (1 + P2(sin_edge)) * gap / (1 + dp0) / P2(rho) / P3(cos_edge) +
            inFringe * (x0 * py0 + y0 * px0) * P2(tan_edge) / rho / (1 + dp0) + inFringe * y0 * px0 / rho / (1 + dp0) +
            k3 * P3(y0) * (2. / 3. / cos_edge - 4. / 3. / P3(cos_edge)) / (1 + dp0) / rho / rho / gap +
            k6 * x0 * y0 / P3(cos_edge) / rho * Rhe;
    }
    if (inFringe == 1.) {
      dx = inFringe * P2(sec_edge) * P2(gap) * k0 / rho / (1 + dp0) + inFringe * P2(x0) * P2(tan_edge) / 2 / rho / (1 + dp0) -
           inFringe * P2(y0) * P2(sec_edge) / 2 / rho / (1 + dp0);
      dy = -inFringe * x0 * y0 * P2(tan_edge) / rho / (1 + dp0);
      dpx = tan_edge * x0 / rho - P2(y0) / 2 * (1 * P3(tan_edge)) / P2(rho) / (1 + dp0) -
            P2(x0) / 2 * (1 * P3(tan_edge)) / P2(rho) / (1 + dp0) - inFringe * (x0 * px0 - y0 * py0) * P2(tan_edge) / rho / (1 + dp0) +
            k4 * P2(sin_edge) * P2(gap) / 2 / P3(cos_edge) / rho * Rhe - k5 * x0 * sin_edge * gap / P3(cos_edge) / rho * Rhe +
            k6 * (y0 * y0 - x0 * x0) / 2 / P3(cos_edge) / rho * Rhe;
      dpy = -1. * tan_edge * y0 / rho + k2 * y0 * (1 + P2(sin_edge)) * gap / (1 + dp0) / P2(rho) / P3(cos_edge) +
            inFringe * (x0 * py0 + y0 * px0) * P2(tan_edge) / rho / (1 + dp0) + inFringe * y0 * px0 / rho / (1 + dp0) +
            x0 * y0 * P2(sec_edge) * tan_edge / P2(rho) / (1 + dp0) +
            k3 * P3(y0) * (2. / 3. / cos_edge - 4. / 3. / P3(cos_edge)) / (1 + dp0) / rho / rho / gap -
            k5 * y0 * sin_edge * gap / P3(cos_edge) / rho * Rhe + k6 * x0 * y0 / P3(cos_edge) / rho * Rhe;
    }
  } else {
    if (inFringe == -1.) {
      dx = inFringe * P2(sec_edge) * P2(gap) * k0 / rho / (1 + dp0);
      dy = 0;
      dpx = -1. * P3(sec_edge) * sin_edge * P2(gap) * k0 / rho / rho / (1 + dp0) + tan_edge * x0 / rho +
            k4 * P2(sin_edge) * P2(gap) / 2 / P3(cos_edge) / rho * Rhe - k5 * x0 * sin_edge * gap / P3(cos_edge) / rho * Rhe;
      dpy = -1. * tan_edge * y0 / rho + k2 * y0 * (1 + P2(sin_edge)) * gap / (1 + dp0) / P2(rho) / P3(cos_edge);
    }
    if (inFringe == 1.) {
      dx = inFringe * P2(sec_edge) * P2(gap) * k0 / rho / (1 + dp0);
      dy = 0;
      dpx = tan_edge * x0 / rho + k4 * P2(sin_edge) * P2(gap) / 2 / P3(cos_edge) / rho * Rhe -
            k5 * x0 * sin_edge * gap / P3(cos_edge) / rho * Rhe;
      dpy = -1. * tan_edge * y0 / rho + k2 * y0 * (1 + P2(sin_edge)) * gap / (1 + dp0) / P2(rho) / P3(cos_edge) -
            k5 * y0 * sin_edge * gap / P3(cos_edge) / rho * Rhe;
    }
  }
  Qf[0] = x0 + dx;
  Qf[1] = px0 + dpx;
  Qf[2] = y0 + dy;
  Qf[3] = py0 + dpy;
  Qf[5] = Qi[5];
}

/* dipoleFringeKHwangRLindberg (src/csbend.c:4413-4520): the symplectic form */
static void fringe_hwang_lindberg(double *Qf, const double *Qi, double rho, double inFringe, double edge, double gap,
                                  double fint, double Rhe) {
  const double k0 = orc_sqr(TRK_PI) / 6., k2 = fint, k3 = 1.0 * 1. / 6., k4 = -1.0 * orc_sqr(TRK_PI) / 3., k5 = 0.0,
               k6 = -1.0;
  const double rho2 = orc_sqr(rho);
  const double x0 = Qi[0], px0 = Qi[1], y0 = Qi[2], py0 = Qi[3], dp0 = Qi[5];
  const double sec_edge = 1. / cos(edge), tan_edge = tan(edge), sin_edge = sin(edge), cos_edge = cos(edge);
  const double sec2_edge = P2(sec_edge), cos3_edge = P3(cos_edge), tan2_edge = P2(tan_edge), tan3_edge = P3(tan_edge);
  double x1, px1, y1, py1, x2, px2, y2, py2, x3, px3, y3, py3, x4, px4, y4, py4, x5, px5, y5, py5, t1, t2;
  if (inFringe == -1) {
    x1 = x0;
    px1 = px0 + tan_edge / rho * x0 + tan_edge / (2 * rho2 * (1 + dp0)) * orc_sqr(y0) -
          tan3_edge / (rho2 * (1 + dp0)) * orc_sqr(x0) - gap * k5 * sin_edge * Rhe / (rho * cos3_edge) * x0 +
          k6 * sec2_edge * Rhe / (2 * rho) * (orc_sqr(y0) - orc_sqr(x0));
    y1 = y0;
    py1 = py0 - tan_edge / rho * y0 + tan_edge / (rho2 * (1 + dp0)) * x0 * y0 +
          gap * k2 * (1 + orc_sqr(sin_edge)) / (rho2 * (1 + dp0) * cos3_edge) * y0 +
          2 * k3 * (orc_sqr(cos_edge) - 2) / (3 * gap * rho2 * cos3_edge) * P3(y0) +
          gap * k5 * sin_edge * Rhe / (rho * cos3_edge) * y0 + k6 * P3(sec_edge) * Rhe / rho * x0 * y0;
    t1 = (1 + tan2_edge / (2 * rho * (1 + dp0)) * x1);
    x2 = x1 / t1;
    px2 = px1 * orc_sqr(t1);
    y2 = y1;
    py2 = py1;
    t1 = sec2_edge / (rho * (1 + dp0));
    x3 = x2 + t1 / 2 * orc_sqr(y2);
    px3 = px2;
    y3 = y2;
    py3 = py2 - t1 * y2 * px2;
    t1 = tan2_edge / (rho * (1 + dp0));
    t2 = orc_exp_sel(t1 * x3);
    x4 = x3;
    px4 = px3 - t1 * y3 * py3;
    y4 = y3 * t2;
    py4 = py3 / t2;
    t1 = orc_sqr(gap) * k0 * sec2_edge / (rho * (1 + dp0));
    x5 = x4 - t1;
    px5 = px4 - t1 * tan_edge / rho + orc_sqr(gap) * k4 * orc_sqr(sin_edge) * Rhe / (2 * rho * cos3_edge);
    y5 = y4;
    py5 = py4;
  } else {
    x1 = x0;
    px1 = px0 + tan_edge / rho * x0 + tan3_edge / (2 * rho2 * (1 + dp0)) * orc_sqr(y0) +
          tan3_edge / (2 * rho2 * (1 + dp0)) * orc_sqr(x0) - gap * k5 * sin_edge * Rhe / (rho * cos3_edge) * x0 +
          k6 * sec2_edge * Rhe / (2 * rho) * (orc_sqr(y0) - orc_sqr(x0));
    y1 = y0;
    py1 = py0 - tan_edge / rho * y0 + tan3_edge / (rho2 * (1 + dp0)) * x0 * y0 +
          gap * k2 * (1 + orc_sqr(sin_edge)) / (rho2 * (1 + dp0) * cos3_edge) * y0 +
          2 * k3 * (orc_sqr(cos_edge) - 2) / (3 * gap * rho2 * cos3_edge) * P3(y0) +
          gap * k5 * sin_edge * Rhe / (rho * cos3_edge) * y0 + k6 * P3(sec_edge) * Rhe / rho * x0 * y0;
    t1 = (1 - tan2_edge / (2 * rho * (1 + dp0)) * x1);
    x2 = x1 / t1;
    px2 = px1 * orc_sqr(t1);
    y2 = y1;
    py2 = py1;
    t1 = sec2_edge / (rho * (1 + dp0));
    x3 = x2 - t1 / 2 * orc_sqr(y2);
    px3 = px2;
    y3 = y2;
    py3 = py2 + t1 * y2 * px2;
    t1 = -tan2_edge / (rho * (1 + dp0));
    t2 = orc_exp_sel(t1 * x3);
    x4 = x3;
    px4 = px3 - t1 * y3 * py3;
    y4 = y3 * t2;
    py4 = py3 / t2;
    x5 = x4 + orc_sqr(gap) * k0 * sec2_edge / (rho * (1 + dp0));
    px5 = px4 + orc_sqr(gap) * k4 * orc_sqr(sin_edge) * Rhe / (2 * rho * cos3_edge);
    y5 = y4;
    py5 = py4;
  }
#undef P2
#undef P3
  Qf[0] = x5;
  Qf[1] = px5;
  Qf[2] = y5;
  Qf[3] = py5;
  Qf[5] = dp0;
}

/* Lindberg's curved-dipole fringe, EDGE_EFFECTS=5 (curvedDipoleFringe,
 * src/csbend.c:5693-5969): in dipole canonical coordinates, with the edge's
 * fringe integrals K0..K6 (FRINGE1K0.. / FRINGE2K0..; no element here is
 * flipped, so no sign changes).  Entrance (inFringe -1) and exit (+1) share
 * the linear map through the fringe field; EDGE_ORDER > 1 adds the
 * second-order terms of the edge, which differ in sign between the two.
 * Written in the reference's operation order, exp/sinh/cosh/cos/tan through
 * the arithmetic-mode selectors. */
static void fringe_curved(double *Qf, const double *Qi, double rho, int inFringe, int edgeOrder, double K1,
                          double edge, const double *K) {
  const double x0 = Qi[0], px0 = Qi[1], y0 = Qi[2], py0 = Qi[3], dp0 = Qi[5];
  const double sec_edge = 1. / orc_cos_sel(edge), tan_edge = orc_tan_sel(edge);
  const double intK0 = K[0], intK1 = K[1], intK2 = K[2], intK3 = K[3], intK4 = K[4], intK5 = K[5], intK6 = K[6];
  double x1, px1, y1, py1, dtau;
  /* the linear map through the fringe field (the same at both ends) */
  const double mx = (intK3 + intK4) / (1.0 + dp0);
  const double my = intK3 / (1.0 + dp0);
  const double delX = intK0 / (1.0 + dp0);
  const double focX = intK1 + tan_edge / rho;
  const double focY = intK2 / (1.0 + dp0);
  if (fabs(mx) < 1.0e-5) {
    x1 = x0 * orc_exp_sel(-mx) + dp0 * delX * (1.0 - 0.5 * mx * (1.0 - mx / 3.0 + mx * mx / 12.0));
    px1 = px0 * orc_exp_sel(mx) + focX * (x0 * (1.0 + mx * mx / 6.0) + dp0 * delX * (0.5 + mx * mx / 24.0));
    dtau = px0 * (mx * x0 + delX) / (1.0 + dp0) + delX * px0 * 0.5 * mx * (1.0 + mx / 3.0 + mx * mx / 12.0) +
           focX * x0 * x0 * mx * (0.5 - (mx - 0.5 * mx * mx) / 3.0) / (1.0 + dp0) +
           dp0 * focX * delX * (delX + mx * x0 / (1.0 + dp0)) * (1.0 + 0.05 * mx * mx) / 6.0 +
           focX * delX * x0 * 0.5 * (1.0 + mx * mx / 12.0) / (1.0 + dp0) +
           dp0 * focX * delX * (2.0 * mx * x0 - dp0 * delX) * (1.0 - mx * (0.75 - mx * (0.35 - 0.125 * mx))) /
             (6.0 * (1.0 + dp0));
  } else {
    x1 = x0 * orc_exp_sel(-mx) + dp0 * delX * (1.0 - orc_exp_sel(-mx)) / mx;
    px1 = px0 * orc_exp_sel(mx) +
          focX * (x0 * orc_sinh_sel(mx) / mx + dp0 * delX * (orc_cosh_sel(mx) - 1.0) / (mx * mx));
    dtau = px0 * (mx * x0 + delX) / (1.0 + dp0) + delX * px0 * (orc_exp_sel(mx) - 1.0 - mx) / mx +
           focX * x0 * x0 * 0.25 * ((orc_exp_sel(-2.0 * mx) - 1.0) / mx + 2.0) / (1.0 + dp0) +
           dp0 * focX * delX * (delX + mx * x0 / (1.0 + dp0)) * (orc_sinh_sel(mx) - mx) / (mx * mx * mx) +
           focX * delX * x0 * (orc_cosh_sel(mx) - 1.0) / (mx * mx * (1.0 + dp0)) +
           dp0 * focX * delX * (2.0 * mx * x0 - dp0 * delX) * 0.25 *
             (2.0 - (3.0 + orc_exp_sel(-2.0 * mx) - 4.0 * orc_exp_sel(-mx)) / mx) / (mx * mx * (1.0 + dp0));
  }
  if (fabs(my) < 1.0e-5) {
    y1 = y0 * orc_exp_sel(my);
    py1 = py0 * orc_exp_sel(-my) + y0 * (focY - focX) * (1.0 + my * my / 6.0);
    dtau += (-my * py0 * y0 + 0.5 * (focY + focX * (my + my * my * (2.0 + my) / 3.0) * y0 * y0)) / (1.0 + dp0);
  } else {
    y1 = y0 * orc_exp_sel(my);
    py1 = py0 * orc_exp_sel(-my) + y0 * (focY - focX) * orc_sinh_sel(my) / my;
    dtau += (-my * py0 * y0 + 0.5 * (focY + 0.5 * focX * ((orc_exp_sel(2.0 * my) - 1.0) / my - 2.0)) * y0 * y0) /
            (1.0 + dp0);
  }
  double xo = x1, pxo = px1, yo = y1, pyo = py1;
  if (edgeOrder > 1) {
    /* second-order terms of the edge itself */
    const double sect2_rho = sec_edge * sec_edge / (rho * (1.0 + dp0));
    const double tant_rho = tan_edge / (rho * (1.0 + dp0));
    double x2, y2, px2, py2;
    if (inFringe == -1) {
      x2 = x1;
      y2 = y1 * orc_exp_sel(tan_edge * tant_rho * x1);
      px2 = px1 - tan_edge * tant_rho * y1 * py1 - (tan_edge * (tan_edge * tant_rho / rho - K1) - 0.5 * intK6) * x1 * x1;
      py2 = py1 * orc_exp_sel(-tan_edge * tant_rho * x1);
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
      y2 = y1 * orc_exp_sel(-tan_edge * tant_rho * x1);
      px2 = px1 + tan_edge * tant_rho * y1 * py1 +
            (tan_edge * (0.5 * tan_edge * tant_rho / rho + K1) + 0.5 * intK6) * x1 * x1;
      py2 = py1 * orc_exp_sel(tan_edge * tant_rho * x1);
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
    xo = x2;
    pxo = px2;
    yo = y2;
    pyo = py2;
  }
  /* the reference adds the differences to the initial values */
  Qf[0] = x0 + (xo - x0);
  Qf[1] = px0 + (pxo - px0);
  Qf[2] = y0 + (yo - y0);
  Qf[3] = py0 + (pyo - py0);
  Qf[4] = -dtau;
  Qf[5] = Qi[5];
}

static void csbend_edge(const orc_csbend_setup *S, int which, double *x, double *xp, double *y, double *yp,
                        double *s, double dp) {
  int eff = which < 0 ? S->edge1_effects : S->edge2_effects;
  double e = which < 0 ? S->e1 : S->e2;
  double psi = which < 0 ? S->psi1 : S->psi2;
  double lim = which < 0 ? S->e1_kick_limit : S->e2_kick_limit;
  double he = which < 0 ? S->he1 : S->he2;
  if (S->edge_order <= 1 && eff == 1) {
    double rho = (1 + dp) * S->rho_actual;
    double delta_xp = tan(e) / rho * *x;
    if (lim > 0 && fabs(delta_xp) > lim)
      delta_xp = SIGN(delta_xp) * lim;
    *xp += delta_xp;
    *yp -= orc_tan_sel(e - psi / (1 + dp)) / rho * *y;
  } else if (S->edge_order >= 2 && eff == 1) {
    double rho = (1 + dp) * S->rho_actual;
    apply_edge_effects(x, xp, y, yp, rho, S->n, e, he, psi * (1 + dp), which);
  } else if (eff == 3) {
    simple_dipole_edge_kick(xp, yp, *x, *y, dp, S->rho_actual, e, psi, lim, S->bd.expanded);
  } else if (eff == 2 || eff == 4 || eff == 5) {
    /* in dipole canonical coordinates (src/csbend.c:1139-1200, :1319-1377) */
    double Qi[6], Qf[6] = {0, 0, 0, 0, 0, 0};
    Qi[0] = *x;
    Qi[1] = *xp;
    Qi[2] = *y;
    Qi[3] = *yp;
    Qi[4] = 0;
    Qi[5] = dp;
    orc_to_dipole_canonical_x(Qi, S->bd.expanded);
    const double fint = which < 0 ? S->fint1 : S->fint2;
    if (eff == 2)
      fringe_hwang(Qf, Qi, S->rho_actual, (double)which, S->edge_order, e, 2 * S->hgap, fint, he);
    else if (eff == 4)
      fringe_hwang_lindberg(Qf, Qi, S->rho_actual, (double)which, e, 2 * S->hgap, fint, he);
    else
      fringe_curved(Qf, Qi, S->rho_actual, which, S->edge_order, S->k1_fringe, e, S->fringe_int[which < 0 ? 0 : 1]);
    orc_from_dipole_canonical_x(Qf, S->bd.expanded);
    *x = Qf[0];
    *xp = Qf[1];
    *y = Qf[2];
    *yp = Qf[3];
    if (eff == 5)
      *s += Qf[4];
  }
}

/* track_through_csbend (src/csbend.c:654-1434), MALIGN_METHOD=0, iSlice=-1 */
static long track_through_csbend(double *coord, long n_part, const trk_lattice *l, int idx, double Po,
                                 double z_start, const orc_maxamp *st, int *err) {
  orc_csbend_setup S;
  const trk_elem *e = &l->e[idx];
  if (csbend_setup(l, idx, Po, &S)) {
    *err = 1;
    return n_part;
  }
  if (S.is_drift) {
    exact_drift(coord, n_part, TRK_P(e, CSBEND_L));
    return n_part;
  }
  orc_aperture ap;
  setup_aperture(&ap, -S.tilt, st);
  long i_top = n_part - 1;
  for (long i_part = 0; i_part <= i_top; i_part++) {
    double *c = ROW(i_part);
    double x, xp, y, yp, s, dp, dp0, Qi[6], Qf[6], dz_lost;
    c[4] += S.dzi * sqrt(1 + orc_sqr(c[1]) + orc_sqr(c[3]));
    c[0] = c[0] + S.dxi + S.dzi * c[1];
    c[2] = c[2] + S.dyi + S.dzi * c[3];
    x = c[0] * S.cos_ttilt + c[2] * S.sin_ttilt;
    y = -c[0] * S.sin_ttilt + c[2] * S.cos_ttilt;
    xp = c[1] * S.cos_ttilt + c[3] * S.sin_ttilt;
    yp = -c[1] * S.sin_ttilt + c[3] * S.cos_ttilt;
    s = c[4];
    dp = dp0 = c[5];
    if (S.edge1)
      csbend_edge(&S, -1, &x, &xp, &y, &yp, &s, dp);
    Qi[0] = x;
    Qi[1] = xp;
    Qi[2] = y;
    Qi[3] = yp;
    Qi[4] = 0;
    Qi[5] = dp;
    if (S.edge1 && S.e1 != 0 && S.bd.rad_coef) {
      /* radiation: pre-adjust delta for the sector integration (src/csbend.c:1215-1222) */
      double Fx, Fy;
      orc_csbend_fields(&S.bd, &Fx, &Fy, x, y);
      double dp_prime =
        -S.bd.rad_coef * (orc_sqr(Fx) + orc_sqr(Fy)) * orc_sqr(1 + dp) * sqrt(orc_sqr(1 + x / S.rho0) + orc_sqr(xp) + orc_sqr(yp));
      Qi[5] -= dp_prime * x * orc_tan_sel(S.e1);
    }
    orc_to_dipole_canonical_x(Qi, S.bd.expanded);
    orc_isr.id = (uint32_t)(long long)c[6];
    int lost = S.bd.expanded ? !orc_integrate_csbend_expanded(Qf, Qi, &S.bd, &ap, &dz_lost)
                             : !orc_integrate_csbend(Qf, Qi, &S.bd, &ap, &dz_lost);
    orc_from_dipole_canonical_x(Qf, S.bd.expanded);
    if (lost) {
      memcpy(c, Qf, sizeof(double) * 6);
      /* convertFromCSBendCoords (src/csbend.c:4527-4548) */
      double X = c[0], XP = c[1], Y = c[2], YP = c[3];
      c[0] = X * S.cos_ttilt - Y * S.sin_ttilt;
      c[2] = X * S.sin_ttilt + Y * S.cos_ttilt;
      c[1] = XP * S.cos_ttilt - YP * S.sin_ttilt;
      c[3] = XP * S.sin_ttilt + YP * S.cos_ttilt;
      swap_rows(ROW(i_part), ROW(i_top));
      ROW(i_top)[4] = z_start + dz_lost;
      ROW(i_top)[5] = Po * (1 + ROW(i_top)[5]);
      i_top--;
      i_part--;
      continue;
    }
    if (S.edge2 && S.e2 != 0 && S.bd.rad_coef) {
      /* radiation: post-adjust delta (src/csbend.c:1270-1281) */
      double Fx, Fy;
      orc_csbend_fields(&S.bd, &Fx, &Fy, Qf[0], Qf[2]);
      double dp_prime = -S.bd.rad_coef * (orc_sqr(Fx) + orc_sqr(Fy)) * orc_sqr(1 + Qf[5]) *
                        sqrt(orc_sqr(1 + Qf[0] / S.rho0) + orc_sqr(Qf[1]) + orc_sqr(Qf[3]));
      Qf[5] -= dp_prime * Qf[0] * orc_tan_sel(S.e2);
    }
    if (S.bd.isr_or_rad) {
      double p0 = Po * (1 + dp0);
      double beta0 = p0 / sqrt(orc_sqr(p0) + 1);
      double p1 = Po * (1 + Qf[5]);
      double beta1 = p1 / sqrt(orc_sqr(p1) + 1);
      s = beta1 * s / beta0 + Qf[4];
    } else
      s += Qf[4];
    x = Qf[0];
    xp = Qf[1];
    y = Qf[2];
    yp = Qf[3];
    dp = Qf[5];
    if (S.edge2)
      csbend_edge(&S, 1, &x, &xp, &y, &yp, &s, dp);
    c[0] = x * S.cos_ttilt - y * S.sin_ttilt + S.dcoord_etilt[0];
    c[2] = x * S.sin_ttilt + y * S.cos_ttilt + S.dcoord_etilt[2];
    c[1] = xp * S.cos_ttilt - yp * S.sin_ttilt + S.dcoord_etilt[1];
    c[3] = xp * S.sin_ttilt + yp * S.cos_ttilt + S.dcoord_etilt[3];
    c[4] = s + S.dcoord_etilt[4];
    c[5] = dp;
    c[0] += S.dxf + S.dzf * c[1];
    c[2] += S.dyf + S.dzf * c[3];
    c[4] += S.dzf * sqrt(1 + orc_sqr(c[1]) + orc_sqr(c[3]));
  }
  return i_top + 1;
}

int orc_csbend_field_table(const trk_lattice *l, int element, double *Fx, double *Fy, int *eo1, int *hasNormal,
                           int *hasSkew) {
  orc_csbend_setup S;
  if (!l || element < 0 || element >= l->n || l->e[element].type != TRK_CSBEND)
    return TRK_ERR_ARG;
  if (csbend_setup(l, element, 1.0, &S) || S.is_drift)
    return TRK_ERR_UNSUPPORTED;
  for (int i = 0; i < 11; i++)
    for (int j = 0; j < 11; j++) {
      Fx[i * 11 + j] = S.bd.Fx_xy[i][j];
      Fy[i * 11 + j] = S.bd.Fy_xy[i][j];
    }
  *eo1 = S.bd.expansionOrder1;
  *hasNormal = S.bd.hasNormal;
  *hasSkew = S.bd.hasSkew;
  return TRK_OK;
}

/* ----------------------------------------------------------------- RFCA */
typedef struct {
  int fiducial_seen;
  double phase_fiducial;
} orc_rf_state;

/* Summation mode for the two beam averages (WAKE mean arrival time, RFCA
 * "tmean" fiducial).  0: as the reference (plain index-order sum for the wake,
 * Kahan for the fiducial); 1: double-double sums rounded once, the value the
 * GPU path computes, for bit-level checks of the downstream arithmetic. */
static int orc_exact_sums = 0;
void orc_set_exact_sums(int on) { orc_exact_sums = on; }
void orc_set_isr_seed(unsigned long long seed) { orc_isr.seed = seed; }
void orc_set_cr_math(int on) { orc_cr_math = on; }
double orc_cr_sin(double x) { return trkcr_sin(x); }
double orc_cr_cos(double x) { return trkcr_cos(x); }
double orc_cr_asin(double x) { return trkcr_asin(x); }
double orc_cr_tan(double x) { return trkcr_tan(x); }
double orc_cr_exp(double x) { return trkcr_exp(x); }
double orc_cr_sinh(double x) { return trkcr_sinh(x); }
double orc_cr_cosh(double x) { return trkcr_cosh(x); }
/* the double-double evaluations behind the fast paths, and the fast paths'
 * parts (hi, L, error bound e; returns the rounding test's verdict), for the
 * tests of the fast paths' error bounds */
double orc_cr_slow(int kind, double x) {
  return kind == 0 ? trkcr_sin_slow(x) : kind == 1 ? trkcr_cos_slow(x) : trkcr_asin_slow(x);
}
int orc_cr_parts(int kind, double x, double *out) {
  double L, e, hi, r;
  const double zh = x * x, zl = fma(x, x, -zh);
  if (kind == 0)
    hi = trkcr_sin_parts(x, zh, zl, &L, &e);
  else if (kind == 1)
    hi = trkcr_cos_parts(zh, zl, &L, &e);
  else
    hi = trkcr_asin_parts(x, zh, zl, &L, &e);
  out[0] = hi;
  out[1] = L;
  out[2] = e;
  return trkcr_round_test(hi, L, e, &r);
}

/* Self-test of the tiered correctly rounded functions: n arguments drawn
 * uniformly from [lo, hi] (log_mag: magnitudes log-uniform in [lo, hi],
 * random sign), each function against its double-double evaluation
 * (trkcr_*_slow, ~2^-100 relative; kind 3: sin and cos together, kind 4:
 * exp).  Returns the number of disagreements;
 * *tiny_hits counts the calls whose tiny-argument test accepted and
 * *max_rel the largest relative error of the tiny path's correction
 * (against the double-double value minus the leading term), which the
 * tiny path's rounding test assumes to be below 2^-50.7. */
static unsigned long long orc_splitmix(unsigned long long *st) {
  unsigned long long z = (*st += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
long orc_cr_selftest(int kind, double lo, double hi, int log_mag, long n, unsigned long long seed, long *tiny_hits,
                     double *max_rel) {
  unsigned long long st = seed;
  long bad = 0, hits = 0;
  double mrel = 0;
  for (long k = 0; k < n; k++) {
    const double u = (double)(orc_splitmix(&st) >> 11) * 0x1p-53;
    double x;
    if (log_mag) {
      x = exp(log(lo) + u * (log(hi) - log(lo)));
      if (orc_splitmix(&st) & 1)
        x = -x;
    } else
      x = lo + u * (hi - lo);
    double got, want, t;
    const double z = x * x, ax = fabs(x);
    if (kind == 4 && ax >= 0x1p-12 && ax <= TRKCR_TINY) {
      /* the tiny path's x^2 P(x) against exp - 1 - x from the double-double
       * (whose absolute accuracy, ~2^-100, resolves x^2 P to 2^-75 here) */
      const trkcr_dd v = trkcr_exp_dd(x);
      const double ce = ((v.hi - 1.0) - x) + v.lo;
      const double rel = fabs(trkcr_exp_tiny_t(x) - ce) / fabs(ce);
      if (rel > mrel)
        mrel = rel;
    }
    if (kind <= 2 && ax >= 0x1p-26 && ax <= TRKCR_TINY) {
      /* the exact correction from the double-double value (hi - lead is
       * exact: hi and the lead are within a factor of two) */
      trkcr_dd v;
      double lead, c;
      if (kind == 0) {
        v = trkcr_sin_dd(x);
        lead = x;
        c = trkcr_sin_tiny_c(x, z);
      } else if (kind == 1) {
        v = trkcr_cos_dd(x);
        lead = 1.0;
        c = trkcr_cos_tiny_c(z);
      } else {
        const double a0 = asin(x);
        const trkcr_dd sa = trkcr_sin_dd(a0);
        /* asin x = a0 + (x - sin a0)/cos a0 to ~2^-100 */
        const double d = ((x - sa.hi) - sa.lo) / cos(a0);
        v = trkcr_two_sum(a0, d);
        lead = x;
        c = trkcr_asin_tiny_c(x, z);
      }
      const double ce = (v.hi - lead) + v.lo;
      const double rel = fabs(c - ce) / fabs(ce);
      if (rel > mrel)
        mrel = rel;
    }
    if (kind == 0) {
      got = trkcr_sin(x);
      want = trkcr_sin_slow(x);
      hits += ax >= 0x1p-26 && ax <= TRKCR_TINY && trkcr_sin_tiny(x, z, &t);
    } else if (kind == 1) {
      got = trkcr_cos(x);
      want = trkcr_cos_slow(x);
      hits += ax >= 0x1p-27 && ax <= TRKCR_TINY && trkcr_cos_tiny(z, &t);
    } else if (kind == 2) {
      got = trkcr_asin(x);
      want = trkcr_asin_slow(x);
      hits += ax >= 0x1p-26 && ax <= TRKCR_TINY && trkcr_asin_tiny(x, z, &t);
    } else if (kind == 4) {
      got = trkcr_exp(x);
      want = trkcr_exp_slow(x);
    } else {
      double s, c;
      trkcr_sincos(x, &s, &c);
      got = s - trkcr_sin_slow(x);
      want = c - trkcr_cos_slow(x);
      bad += !(got == 0 && want == 0);
      continue;
    }
    if (!(got == want) && !(got != got && want != want))
      bad++;
  }
  if (tiny_hits)
    *tiny_hits = hits;
  if (max_rel)
    *max_rel = mrel;
  return bad;
}

/* Self-test of trkcr_div_rcp (the parity build's division by a divisor
 * with a precomputed correctly rounded reciprocal) against the IEEE
 * quotient: n random pairs over 2^-20..2^20 with random signs, one in four
 * divisors with a run of trailing ones, one in four dividends placed on a
 * rounding midpoint of the quotient, and zeros.  Returns disagreements. */
long orc_div_rcp_selftest(long n, unsigned long long seed) {
  unsigned long long st = seed;
  long bad = 0;
  for (long k = 0; k < n; k++) {
    const unsigned long long r1 = orc_splitmix(&st), r2 = orc_splitmix(&st), r3 = orc_splitmix(&st);
    double a = ldexp(1.0 + (double)(r1 >> 12) * 0x1p-52, (int)(r3 % 41) - 20);
    double b = ldexp(1.0 + (double)(r2 >> 12) * 0x1p-52, (int)((r3 >> 8) % 41) - 20);
    if (r3 & (1ULL << 20))
      a = -a;
    if (r3 & (1ULL << 21))
      b = -b;
    if ((k & 3) == 1) {
      uint64_t bits;
      memcpy(&bits, &b, 8);
      bits |= (1ULL << 52) - (1ULL << ((r3 >> 24) % 9));
      memcpy(&b, &bits, 8);
    } else if ((k & 3) == 2) {
      const double q = a / b, m = q + (nextafter(q, INFINITY) - q) / 2;
      a = m * b;
    } else if ((k & 1023) == 3) {
      a = (r3 & 1) ? 0.0 : -0.0;
    }
    const double got = trkcr_div_rcp(a, b, 1.0 / b), want = a / b;
    if (memcmp(&got, &want, 8) != 0)
      bad++;
  }
  return bad;
}

static void dd_acc(double *hi, double *lo, double v) {
  double s = *hi + v, bb = s - *hi, e = (*hi - (s - bb)) + (v - bb);
  e += *lo;
  double h = s + e;
  *lo = e - (h - s);
  *hi = h;
}

/* KahanPlus: compensated summation (SDDS mdbmth, not shipped with the
 * reference; the published algorithm of W. Kahan, 1965). */
static double kahan_plus(double sum, double b, double *error) {
  double y = b - *error;
  double t = sum + y;
  *error = (t - sum) - y;
  return t;
}

/* ------------------------------------------------------- sharded runs
 * The particle-sharded decomposition the multi-GPU library uses, restated
 * so it can be tested on CPU ranks: each rank tracks its own particles and
 * exchanges only beam time statistics ({sum as double-double, count, min,
 * max}, gathered and combined in rank order), the wake histograms (summed)
 * and the CHARGE particle count (summed) -- Pelegant's exchanges
 * (src/wake.c:226-233, src/trwake.c:195-204, src/simple_rfca.c:222-230,
 * src/do_tracking.c:1378-1381). */
static int orc_world = 1;
static orc_gather_fn orc_gather_cb = NULL;
static orc_sum_fn orc_sum_cb = NULL;

void orc_set_collective(int world, orc_gather_fn gather, orc_sum_fn sum) {
  orc_world = (world > 1 && gather && sum) ? world : 1;
  orc_gather_cb = gather;
  orc_sum_cb = sum;
}

/* {hi, lo} double-double sum, count, min, max of this rank -> of all ranks */
static void shard_stats(double *hi, double *lo, double *n, double *tmin, double *tmax) {
  if (orc_world <= 1)
    return;
  double send[6] = {*hi + *lo, *n, *tmin, *tmax, *hi, *lo};
  double *recv = (double *)malloc(sizeof(double) * 6 * orc_world);
  orc_gather_cb(send, recv, 6);
  trkcr_dd acc = trkcr_make(0.0, 0.0);
  double N = 0, mn = DBL_MAX, mx = -DBL_MAX;
  for (int r = 0; r < orc_world; r++) {
    const double *g = recv + 6 * r;
    acc = trkcr_add(acc, trkcr_make(g[4], g[5]));
    N += g[1];
    if (g[2] < mn)
      mn = g[2];
    if (g[3] > mx)
      mx = g[3];
  }
  free(recv);
  *hi = acc.hi;
  *lo = acc.lo;
  *n = N;
  *tmin = mn;
  *tmax = mx;
}

static void shard_sum(double *buf, long n) {
  if (orc_world > 1)
    orc_sum_cb(buf, n);
}

/* beta_from_delta (src/do_tracking.c:95-98) */
static double beta_from_delta(double p, double delta) {
  p *= 1 + delta;
  return p / sqrt(p * p + 1);
}

void orc_match_energy(double *coord, long np, double *P_central, int change_beam);

/* simple_rf_cavity -> trackRfCavityWithWakes (src/simple_rfca.c:264-985):
 * traveling-wave kick method (no matrix method, no backtracking), fiducial
 * mode "tmean" with Kahan summation; LOCK_PHASE and LINEARIZE with the beam's
 * mean arrival time of each pass (:500-556). */
static long rf_cavity(double *coord, long np, const trk_elem *e, orc_rf_state *rs, double *P_central, double zEnd,
                      int *err) {
  double length = TRK_P(e, RFCA_L);
  long nKicks;
  double omega, volt, tau, dtLight, phase, t0, To;
  (void)To;
  if (np <= 0 && orc_world <= 1)
    return np;
  const int lock = TRK_P(e, RFCA_LOCK_PHASE) != 0, linearize = TRK_P(e, RFCA_LINEARIZE) != 0;
  if (TRK_P(e, RFCA_CHANGE_T) || TRK_P(e, RFCA_STANDING_WAVE) || (TRK_P(e, RFCA_CHANGE_P0) && orc_world > 1)) {
    *err = 1;
    return np;
  }
  if (TRK_P(e, RFCA_VOLT) == 0) {
    if (length) {
      for (long ip = 0; ip < np; ip++) {
        double *c = ROW(ip);
        c[0] += c[1] * length;
        c[2] += c[3] * length;
        c[4] += length * sqrt(1 + orc_sqr(c[1]) + orc_sqr(c[3]));
      }
    }
    return np;
  }
  omega = TRK_PIx2 * TRK_P(e, RFCA_FREQ);
  volt = TRK_P(e, RFCA_VOLT) / (1e6 * TRK_ME_MEV * TRK_PARTICLE_REL_SIGN);
  tau = omega ? TRK_P(e, RFCA_Q) / omega : 0;
  nKicks = length ? (long)TRK_P(e, RFCA_N_KICKS) : 1;
  if (nKicks <= 0) {
    *err = 1; /* matrix method: not on this path */
    return np;
  }
  if ((lock || linearize) && nKicks != 1) {
    *err = 1; /* "Must use n_kicks=1 for linearized rf cavity" (src/simple_rfca.c:505-506) */
    return np;
  }
  length /= nKicks;
  volt /= nKicks;
  dtLight = length / TRK_C_MKS;
  if (!rs->fiducial_seen) {
    if (TRK_P(e, RFCA_T_REFERENCE) != -1)
      t0 = TRK_P(e, RFCA_T_REFERENCE);
    else {
      /* findFiducialTime, FID_MODE_TMEAN (src/simple_rfca.c:191-230) */
      double tsum = 0, error = 0, sOffset = length / 2;
      long nsum = 0;
      double hi = 0, lo = 0;
      for (long ip = 0; ip < np; ip++) {
        double t = (ROW(ip)[4] + sOffset) / (TRK_C_MKS * beta_from_delta(*P_central, ROW(ip)[5]));
        if (orc_exact_sums)
          dd_acc(&hi, &lo, t);
        else
          tsum = kahan_plus(tsum, t, &error);
        nsum++;
      }
      if (orc_exact_sums)
        tsum = hi + lo;
      if (orc_world > 1) {
        /* KahanParallel over ranks (src/simple_rfca.c:222-230) */
        double dn = (double)nsum, mn = DBL_MAX, mx = -DBL_MAX;
        if (!orc_exact_sums) {
          hi = tsum;
          lo = 0;
        }
        shard_stats(&hi, &lo, &dn, &mn, &mx);
        tsum = hi + lo;
        nsum = (long)dn;
      }
      t0 = tsum / nsum;
    }
    rs->phase_fiducial = -omega * t0;
    rs->fiducial_seen = 1;
  }
  phase = rs->phase_fiducial;
  if (omega) {
    t0 = -rs->phase_fiducial / omega;
    To = TRK_PIx2 / omega;
  } else
    t0 = To = 0;
  phase += TRK_P(e, RFCA_PHASE) * TRK_PI / 180.0;
  int same_dgamma = 0;
  double dgamma = 0;
  if (omega == 0 && tau == 0) {
    dgamma = volt * orc_sin_sel(phase);
    same_dgamma = 1;
  }
  double timeOffset = 0;
  double tAve = 0, dgammaAve = 0;
  if (linearize || lock) {
    /* the mean arrival time (src/simple_rfca.c:503-556) */
    double error = 0, hi = 0, lo = 0;
    for (long ip = 0; ip < np; ip++) {
      double *c = ROW(ip);
      double P = *P_central * (1 + c[5]), gamma;
      double beta_i = P / (gamma = sqrt(orc_sqr(P) + 1));
      double t = (c[4] + length / 2) / (TRK_C_MKS * beta_i) - timeOffset;
      if (orc_exact_sums)
        dd_acc(&hi, &lo, t);
      else
        tAve = kahan_plus(tAve, t, &error);
    }
    if (orc_exact_sums)
      tAve = hi + lo;
    double nt = (double)np;
    if (orc_world > 1) {
      double mn = DBL_MAX, mx = -DBL_MAX;
      if (!orc_exact_sums) {
        hi = tAve;
        lo = 0;
      }
      shard_stats(&hi, &lo, &nt, &mn, &mx);
      tAve = hi + lo;
    }
    tAve /= nt;
    if (lock) {
      phase = TRK_PI / 180 * TRK_P(e, RFCA_PHASE);
      dgammaAve = volt * orc_sin_sel(phase);
    } else
      dgammaAve = volt * orc_sin_sel(omega * (tAve - timeOffset) + phase);
  }
  for (long ip = 0; ip < np; ip++) {
    ROW(ip)[0] -= TRK_P(e, RFCA_DX);
    ROW(ip)[2] -= TRK_P(e, RFCA_DY);
  }
  double *inverseF = (double *)calloc(sizeof(double), np);
  for (long ik = 0; ik < nKicks; ik++) {
    for (long ip = 0; ip < np; ip++) {
      double *c = ROW(ip);
      double dc4, P, gamma, beta_i, t, dt, gamma1;
      if (c[5] == -1)
        continue;
      if (length)
        dc4 = length / 2 * sqrt(1 + orc_sqr(c[1]) + orc_sqr(c[3]));
      else
        dc4 = 0;
      P = *P_central * (1 + c[5]);
      beta_i = P / (gamma = sqrt(orc_sqr(P) + 1));
      t = (c[4] + dc4) / (TRK_C_MKS * beta_i) - timeOffset;
      if ((dt = t - t0) < 0)
        dt = 0;
      if (!same_dgamma) {
        if (!linearize) {
          double phi = omega * (t - (lock ? tAve : 0) - ik * dtLight) + phase;
          double dfactor = tau ? sqrt(1 - exp(-dt / tau)) : 1;
          dgamma = volt * orc_sin_sel(phi) * dfactor;
        } else
          dgamma = dgammaAve + volt * omega * (t - tAve) * orc_cos_sel(omega * (tAve - timeOffset) + phase);
      }
      if (length) {
        if (TRK_P(e, RFCA_END1_FOCUS) && ik == 0) {
          inverseF[ip] = dgamma / (2 * gamma * length);
          c[1] -= c[0] * inverseF[ip];
          c[3] -= c[2] * inverseF[ip];
        }
        c[0] += c[1] * length / 2;
        c[2] += c[3] * length / 2;
        c[4] += length / 2 * sqrt(1 + orc_sqr(c[1]) + orc_sqr(c[3]));
      }
      orc_add_to_particle_energy(c, t, *P_central, dgamma);
      if ((gamma1 = gamma + dgamma) <= 1)
        c[5] = -1;
      else
        inverseF[ip] = -dgamma / (2 * gamma1 * length);
    }
    if (length) {
      for (long ip = 0; ip < np; ip++) {
        double *c = ROW(ip);
        c[0] += c[1] * length / 2;
        c[2] += c[3] * length / 2;
        c[4] += length / 2 * sqrt(1 + orc_sqr(c[1]) + orc_sqr(c[3]));
        if (TRK_P(e, RFCA_END2_FOCUS) && (ik == nKicks - 1)) {
          c[1] -= c[0] * inverseF[ip];
          c[3] -= c[2] * inverseF[ip];
        }
      }
    }
  }
  free(inverseF);
  for (long ip = 0; ip < np; ip++) {
    ROW(ip)[0] += TRK_P(e, RFCA_DX);
    ROW(ip)[2] += TRK_P(e, RFCA_DY);
  }
  np = remove_invalid(coord, np, zEnd, *P_central);
  if (TRK_P(e, RFCA_CHANGE_P0)) /* src/simple_rfca.c:977-978 */
    orc_match_energy(coord, np, P_central, 0);
  return np;
}

/* ----------------------------------------------------------------- wakes */
typedef struct {
  double macroParticleCharge;
  int charge_set;
} orc_wake_state;

/* convolveArrays (src/wake.c:480-496) */
static void convolve_arrays(double *output, long outputs, const double *a1, long n1, const double *a2, long n2,
                            long di2) {
  for (long ib = 0; ib < outputs; ib++) {
    long ib2 = ib + di2, ib1 = 0, di;
    output[ib] = 0;
    if (ib2 >= n2) {
      di = ib2 - n2 + 1;
      ib1 += di;
      ib2 -= di;
    }
    for (; ib1 < n1 && ib2 >= 0; ib1++, ib2--)
      output[ib] += a1[ib1] * a2[ib2];
  }
}

/* wake table set-up shared by WAKE and TRWAKE (src/wake.c:434-477,
 * src/trwake.c:460-517): dt from the table span, i0 for acausal tables. */
static int wake_table_setup(const trk_elem *e, double *dt, long *i0, int acausal) {
  double tmin = DBL_MAX, tmax = -DBL_MAX;
  if (!e->wake_t || e->wake_points < 2)
    return 1;
  for (long i = 0; i < e->wake_points; i++) {
    if (e->wake_t[i] < tmin)
      tmin = e->wake_t[i];
    if (e->wake_t[i] > tmax)
      tmax = e->wake_t[i];
  }
  if (tmin >= tmax)
    return 1;
  *dt = (tmax - tmin) / (e->wake_points - 1);
  *i0 = 0;
  if (tmin != 0) {
    if (!acausal)
      return 1;
    *i0 = -1;
    for (long iw = 0; iw < e->wake_points; iw++)
      if (fabs(e->wake_t[iw]) < 1e-6 * *dt) {
        *i0 = iw;
        break;
      }
    if (*i0 == -1 || fabs(tmin) > tmax)
      return 1;
  }
  return 0;
}

/* track_through_wake (src/wake.c:23-304), one bunch, no smoothing */
static int track_through_wake(double *coord, long np, const trk_elem *e, double *P_central, long i_pass,
                              orc_wake_state *ws, const double *chargeMacro) {
  double dt, tmean, tmin, tmax, factor, rampFactor;
  long i0, nb;
  const double Po = *P_central;
  if (TRK_P(e, WAKE_SMOOTHING) || (TRK_P(e, WAKE_CHANGE_P0) && orc_world > 1))
    return 1;
  if (wake_table_setup(e, &dt, &i0, (int)TRK_P(e, WAKE_ACAUSAL_ALLOWED)))
    return 1;
  long rampPasses = (long)TRK_P(e, WAKE_RAMP_PASSES);
  if (i_pass >= rampPasses - 1)
    rampFactor = 1;
  else
    rampFactor = (i_pass + 1.0) / rampPasses;
  if (np <= 0 && orc_world <= 1) {
    if (!chargeMacro && i_pass == 0)
      ws->macroParticleCharge = 0;
    else if (chargeMacro)
      ws->macroParticleCharge = *chargeMacro;
    return 0;
  }
  double *time = (double *)malloc(sizeof(double) * (np > 0 ? np : 1));
  long *pbin = (long *)malloc(sizeof(long) * (np > 0 ? np : 1));
  /* computeTimeCoordinatesOnly (src/trwake.c:519-527) */
  for (long ip = 0; ip < np; ip++) {
    double P = Po * (ROW(ip)[5] + 1);
    time[ip] = ROW(ip)[4] * sqrt(orc_sqr(P) + 1) / (TRK_C_MKS * P);
  }
  /* compute_average (SDDS mdbmth, not shipped): arithmetic mean, summed in
   * index order */
  double sum = 0, slo = 0;
  for (long ip = 0; ip < np; ip++) {
    if (orc_exact_sums)
      dd_acc(&sum, &slo, time[ip]);
    else
      sum += time[ip];
  }
  tmin = DBL_MAX;
  tmax = -DBL_MAX;
  for (long ip = 0; ip < np; ip++) {
    if (time[ip] < tmin)
      tmin = time[ip];
    if (time[ip] > tmax)
      tmax = time[ip];
  }
  double n_all = (double)np;
  shard_stats(&sum, &slo, &n_all, &tmin, &tmax);
  if (orc_exact_sums || orc_world > 1)
    sum = sum + slo;
  tmean = sum / n_all;
  /* set_up_wake (src/wake.c:340-372) */
  if (chargeMacro)
    ws->macroParticleCharge = *chargeMacro;
  else if (i_pass == 0) {
    ws->macroParticleCharge = 0;
    if (n_all)
      ws->macroParticleCharge = TRK_P(e, WAKE_CHARGE) / n_all;
  }
  if ((tmax - tmin) > (e->wake_t[e->wake_points - 1] - e->wake_t[0]) && !TRK_P(e, WAKE_ALLOW_LONG_BEAM)) {
    free(time);
    free(pbin);
    return 2; /* the reference exits: beam longer than the wake */
  }
  if (TRK_P(e, WAKE_N_BINS)) {
    nb = (long)TRK_P(e, WAKE_N_BINS);
    tmin = tmean - dt * nb / 2.0;
  } else {
    nb = (long)((tmax - tmin) / dt + 3);
    tmin -= dt;
  }
  if (nb <= 0) {
    free(time);
    free(pbin);
    return 0;
  }
  double *Itime = (double *)calloc(nb, sizeof(double));
  double *Vtime = (double *)calloc(nb + 1, sizeof(double));
  /* binTimeDistribution (src/wake.c:498-518) */
  for (long ip = 0; ip < np; ip++) {
    long ib;
    pbin[ip] = -1;
    ib = (long)((time[ip] - tmin) / dt + 0.5);
    if (ib < 0 || ib > nb - 1)
      continue;
    Itime[ib] += 1;
    pbin[ip] = ib;
  }
  shard_sum(Itime, nb); /* src/wake.c:226-233 */
  Vtime[nb] = 0;
  convolve_arrays(Vtime, nb, Itime, nb, e->wake_w0, e->wake_points, i0);
  factor = ws->macroParticleCharge * TRK_PARTICLE_REL_SIGN * TRK_P(e, WAKE_FACTOR) * rampFactor;
  for (long ib = 0; ib < nb; ib++)
    Vtime[ib] *= factor;
  /* applyLongitudinalWakeKicks (src/wake.c:306-330) */
  int interpolate = (int)TRK_P(e, WAKE_INTERPOLATE);
  for (long ip = 0; ip < np; ip++) {
    long ib = pbin[ip];
    double dgam, dt1;
    if (ib >= 0 && ib <= nb - 1) {
      if (interpolate) {
        dt1 = time[ip] - (tmin + dt * ib);
        if ((dt1 < 0 && ib) || ib == nb - 1) {
          ib--;
          dt1 += dt;
        }
        dgam = (Vtime[ib] + (Vtime[ib + 1] - Vtime[ib]) / dt * dt1) / (1e6 * TRK_ME_MEV * TRK_PARTICLE_REL_SIGN);
      } else
        dgam = Vtime[ib] / (1e6 * TRK_ME_MEV * TRK_PARTICLE_REL_SIGN);
      if (dgam)
        orc_add_to_particle_energy(ROW(ip), time[ip], Po, -dgam);
    }
  }
  free(Itime);
  free(Vtime);
  free(time);
  free(pbin);
  if (TRK_P(e, WAKE_CHANGE_P0)) /* src/wake.c:289-290 */
    orc_match_energy(coord, np, P_central, 0);
  return 0;
}

/* track_through_trwake (src/trwake.c:22-287), one bunch, no smoothing.
 * With one bunch the reference leaves tmean at 0 (it is only computed for
 * multi-bunch beams, src/trwake.c:70-95), so N_BINS>0 bins around t=0. */
static int track_through_trwake(double *coord, long np, const trk_elem *e, double Po, long i_pass,
                                orc_wake_state *ws, const double *chargeMacro) {
  double dt, tmean = 0, tmin, tmax, rampFactor = 1;
  long i0, nb;
  if (TRK_P(e, TRWAKE_SMOOTHING))
    return 1;
  if (wake_table_setup(e, &dt, &i0, (int)TRK_P(e, TRWAKE_ACAUSAL_ALLOWED)))
    return 1;
  long rampPasses = (long)TRK_P(e, TRWAKE_RAMP_PASSES);
  if (i_pass >= rampPasses - 1)
    rampFactor = 1;
  else
    rampFactor = (i_pass + 1.0) / rampPasses;
  if (np <= 0 && orc_world <= 1) {
    if (chargeMacro)
      ws->macroParticleCharge = *chargeMacro;
    else if (i_pass == 0)
      ws->macroParticleCharge = 0;
    return 0;
  }
  double *time = (double *)malloc(sizeof(double) * (np > 0 ? np : 1));
  long *pbin = (long *)malloc(sizeof(long) * (np > 0 ? np : 1));
  double *pz = (double *)calloc(np > 0 ? np : 1, sizeof(double));
  for (long ip = 0; ip < np; ip++) {
    double P = Po * (ROW(ip)[5] + 1);
    time[ip] = ROW(ip)[4] * sqrt(orc_sqr(P) + 1) / (TRK_C_MKS * P);
  }
  tmin = DBL_MAX;
  tmax = -DBL_MAX;
  for (long ip = 0; ip < np; ip++) {
    if (time[ip] < tmin)
      tmin = time[ip];
    if (time[ip] > tmax)
      tmax = time[ip];
  }
  double shi = 0, slo = 0, n_all = (double)np;
  shard_stats(&shi, &slo, &n_all, &tmin, &tmax);
  if (chargeMacro)
    ws->macroParticleCharge = *chargeMacro;
  else if (i_pass == 0) {
    ws->macroParticleCharge = 0;
    if (n_all)
      ws->macroParticleCharge = TRK_P(e, TRWAKE_CHARGE) / n_all;
  }
  if ((tmax - tmin) > (e->wake_t[e->wake_points - 1] - e->wake_t[0])) {
    free(time);
    free(pbin);
    free(pz);
    return 2;
  }
  if (TRK_P(e, TRWAKE_N_BINS)) {
    tmin = tmean - dt * TRK_P(e, TRWAKE_N_BINS) / 2.0;
    nb = (long)TRK_P(e, TRWAKE_N_BINS);
  } else {
    nb = (long)((tmax - tmin) / dt + 3);
    tmin -= dt;
    tmax += dt;
  }
  if (tmin > tmax || nb <= 0) {
    free(time);
    free(pbin);
    free(pz);
    return 2;
  }
  double tilt = TRK_P(e, TRWAKE_TILT);
  if (tilt)
    rotate_beam(coord, np, tilt);
  double *posItime[2];
  posItime[0] = (double *)calloc(nb, sizeof(double));
  posItime[1] = (double *)calloc(nb, sizeof(double));
  double *Vtime = (double *)calloc(nb + 1, sizeof(double));
  long xPower = (long)TRK_P(e, TRWAKE_X_DRIVE_EXPONENT), yPower = (long)TRK_P(e, TRWAKE_Y_DRIVE_EXPONENT);
  double dx = TRK_P(e, TRWAKE_DX), dy = TRK_P(e, TRWAKE_DY);
  /* binTransverseTimeDistribution (src/trwake.c:610-641) */
  for (long ip = 0; ip < np; ip++) {
    double *c = ROW(ip);
    long ib;
    pbin[ip] = -1;
    ib = (long)((time[ip] - tmin) / dt + 0.5);
    if (ib < 0 || ib > nb - 1)
      continue;
    if (xPower == 1)
      posItime[0][ib] += c[0] - dx;
    else if (xPower < 1)
      posItime[0][ib] += 1;
    else
      posItime[0][ib] += orc_ipow(c[0] - dx, xPower);
    if (yPower == 1)
      posItime[1][ib] += c[2] - dy;
    else if (yPower < 1)
      posItime[1][ib] += 1;
    else
      posItime[1][ib] += orc_ipow(c[2] - dy, yPower);
    pbin[ip] = ib;
    pz[ip] = Po * (1 + c[5]) / sqrt(1 + orc_sqr(c[1]) + orc_sqr(c[3]));
  }
  shard_sum(posItime[0], nb); /* src/trwake.c:195-204 */
  shard_sum(posItime[1], nb);
  for (int plane = 0; plane < 2; plane++) {
    const double *W = plane ? e->wake_w1 : e->wake_w0;
    double factor = ws->macroParticleCharge * TRK_PARTICLE_REL_SIGN * TRK_P(e, TRWAKE_FACTOR);
    if (plane == 0)
      factor *= TRK_P(e, TRWAKE_XFACTOR) * rampFactor;
    else
      factor *= TRK_P(e, TRWAKE_YFACTOR) * rampFactor;
    if (!factor)
      continue;
    Vtime[nb] = 0;
    convolve_arrays(Vtime, nb, posItime[plane], nb, W, e->wake_points, i0);
    for (long ib = 0; ib < nb; ib++)
      Vtime[ib] *= factor;
    /* applyTransverseWakeKicks (src/trwake.c:289-314) */
    int interpolate = (int)TRK_P(e, TRWAKE_INTERPOLATE);
    long exponent = (long)(plane == 0 ? TRK_P(e, TRWAKE_X_PROBE_EXPONENT) : TRK_P(e, TRWAKE_Y_PROBE_EXPONENT));
    int offset = 2 * plane + 1;
    for (long ip = 0; ip < np; ip++) {
      long ib = pbin[ip];
      double dt1, Vinterp;
      if (ib >= 0 && ib <= nb - 1) {
        if (interpolate) {
          dt1 = time[ip] - (tmin + dt * ib);
          if ((dt1 < 0 && ib) || ib == nb - 1) {
            ib--;
            dt1 += dt;
          }
          Vinterp = Vtime[ib] + (Vtime[ib + 1] - Vtime[ib]) / dt * dt1;
        } else
          Vinterp = Vtime[ib];
        if (exponent)
          Vinterp *= orc_ipow(ROW(ip)[offset - 1], exponent);
        if (Vinterp)
          ROW(ip)[offset] += Vinterp / (1e6 * TRK_ME_MEV * TRK_PARTICLE_REL_SIGN) / pz[ip];
      }
    }
  }
  if (tilt)
    rotate_beam(coord, np, -tilt);
  free(posItime[0]);
  free(posItime[1]);
  free(Vtime);
  free(time);
  free(pbin);
  free(pz);
  return 0;
}

/* ------------------------------------------------------------- driver */
typedef struct {
  orc_maxamp maxamp;
  orc_rf_state *rf;     /* per element */
  orc_wake_state *wake; /* per element */
  int have_charge;
  double chargeMacro;
} orc_run_state;

/* The body of do_tracking's element switch (src/do_tracking.c:1239-2495) and
 * the after-element filters (:2506-2524 aperture, :2676 NaN/inf filter). */
static int track_one_element(const trk_lattice *l, int idx, double *coord, long nToTrack, long i_pass, double last_z,
                             double z, double *P_central, orc_run_state *rs, long *nLeft_out) {
  const trk_elem *e = &l->e[idx];
  long nLeft = nToTrack;
  int err = 0;
  orc_isr.pass = (uint32_t)i_pass;
  orc_isr.elem = (uint32_t)idx;
  switch (e->type) {
  case TRK_MARK:
  case TRK_CHARGE:
    break;
  case TRK_DRIF:
    drift_matrix_track(coord, nToTrack, TRK_P(e, DRIF_L), (long)TRK_P(e, DRIF_ORDER));
    break;
  case TRK_EDRIFT:
    exact_drift(coord, nToTrack, TRK_P(e, EDRIFT_L));
    break;
  case TRK_KQUAD:
  case TRK_KSEXT:
  case TRK_KOCT:
    nLeft = multipole_tracking2(coord, nToTrack, e, *P_central, last_z, &rs->maxamp, &err);
    break;
  case TRK_CSBEND:
    nLeft = track_through_csbend(coord, nToTrack, l, idx, *P_central, last_z, &rs->maxamp, &err);
    break;
  case TRK_RFCA:
    nLeft = rf_cavity(coord, nToTrack, e, &rs->rf[idx], P_central, z, &err);
    break;
  case TRK_WAKE:
    err = track_through_wake(coord, nToTrack, e, P_central, i_pass, &rs->wake[idx],
                             rs->have_charge ? &rs->chargeMacro : NULL);
    break;
  case TRK_TRWAKE:
    err = track_through_trwake(coord, nToTrack, e, *P_central, i_pass, &rs->wake[idx],
                               rs->have_charge ? &rs->chargeMacro : NULL);
    break;
  case TRK_MAXAMP:
    maxamp_update(&rs->maxamp, e);
    break;
  default:
    err = 1;
  }
  if (err)
    return err == 2 ? TRK_ERR_PHYSICS : TRK_ERR_UNSUPPORTED;
  if (e->type != TRK_MARK && e->type != TRK_CHARGE) {
    const orc_maxamp *st = &rs->maxamp;
    if (st->x_max || st->y_max) {
      if (!st->elliptical)
        nLeft = limit_amplitudes(coord, st->x_max, st->y_max, nLeft, z, *P_central, e->type == TRK_DRIF);
      else {
        int e2 = 0;
        nLeft = elimit_amplitudes(coord, st->x_max, st->y_max, nLeft, z, *P_central, e->type == TRK_DRIF,
                                  st->exponent, st->yExponent, &e2);
        if (e2)
          return TRK_ERR_UNSUPPORTED;
      }
    }
  }
  nLeft = limit_amplitudes(coord, DBL_MAX, DBL_MAX, nLeft, z, *P_central, 0);
  *nLeft_out = nLeft;
  return TRK_OK;
}

static int run_state_init(const trk_lattice *l, long nOriginal, orc_run_state *rs) {
  memset(rs, 0, sizeof(*rs));
  rs->rf = (orc_rf_state *)calloc(l->n > 0 ? l->n : 1, sizeof(orc_rf_state));
  rs->wake = (orc_wake_state *)calloc(l->n > 0 ? l->n : 1, sizeof(orc_wake_state));
  if (!rs->rf || !rs->wake)
    return TRK_ERR_NOMEM;
  /* CHARGE element (src/do_tracking.c:780-815) */
  for (int i = 0; i < l->n; i++)
    if (l->e[i].type == TRK_CHARGE) {
      const trk_elem *e = &l->e[i];
      rs->have_charge = 1;
      rs->chargeMacro = 0;
      double nAll = (double)nOriginal;
      shard_sum(&nAll, 1); /* total_nOriginal (src/do_tracking.c:1378-1381) */
      if (nAll)
        rs->chargeMacro = TRK_P(e, CHARGE_TOTAL) / nAll;
      if (TRK_P(e, CHARGE_PER_PARTICLE))
        rs->chargeMacro = TRK_P(e, CHARGE_PER_PARTICLE);
    }
  return TRK_OK;
}

static void run_state_free(orc_run_state *rs) {
  free(rs->rf);
  free(rs->wake);
}

int orc_track(const trk_lattice *l, double *coord, long np, long n_passes, long pass_offset, double *p_central,
              orc_result *result) {
  orc_run_state rs;
  int rc;
  if (!l || (!coord && np) || !p_central)
    return TRK_ERR_ARG;
  orc_isr.single = np == 1;
  if ((rc = run_state_init(l, np, &rs)))
    return rc;
  for (long ip = 0; ip < np; ip++) {
    ROW(ip)[7] = -1;
    ROW(ip)[8] = -1;
  }
  long nToTrack = np, effort = 0;
  /* initial NaN screen (src/do_tracking.c:478-484) */
  long nLeft = limit_amplitudes(coord, DBL_MAX, DBL_MAX, nToTrack, 0.0, *p_central, 0);
  for (long k = nLeft; k < nToTrack; k++) {
    ROW(k)[7] = pass_offset;
    ROW(k)[8] = -1;
  }
  nToTrack = nLeft;
  for (long i_pass = pass_offset; i_pass < pass_offset + n_passes; i_pass++) {
    double z = 0, last_z;
    for (int idx = 0; idx < l->n; idx++) {
      last_z = z;
      z += trk_elem_length(&l->e[idx]);
      rc = track_one_element(l, idx, coord, nToTrack, i_pass, last_z, z, p_central, &rs, &nLeft);
      if (rc) {
        run_state_free(&rs);
        return rc;
      }
      /* recordLostParticles (src/do_tracking.c:4669-4731) */
      for (long k = nLeft; k < nToTrack; k++) {
        ROW(k)[7] = i_pass;
        ROW(k)[8] = idx;
      }
      nToTrack = nLeft;
    }
    effort += nLeft; /* src/do_tracking.c:2812-2819 */
  }
  run_state_free(&rs);
  if (result) {
    result->n_left = nToTrack;
    result->particle_passes = effort;
    result->p_central = *p_central;
  }
  return TRK_OK;
}

int orc_track_element(const trk_lattice *l, int element, double *coord, long np, long pass, double *p_central,
                      long *n_left) {
  orc_run_state rs;
  int rc;
  if (!l || element < 0 || element >= l->n || !p_central || !n_left)
    return TRK_ERR_ARG;
  if ((rc = run_state_init(l, np, &rs)))
    return rc;
  /* sticky MAXAMP state before this element */
  double z = 0;
  for (int i = 0; i < element; i++) {
    if (l->e[i].type == TRK_MAXAMP)
      maxamp_update(&rs.maxamp, &l->e[i]);
    z += trk_elem_length(&l->e[i]);
  }
  if (pass > 0 && !rs.maxamp.seen)
    for (int i = element; i < l->n; i++)
      if (l->e[i].type == TRK_MAXAMP)
        maxamp_update(&rs.maxamp, &l->e[i]);
  double last_z = z;
  z += trk_elem_length(&l->e[element]);
  rc = track_one_element(l, element, coord, np, pass, last_z, z, p_central, &rs, n_left);
  run_state_free(&rs);
  return rc;
}

/* ------------------------------------------------------ beam observers
 * On rows of ORC_STRIDE doubles, survivors first (np of them).  Kahan sums
 * of the reference become double-double sums in exact-sums mode, as above. */

/* compute_centroids (src/compute_centroids.c:53-160, serial branch) */
void orc_beam_centroids(const double *coord, long np, double *centroid) {
  double sum[6], error[6], lo[6];
  for (int c = 0; c < 6; c++)
    sum[c] = centroid[c] = error[c] = lo[c] = 0;
  for (long i = 0; i < np; i++)
    for (int c = 0; c < 6; c++) {
      const double v = coord[(size_t)i * ORC_STRIDE + c];
      if (orc_exact_sums)
        dd_acc(&sum[c], &lo[c], v);
      else
        sum[c] = kahan_plus(sum[c], v, &error[c]);
    }
  if (np)
    for (int c = 0; c < 6; c++)
      centroid[c] = sum[c] / np;
}

/* computeTimeCoordinates' per-particle time (src/trwake.c:533-548) */
static double orc_time(const double *r, double Po) {
  const double P = Po * (r[5] + 1);
  return r[4] * sqrt(P * P + 1) / (TRK_C_MKS * P);
}

/* accumulate_beam_sums (src/compute_centroids.c:286-461, the serial
 * version): sums of the chosen particles folded into *s.  The sigma sums
 * are the reference's in-line Kahan sums (not switchable to double-double
 * there either); only the centroid sums follow the exact-sums mode. */
void orc_accumulate_beam_sums(const double *coord, long np, orc_beam_sums *s, double Po, double mp_charge,
                              const double *time_value, double tMin, double tMax, long startPID, long endPID,
                              unsigned flags) {
  static const short sparse[7][7] = {{1, 1, 0, 0, 0, 1, 0}, {0, 1, 0, 0, 0, 1, 0}, {0, 0, 1, 1, 0, 1, 0},
                                     {0, 0, 0, 1, 0, 1, 0}, {0, 0, 0, 0, 1, 1, 1}, {0, 0, 0, 0, 0, 1, 0},
                                     {0, 0, 0, 0, 0, 0, 1}};
  const int second = (flags & 0x8u) != 0, exact_emit = (flags & 0x4u) != 0;
  double *t = (double *)malloc(sizeof(double) * (np > 0 ? np : 1));
  short *chosen = (short *)malloc(sizeof(short) * (np > 0 ? np : 1));
  double *pz = exact_emit ? (double *)malloc(sizeof(double) * (np > 0 ? np : 1)) : NULL;
  for (long i = 0; i < np; i++) {
    const double *r = coord + (size_t)i * ORC_STRIDE;
    t[i] = time_value ? time_value[i] : orc_time(r, Po);
    if (pz)
      pz[i] = Po * (1 + r[5]) / sqrt(1 + r[1] * r[1] + r[3] * r[3]);
  }
  if (!s->n_part)
    s->p0 = Po;
  long npCount = 0;
  if (np) {
    for (long i = 0; i < np; i++) {
      const double id = coord[(size_t)i * ORC_STRIDE + 6];
      chosen[i] = ((startPID < 0 && endPID < 0) || (id >= startPID && id <= endPID)) &&
                  (tMin >= tMax || (t[i] >= tMin && t[i] <= tMax));
      npCount += chosen[i];
    }
    if (!(flags & 0x2u) && second)
      for (int c = 0; c < 6; c++) {
        if (c == 4)
          continue;
        for (long i = 0; i < np; i++)
          if (chosen[i]) {
            const double v = coord[(size_t)i * ORC_STRIDE + c];
            if (fabs(v) > s->maxabs[c])
              s->maxabs[c] = fabs(v);
            if (v > s->max[c])
              s->max[c] = v;
            if (v < s->min[c])
              s->min[c] = v;
          }
      }
    double cen[7], cenn[7];
    for (int c = 0; c < 7; c++) {
      double err = 0, errn = 0, lo = 0, lon = 0;
      cen[c] = cenn[c] = 0;
      for (long i = 0; i < np; i++)
        if (chosen[i]) {
          const double *r = coord + (size_t)i * ORC_STRIDE;
          if (exact_emit && (c == 1 || c == 3)) {
            if (orc_exact_sums)
              dd_acc(&cenn[c], &lon, r[c] * pz[i]);
            else
              cenn[c] = kahan_plus(cenn[c], r[c] * pz[i], &errn);
          }
          const double v = c < 6 ? r[c] : t[i];
          if (orc_exact_sums)
            dd_acc(&cen[c], &lo, v);
          else
            cen[c] = kahan_plus(cen[c], v, &err);
        }
      if (npCount) {
        s->centroid[c] = (s->centroid[c] * s->n_part + cen[c]) / (s->n_part + npCount);
        cen[c] /= npCount;
        cenn[c] /= npCount;
      }
    }
    for (int c = 0; c < 7; c++)
      if (c != 1 && c != 3)
        cenn[c] = cen[c];
    for (long i = 0; i < np; i++)
      t[i] -= cen[6];
    if (!(flags & 0x2u) && second)
      for (long i = 0; i < np; i++)
        if (chosen[i]) {
          double v = coord[(size_t)i * ORC_STRIDE + 4] - cen[4];
          if (fabs(v) > s->maxabs[4])
            s->maxabs[4] = fabs(v);
          if (v > s->max[4])
            s->max[4] = v;
          if (v < s->min[4])
            s->min[4] = v;
          v = t[i];
          if (fabs(v) > s->maxabs[6])
            s->maxabs[6] = fabs(v);
          if (v > s->max[6])
            s->max[6] = v;
          if (v < s->min[6])
            s->min[6] = v;
        }
    if (second)
      for (int a = 0; a < 7; a++)
        for (int b = a; b < 7; b++) {
          double Sij = 0, Sijn = 0, e = 0, en = 0;
          if ((flags & 0x1u) && !sparse[a][b]) {
            s->sigma[b][a] = s->sigma[a][b] = 0;
            s->sigman[b][a] = s->sigman[a][b] = 0;
            continue;
          }
          for (long i = 0; i < np; i++)
            if (chosen[i]) {
              const double *r = coord + (size_t)i * ORC_STRIDE;
              const double bv = (a < 6 ? r[a] - cen[a] : t[i]) * (b < 6 ? r[b] - cen[b] : t[i]);
              /* in-line Kahan (src/compute_centroids.c:424-436) */
              double Y = bv + e, old = Sij;
              Sij += Y;
              e = Y - (Sij - old);
              if (exact_emit) {
                const double bn = (r[a] * (a == 1 || a == 3 ? pz[i] : 1) - cenn[a]) * (r[b] * (b == 1 || b == 3 ? pz[i] : 1));
                double Yn = bn + en, oldn = Sijn;
                Sijn += Yn;
                en = Yn - (Sijn - oldn);
              }
            }
          s->sigma[b][a] = (s->sigma[a][b] = (s->sigma[a][b] * s->n_part + Sij) / (s->n_part + npCount));
          if (exact_emit)
            s->sigman[b][a] = (s->sigman[a][b] = (s->sigman[a][b] * s->n_part + Sijn) / (s->n_part + npCount));
        }
  }
  s->charge = mp_charge * npCount;
  s->n_part += npCount;
  free(t);
  free(chosen);
  free(pz);
}

/* do_match_energy (src/do_tracking.c:3376-3546, the serial branches) */
void orc_match_energy(double *coord, long np, double *P_central, int change_beam) {
  if (!np)
    return;
  double P_average = 0, error = 0, lo = 0;
  for (long i = 0; i < np; i++) {
    const double v = (*P_central) * (1 + coord[(size_t)i * ORC_STRIDE + 5]);
    if (orc_exact_sums)
      dd_acc(&P_average, &lo, v);
    else
      P_average = kahan_plus(P_average, v, &error);
  }
  P_average /= np;
  if (!change_beam) {
    if (fabs(P_average - (*P_central)) / (*P_central) > 1e-14) {
      const double dp = (*P_central - P_average) / P_average;
      const double dr = (*P_central) / P_average;
      for (long i = 0; i < np; i++)
        coord[(size_t)i * ORC_STRIDE + 5] = dp + coord[(size_t)i * ORC_STRIDE + 5] * dr;
      *P_central = P_average;
    }
  } else {
    const double dP_centroid = *P_central - P_average;
    for (long i = 0; i < np; i++) {
      double *r = coord + (size_t)i * ORC_STRIDE;
      double P = (1 + r[5]) * (*P_central);
      const double tt = r[4] / (P / sqrt(P * P + 1));
      P += dP_centroid;
      r[5] = (P - *P_central) / (*P_central);
      r[4] = tt * (P / sqrt(P * P + 1));
    }
  }
}
