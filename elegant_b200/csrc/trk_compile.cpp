/*
 * trk_compile.cpp -- turns a trk_lattice into the device op table.
 *
 * For every element this evaluates, on the host and with the reference's own
 * expressions, what the reference computes once per element call before its
 * per-particle loop: strengths divided by slices, substep lengths, edge
 * tangents, misalignment rotations, aperture state, field-expansion tables.
 * The kernels then only run the per-particle arithmetic.
 */
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "trk_compile.h"
#include "trk_constants.h"
#include "trk_crmath.h"
#include "trk_lattice.h"

namespace {

/* integrator substep tables (src/multipole.c:1118-1141, src/csbend.c:1480-1503) */
const double driftFrac2[2] = {0.5, 0.5};
const double kickFrac2[2] = {1.0, 0.0};
const double driftFrac4[4] = {0.5 / (2 - TRK_BETA), (1 - TRK_BETA) / (2 - TRK_BETA) / 2,
                              (1 - TRK_BETA) / (2 - TRK_BETA) / 2, 0.5 / (2 - TRK_BETA)};
const double kickFrac4[4] = {1. / (2 - TRK_BETA), -TRK_BETA / (2 - TRK_BETA), 1 / (2 - TRK_BETA), 0};
const double driftFrac6[8] = {0.39225680523878,   0.5100434119184585, -0.47105338540975655, 0.0687531682525181,
                              0.0687531682525181, -0.47105338540975655, 0.5100434119184585, 0.39225680523878};
const double kickFrac6[8] = {0.784513610477560,  0.235573213359357, -1.17767998417887, 1.3151863206839063,
                             -1.17767998417887, 0.235573213359357, 0.784513610477560,  0};

int substeps(int order, const double **df, const double **kf) {
  switch (order) {
  case 2:
    *df = driftFrac2;
    *kf = kickFrac2;
    return 2;
  case 4:
    *df = driftFrac4;
    *kf = kickFrac4;
    return 4;
  case 6:
    *df = driftFrac6;
    *kf = kickFrac6;
    return 8;
  default:
    return 0;
  }
}

double sgn(double x) { return x < 0 ? -1 : 1; }

/* cos/sin used by rotateBeamCoordinatesForMisalignment (src/tilt_matrices.c:161-175) */
bool rotation(double angle, double *c, double *s) {
  if (!angle || std::fabs(std::fabs(angle) - TRK_PIx2) < 1e-12)
    return false;
  if (std::fabs(std::fabs(angle) - TRK_PI) < 1e-12) {
    *c = -1;
    *s = 0;
  } else if (std::fabs(angle - TRK_PIo2) < 1e-12) {
    *c = 0;
    *s = 1;
  } else if (std::fabs(angle + TRK_PIo2) < 1e-12) {
    *c = 0;
    *s = -1;
  } else {
    *c = std::cos(angle);
    *s = std::sin(angle);
  }
  return true;
}


struct MaxampState {
  int idx = -1; /* aperture record, -1 none */
  double x_max = 0, y_max = 0;
};

} // namespace

/* integer power by recursive squaring, the oracle's and the compiled SDDS
 * shim's definition (src/multipole.c and src/limit_amplitudes.c call ipow) */
double ipow_h(double x, long p) {
  if (p == 0)
    return 1.0;
  if (p == 1)
    return x;
  if (p == 2)
    return x * x;
  if (p < 0)
    return 1.0 / ipow_h(x, -p);
  const double h = ipow_h(x, p / 2);
  return (p & 1) ? h * h * x : h * h;
}

/* Field-expansion coefficients of a curved magnet from the recursion
 * Laplace's equation imposes in the curvilinear frame with curvature h
 * (the reference evaluates the same coefficients in closed form,
 * src/csbend.c:175-~650):
 *   curl:  (i+1) a[i+1][j] = (j+1) c[i][j+1]
 *   div :  (i+1) (c[i+1][j] + h c[i][j]) + (j+1) (a[i][j+1] + h a[i-1][j+1]) = 0
 * a[i][j], c[i][j]: coefficients of x^i y^j in Fy, Fx; mid-plane data
 * a[i][0] = b_i / i!, c[i][0] = -c_i / i!; steering terms only in [0][0]. */
int trk_csbend_field_table(const double *b, const double *c, double h, int nonlinear, long expansionOrder,
                           double *Fx, double *Fy, int *eo1, int *hasNormal, int *hasSkew) {
  double a[12][12], cx[12][12];
  int i, j;
  if (expansionOrder == 0) {
    for (i = 8; i >= 0; i--)
      if (b[i] || c[i])
        break;
    if ((expansionOrder = i + 2) < 4)
      expansionOrder = 4;
  }
  if (expansionOrder + 1 > 11)
    return 1;
  *eo1 = (int)expansionOrder + 1;
  *hasNormal = *hasSkew = 0;
  for (i = 0; i < 9; i++) {
    if (b[i])
      *hasNormal = 1;
    if (c[i])
      *hasSkew = 1;
  }
  std::memset(a, 0, sizeof(a));
  std::memset(cx, 0, sizeof(cx));
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
  for (i = 0; i < 121; i++)
    Fx[i] = Fy[i] = 0;
  if (nonlinear) {
    for (i = 0; i <= 10; i++)
      for (j = 0; i + j <= 10; j++) {
        Fx[i * 11 + j] = cx[i][j];
        Fy[i * 11 + j] = a[i][j];
      }
  } else {
    Fx[0 * 11 + 1] = cx[0][1];
    Fy[1 * 11 + 0] = a[1][0];
    Fy[0 * 11 + 1] = a[0][1];
    Fx[1 * 11 + 0] = cx[1][0];
  }
  Fx[0] = c[0];
  Fy[0] = 1 - b[0];
  return 0;
}

namespace {

/* quadPartialFringeMatrix (src/fringe.c:231-275): the 2x2 blocks
 * {R00, R01, R10, R11, R22, R23, R32, R33} of one linear fringe part; the
 * exponentials correctly rounded, as the parity build's arithmetic is */
static void quad_partial_fringe(double *R, double K1, long inFringe, const double *fi, long part) {
  double J1x, J2x, J3x, J1y, J2y, J3y;
  const double K1sqr = K1 * K1;
  if (part == 1) {
    J1x = inFringe * (K1 * fi[1] - 2 * K1sqr * fi[3] / 3. - K1sqr * fi[0] * fi[2] / 2);
    J2x = inFringe * K1 * fi[2];
    J3x = inFringe * K1sqr * (fi[2] + fi[4] + fi[0] * fi[1]);
    J1y = inFringe * (-K1 * fi[1] - 2 * K1sqr * fi[3] / 3. - K1sqr * fi[0] * fi[2] / 2);
  } else {
    J1x = inFringe * (K1 * fi[1] + K1sqr * fi[0] * fi[2] / 2);
    J2x = inFringe * K1 * fi[2];
    J3x = inFringe * K1sqr * (fi[4] - fi[0] * fi[1]);
    J1y = inFringe * (-K1 * fi[1] + K1sqr * fi[0] * fi[2] / 2);
  }
  J2y = -J2x;
  J3y = J3x;
  const double ex = trkcr_exp(J1x), ey = trkcr_exp(J1y);
  R[0] = ex;
  R[1] = J2x / ex;
  R[2] = ex * J3x;
  R[3] = (1 + J2x * J3x) / ex;
  R[4] = ey;
  R[5] = J2y / ey;
  R[6] = ey * J3y;
  R[7] = (1 + J2y * J3y) / ey;
}

/* the two linear parts quadFringe applies at one edge (src/fringe.c:47-90):
 * M1 from the I-m integrals, M2 from the I+m ones, diagonal entries swapped
 * and the parts exchanged at an entrance, inverted for a backward magnet */
static void quad_fringe_matrices(double K1, const double *fint_m, const double *fint_p, int backtrack, int inFringe,
                          double *M1, double *M2) {
  quad_partial_fringe(M1, K1, 1, fint_m, 1);
  quad_partial_fringe(M2, K1, 1, fint_p, 2);
  if (inFringe * (backtrack ? -1 : 1) == -1) {
    std::swap(M1[0], M1[3]);
    std::swap(M1[4], M1[7]);
    std::swap(M2[0], M2[3]);
    std::swap(M2[4], M2[7]);
    for (int k = 0; k < 8; k++)
      std::swap(M1[k], M2[k]);
  }
  if (backtrack) {
    for (double *M : {M1, M2}) {
      std::swap(M[0], M[3]);
      std::swap(M[4], M[7]);
      M[1] *= -1;
      M[2] *= -1;
      M[5] *= -1;
      M[6] *= -1;
    }
  }
}

int compile_mult(const trk_elem *e, double Po, trk_op *op) {
  double KnL[3] = {0, 0, 0}, drift, tilt, dx, dy, dz, xkick = 0, ykick = 0, lEnd = 0;
  int order[3] = {0, 0, 0}, skew[3] = {0, 0, 0}, integ, expand;
  long n_kicks, nSlices;
  int doEndDrift = 0, synch_rad = 0, isr = 0, isr1 = 1;
  double elem_length = 0;
  double cfac = TRK_E_MKS / (TRK_ME_MKS * TRK_C_MKS * Po);
  switch (e->type) {
  case TRK_KQUAD: {
    if (TRK_P(e, KQUAD_RADIAL) || TRK_P(e, KQUAD_MALIGN_METHOD))
      return trk_set_error(TRK_ERR_UNSUPPORTED, "KQUAD %s: RADIAL and MALIGN_METHOD!=0 are not on this path",
                           e->name);
    synch_rad = TRK_P(e, KQUAD_SYNCH_RAD) != 0;
    isr = TRK_P(e, KQUAD_ISR) != 0;
    isr1 = TRK_P(e, KQUAD_ISR1PART) != 0;
    elem_length = TRK_P(e, KQUAD_L);
    nSlices = (long)TRK_P(e, KQUAD_N_SLICES);
    n_kicks = (long)TRK_P(e, KQUAD_N_KICKS);
    expand = (int)TRK_P(e, KQUAD_EXPAND_HAMILTONIAN);
    order[0] = 1;
    double lEff = TRK_P(e, KQUAD_LEFFECTIVE);
    if (lEff <= 0)
      lEff = TRK_P(e, KQUAD_L);
    else {
      lEnd = (TRK_P(e, KQUAD_L) - lEff) / 2;
      doEndDrift = 1;
    }
    if (TRK_P(e, KQUAD_BORE))
      KnL[0] = TRK_P(e, KQUAD_B) / TRK_P(e, KQUAD_BORE) * cfac * lEff * (1 + TRK_P(e, KQUAD_FSE));
    else
      KnL[0] = TRK_P(e, KQUAD_K1) * lEff * (1 + TRK_P(e, KQUAD_FSE));
    drift = lEff;
    tilt = TRK_P(e, KQUAD_TILT);
    dx = TRK_P(e, KQUAD_DX);
    dy = TRK_P(e, KQUAD_DY);
    dz = TRK_P(e, KQUAD_DZ);
    xkick = TRK_P(e, KQUAD_HKICK) * TRK_P(e, KQUAD_HCALIBRATION);
    ykick = TRK_P(e, KQUAD_VKICK) * TRK_P(e, KQUAD_VCALIBRATION);
    integ = (int)TRK_P(e, KQUAD_INTEGRATION_ORDER);
    break;
  }
  case TRK_KSEXT:
    if (TRK_P(e, KSEXT_MALIGN_METHOD))
      return trk_set_error(TRK_ERR_UNSUPPORTED, "KSEXT %s: MALIGN_METHOD!=0 is not on this path", e->name);
    synch_rad = TRK_P(e, KSEXT_SYNCH_RAD) != 0;
    isr = TRK_P(e, KSEXT_ISR) != 0;
    isr1 = TRK_P(e, KSEXT_ISR1PART) != 0;
    elem_length = TRK_P(e, KSEXT_L);
    n_kicks = (long)TRK_P(e, KSEXT_N_KICKS);
    nSlices = (long)TRK_P(e, KSEXT_N_SLICES);
    expand = (int)TRK_P(e, KSEXT_EXPAND_HAMILTONIAN);
    order[0] = 2;
    if (TRK_P(e, KSEXT_BORE))
      KnL[0] = 2 * TRK_P(e, KSEXT_B) / (TRK_P(e, KSEXT_BORE) * TRK_P(e, KSEXT_BORE)) * cfac * TRK_P(e, KSEXT_L) *
               (1 + TRK_P(e, KSEXT_FSE));
    else
      KnL[0] = TRK_P(e, KSEXT_K2) * TRK_P(e, KSEXT_L) * (1 + TRK_P(e, KSEXT_FSE));
    drift = TRK_P(e, KSEXT_L);
    tilt = TRK_P(e, KSEXT_TILT);
    dx = TRK_P(e, KSEXT_DX);
    dy = TRK_P(e, KSEXT_DY);
    dz = TRK_P(e, KSEXT_DZ);
    xkick = TRK_P(e, KSEXT_HKICK) * TRK_P(e, KSEXT_HCALIBRATION);
    ykick = TRK_P(e, KSEXT_VKICK) * TRK_P(e, KSEXT_VCALIBRATION);
    integ = (int)TRK_P(e, KSEXT_INTEGRATION_ORDER);
    if (TRK_P(e, KSEXT_K1)) {
      KnL[1] = TRK_P(e, KSEXT_K1) * TRK_P(e, KSEXT_L);
      order[1] = 1;
    }
    if (TRK_P(e, KSEXT_J1)) {
      KnL[2] = TRK_P(e, KSEXT_J1) * TRK_P(e, KSEXT_L);
      order[2] = 1;
      skew[2] = 1;
    }
    break;
  case TRK_KOCT:
    if (TRK_P(e, KOCT_MALIGN_METHOD))
      return trk_set_error(TRK_ERR_UNSUPPORTED, "KOCT %s: MALIGN_METHOD!=0 is not on this path", e->name);
    synch_rad = TRK_P(e, KOCT_SYNCH_RAD) != 0;
    isr = TRK_P(e, KOCT_ISR) != 0;
    isr1 = TRK_P(e, KOCT_ISR1PART) != 0;
    elem_length = TRK_P(e, KOCT_L);
    n_kicks = (long)TRK_P(e, KOCT_N_KICKS);
    nSlices = (long)TRK_P(e, KOCT_N_SLICES);
    expand = (int)TRK_P(e, KOCT_EXPAND_HAMILTONIAN);
    order[0] = 3;
    if (TRK_P(e, KOCT_BORE))
      KnL[0] = 6 * TRK_P(e, KOCT_B) / ipow_h(TRK_P(e, KOCT_BORE), 3) * cfac * TRK_P(e, KOCT_L) * (1 + TRK_P(e, KOCT_FSE));
    else
      KnL[0] = TRK_P(e, KOCT_K3) * TRK_P(e, KOCT_L) * (1 + TRK_P(e, KOCT_FSE));
    drift = TRK_P(e, KOCT_L);
    tilt = TRK_P(e, KOCT_TILT);
    dx = TRK_P(e, KOCT_DX);
    dy = TRK_P(e, KOCT_DY);
    dz = TRK_P(e, KOCT_DZ);
    integ = (int)TRK_P(e, KOCT_INTEGRATION_ORDER);
    break;
  default:
    return trk_set_error(TRK_ERR_ARG, "not a multipole");
  }
  const double *df, *kf;
  int nSub = substeps(integ, &df, &kf);
  if (!nSub)
    return trk_set_error(TRK_ERR_PHYSICS, "%s: multipole integration_order must be 2, 4, or 6", e->name);
  if (n_kicks <= 0) {
    if (nSlices <= 0)
      return trk_set_error(TRK_ERR_PHYSICS, "%s: N_KICKS<=0 and N_SLICES<=0 in multipole tracking", e->name);
  } else {
    if (integ > 2) {
      if ((nSlices = (long)std::ceil(n_kicks / (1.0 * integ))) < 1)
        nSlices = 1;
    } else
      nSlices = n_kicks;
  }
  op->kind = OPK_MULT;
  op->i[0] = (int)nSlices;
  op->i[1] = nSub;
  op->i[2] = expand;
  op->i[3] = std::max(order[0], std::max(order[1], order[2]));
  op->i[4] = order[0] | (order[1] << 8) | (order[2] << 16);
  op->i[5] = skew[0] | (skew[1] << 1) | (skew[2] << 2);
  int flags = 0;
  if (dx || dy || dz)
    flags |= MF_OFFSET;
  double c, s;
  if (rotation(tilt, &c, &s)) {
    flags |= MF_TILT;
    op->d[MD_TC] = c;
    op->d[MD_TS] = s;
  }
  if (rotation(-tilt, &c, &s)) {
    op->d[MD_XC] = c;
    op->d[MD_XS] = s;
  }
  if (doEndDrift)
    flags |= MF_ENDDRIFT;
  op->d[MD_DX] = dx;
  op->d[MD_DY] = dy;
  op->d[MD_DZ] = dz;
  op->d[MD_LEND] = lEnd;
  /* setupMultApertureData(..., -tilt, ...) (src/multipole.c:990) */
  double rt = -tilt;
  if (rt) {
    flags |= MF_APTILT;
    op->d[MD_APC] = std::cos(rt);
    op->d[MD_APS] = std::sin(rt);
  }
  const long n_parts = nSlices;
  double driftp = drift / n_parts;
  double xk = xkick / n_parts, yk = ykick / n_parts;
  op->d[MD_DRIFT] = driftp;
  for (int st = 0; st < nSub; st++) {
    op->d[MD_DSH + st] = driftp * df[st];
    for (int o = 0; o < 3; o++)
      op->d[MD_KQ + st * 3 + o] = (KnL[o] / n_parts) * kf[st];
    op->d[MD_KX + st] = -xk * kf[st];
    op->d[MD_KY + st] = -yk * kf[st];
  }
  /* multipole_tracking2 keeps one dzLoss for all particles of a call and
   * integrate_kick_multipole_ordn resets it only after its entry checks
   * (src/multipole.c:686, :1179-1186, :1232): a particle rejected at entry is
   * recorded at z_start + the previous particle's dzLoss, which is this sum
   * whenever that particle went through the body */
  double dzfull = 0;
  if (driftp != 0)
    for (long k = 0; k < n_parts; k++)
      for (int st = 0; st < nSub; st++)
        dzfull += op->d[MD_DSH + st];
  op->d[MD_DZFULL] = dzfull;
  if (KnL[0])
    flags |= MF_KNL0;
  if (KnL[1])
    flags |= MF_KNL1;
  if (KnL[2])
    flags |= MF_KNL2;
  if (xk)
    flags |= MF_XKICK;
  if (yk)
    flags |= MF_YKICK;
  /* classical radiation: rad_coef = e^2 Po^3 / (6 pi eps0 c^2 m), zero for
   * elements shorter than 1e-6 m (src/multipole.c:755-763) */
  /* and incoherent radiation: isr_coef = r_e sqrt(55/(24 sqrt 3) Po^5 137.0359895)
   * (src/multipole.c:757-760) */
  if ((synch_rad || isr) && !(elem_length < 1e-6)) {
    const double rad_coef = synch_rad ? (TRK_E_MKS * TRK_E_MKS) * (Po * Po * Po) /
                                          (6 * TRK_PI * TRK_EPSILON_O * (TRK_C_MKS * TRK_C_MKS) * TRK_ME_MKS)
                                      : 0.0;
    const double isr_coef = isr ? TRK_RE_MKS * std::sqrt(55.0 / (24 * std::sqrt(3.0)) * ipow_h(Po, 5) * 137.0359895)
                                : 0.0;
    if (rad_coef || isr_coef > 0) {
      flags |= MF_RAD;
      op->d[MD_RAD] = rad_coef;
      op->d[MD_XKR] = xk;
      op->d[MD_YKR] = yk;
      for (int st = 0; st < nSub && st < 8; st++)
        op->d[MD_KFRAC + st] = kf[st];
      if (isr_coef > 0) {
        flags |= MF_ISR;
        op->d[MD_ISR] = isr_coef;
        if (!isr1)
          flags |= MF_ISR1OFF;
      }
    }
  }
  /* KQUAD hard-edge fringe (src/multipole.c:999-1006, :1054-1061; src/fringe.c) */
  if (e->type == TRK_KQUAD) {
    for (int edge = 0; edge < 2; edge++) {
      const int eff = (int)(edge ? TRK_P(e, KQUAD_EDGE2_EFFECTS) : TRK_P(e, KQUAD_EDGE1_EFFECTS));
      if (eff <= 0)
        continue;
      flags |= edge ? MF_FRINGE2 : MF_FRINGE1;
      double *fr = op->d + (edge ? MD_FR2 : MD_FR1);
      const int linear = (int)(edge ? TRK_P(e, KQUAD_EDGE2_LINEAR) : TRK_P(e, KQUAD_EDGE1_LINEAR));
      if (linear)
        quad_fringe_matrices(TRK_P(e, KQUAD_K1), &TRK_P(e, KQUAD_I0M), &TRK_P(e, KQUAD_I0P), TRK_P(e, KQUAD_L) < 0,
                             edge ? 1 : -1, fr, fr + 8);
      fr[16] = edge ? TRK_P(e, KQUAD_EDGE2_NONLINEAR_FACTOR) : TRK_P(e, KQUAD_EDGE1_NONLINEAR_FACTOR);
      fr[17] = eff;
      fr[18] = linear;
    }
    op->d[MD_FRK1] = TRK_P(e, KQUAD_K1);
  }
  op->i[6] = flags;
  return TRK_OK;
}

/* determine_bend_flags (src/bend_matrix.c:1347-1394) */
void bend_edge_flags(const trk_lattice *l, int idx, int *edge1, int *edge2) {
  const trk_elem *e = &l->e[idx];
  int precedes = 0, follows = 0;
  for (int k = idx - 1; k >= 0; k--) {
    if (l->e[k].type == e->type && std::strcmp(l->e[k].name, e->name) == 0) {
      precedes = 1;
      break;
    }
    if (l->e[k].type != TRK_MARK)
      break;
  }
  for (int k = idx + 1; k < l->n; k++) {
    if (l->e[k].type == e->type && std::strcmp(l->e[k].name, e->name) == 0) {
      follows = 1;
      break;
    }
    if (l->e[k].type != TRK_MARK)
      break;
  }
  *edge1 = TRK_P(e, CSBEND_EDGE1_EFFECTS) && !precedes;
  *edge2 = TRK_P(e, CSBEND_EDGE2_EFFECTS) && !follows;
}

/* computeEtiltCentroidOffset (src/csbend.c:4748-4790) */
void etilt_offset(double *d, double rho0, double angle, double etilt) {
  if (!etilt) {
    for (int i = 0; i < 6; i++)
      d[i] = 0;
    return;
  }
  etilt *= -1;
  double q1a = (1 - std::cos(angle)) * rho0 * (std::cos(etilt) - 1);
  double q2a = 0;
  double q3a = (1 - std::cos(angle)) * rho0 * std::sin(etilt);
  double qp1 = std::sin(angle) * std::cos(etilt);
  double qp2 = std::cos(angle);
  double k = std::sqrt(qp1 * qp1 + qp2 * qp2);
  qp1 /= k;
  qp2 /= k;
  double qp3 = std::sin(angle) * std::sin(etilt) / k;
  double tan_alpha = 1. / std::tan(angle) / std::cos(etilt);
  double q1b = q1a * tan_alpha / (std::tan(angle) + tan_alpha);
  double q2b = -q1b * std::tan(angle);
  double dz = std::sqrt((q1b - q1a) * (q1b - q1a) + (q2b - q2a) * (q2b - q2a));
  double q3b = q3a + qp3 * dz;
  d[0] = std::sqrt(q1b * q1b + q2b * q2b);
  d[1] = std::tan(std::atan(tan_alpha) - (TRK_PIo2 - angle));
  d[2] = q3b;
  d[3] = qp3;
  d[4] = dz * std::sqrt(1 + qp3 * qp3);
  d[5] = 0;
}

int edge_mode(int on, int effects, int edge_order, const char *name) {
  if (!on || effects == 0)
    return EDGE_NONE;
  if (effects == 1)
    return edge_order <= 1 ? EDGE_LIN1 : EDGE_LIN2;
  if (effects == 3)
    return EDGE_SYMP;
  if (effects == 2)
    return edge_order <= 1 ? EDGE_HWANG1 : EDGE_HWANG2;
  if (effects == 4)
    return EDGE_HWANGL;
  if (effects == 5)
    return edge_order <= 1 ? EDGE_CURV1 : EDGE_CURV2;
  trk_set_error(TRK_ERR_UNSUPPORTED, "CSBEND %s: EDGE_EFFECTS=%d is not on this path (0 to 5 are)", name, effects);
  return -1;
}

/* set-up of track_through_csbend (src/csbend.c:654-1078) */
int compile_bend(const trk_lattice *l, int idx, double Po, trk_op *op, std::vector<double> &field) {
  const trk_elem *e = &l->e[idx];
  if (TRK_P(e, CSBEND_REFERENCE_CORRECTION) || TRK_P(e, CSBEND_FSE_CORRECTION) || TRK_P(e, CSBEND_MALIGN_METHOD) ||
      TRK_P(e, CSBEND_USE_RAD_DIST))
    return trk_set_error(TRK_ERR_UNSUPPORTED,
                         "CSBEND %s: REFERENCE_CORRECTION, FSE_CORRECTION, MALIGN_METHOD!=0 and "
                         "USE_RAD_DIST (photon-based radiation) are not on this path",
                         e->name);
  const double L = TRK_P(e, CSBEND_L), ANGLE = TRK_P(e, CSBEND_ANGLE);
  if (ANGLE == 0) {
    op->kind = OPK_EDRIFT;
    op->d[DD_L] = L;
    return TRK_OK;
  }
  const double *df, *kf;
  int integ = (int)TRK_P(e, CSBEND_INTEGRATION_ORDER);
  int nSub = substeps(integ, &df, &kf);
  if (!nSub)
    return trk_set_error(TRK_ERR_PHYSICS, "CSBEND integration_order is invalid--must be 2, 4, or 6");
  double b[9], c[9];
  double rho0 = L / ANGLE;
  b[0] = 0;
  for (int i = 1; i <= 8; i++)
    b[i] = TRK_P(e, CSBEND_USE_BN) ? e->p[P_CSBEND_B1 + i - 1] : e->p[P_CSBEND_K1 + i - 1] * rho0;
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
  const double fse_ = TRK_P(e, CSBEND_FSE), fseD = TRK_P(e, CSBEND_FSE_DIPOLE), fseQ = TRK_P(e, CSBEND_FSE_QUADRUPOLE);
  b[1] *= (1 + fse_ + fseQ) / (1 + fse_ + fseD);
  c[1] *= (1 + fse_ + fseQ) / (1 + fse_ + fseD);
  b[2] *= (1 + fse_) / (1 + fse_ + fseD);
  c[2] *= (1 + fse_) / (1 + fse_ + fseD);
  b[0] = TRK_P(e, CSBEND_XKICK) / ANGLE;
  c[0] = TRK_P(e, CSBEND_YKICK) / ANGLE;
  double angle, e1, e2, etilt, tilt;
  const double he1 = TRK_P(e, CSBEND_H1), he2 = TRK_P(e, CSBEND_H2);
  if (ANGLE < 0) {
    angle = -ANGLE;
    e1 = -TRK_P(e, CSBEND_E1);
    e2 = -TRK_P(e, CSBEND_E2);
    etilt = TRK_P(e, CSBEND_ETILT) * TRK_P(e, CSBEND_ETILT_SIGN);
    tilt = TRK_P(e, CSBEND_TILT) + TRK_PI;
    rho0 = L / angle;
    for (int i = 1; i < 9; i += 2) {
      b[i] *= -1;
      c[i] *= -1;
    }
  } else {
    angle = ANGLE;
    e1 = TRK_P(e, CSBEND_E1);
    e2 = TRK_P(e, CSBEND_E2);
    etilt = TRK_P(e, CSBEND_ETILT) * TRK_P(e, CSBEND_ETILT_SIGN);
    tilt = TRK_P(e, CSBEND_TILT);
    rho0 = L / angle;
  }
  if (std::fabs(rho0) > 1e6) {
    if (TRK_P(e, CSBEND_K1) != 0 || TRK_P(e, CSBEND_K2) != 0)
      return trk_set_error(TRK_ERR_UNSUPPORTED, "CSBEND %s: radius > 1e6 with K1/K2 is tracked as KQUAD by the reference",
                           e->name);
    op->kind = OPK_EDRIFT;
    op->d[DD_L] = L;
    return TRK_OK;
  }
  double fse = fse_ + fseD;
  const double h = 1 / rho0;
  const double n = -b[1] / h;
  if (std::fabs(fse + 1) < 1e-12)
    fse = -1 + 1e-12;
  const double rho_actual = 1 / ((1 + fse) * h);
  double lim1 = TRK_P(e, CSBEND_EDGE1_KICK_LIMIT), lim2 = TRK_P(e, CSBEND_EDGE2_KICK_LIMIT);
  if (TRK_P(e, CSBEND_KICK_LIMIT_SCALING)) {
    lim1 *= rho0 / rho_actual;
    lim2 *= rho0 / rho_actual;
  }
  const double hgap = TRK_P(e, CSBEND_HGAP);
  const double fint1 = TRK_P(e, CSBEND_FINT1) >= 0 ? TRK_P(e, CSBEND_FINT1) : TRK_P(e, CSBEND_FINT);
  const double fint2 = TRK_P(e, CSBEND_FINT2) >= 0 ? TRK_P(e, CSBEND_FINT2) : TRK_P(e, CSBEND_FINT);
  const double Kg1 = 2 * hgap * fint1 * sgn(rho0);
  double psi1 = Kg1 / std::fabs(rho_actual) / std::cos(e1) * (1 + std::sin(e1) * std::sin(e1));
  const double Kg2 = 2 * hgap * fint2 * sgn(rho0);
  double psi2 = Kg2 / std::fabs(rho_actual) / std::cos(e2) * (1 + std::sin(e2) * std::sin(e2));
  if (L < 0) {
    psi1 *= -1;
    psi2 *= -1;
  }
  const long nSlices = (long)TRK_P(e, CSBEND_N_SLICES);
  if (nSlices < 1)
    return trk_set_error(TRK_ERR_PHYSICS, "CSBEND %s: invalid number of steps", e->name);
  double Fx[121], Fy[121];
  int eo1, hasN, hasS;
  if (trk_csbend_field_table(b, c, h, (int)TRK_P(e, CSBEND_NONLINEAR), (long)TRK_P(e, CSBEND_EXPANSION_ORDER), Fx, Fy,
                             &eo1, &hasN, &hasS))
    return trk_set_error(TRK_ERR_PHYSICS, "expansion order >10 for CSBEND %s", e->name);
  op->kind = OPK_BEND;
  op->i[0] = (int)nSlices;
  op->i[1] = nSub;
  op->i[2] = hasS ? 2 : (hasN ? 1 : 0);
  op->i[3] = eo1;
  op->i[4] = (int)field.size();
  if (hasN || hasS) {
    field.insert(field.end(), Fx, Fx + 121);
    field.insert(field.end(), Fy, Fy + 121);
  }
  int ed1, ed2;
  bend_edge_flags(l, idx, &ed1, &ed2);
  int eo = (int)TRK_P(e, CSBEND_EDGE_ORDER);
  int m1 = edge_mode(ed1, (int)TRK_P(e, CSBEND_EDGE1_EFFECTS), eo, e->name);
  int m2 = edge_mode(ed2, (int)TRK_P(e, CSBEND_EDGE2_EFFECTS), eo, e->name);
  if (m1 < 0 || m2 < 0)
    return TRK_ERR_UNSUPPORTED;
  if (eo > 1 && (TRK_P(e, CSBEND_EDGE1_EFFECTS) == 2 || TRK_P(e, CSBEND_EDGE2_EFFECTS) == 2) &&
      TRK_P(e, CSBEND_HGAP) == 0)
    return trk_set_error(TRK_ERR_PHYSICS, /* src/csbend.c:711-712 */
                         "CSBEND %s has EDGE_ORDER>1 and EDGE[12]_EFFECTS==2, but HGAP=0. This gives undefined "
                         "results.",
                         e->name);
  op->i[5] = m1;
  op->i[6] = m2;
  double *d = op->d;
  d[BD_RHO0] = rho0;
  d[BD_RHOA] = rho_actual;
  const double s = L / nSlices;
  d[BD_SLICE] = s;
  for (int j = 0; j < nSub; j++) {
    double dsh = s * df[j];
    d[BD_DSH + j] = dsh;
    d[BD_ARG + j] = dsh / rho0;
    d[BD_DS + j] = s * kf[j];
    d[BD_SA + j] = std::sin(dsh / rho0);
    d[BD_CA + j] = std::cos(dsh / rho0);
    d[BD_SH + j] = std::sin(dsh / (2 * rho0));
    d[BD_CH + j] = std::cos(dsh / (2 * rho0));
  }
  /* total tilt (src/csbend.c:1039-1055) */
  const double ttilt = tilt + etilt;
  double ct, st;
  if (ttilt == 0) {
    ct = 1;
    st = 0;
  } else if (std::fabs(std::fabs(ttilt) - TRK_PI) < 1e-12) {
    ct = -1;
    st = 0;
  } else if (std::fabs(ttilt - TRK_PIo2) < 1e-12) {
    ct = 0;
    st = 1;
  } else if (std::fabs(ttilt + TRK_PIo2) < 1e-12) {
    ct = 0;
    st = -1;
  } else {
    ct = std::cos(ttilt);
    st = std::sin(ttilt);
  }
  d[BD_CT] = ct;
  d[BD_ST] = st;
  double det[6];
  etilt_offset(det, rho0, angle, etilt);
  for (int k = 0; k < 5; k++)
    d[BD_ET + k] = det[k];
  const double dx = TRK_P(e, CSBEND_DX), dy = TRK_P(e, CSBEND_DY), dz = TRK_P(e, CSBEND_DZ);
  d[BD_DXI] = -dx;
  d[BD_DYI] = -dy;
  d[BD_DZI] = dz;
  d[BD_DXF] = dx * std::cos(ANGLE) + dz * std::sin(ANGLE);
  d[BD_DZF] = dx * std::sin(ANGLE) - dz * std::cos(ANGLE);
  d[BD_DYF] = dy;
  int flags = 0;
  if (Po > 0)
    flags |= BF_ISR_ROUNDTRIP; /* isrConstant < 0 but nonzero (src/csbend.c:931-934) */
  if (dx || dy || dz || ttilt || etilt)
    flags |= BF_MISALIGN;
  if (TRK_P(e, CSBEND_EXPAND_HAMILTONIAN))
    flags |= BF_EXPAND; /* integrate_csbend_ordn_expanded (src/csbend.c:1227-1229) */
  /* classical radiation (src/csbend.c:953-959) */
  if (TRK_P(e, CSBEND_SYNCH_RAD)) {
    const double rad_coef = (TRK_E_MKS * TRK_E_MKS) * (Po * Po * Po) * ((1 + fse) * (1 + fse)) /
                            (6 * TRK_PI * TRK_EPSILON_O * (TRK_C_MKS * TRK_C_MKS) * TRK_ME_MKS * (rho0 * rho0));
    if (rad_coef) {
      flags |= BF_RAD;
      d[BD_RAD] = rad_coef;
      /* delta adjusted at edges with nonzero angles (src/csbend.c:1215-1222, :1270-1281) */
      if (ed1 && e1 != 0)
        flags |= BF_RADE1;
      if (ed2 && e2 != 0)
        flags |= BF_RADE2;
    }
  }
  /* incoherent radiation: isrConstant (src/csbend.c:961-964) */
  if (TRK_P(e, CSBEND_ISR)) {
    const double ra = std::fabs(rho_actual);
    const double isr_constant =
      TRK_RE_MKS * std::sqrt(55.0 / (24 * std::sqrt(3.0)) * ipow_h(Po, 5) * 137.0359895 / (ra * ra * ra));
    if (isr_constant > 0) {
      flags |= BF_RAD | BF_ISR;
      d[BD_ISR] = isr_constant;
      if (TRK_P(e, CSBEND_ISR1PART) == 0)
        flags |= BF_ISR1OFF;
    }
  }
  const double rt = -tilt;
  if (rt) {
    flags |= BF_APTILT;
    d[BD_APC] = std::cos(rt);
    d[BD_APS] = std::sin(rt);
  }
  op->i[7] = flags;
  d[BD_E1] = e1;
  d[BD_TE1] = trkcr_tan(e1); /* tan and sec of the edge angles rounded once */
  d[BD_PSI1] = psi1;
  d[BD_LIM1] = lim1;
  d[BD_HE1] = he1;
  d[BD_SE1] = 1. / trkcr_cos(e1);
  d[BD_E2] = e2;
  d[BD_TE2] = trkcr_tan(e2);
  d[BD_PSI2] = psi2;
  d[BD_LIM2] = lim2;
  d[BD_HE2] = he2;
  d[BD_SE2] = 1. / trkcr_cos(e2);
  /* Hwang fringes: the values dipoleFringeKHwang / ...RLindberg form per call
   * (src/csbend.c:4360-4363, :4443-4446); FINT1/FINT2 where >= 0, else FINT
   * (src/csbend.c:1150, :1329) */
  d[BD_FS1] = std::sin(e1);
  d[BD_FC1] = std::cos(e1);
  d[BD_FS2] = std::sin(e2);
  d[BD_FC2] = std::cos(e2);
  d[BD_FF1] = TRK_P(e, CSBEND_FINT1) >= 0 ? TRK_P(e, CSBEND_FINT1) : TRK_P(e, CSBEND_FINT);
  d[BD_FF2] = TRK_P(e, CSBEND_FINT2) >= 0 ? TRK_P(e, CSBEND_FINT2) : TRK_P(e, CSBEND_FINT);
  d[BD_GAP] = 2 * TRK_P(e, CSBEND_HGAP);
  /* curved-dipole fringe: K1 as track_through_csbend passes it (b[1]/rho0
   * after the sign change of a negative bend, src/csbend.c:1193, :1370), the
   * FRINGE1K0..6 / FRINGE2K0..6 integrals and the edge angle's tan and sec,
   * rounded once as curvedDipoleFringe forms them (src/csbend.c:5720-5721) */
  d[BD_K1F] = b[1] / rho0;
  if (m1 == EDGE_CURV1 || m1 == EDGE_CURV2 || m2 == EDGE_CURV1 || m2 == EDGE_CURV2) {
    for (int k = 0; k < 2; k++) {
      const double ek = k ? e2 : e1;
      for (int j = 0; j < 7; j++)
        field.push_back(e->p[(k ? P_CSBEND_FRINGE2K0 : P_CSBEND_FRINGE1K0) + j]);
      field.push_back(trkcr_tan(ek));
      field.push_back(1. / trkcr_cos(ek));
    }
  }
  d[BD_N] = n;
  d[BD_RHOINV] = 1.0 / rho0;
  d[BD_INVRHOA] = 1.0 / rho_actual;
  for (int j = 0; j < nSub; j++) {
    d[BD_OMC + j] = 2 * d[BD_SH + j] * d[BD_SH + j];
    d[BD_C1 + j] = d[BD_DS + j] * d[BD_INVRHOA];
    d[BD_C2 + j] = d[BD_C1 + j] * d[BD_RHOINV];
  }
  return TRK_OK;
}

int compile_rf(const trk_elem *e, trk_op *op, int slot) {
  if (TRK_P(e, RFCA_CHANGE_T) || TRK_P(e, RFCA_STANDING_WAVE))
    return trk_set_error(TRK_ERR_UNSUPPORTED, "RFCA %s: CHANGE_T and STANDING_WAVE are not on this path", e->name);
  double length = TRK_P(e, RFCA_L);
  if (TRK_P(e, RFCA_VOLT) == 0) {
    op->kind = OPK_RFDRIFT; /* src/simple_rfca.c:389-401 */
    op->d[DD_L] = length;
    return TRK_OK;
  }
  long nKicks = length ? (long)TRK_P(e, RFCA_N_KICKS) : 1;
  if (nKicks <= 0)
    return trk_set_error(TRK_ERR_UNSUPPORTED, "RFCA %s: L>0 with N_KICKS=0 (matrix method) is not on this path",
                         e->name);
  const bool lock = TRK_P(e, RFCA_LOCK_PHASE) != 0, linearize = TRK_P(e, RFCA_LINEARIZE) != 0;
  if ((lock || linearize) && nKicks != 1)
    return trk_set_error(TRK_ERR_PHYSICS, "Must use n_kicks=1 for linearized rf cavity"); /* src/simple_rfca.c:505 */
  double omega = TRK_PIx2 * TRK_P(e, RFCA_FREQ);
  double volt = TRK_P(e, RFCA_VOLT) / (1e6 * TRK_ME_MEV * TRK_PARTICLE_REL_SIGN);
  double tau = omega ? TRK_P(e, RFCA_Q) / omega : 0;
  length /= nKicks;
  volt /= nKicks;
  op->kind = OPK_RF;
  op->i[0] = (int)nKicks;
  op->i[1] = slot;
  int flags = 0;
  if (omega == 0 && tau == 0)
    flags |= RF_SAME_DGAMMA;
  if (TRK_P(e, RFCA_END1_FOCUS))
    flags |= RF_END1;
  if (TRK_P(e, RFCA_END2_FOCUS))
    flags |= RF_END2;
  if (TRK_P(e, RFCA_DX) || TRK_P(e, RFCA_DY))
    flags |= RF_OFFSET;
  if (lock)
    flags |= RF_LOCK;
  if (linearize)
    flags |= RF_LINEAR;
  if (TRK_P(e, RFCA_CHANGE_P0))
    flags |= RF_CHANGE_P0; /* do_match_energy after the cavity (src/simple_rfca.c:977-978) */
  op->i[3] = flags;
  op->d[RD_OMEGA] = omega;
  op->d[RD_VOLT] = volt;
  op->d[RD_LEN] = length;
  op->d[RD_DTL] = length / TRK_C_MKS;
  op->d[RD_TAU] = tau;
  op->d[RD_PHASE_ADD] = TRK_P(e, RFCA_PHASE) * TRK_PI / 180.0;
  op->d[RD_DX] = TRK_P(e, RFCA_DX);
  op->d[RD_DY] = TRK_P(e, RFCA_DY);
  op->d[RD_SOFF] = length / 2;
  op->d[RD_TREF] = TRK_P(e, RFCA_T_REFERENCE);
  op->d[RD_PHASE_LOCK] = TRK_PI / 180 * TRK_P(e, RFCA_PHASE);
  return TRK_OK;
}

int compile_wake(const trk_elem *e, trk_op *op, CompiledWake &w) {
  const bool tr = e->type == TRK_TRWAKE;
  if (!e->wake_t || e->wake_points < 2)
    return trk_set_error(TRK_ERR_ARG, "%s %s: no wake table (trk_lattice_set_wake)", tr ? "TRWAKE" : "WAKE", e->name);
  if (tr ? TRK_P(e, TRWAKE_SMOOTHING) : TRK_P(e, WAKE_SMOOTHING))
    return trk_set_error(TRK_ERR_UNSUPPORTED, "%s: SMOOTHING is not on this path", e->name);
  if ((tr ? TRK_P(e, TRWAKE_START_BUNCH) : TRK_P(e, WAKE_START_BUNCH)) >= 0 ||
      (tr ? TRK_P(e, TRWAKE_END_BUNCH) : TRK_P(e, WAKE_END_BUNCH)) >= 0)
    return trk_set_error(TRK_ERR_UNSUPPORTED, "%s: START_BUNCH/END_BUNCH (bunched-beam mode) are not on this path",
                         e->name);
  long nbins = (long)(tr ? TRK_P(e, TRWAKE_N_BINS) : TRK_P(e, WAKE_N_BINS));
  if (nbins < 2 && nbins != 0)
    return trk_set_error(TRK_ERR_PHYSICS, "n_bins must be >=2 or else 0 (autoscale) for WAKE element %s", e->name);
  /* set_up_wake (src/wake.c:434-477) */
  double tmin = 1.7976931348623157e308, tmax = -1.7976931348623157e308;
  for (long i = 0; i < e->wake_points; i++) {
    tmin = std::min(tmin, e->wake_t[i]);
    tmax = std::max(tmax, e->wake_t[i]);
  }
  if (tmin >= tmax)
    return trk_set_error(TRK_ERR_PHYSICS, "zero or negative time span in wake table of %s", e->name);
  w.dt = (tmax - tmin) / (e->wake_points - 1);
  w.i0 = 0;
  int acausal = (int)(tr ? TRK_P(e, TRWAKE_ACAUSAL_ALLOWED) : TRK_P(e, WAKE_ACAUSAL_ALLOWED));
  if (tmin != 0) {
    if (!acausal)
      return trk_set_error(TRK_ERR_PHYSICS, "wake function of %s does not start at t=0 (set ACAUSAL_ALLOWED=1)", e->name);
    w.i0 = -1;
    for (long iw = 0; iw < e->wake_points; iw++)
      if (std::fabs(e->wake_t[iw]) < 1e-6 * w.dt) {
        w.i0 = iw;
        break;
      }
    if (w.i0 == -1 || std::fabs(tmin) > tmax)
      return trk_set_error(TRK_ERR_PHYSICS, "bad acausal wake table for %s", e->name);
  }
  w.span = e->wake_t[e->wake_points - 1] - e->wake_t[0];
  w.points = e->wake_points;
  w.n_bins = nbins;
  int allow_long = tr ? 0 : (int)TRK_P(e, WAKE_ALLOW_LONG_BEAM);
  w.allow_long_beam = allow_long;
  w.max_bins = nbins ? nbins : (allow_long ? 16 * (e->wake_points + 3) : e->wake_points + 3);
  w.t = e->wake_t;
  w.W = e->wake_w0;
  w.Wy = e->wake_w1;
  w.transverse = tr;
  w.change_p0 = !tr && TRK_P(e, WAKE_CHANGE_P0) != 0; /* src/wake.c:289-290 */
  w.factor = tr ? TRK_P(e, TRWAKE_FACTOR) : TRK_P(e, WAKE_FACTOR);
  w.xfactor = tr ? TRK_P(e, TRWAKE_XFACTOR) : 1;
  w.yfactor = tr ? TRK_P(e, TRWAKE_YFACTOR) : 1;
  w.interpolate = (int)(tr ? TRK_P(e, TRWAKE_INTERPOLATE) : TRK_P(e, WAKE_INTERPOLATE));
  w.ramp_passes = (long)(tr ? TRK_P(e, TRWAKE_RAMP_PASSES) : TRK_P(e, WAKE_RAMP_PASSES));
  w.charge = tr ? TRK_P(e, TRWAKE_CHARGE) : TRK_P(e, WAKE_CHARGE);
  if (tr) {
    w.x_power = (int)TRK_P(e, TRWAKE_X_DRIVE_EXPONENT);
    w.y_power = (int)TRK_P(e, TRWAKE_Y_DRIVE_EXPONENT);
    w.x_probe = (int)TRK_P(e, TRWAKE_X_PROBE_EXPONENT);
    w.y_probe = (int)TRK_P(e, TRWAKE_Y_PROBE_EXPONENT);
    w.tdx = TRK_P(e, TRWAKE_DX);
    w.tdy = TRK_P(e, TRWAKE_DY);
    w.tilt = TRK_P(e, TRWAKE_TILT);
  }
  op->kind = tr ? OPK_TRWAKE : OPK_WAKE;
  return TRK_OK;
}

} // namespace

int trk_compile(const trk_lattice *l, double Po, CompiledLattice &out) {
  out = CompiledLattice();
  if (!l)
    return trk_set_error(TRK_ERR_ARG, "null lattice");
  const int n = l->n;
  out.ops.resize(n);
  /* aperture record 0..: one per MAXAMP element (sticky state, src/do_tracking.c:1883-1893) */
  std::vector<int> ap_of_elem(n, -1);
  for (int i = 0; i < n; i++) {
    const trk_elem *e = &l->e[i];
    if (e->type != TRK_MAXAMP)
      continue;
    trk_aperture a;
    std::memset(&a, 0, sizeof(a));
    a.x_max = TRK_P(e, MAXAMP_X_MAX);
    a.y_max = TRK_P(e, MAXAMP_Y_MAX);
    a.elliptical = (int)TRK_P(e, MAXAMP_ELLIPTICAL);
    long xe = (long)TRK_P(e, MAXAMP_EXPONENT), ye = (long)TRK_P(e, MAXAMP_YEXPONENT);
    a.xexp = (int)xe;
    a.yexp = (int)(ye ? ye : xe);
    if (a.elliptical && (a.x_max || a.y_max)) {
      /* elimit_amplitudes exits on a bad exponent (src/limit_amplitudes.c:523-538) */
      if (xe < 2 || xe % 2 || (ye && (ye < 2 || ye % 2)))
        return trk_set_error(TRK_ERR_PHYSICS, "MAXAMP %s: exponent is not valid. Give even integer >=2", e->name);
    }
    a.valid = 1;
    a.a2 = ipow_h(a.x_max, a.xexp);
    a.b2 = ipow_h(a.y_max, a.yexp);
    ap_of_elem[i] = (int)out.aps.size();
    out.aps.push_back(a);
  }
  int last_maxamp = -1;
  for (int i = 0; i < n; i++)
    if (l->e[i].type == TRK_MAXAMP)
      last_maxamp = i;

  std::vector<int> rf_slot_of_ref; /* PHASE_REFERENCE -> slot */
  std::vector<long> rf_ref_ids;
  double z = 0;
  int cur_maxamp = -1;
  for (int i = 0; i < n; i++) {
    const trk_elem *e = &l->e[i];
    trk_op &op = out.ops[i];
    std::memset(&op, 0, sizeof(op));
    op.elem = i;
    op.z_start = z;
    z += trk_elem_length(e);
    op.z_end = z;
    op.ap_post[0] = op.ap_post[1] = op.ap_in[0] = op.ap_in[1] = -1;
    op.no_aperture = (e->type == TRK_MARK || e->type == TRK_CHARGE);
    op.extrapolate = (e->type == TRK_DRIF);
    int rc = TRK_OK;
    switch (e->type) {
    case TRK_MARK:
    case TRK_CHARGE:
    case TRK_MAXAMP:
      op.kind = OPK_NOP;
      break;
    case TRK_DRIF: {
      long order = (long)TRK_P(e, DRIF_ORDER);
      if (order == 0)
        order = 2; /* run->default_order (src/elegant.nl:43) */
      if (order > 2)
        order = 2;
      op.kind = OPK_DRIFT;
      op.i[0] = (int)order;
      op.d[DD_L] = TRK_P(e, DRIF_L);
      op.d[DD_T] = TRK_P(e, DRIF_L) / 2;
      break;
    }
    case TRK_EDRIFT:
      op.kind = OPK_EDRIFT;
      op.d[DD_L] = TRK_P(e, EDRIFT_L);
      break;
    case TRK_KQUAD:
    case TRK_KSEXT:
    case TRK_KOCT:
      rc = compile_mult(e, Po, &op);
      if (rc == TRK_OK)
        out.n_mult++;
      break;
    case TRK_CSBEND:
      rc = compile_bend(l, i, Po, &op, out.field);
      break;
    case TRK_RFCA: {
      long ref = (long)TRK_P(e, RFCA_PHASE_REFERENCE);
      int slot = -1;
      if (ref != 0)
        for (size_t k = 0; k < rf_ref_ids.size(); k++)
          if (rf_ref_ids[k] == ref)
            slot = (int)k;
      if (slot < 0) {
        slot = (int)rf_ref_ids.size();
        rf_ref_ids.push_back(ref != 0 ? ref : -1 - i);
        out.rf_first_op.push_back(i);
      }
      rc = compile_rf(e, &op, slot);
      break;
    }
    case TRK_WAKE:
    case TRK_TRWAKE: {
      CompiledWake w;
      rc = compile_wake(e, &op, w);
      if (rc == TRK_OK) {
        w.op = i;
        out.wakes.push_back(w);
        op.i[0] = (int)out.wakes.size() - 1;
      }
      break;
    }
    default:
      rc = trk_set_error(TRK_ERR_UNKNOWN_TYPE, "element type %d not supported", e->type);
    }
    if (rc != TRK_OK)
      return rc;
    /* kinds with a specialized fast-build body (the parity build runs the
     * general body for them) */
    if (op.kind == OPK_MULT) {
      const int f = op.i[6];
      const int o = op.i[4] & 0xff;
      if (op.i[1] == 4 && !op.i[2] && op.d[MD_DRIFT] != 0 && o >= 1 && o <= 3 && !(op.i[5] & 1) &&
          !(f & (MF_KNL1 | MF_KNL2 | MF_XKICK | MF_YKICK | MF_OFFSET | MF_TILT | MF_ENDDRIFT | MF_RAD | MF_FRINGE1 |
                 MF_FRINGE2)))
        op.kind = OPK_MULT1;
    } else if (op.kind == OPK_BEND) {
      const bool e1_noop = op.i[5] == EDGE_NONE ||
                           (op.i[5] == EDGE_LIN1 && op.d[BD_TE1] == 0 && op.d[BD_PSI1] == 0 && op.d[BD_LIM1] <= 0);
      const bool e2_noop = op.i[6] == EDGE_NONE ||
                           (op.i[6] == EDGE_LIN1 && op.d[BD_TE2] == 0 && op.d[BD_PSI2] == 0 && op.d[BD_LIM2] <= 0);
      const bool plain =
        op.i[1] == 4 && !(op.i[7] & (BF_MISALIGN | BF_APTILT | BF_RAD | BF_EXPAND)) && e1_noop && e2_noop;
      if (plain && op.i[2] == 0)
        op.kind = OPK_DIPOLE;
      else if (plain && op.i[2] == 1 && op.i[3] == 5) {
        op.kind = OPK_CFBEND;
        out.has_cfbend = true;
      }
    }
    if (op.kind != OPK_NOP && op.kind != OPK_DRIFT && op.kind != OPK_EDRIFT && op.kind != OPK_RFDRIFT &&
        op.kind != OPK_MULT1 && op.kind != OPK_DIPOLE && op.kind != OPK_CFBEND && op.kind != OPK_RF &&
        op.kind != OPK_WAKE && op.kind != OPK_TRWAKE)
      out.lean = false;
    if (e->type == TRK_MAXAMP)
      cur_maxamp = i;
    /* aperture state for the first pass of a run and for later passes */
    int st0 = cur_maxamp;
    int stN = cur_maxamp >= 0 ? cur_maxamp : last_maxamp;
    int states[2] = {st0, stN};
    for (int v = 0; v < 2; v++) {
      int m = states[v];
      if (m < 0)
        continue;
      const trk_aperture &a = out.aps[ap_of_elem[m]];
      bool active = a.x_max > 0 || a.y_max > 0;
      /* in-element checks (checkMultAperture) only matter with a positive limit */
      if (active && (op.kind == OPK_MULT || op.kind == OPK_BEND || op.kind == OPK_MULT1 || op.kind == OPK_DIPOLE ||
                     op.kind == OPK_CFBEND))
        op.ap_in[v] = ap_of_elem[m];
      /* after-element limit if (x_max || y_max) (src/do_tracking.c:2508) */
      if (a.x_max || a.y_max)
        op.ap_post[v] = ap_of_elem[m];
    }
  }
  out.total_length = z;
  out.n_rf_slots = (int)rf_ref_ids.size();
  /* CHANGE_P0 moves the central momentum inside the run; the radiation
   * constants are formed from it once, at compile time */
  bool change_p0 = false;
  for (const trk_op &op : out.ops)
    change_p0 = change_p0 || (op.kind == OPK_RF && (op.i[3] & RF_CHANGE_P0));
  for (const CompiledWake &w : out.wakes)
    change_p0 = change_p0 || w.change_p0;
  if (change_p0)
    for (const trk_op &op : out.ops)
      if ((op.kind == OPK_BEND && (op.i[7] & BF_RAD)) || (op.kind == OPK_MULT && (op.i[6] & MF_RAD)))
        return trk_set_error(TRK_ERR_UNSUPPORTED,
                             "CHANGE_P0 with radiating elements (SYNCH_RAD, ISR) is not on this path");
  return TRK_OK;
}

void trk_expansion_coefficients(double *coef10) {
  /* expansion_coefficients(n), n = 0..3 (src/multipole.h:76-146):
   * (-1)^(i/2) / (i! (n-i)!) with orders 0..2 as literal tables */
  const double c0[] = {1.};
  const double c1[] = {1., 1.};
  const double c2[] = {1. / 2, 1., -1. / 2};
  coef10[0] = c0[0];
  coef10[1] = c1[0];
  coef10[2] = c1[1];
  for (int i = 0; i < 3; i++)
    coef10[3 + i] = c2[i];
  for (int i = 0; i <= 3; i++) {
    double fi = 1, fn = 1;
    for (long k = i; k > 1; k--)
      fi *= k;
    for (long k = 3 - i; k > 1; k--)
      fn *= k;
    coef10[6 + i] = (((i / 2) & 1) ? -1.0 : 1.0) / (fi * fn);
  }
}
