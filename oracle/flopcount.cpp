// TEST INFRASTRUCTURE: counts the algorithmic FP64 operations per particle of
// the reference formulation of each element, by compiling the oracle's
// per-particle maps (trk_oracle_core.h) with a counting number type.
//
// Convention: add, sub, mul, div and sqrt of particle-dependent values count
// 1 each (the reference build has no FMA); sin, cos, asin count 1 each and are
// also listed separately; comparisons and per-element constants (products of
// element parameters that a compiler hoists) are not counted.  DRIF, EDRIFT
// and the RFCA/WAKE per-particle arithmetic are counted from their formulas
// (structural zeros of the DRIF matrix removed).
//
// Writes oracle/flops.json: per-element counts and F per particle-turn for
// the benchmark lattices.
#include <cmath>
#include <cstdio>
#include <cstring>

struct Count {
  long add = 0, mul = 0, div = 0, sqrt = 0, trans = 0;
  long total() const { return add + mul + div + sqrt + trans; }
};
static Count g;

struct FR {
  double v;
  FR() : v(0) {}
  FR(double x) : v(x) {}
  FR &operator+=(const FR &o) { g.add++; v += o.v; return *this; }
  FR &operator-=(const FR &o) { g.add++; v -= o.v; return *this; }
  FR &operator*=(const FR &o) { g.mul++; v *= o.v; return *this; }
  FR &operator/=(const FR &o) { g.div++; v /= o.v; return *this; }
  FR operator-() const { return FR(-v); }
};
static FR operator+(const FR &a, const FR &b) { g.add++; return FR(a.v + b.v); }
static FR operator-(const FR &a, const FR &b) { g.add++; return FR(a.v - b.v); }
static FR operator*(const FR &a, const FR &b) { g.mul++; return FR(a.v * b.v); }
static FR operator/(const FR &a, const FR &b) { g.div++; return FR(a.v / b.v); }
static FR operator+(double a, const FR &b) { g.add++; return FR(a + b.v); }
static FR operator-(double a, const FR &b) { g.add++; return FR(a - b.v); }
static FR operator*(double a, const FR &b) { g.mul++; return FR(a * b.v); }
static FR operator/(double a, const FR &b) { g.div++; return FR(a / b.v); }
static FR operator+(const FR &a, double b) { g.add++; return FR(a.v + b); }
static FR operator-(const FR &a, double b) { g.add++; return FR(a.v - b); }
static FR operator*(const FR &a, double b) { g.mul++; return FR(a.v * b); }
static FR operator/(const FR &a, double b) { g.div++; return FR(a.v / b); }
static FR operator+(int a, const FR &b) { return double(a) + b; }
static FR operator-(int a, const FR &b) { return double(a) - b; }
static FR operator*(int a, const FR &b) { return double(a) * b; }
static FR operator/(int a, const FR &b) { return double(a) / b; }
static bool operator<(const FR &a, const FR &b) { return a.v < b.v; }
static bool operator>(const FR &a, const FR &b) { return a.v > b.v; }
static FR fr_sqrt(const FR &a) { g.sqrt++; return FR(std::sqrt(a.v)); }
static FR fr_sin(const FR &a) { g.trans++; return FR(std::sin(a.v)); }
static FR fr_cos(const FR &a) { g.trans++; return FR(std::cos(a.v)); }
static FR fr_asin(const FR &a) { g.trans++; return FR(std::asin(a.v)); }
static FR fr_tan(const FR &a) { g.trans++; return FR(std::tan(a.v)); }
static FR fr_fabs(const FR &a) { return FR(std::fabs(a.v)); }

#define ORC_R FR
#define ORC_SQRT(x) fr_sqrt(x)
#define ORC_SIN(x) fr_sin(x)
#define ORC_COS(x) fr_cos(x)
#define ORC_TAN(x) fr_tan(x)
#define ORC_ASIN(x) fr_asin(x)
#define ORC_FABS(x) fr_fabs(x)
#define ORC_ISNAN(x) std::isnan((x).v)
#define ORC_ISINF(x) std::isinf((x).v)
#define ORC_VAL(x) ((x).v)
#include "trk_oracle_core.h"

static const double BETA_P = 13700.0;

struct Res {
  const char *name;
  Count c;
};

static Count count_mult(int order, double KnL, int nSlices) {
  orc_mult m;
  std::memset((void *)&m, 0, sizeof(m));
  m.order[0] = order;
  m.KnL[0] = KnL;
  m.drift = order == 1 ? 0.3 : 0.2;
  m.nSlices = nSlices;
  m.integ_order = 4;
  m.maxOrder = order;
  FR c[7] = {1e-4, 1e-5, -2e-4, 2e-5, 0.1, 1e-3, 1};
  FR dz;
  g = Count();
  orc_integrate_kick_multipole(c, &m, BETA_P, nullptr, &dz);
  return g;
}

static Count count_bend(int nSlices, double K1, double rho0) {
  static orc_bend b;
  std::memset((void *)&b, 0, sizeof(b));
  b.rho0 = rho0;
  b.rho_actual = rho0;
  b.length = 1.0;
  b.nSlices = nSlices;
  b.integ_order = 4;
  b.isr_or_rad = 1;
  if (K1) {
    /* K1-only table: Fy = 1 + K1 rho0 x + ..., evaluated over i+j < 5 */
    b.hasNormal = 1;
    b.expansionOrder1 = 5;
    b.Fy_xy[0][0] = 1;
    b.Fy_xy[1][0] = K1 * rho0;
    b.Fx_xy[0][1] = K1 * rho0;
  }
  FR Qi[6] = {1e-4, 1e-5, -2e-4, 2e-5, 0, 1e-3}, Qf[6];
  FR dz;
  g = Count();
  /* entry: edge kick with E1=0 (reference still multiplies), canonical in/out */
  orc_to_dipole_canonical(Qi);
  orc_integrate_csbend(Qf, Qi, &b, nullptr, &dz);
  orc_from_dipole_canonical(Qf);
  return g;
}

int main(int argc, char **argv) {
  const char *out = argc > 1 ? argv[1] : "flops.json";
  Count quad = count_mult(1, 1.2 * 0.3, 2);       /* KQUAD N_KICKS=8 -> 2 slices */
  Count sext = count_mult(2, 40 * 0.2, 1);        /* KSEXT N_KICKS=4 -> 1 slice */
  Count oct = count_mult(3, 500 * 0.2, 1);        /* KOCT default 1 slice */
  Count bend16 = count_bend(16, 0.0, 1.0 / (2 * M_PI / 80));
  Count bend32k1 = count_bend(32, -0.4, 1.0 / (2 * M_PI / 280));
  Count mba_quad = count_mult(1, 3.0 * 0.3, 2);
  /* DRIF order 2 without structural zeros: x += L x', y += L y',
   * s = (L + s) + (L/2 y') y' + (L/2 x') x' */
  Count drift;
  drift.add = 5;
  drift.mul = 6;
  /* RFCA L=0: P, gamma, beta, t, phi, sin, add_to_particle_energy */
  Count rf;
  rf.add = 8;
  rf.mul = 9;
  rf.div = 5;
  rf.sqrt = 4;
  rf.trans = 1;
  /* WAKE per particle: time (2 stats + bin + kick), bin index, energy kick */
  Count wake;
  wake.add = 12;
  wake.mul = 14;
  wake.div = 8;
  wake.sqrt = 6;
  auto tot = [](const Count &c, long n) { return (double)c.total() * n; };
  double f_c1 = tot(quad, 80) + tot(bend16, 80) + tot(drift, 160);
  double f_c2 = f_c1 + tot(sext, 80) + tot(rf, 1) + tot(wake, 1);
  double f_c5 = 40 * (tot(bend32k1, 7) + tot(mba_quad, 12) + tot(sext, 6) + tot(oct, 2) + tot(drift, 27)) +
                tot(rf, 1) + 2 * tot(wake, 1);
  long tr_c2 = bend16.trans * 80 + rf.trans;
  FILE *f = std::fopen(out, "w");
  if (!f)
    return 1;
  auto put = [&](const char *n, const Count &c, bool comma) {
    std::fprintf(f, "    \"%s\": {\"add\": %ld, \"mul\": %ld, \"div\": %ld, \"sqrt\": %ld, \"transcendental\": %ld, "
                 "\"total\": %ld}%s\n", n, c.add, c.mul, c.div, c.sqrt, c.trans, c.total(), comma ? "," : "");
  };
  std::fprintf(f, "{\n  \"convention\": \"add/sub/mul/div/sqrt of particle-dependent values = 1 flop each, sin/cos/asin = 1 "
                  "each (also listed); reference formulation (no FMA); per-element constants not counted\",\n");
  std::fprintf(f, "  \"generated_by\": \"oracle/flopcount.cpp (make -C oracle flops)\",\n");
  std::fprintf(f, "  \"per_particle\": {\n");
  put("KQUAD_N_KICKS8", quad, true);
  put("KSEXT_N_KICKS4", sext, true);
  put("KOCT_default", oct, true);
  put("CSBEND_16_slices_dipole", bend16, true);
  put("CSBEND_32_slices_K1", bend32k1, true);
  put("DRIF_order2", drift, true);
  put("RFCA_L0", rf, true);
  put("WAKE", wake, false);
  std::fprintf(f, "  },\n  \"flops_per_particle_turn\": {\"c1\": %.0f, \"c2\": %.0f, \"c5\": %.0f},\n", f_c1, f_c2, f_c5);
  std::fprintf(f, "  \"transcendentals_per_particle_turn\": {\"c2\": %ld}\n}\n", tr_c2);
  std::fclose(f);
  std::printf("C1 %.0f  C2 %.0f  C5 %.0f flops/particle-turn\n", f_c1, f_c2, f_c5);
  return 0;
}
