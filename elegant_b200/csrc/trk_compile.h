/*
 * trk_compile.h -- lattice compiler (host side of libtrkgpu.so).
 */
#ifndef TRK_COMPILE_H
#define TRK_COMPILE_H

#include <vector>

#include "trk.h"
#include "trk_ops.h"

struct CompiledWake {
  int op = -1;
  int transverse = 0;
  double dt = 0, span = 0;
  long i0 = 0, points = 0, n_bins = 0, max_bins = 0;
  int allow_long_beam = 0;
  const double *t = nullptr, *W = nullptr, *Wy = nullptr;
  double factor = 1, xfactor = 1, yfactor = 1, charge = 0;
  int interpolate = 0;
  long ramp_passes = 0;
  int x_power = 1, y_power = 1, x_probe = 0, y_probe = 0;
  double tdx = 0, tdy = 0, tilt = 0;
  int change_p0 = 0; /* WAKE CHANGE_P0: match the central momentum to the beam's after the kick */
};

struct CompiledLattice {
  std::vector<trk_op> ops;
  std::vector<trk_aperture> aps;
  std::vector<double> field;
  std::vector<CompiledWake> wakes;
  std::vector<int> rf_first_op; /* op index of the first RFCA of each fiducial slot */
  int n_rf_slots = 0;
  int n_mult = 0;
  double total_length = 0;
  bool lean = true; /* every op has a kind the lean kernel variant handles */
  bool has_cfbend = false; /* some op is a combined-function CSBEND (OPK_CFBEND) */
};

/* Launch shape of the tracking kernel when the caller names none, measured on
 * B200: fast build (128 threads, 6 blocks/SM; 80 registers) for lean
 * lattices, (128, 5; 102 registers) for lean lattices with combined-function
 * bends, whose body spills at 80 registers; parity build (128, 6) for lean
 * lattices without combined-function bends (the FODO ring with RF and wake:
 * 94.6 ms per turn of 1e6 particles against 104.6 ms at (128, 4) and
 * 95.6 ms at (256, 3)); (128, 4) otherwise. */
/* lean kernel flavour of a compiled lattice: 0 general, 1 lean, 2 lean with
 * combined-function bends */
inline int trk_lean_flavor(const CompiledLattice &c) { return c.lean ? (c.has_cfbend ? 2 : 1) : 0; }

inline int trk_default_variant(bool fast, const CompiledLattice &c) {
  if (c.lean && (fast || !c.has_cfbend))
    return fast && c.has_cfbend ? 4 : 7;
  return 1;
}

int trk_compile(const trk_lattice *l, double Po, CompiledLattice &out);
void trk_expansion_coefficients(double *coef10);
double ipow_h(double x, long p);
extern "C" int trk_csbend_field_table(const double *b, const double *c, double h, int nonlinear, long expansionOrder,
                                      double *Fx, double *Fy, int *eo1, int *hasNormal, int *hasSkew);

#endif
