/*
 * trk_params.h -- element parameter tables.
 *
 * Each list names the parameters an element of that type accepts, with the
 * reference's parameter name and default value (src/track_data.c):
 *   DRIF   drift_param   :452      EDRIFT edrift_param :3194
 *   KQUAD  kquad_param   :1227     KSEXT  ksext_param  :1125
 *   KOCT   koct_param    :1169     CSBEND csbend_param :1898
 *   RFCA   rfca_param    :579      WAKE   wake_param   :2415
 *   TRWAKE trwake_param  :2477     MAXAMP maxamp_param :994
 *   CHARGE charge_param  :2507
 * Only parameters that change tracking on this path are listed; string
 * parameters (file names, FIDUCIAL, OPEN_SIDE) are not, and their defaults are
 * the only behaviour implemented.  The order inside each list is this
 * library's storage order, not the reference's.
 *
 * X(ENUM, "NAME", default)
 */
#ifndef TRK_PARAMS_H
#define TRK_PARAMS_H

#define TRK_PARAMS_DRIF(X) \
  X(DRIF_L, "L", 0.0)      \
  X(DRIF_ORDER, "ORDER", 0.0)

#define TRK_PARAMS_EDRIFT(X) X(EDRIFT_L, "L", 0.0)

#define TRK_PARAMS_KQUAD(X)                        \
  X(KQUAD_L, "L", 0.0)                             \
  X(KQUAD_K1, "K1", 0.0)                           \
  X(KQUAD_TILT, "TILT", 0.0)                       \
  X(KQUAD_PITCH, "PITCH", 0.0)                     \
  X(KQUAD_YAW, "YAW", 0.0)                         \
  X(KQUAD_BORE, "BORE", 0.0)                       \
  X(KQUAD_B, "B", 0.0)                             \
  X(KQUAD_DX, "DX", 0.0)                           \
  X(KQUAD_DY, "DY", 0.0)                           \
  X(KQUAD_DZ, "DZ", 0.0)                           \
  X(KQUAD_FSE, "FSE", 0.0)                         \
  X(KQUAD_N_KICKS, "N_KICKS", 0.0)                 \
  X(KQUAD_N_SLICES, "N_SLICES", 1.0)               \
  X(KQUAD_HKICK, "HKICK", 0.0)                     \
  X(KQUAD_VKICK, "VKICK", 0.0)                     \
  X(KQUAD_HCALIBRATION, "HCALIBRATION", 1.0)       \
  X(KQUAD_VCALIBRATION, "VCALIBRATION", 1.0)       \
  X(KQUAD_SYNCH_RAD, "SYNCH_RAD", 0.0)             \
  X(KQUAD_INTEGRATION_ORDER, "INTEGRATION_ORDER", 4.0) \
  X(KQUAD_ISR, "ISR", 0.0)                         \
  X(KQUAD_ISR1PART, "ISR1PART", 1.0)               \
  X(KQUAD_EDGE1_EFFECTS, "EDGE1_EFFECTS", 0.0)     \
  X(KQUAD_EDGE2_EFFECTS, "EDGE2_EFFECTS", 0.0)     \
  X(KQUAD_LEFFECTIVE, "LEFFECTIVE", 0.0)           \
  X(KQUAD_RADIAL, "RADIAL", 0.0)                   \
  X(KQUAD_EXPAND_HAMILTONIAN, "EXPAND_HAMILTONIAN", 0.0) \
  X(KQUAD_MALIGN_METHOD, "MALIGN_METHOD", 0.0)     \
  X(KQUAD_I0P, "I0P", 0.0)                         \
  X(KQUAD_I1P, "I1P", 0.0)                         \
  X(KQUAD_I2P, "I2P", 0.0)                         \
  X(KQUAD_I3P, "I3P", 0.0)                         \
  X(KQUAD_LAMBDA2P, "LAMBDA2P", 0.0)               \
  X(KQUAD_I0M, "I0M", 0.0)                         \
  X(KQUAD_I1M, "I1M", 0.0)                         \
  X(KQUAD_I2M, "I2M", 0.0)                         \
  X(KQUAD_I3M, "I3M", 0.0)                         \
  X(KQUAD_LAMBDA2M, "LAMBDA2M", 0.0)               \
  X(KQUAD_EDGE1_LINEAR, "EDGE1_LINEAR", 1.0)       \
  X(KQUAD_EDGE2_LINEAR, "EDGE2_LINEAR", 1.0)       \
  X(KQUAD_EDGE1_NONLINEAR_FACTOR, "EDGE1_NONLINEAR_FACTOR", 1.0) \
  X(KQUAD_EDGE2_NONLINEAR_FACTOR, "EDGE2_NONLINEAR_FACTOR", 1.0) \
  X(KQUAD_HSTEERING, "HSTEERING", 0.0) \
  X(KQUAD_VSTEERING, "VSTEERING", 0.0) \
  X(KQUAD_SYSTEMATIC_MULTIPOLE_FACTOR, "SYSTEMATIC_MULTIPOLE_FACTOR", 1.0) \
  X(KQUAD_RANDOM_MULTIPOLE_FACTOR, "RANDOM_MULTIPOLE_FACTOR", 1.0) \
  X(KQUAD_STEERING_MULTIPOLE_FACTOR, "STEERING_MULTIPOLE_FACTOR", 1.0) \
  X(KQUAD_MIN_NORMAL_ORDER, "MIN_NORMAL_ORDER", -1.0) \
  X(KQUAD_MIN_SKEW_ORDER, "MIN_SKEW_ORDER", -1.0) \
  X(KQUAD_MAX_NORMAL_ORDER, "MAX_NORMAL_ORDER", -1.0) \
  X(KQUAD_MAX_SKEW_ORDER, "MAX_SKEW_ORDER", -1.0) \
  X(KQUAD_SQRT_ORDER, "SQRT_ORDER", 0.0) \
  X(KQUAD_SR_IN_ORDINARY_MATRIX, "SR_IN_ORDINARY_MATRIX", 0.0) \
  X(KQUAD_TRACKING_MATRIX, "TRACKING_MATRIX", 0.0)

#define TRK_PARAMS_KSEXT(X)                        \
  X(KSEXT_L, "L", 0.0)                             \
  X(KSEXT_K2, "K2", 0.0)                           \
  X(KSEXT_K1, "K1", 0.0)                           \
  X(KSEXT_J1, "J1", 0.0)                           \
  X(KSEXT_TILT, "TILT", 0.0)                       \
  X(KSEXT_PITCH, "PITCH", 0.0)                     \
  X(KSEXT_YAW, "YAW", 0.0)                         \
  X(KSEXT_BORE, "BORE", 0.0)                       \
  X(KSEXT_B, "B", 0.0)                             \
  X(KSEXT_N_KICKS, "N_KICKS", 0.0)                 \
  X(KSEXT_N_SLICES, "N_SLICES", 1.0)               \
  X(KSEXT_DX, "DX", 0.0)                           \
  X(KSEXT_DY, "DY", 0.0)                           \
  X(KSEXT_DZ, "DZ", 0.0)                           \
  X(KSEXT_FSE, "FSE", 0.0)                         \
  X(KSEXT_HKICK, "HKICK", 0.0)                     \
  X(KSEXT_VKICK, "VKICK", 0.0)                     \
  X(KSEXT_HCALIBRATION, "HCALIBRATION", 1.0)       \
  X(KSEXT_VCALIBRATION, "VCALIBRATION", 1.0)       \
  X(KSEXT_SYNCH_RAD, "SYNCH_RAD", 0.0)             \
  X(KSEXT_INTEGRATION_ORDER, "INTEGRATION_ORDER", 4.0) \
  X(KSEXT_ISR, "ISR", 0.0)                         \
  X(KSEXT_ISR1PART, "ISR1PART", 1.0)               \
  X(KSEXT_EXPAND_HAMILTONIAN, "EXPAND_HAMILTONIAN", 0.0) \
  X(KSEXT_MALIGN_METHOD, "MALIGN_METHOD", 0.0) \
  X(KSEXT_HSTEERING, "HSTEERING", 0.0) \
  X(KSEXT_VSTEERING, "VSTEERING", 0.0) \
  X(KSEXT_SYSTEMATIC_MULTIPOLE_FACTOR, "SYSTEMATIC_MULTIPOLE_FACTOR", 1.0) \
  X(KSEXT_RANDOM_MULTIPOLE_FACTOR, "RANDOM_MULTIPOLE_FACTOR", 1.0) \
  X(KSEXT_STEERING_MULTIPOLE_FACTOR, "STEERING_MULTIPOLE_FACTOR", 1.0) \
  X(KSEXT_MIN_NORMAL_ORDER, "MIN_NORMAL_ORDER", -1.0) \
  X(KSEXT_MIN_SKEW_ORDER, "MIN_SKEW_ORDER", -1.0) \
  X(KSEXT_MAX_NORMAL_ORDER, "MAX_NORMAL_ORDER", -1.0) \
  X(KSEXT_MAX_SKEW_ORDER, "MAX_SKEW_ORDER", -1.0) \
  X(KSEXT_SQRT_ORDER, "SQRT_ORDER", 0.0)

#define TRK_PARAMS_KOCT(X)                         \
  X(KOCT_L, "L", 0.0)                              \
  X(KOCT_K3, "K3", 0.0)                            \
  X(KOCT_TILT, "TILT", 0.0)                        \
  X(KOCT_PITCH, "PITCH", 0.0)                      \
  X(KOCT_YAW, "YAW", 0.0)                          \
  X(KOCT_BORE, "BORE", 0.0)                        \
  X(KOCT_B, "B", 0.0)                              \
  X(KOCT_DX, "DX", 0.0)                            \
  X(KOCT_DY, "DY", 0.0)                            \
  X(KOCT_DZ, "DZ", 0.0)                            \
  X(KOCT_FSE, "FSE", 0.0)                          \
  X(KOCT_N_KICKS, "N_KICKS", 4.0)                  \
  X(KOCT_N_SLICES, "N_SLICES", 4.0)                \
  X(KOCT_INTEGRATION_ORDER, "INTEGRATION_ORDER", 4.0) \
  X(KOCT_SYNCH_RAD, "SYNCH_RAD", 0.0)              \
  X(KOCT_ISR, "ISR", 0.0)                          \
  X(KOCT_ISR1PART, "ISR1PART", 1.0)                \
  X(KOCT_EXPAND_HAMILTONIAN, "EXPAND_HAMILTONIAN", 0.0) \
  X(KOCT_MALIGN_METHOD, "MALIGN_METHOD", 0.0) \
  X(KOCT_SQRT_ORDER, "SQRT_ORDER", 0.0)

#define TRK_PARAMS_CSBEND(X)                       \
  X(CSBEND_L, "L", 0.0)                            \
  X(CSBEND_ANGLE, "ANGLE", 0.0)                    \
  X(CSBEND_K1, "K1", 0.0)                          \
  X(CSBEND_K2, "K2", 0.0)                          \
  X(CSBEND_K3, "K3", 0.0)                          \
  X(CSBEND_K4, "K4", 0.0)                          \
  X(CSBEND_K5, "K5", 0.0)                          \
  X(CSBEND_K6, "K6", 0.0)                          \
  X(CSBEND_K7, "K7", 0.0)                          \
  X(CSBEND_K8, "K8", 0.0)                          \
  X(CSBEND_E1, "E1", 0.0)                          \
  X(CSBEND_E2, "E2", 0.0)                          \
  X(CSBEND_TILT, "TILT", 0.0)                      \
  X(CSBEND_H1, "H1", 0.0)                          \
  X(CSBEND_H2, "H2", 0.0)                          \
  X(CSBEND_HGAP, "HGAP", 0.0)                      \
  X(CSBEND_FINT, "FINT", 0.5)                      \
  X(CSBEND_FINT1, "FINT1", -1.0)                   \
  X(CSBEND_FINT2, "FINT2", -1.0)                   \
  X(CSBEND_DX, "DX", 0.0)                          \
  X(CSBEND_DY, "DY", 0.0)                          \
  X(CSBEND_DZ, "DZ", 0.0)                          \
  X(CSBEND_XKICK, "XKICK", 0.0)                    \
  X(CSBEND_YKICK, "YKICK", 0.0)                    \
  X(CSBEND_FSE, "FSE", 0.0)                        \
  X(CSBEND_FSE_DIPOLE, "FSE_DIPOLE", 0.0)          \
  X(CSBEND_FSE_QUADRUPOLE, "FSE_QUADRUPOLE", 0.0)  \
  X(CSBEND_ETILT, "ETILT", 0.0)                    \
  X(CSBEND_N_SLICES, "N_SLICES", 4.0)              \
  X(CSBEND_ETILT_SIGN, "ETILT_SIGN", 1.0)          \
  X(CSBEND_NONLINEAR, "NONLINEAR", 1.0)            \
  X(CSBEND_SYNCH_RAD, "SYNCH_RAD", 0.0)            \
  X(CSBEND_EDGE1_EFFECTS, "EDGE1_EFFECTS", 1.0)    \
  X(CSBEND_EDGE2_EFFECTS, "EDGE2_EFFECTS", 1.0)    \
  X(CSBEND_EDGE_ORDER, "EDGE_ORDER", 1.0)          \
  X(CSBEND_INTEGRATION_ORDER, "INTEGRATION_ORDER", 4.0) \
  X(CSBEND_EXPAND_HAMILTONIAN, "EXPAND_HAMILTONIAN", 0.0) \
  X(CSBEND_EDGE1_KICK_LIMIT, "EDGE1_KICK_LIMIT", -1.0) \
  X(CSBEND_EDGE2_KICK_LIMIT, "EDGE2_KICK_LIMIT", -1.0) \
  X(CSBEND_KICK_LIMIT_SCALING, "KICK_LIMIT_SCALING", 0.0) \
  X(CSBEND_USE_BN, "USE_BN", 0.0)                  \
  X(CSBEND_EXPANSION_ORDER, "EXPANSION_ORDER", 0.0) \
  X(CSBEND_B1, "B1", 0.0)                          \
  X(CSBEND_B2, "B2", 0.0)                          \
  X(CSBEND_B3, "B3", 0.0)                          \
  X(CSBEND_B4, "B4", 0.0)                          \
  X(CSBEND_B5, "B5", 0.0)                          \
  X(CSBEND_B6, "B6", 0.0)                          \
  X(CSBEND_B7, "B7", 0.0)                          \
  X(CSBEND_B8, "B8", 0.0)                          \
  X(CSBEND_ISR, "ISR", 0.0)                        \
  X(CSBEND_ISR1PART, "ISR1PART", 1.0)              \
  X(CSBEND_REFERENCE_CORRECTION, "REFERENCE_CORRECTION", 0.0) \
  X(CSBEND_FSE_CORRECTION, "FSE_CORRECTION", 0.0)  \
  X(CSBEND_MALIGN_METHOD, "MALIGN_METHOD", 0.0) \
  X(CSBEND_FRINGE1K0, "FRINGE1K0", 0.0) \
  X(CSBEND_FRINGE1K1, "FRINGE1K1", 0.0) \
  X(CSBEND_FRINGE1K2, "FRINGE1K2", 0.0) \
  X(CSBEND_FRINGE1K3, "FRINGE1K3", 0.0) \
  X(CSBEND_FRINGE1K4, "FRINGE1K4", 0.0) \
  X(CSBEND_FRINGE1K5, "FRINGE1K5", 0.0) \
  X(CSBEND_FRINGE1K6, "FRINGE1K6", 0.0) \
  X(CSBEND_FRINGE2K0, "FRINGE2K0", 0.0) \
  X(CSBEND_FRINGE2K1, "FRINGE2K1", 0.0) \
  X(CSBEND_FRINGE2K2, "FRINGE2K2", 0.0) \
  X(CSBEND_FRINGE2K3, "FRINGE2K3", 0.0) \
  X(CSBEND_FRINGE2K4, "FRINGE2K4", 0.0) \
  X(CSBEND_FRINGE2K5, "FRINGE2K5", 0.0) \
  X(CSBEND_FRINGE2K6, "FRINGE2K6", 0.0) \
  X(CSBEND_EPITCH, "EPITCH", 0.0) \
  X(CSBEND_EYAW, "EYAW", 0.0) \
  X(CSBEND_SR_IN_ORDINARY_MATRIX, "SR_IN_ORDINARY_MATRIX", 0.0) \
  X(CSBEND_XREFERENCE, "XREFERENCE", 0.0) \
  X(CSBEND_F1, "F1", 0.0) \
  X(CSBEND_F2, "F2", 0.0) \
  X(CSBEND_F3, "F3", 0.0) \
  X(CSBEND_F4, "F4", 0.0) \
  X(CSBEND_F5, "F5", 0.0) \
  X(CSBEND_F6, "F6", 0.0) \
  X(CSBEND_F7, "F7", 0.0) \
  X(CSBEND_F8, "F8", 0.0) \
  X(CSBEND_G1, "G1", 0.0) \
  X(CSBEND_G2, "G2", 0.0) \
  X(CSBEND_G3, "G3", 0.0) \
  X(CSBEND_G4, "G4", 0.0) \
  X(CSBEND_G5, "G5", 0.0) \
  X(CSBEND_G6, "G6", 0.0) \
  X(CSBEND_G7, "G7", 0.0) \
  X(CSBEND_G8, "G8", 0.0) \
  X(CSBEND_SQRT_ORDER, "SQRT_ORDER", 0.0) \
  X(CSBEND_USE_RAD_DIST, "USE_RAD_DIST", 0.0) \
  X(CSBEND_ADD_OPENING_ANGLE, "ADD_OPENING_ANGLE", 1.0) \
  X(CSBEND_PHOTON_LOW_ENERGY_CUTOFF, "PHOTON_LOW_ENERGY_CUTOFF", 0.0) \
  X(CSBEND_TRACKING_MATRIX, "TRACKING_MATRIX", 0.0) \
  X(CSBEND_XSTEERING, "XSTEERING", 0.0) \
  X(CSBEND_YSTEERING, "YSTEERING", 0.0)

#define TRK_PARAMS_RFCA(X)                         \
  X(RFCA_L, "L", 0.0)                              \
  X(RFCA_VOLT, "VOLT", 0.0)                        \
  X(RFCA_PHASE, "PHASE", 0.0)                      \
  X(RFCA_FREQ, "FREQ", 500.0e6)                    \
  X(RFCA_Q, "Q", 0.0)                              \
  X(RFCA_PHASE_REFERENCE, "PHASE_REFERENCE", 0.0)  \
  X(RFCA_CHANGE_P0, "CHANGE_P0", 0.0)              \
  X(RFCA_CHANGE_T, "CHANGE_T", 0.0)                \
  X(RFCA_END1_FOCUS, "END1_FOCUS", 0.0)            \
  X(RFCA_END2_FOCUS, "END2_FOCUS", 0.0)            \
  X(RFCA_STANDING_WAVE, "STANDING_WAVE", 0.0)      \
  X(RFCA_N_KICKS, "N_KICKS", 0.0)                  \
  X(RFCA_DX, "DX", 0.0)                            \
  X(RFCA_DY, "DY", 0.0)                            \
  X(RFCA_T_REFERENCE, "T_REFERENCE", -1.0)         \
  X(RFCA_LINEARIZE, "LINEARIZE", 0.0)              \
  X(RFCA_LOCK_PHASE, "LOCK_PHASE", 0.0)

#define TRK_PARAMS_WAKE(X)                         \
  X(WAKE_CHARGE, "CHARGE", 0.0)                    \
  X(WAKE_FACTOR, "FACTOR", 1.0)                    \
  X(WAKE_N_BINS, "N_BINS", 0.0)                    \
  X(WAKE_INTERPOLATE, "INTERPOLATE", 0.0)          \
  X(WAKE_SMOOTHING, "SMOOTHING", 0.0)              \
  X(WAKE_CHANGE_P0, "CHANGE_P0", 0.0)              \
  X(WAKE_ALLOW_LONG_BEAM, "ALLOW_LONG_BEAM", 0.0)  \
  X(WAKE_RAMP_PASSES, "RAMP_PASSES", 0.0)          \
  X(WAKE_BUNCHED_BEAM_MODE, "BUNCHED_BEAM_MODE", 1.0) \
  X(WAKE_ACAUSAL_ALLOWED, "ACAUSAL_ALLOWED", 0.0) \
  X(WAKE_SG_HALFWIDTH, "SG_HALFWIDTH", 4.0) \
  X(WAKE_SG_ORDER, "SG_ORDER", 1.0) \
  X(WAKE_START_BUNCH, "START_BUNCH", -1.0) \
  X(WAKE_END_BUNCH, "END_BUNCH", -1.0)

#define TRK_PARAMS_TRWAKE(X)                       \
  X(TRWAKE_CHARGE, "CHARGE", 0.0)                  \
  X(TRWAKE_FACTOR, "FACTOR", 1.0)                  \
  X(TRWAKE_XFACTOR, "XFACTOR", 1.0)                \
  X(TRWAKE_YFACTOR, "YFACTOR", 1.0)                \
  X(TRWAKE_N_BINS, "N_BINS", 0.0)                  \
  X(TRWAKE_INTERPOLATE, "INTERPOLATE", 0.0)        \
  X(TRWAKE_SMOOTHING, "SMOOTHING", 0.0)            \
  X(TRWAKE_DX, "DX", 0.0)                          \
  X(TRWAKE_DY, "DY", 0.0)                          \
  X(TRWAKE_TILT, "TILT", 0.0)                      \
  X(TRWAKE_X_DRIVE_EXPONENT, "X_DRIVE_EXPONENT", 1.0) \
  X(TRWAKE_Y_DRIVE_EXPONENT, "Y_DRIVE_EXPONENT", 1.0) \
  X(TRWAKE_X_PROBE_EXPONENT, "X_PROBE_EXPONENT", 0.0) \
  X(TRWAKE_Y_PROBE_EXPONENT, "Y_PROBE_EXPONENT", 0.0) \
  X(TRWAKE_RAMP_PASSES, "RAMP_PASSES", 0.0)        \
  X(TRWAKE_BUNCHED_BEAM_MODE, "BUNCHED_BEAM_MODE", 1.0) \
  X(TRWAKE_ACAUSAL_ALLOWED, "ACAUSAL_ALLOWED", 0.0) \
  X(TRWAKE_SG_HALFWIDTH, "SG_HALFWIDTH", 4.0) \
  X(TRWAKE_SG_ORDER, "SG_ORDER", 1.0) \
  X(TRWAKE_START_BUNCH, "START_BUNCH", -1.0) \
  X(TRWAKE_END_BUNCH, "END_BUNCH", -1.0)

#define TRK_PARAMS_MAXAMP(X)                       \
  X(MAXAMP_X_MAX, "X_MAX", 0.0)                    \
  X(MAXAMP_Y_MAX, "Y_MAX", 0.0)                    \
  X(MAXAMP_ELLIPTICAL, "ELLIPTICAL", 0.0)          \
  X(MAXAMP_EXPONENT, "EXPONENT", 2.0)              \
  X(MAXAMP_YEXPONENT, "YEXPONENT", 0.0)

#define TRK_PARAMS_CHARGE(X)                       \
  X(CHARGE_TOTAL, "TOTAL", 0.0)                    \
  X(CHARGE_PER_PARTICLE, "PER_PARTICLE", 0.0)

#define TRK_PARAMS_MARK(X)                         \
  X(MARK_DX, "DX", 0.0)                            \
  X(MARK_DY, "DY", 0.0)                            \
  X(MARK_FITPOINT, "FITPOINT", 0.0)

#define TRK_ENUM_ENTRY(e, n, d) P_##e,
enum {
  TRK_PARAMS_MARK(TRK_ENUM_ENTRY) P_MARK_COUNT_
};
enum {
  TRK_PARAMS_DRIF(TRK_ENUM_ENTRY) P_DRIF_COUNT_
};
enum {
  TRK_PARAMS_EDRIFT(TRK_ENUM_ENTRY) P_EDRIFT_COUNT_
};
enum {
  TRK_PARAMS_KQUAD(TRK_ENUM_ENTRY) P_KQUAD_COUNT_
};
enum {
  TRK_PARAMS_KSEXT(TRK_ENUM_ENTRY) P_KSEXT_COUNT_
};
enum {
  TRK_PARAMS_KOCT(TRK_ENUM_ENTRY) P_KOCT_COUNT_
};
enum {
  TRK_PARAMS_CSBEND(TRK_ENUM_ENTRY) P_CSBEND_COUNT_
};
enum {
  TRK_PARAMS_RFCA(TRK_ENUM_ENTRY) P_RFCA_COUNT_
};
enum {
  TRK_PARAMS_WAKE(TRK_ENUM_ENTRY) P_WAKE_COUNT_
};
enum {
  TRK_PARAMS_TRWAKE(TRK_ENUM_ENTRY) P_TRWAKE_COUNT_
};
enum {
  TRK_PARAMS_MAXAMP(TRK_ENUM_ENTRY) P_MAXAMP_COUNT_
};
enum {
  TRK_PARAMS_CHARGE(TRK_ENUM_ENTRY) P_CHARGE_COUNT_
};
#undef TRK_ENUM_ENTRY

#define TRK_MAX_PARAMS 128

#endif
