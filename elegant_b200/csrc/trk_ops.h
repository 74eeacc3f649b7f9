/*
 * trk_ops.h -- the compiled lattice as the kernels read it.
 *
 * The host turns each lattice element into one trk_op record whose constants
 * are everything the reference computes once per element call (strengths
 * divided by slices, substep lengths, edge tangents, misalignment cos/sin,
 * ...), evaluated on the host with the reference's expressions so the device
 * only runs the per-particle arithmetic.  Records are 1 KB-aligned-free POD,
 * read with uniform (warp-broadcast) loads.
 */
#ifndef TRK_OPS_H
#define TRK_OPS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum trk_op_kind {
  OPK_NOP = 0,    /* MARK, CHARGE, MAXAMP (state is baked into aperture indices) */
  OPK_DRIFT = 1,  /* DRIF, order-1/2 transport matrix */
  OPK_EDRIFT = 2, /* EDRIFT, and CSBEND with ANGLE=0 */
  OPK_MULT = 3,   /* KQUAD, KSEXT, KOCT */
  OPK_BEND = 4,   /* CSBEND */
  OPK_RF = 5,     /* RFCA */
  OPK_WAKE = 6,   /* WAKE (collective: ends a fused segment) */
  OPK_TRWAKE = 7, /* TRWAKE (collective) */
  OPK_RFDRIFT = 8, /* RFCA with VOLT=0: drift of length L */
  OPK_MULT1 = 9,   /* KQUAD/KSEXT/KOCT with one normal multipole, 4th-order integrator, no
                      misalignment, steering or end drifts (specialized fast-build body) */
  OPK_DIPOLE = 10, /* CSBEND: pure dipole, 4th-order integrator, no misalignment, edge kicks
                      that are exact no-ops (E=0, no fringe) or absent (specialized fast-build body) */
  OPK_CFBEND = 11  /* CSBEND: combined function (normal field expansion of order 4: K1 and/or K2),
                      otherwise as OPK_DIPOLE (specialized fast-build body) */
};

/* multipole flags (i[6]) */
#define MF_OFFSET 1   /* DX/DY/DZ nonzero */
#define MF_TILT 2     /* TILT nonzero */
#define MF_ENDDRIFT 4 /* LEFFECTIVE end drifts */
#define MF_XKICK 8
#define MF_YKICK 16
#define MF_KNL0 32
#define MF_KNL1 64
#define MF_KNL2 128
#define MF_APTILT 256 /* aperture check rotates by -TILT */
#define MF_RAD 512    /* radiation block after each kick (SYNCH_RAD and/or ISR) */
#define MF_ISR 1024   /* incoherent synchrotron radiation (ISR) */
#define MF_ISR1OFF 2048 /* ISR1PART=0: no ISR when a single particle is tracked */
#define MF_FRINGE1 4096 /* KQUAD entrance fringe (EDGE1_EFFECTS > 0) */
#define MF_FRINGE2 8192 /* KQUAD exit fringe (EDGE2_EFFECTS > 0) */

/* bend flags (i[7]) */
#define BF_ISR_ROUNDTRIP 1 /* reference's (1+DPoP) divide/multiply round trip */
#define BF_MISALIGN 2      /* entry/exit offsets or tilt not all zero */
#define BF_APTILT 4
#define BF_RAD 8       /* radiation block after each kick (SYNCH_RAD and/or ISR) */
#define BF_ISR 16      /* incoherent synchrotron radiation (ISR) */
#define BF_ISR1OFF 32  /* ISR1PART=0: no ISR when a single particle is tracked */
#define BF_EXPAND 64   /* EXPAND_HAMILTONIAN: leading-order drift, (1+delta) coordinate factors */
#define BF_RADE1 128   /* SYNCH_RAD with an entrance edge angle: delta pre-adjusted at the entrance */
#define BF_RADE2 256   /* ... and post-adjusted at the exit */

/* RF flags (i[3]) */
#define RF_SAME_DGAMMA 1
#define RF_END1 2
#define RF_END2 4
#define RF_OFFSET 8
#define RF_LOCK 16   /* LOCK_PHASE: phase PHASE only, kick at t - <t> of the pass */
#define RF_LINEAR 32 /* LINEARIZE: kick linear in t - <t> about the mean */
#define RF_CHANGE_P0 64 /* CHANGE_P0: the central momentum follows the beam's after the cavity */

typedef struct {
  int32_t kind;
  int32_t elem;        /* lattice element index (loss bookkeeping) */
  int32_t ap_post[2];  /* after-element aperture record for pass 0 / later passes (-1 none) */
  int32_t ap_in[2];    /* in-element (per slice) aperture record, pass 0 / later (-1 none) */
  int32_t extrapolate; /* limit_amplitudes extrapolate_z (DRIF) */
  int32_t no_aperture; /* NO_APERTURE element class (MARK, CHARGE) */
  int32_t i[8];
  double z_start, z_end;
  double d[128];
} trk_op;

/* after-element / in-element aperture from the sticky MAXAMP state */
typedef struct {
  double x_max, y_max;
  int32_t elliptical;
  int32_t xexp, yexp;
  int32_t valid;       /* elimit exponents valid */
  double a2, b2;       /* ipow(x_max, xexp), ipow(y_max, yexp) for elimit */
} trk_aperture;

/* Index layout of trk_op.d / .i per kind (documented with the producer in
 * trk_host.cu). */
/* MULT */
#define MD_DX 0
#define MD_DY 1
#define MD_DZ 2
#define MD_TC 3   /* cos/sin of TILT (entry rotation) */
#define MD_TS 4
#define MD_XC 5   /* cos/sin of -TILT (exit rotation) */
#define MD_XS 6
#define MD_LEND 7
#define MD_APC 8  /* aperture reverse tilt cos/sin */
#define MD_APS 9
#define MD_DSH 10 /* 8 drift substep lengths */
#define MD_KQ 18  /* [step*3 + order] kick strengths, 24 values */
#define MD_KX 42  /* 8 values -xkick*kickFrac */
#define MD_KY 50  /* 8 values -ykick*kickFrac */
#define MD_DRIFT 58 /* drift per slice (nonzero test) */
#define MD_COEF 59  /* expansion coefficients for orders 0..3 packed: order n at MD_COEF + n*(n+1)/2 */
#define MD_DZFULL 70 /* dzLoss of a particle that went through the whole body (substep lengths summed in order) */
#define MD_KFRAC 71  /* 8 kick fractions of the integrator (radiation) */
#define MD_RAD 79    /* rad_coef (src/multipole.c:755-756) */
#define MD_XKR 80    /* xkick / n_parts, ykick / n_parts (radiation field strength) */
#define MD_YKR 81
#define MD_ISR 82    /* isr_coef (src/multipole.c:757) */
/* KQUAD fringe, per edge (entrance at MD_FR1, exit at MD_FR2): the linear
 * parts M1 and M2 as they apply to that edge (R00 R01 R10 R11 R22 R23 R32
 * R33 each), the nonlinear factor, EDGE_EFFECTS (higherOrder), EDGE_LINEAR;
 * K1 at MD_FRK1 */
#define MD_FR1 83
#define MD_FR2 102
#define MD_FRLEN 19
#define MD_FRK1 121
/* i: 0 n_parts, 1 nSub, 2 expand, 3 maxOrder, 4 orders (o0 | o1<<8 | o2<<16), 5 skew bits, 6 flags */

/* BEND */
#define BD_RHO0 0
#define BD_RHOA 1
#define BD_SLICE 2   /* s/n */
#define BD_DSH 3     /* 8 substep drift lengths */
#define BD_ARG 11    /* 8 values dsh/rho0 */
#define BD_DS 19     /* 8 kick lengths s*kickFrac */
#define BD_SA 27     /* 8 sin(dsh/rho0) */
#define BD_CA 35     /* 8 cos(dsh/rho0) */
#define BD_SH 43     /* 8 sin(dsh/(2 rho0)) */
#define BD_CH 51     /* 8 cos(dsh/(2 rho0)) */
#define BD_DXI 59
#define BD_DYI 60
#define BD_DZI 61
#define BD_CT 62     /* cos/sin total tilt */
#define BD_ST 63
#define BD_ET 64     /* dcoord_etilt[0..4] */
#define BD_DXF 69
#define BD_DYF 70
#define BD_DZF 71
#define BD_APC 72
#define BD_APS 73
#define BD_E1 74      /* edge angle, tan, psi, kick limit, h (pole curvature), 1/cos */
#define BD_TE1 75
#define BD_PSI1 76
#define BD_LIM1 77
#define BD_HE1 78
#define BD_SE1 79
#define BD_E2 80
#define BD_TE2 81
#define BD_PSI2 82
#define BD_LIM2 83
#define BD_HE2 84
#define BD_SE2 85
#define BD_N 86       /* field index n = -b1/h for order-2 edges */
#define BD_RHOINV 87  /* 1/rho0 (fast build) */
#define BD_INVRHOA 88 /* 1/rho_actual (fast build) */
#define BD_OMC 89     /* 8 values 1 - cos(dsh/rho0) = 2 sin^2(dsh/(2 rho0)) (fast build) */
#define BD_C1 97      /* 8 values ds/rho_actual (fast build kick) */
#define BD_C2 105     /* 8 values ds/(rho_actual rho0) (fast build kick) */
#define BD_RAD 113    /* rad_coef (src/csbend.c:956-959) */
#define BD_ISR 114    /* isrConstant (src/csbend.c:961) */
/* Hwang fringes (EDGE_EFFECTS 2 and 4): sin and cos of each edge angle, its
 * FINT, and the full gap 2 HGAP (sec and tan are BD_SE1/2, BD_TE1/2, the
 * pole-face curvature BD_HE1/2) */
#define BD_FS1 115
#define BD_FC1 116
#define BD_FF1 117
#define BD_FS2 118
#define BD_FC2 119
#define BD_FF2 120
#define BD_GAP 121
/* Lindberg's curved-dipole fringe (EDGE_EFFECTS 5): the body gradient
 * b[1]/rho0 the edge maps take; the edges' records (FR_CURV_LEN values each:
 * integrals K0..K6, tan and sec of the edge angle, entrance then exit) sit in
 * the field pool after the bend's field table (at i[4], + 242 where i[2] != 0) */
#define BD_K1F 122
#define FR_CURV_LEN 9
/* i: 0 nSlices, 1 nSub, 2 field mode (0 dipole, 1 normal, 2 skew), 3 expansionOrder1,
 *    4 field pool offset, 5 edge1 mode, 6 edge2 mode, 7 flags */
#define EDGE_NONE 0
#define EDGE_LIN1 1 /* EDGE_EFFECTS=1, EDGE_ORDER<=1 */
#define EDGE_LIN2 2 /* EDGE_EFFECTS=1, EDGE_ORDER>=2 (apply_edge_effects) */
#define EDGE_SYMP 3 /* EDGE_EFFECTS=3 */
#define EDGE_HWANG1 4 /* EDGE_EFFECTS=2, EDGE_ORDER<=1 (dipoleFringeKHwang, linear terms) */
#define EDGE_HWANG2 5 /* EDGE_EFFECTS=2, EDGE_ORDER>=2 */
#define EDGE_HWANGL 6 /* EDGE_EFFECTS=4 (dipoleFringeKHwangRLindberg) */
#define EDGE_CURV1 7 /* EDGE_EFFECTS=5, EDGE_ORDER<=1 (curvedDipoleFringe, linear map) */
#define EDGE_CURV2 8 /* EDGE_EFFECTS=5, EDGE_ORDER>=2 (with the edge's second-order terms) */

/* RF */
#define RD_OMEGA 0
#define RD_VOLT 1
#define RD_LEN 2    /* length per kick */
#define RD_DTL 3
#define RD_TAU 4
#define RD_PHASE_ADD 5 /* PHASE*PI/180 */
#define RD_DX 6
#define RD_DY 7
#define RD_HALF 8   /* length/2 */
#define RD_SOFF 9   /* fiducial sOffset = length/2 */
#define RD_TREF 10  /* T_REFERENCE or -1 */
#define RD_PHASE_LOCK 11 /* PI/180*PHASE, LOCK_PHASE's phase (src/simple_rfca.c:551) */
/* i: 0 nKicks, 1 rf state slot, 2 unused, 3 flags */

/* DRIFT */
#define DD_L 0
#define DD_T 1  /* L/2 */
/* i: 0 order */

#ifdef __cplusplus
}
#endif
#endif
