"""Single-element lattices shared by the parity suites (GPU vs oracle,
oracle vs the reference's own code)."""
import math

from elegant_b200 import Lattice


def single(type_name, **params):
    lat = Lattice()
    lat.add(type_name, type_name, **params)
    return lat


QUAD_FRINGE_INTEGRALS = dict(I0P=0.01, I1P=2e-5, I2P=1e-7, I3P=5e-10, LAMBDA2P=3e-7, I0M=0.012, I1M=-1.5e-5,
                             I2M=8e-8, I3M=-4e-10, LAMBDA2M=2e-7)


# Lindberg's edge integrals K0..K6 for both ends of a bend (EDGE_EFFECTS=5)
CURVED_FRINGE = dict(FRINGE1K0=2e-3, FRINGE1K1=0.01, FRINGE1K2=0.02, FRINGE1K3=3e-3, FRINGE1K4=-1e-3,
                     FRINGE1K5=0.05, FRINGE1K6=0.1, FRINGE2K0=1.5e-3, FRINGE2K1=-0.02, FRINGE2K2=0.015,
                     FRINGE2K3=2e-3, FRINGE2K4=5e-4, FRINGE2K5=-0.04, FRINGE2K6=0.3)

def fringe_ring(cells=2):
    """A small FODO ring whose bends mix every dipole-edge model (curved-dipole
    fringe of both orders with and without a field table, Hwang-Lindberg,
    symplectic kick, plain linear edge) among fringed quadrupoles and weak
    sextupoles, so that several fringe records share the field pool."""
    lat = Lattice()
    a = 2 * math.pi / 80
    for c in range(cells):
        lat.add("KQUAD", f"QF{c}", L=0.3, K1=1.2, N_KICKS=8, EDGE1_EFFECTS=2, EDGE2_EFFECTS=2,
                **QUAD_FRINGE_INTEGRALS)
        lat.add("DRIF", f"D1{c}", L=1.0)
        lat.add("CSBEND", f"BA{c}", L=1.0, ANGLE=a, E1=a / 2, E2=a / 2, K1=-0.05, EDGE1_EFFECTS=5,
                EDGE2_EFFECTS=5, EDGE_ORDER=2, N_SLICES=8, **CURVED_FRINGE)
        lat.add("DRIF", f"D2{c}", L=1.0)
        lat.add("KQUAD", f"QD{c}", L=0.3, K1=-1.2, N_KICKS=8)
        lat.add("KSEXT", f"SD{c}", L=0.2, K2=-4.0, N_KICKS=4)
        lat.add("DRIF", f"D3{c}", L=1.0)
        lat.add("CSBEND", f"BB{c}", L=1.0, ANGLE=a, E1=a / 2, E2=0.0, EDGE1_EFFECTS=5, EDGE2_EFFECTS=3,
                N_SLICES=8, **CURVED_FRINGE)
        lat.add("DRIF", f"D4{c}", L=1.0)
        lat.add("KQUAD", f"QF2{c}", L=0.3, K1=1.2, N_KICKS=8)
        lat.add("KSEXT", f"SF{c}", L=0.2, K2=4.0, N_KICKS=4)
        lat.add("DRIF", f"D5{c}", L=1.0)
        lat.add("CSBEND", f"BC{c}", L=1.0, ANGLE=a, E1=0.03, E2=0.05, HGAP=0.02, FINT=0.5, K2=3.0,
                EDGE1_EFFECTS=4, EDGE2_EFFECTS=5, N_SLICES=8, **CURVED_FRINGE)
        lat.add("DRIF", f"D6{c}", L=1.0)
        lat.add("KQUAD", f"QD2{c}", L=0.3, K1=-1.2, N_KICKS=8)
        lat.add("DRIF", f"D7{c}", L=1.0)
        lat.add("CSBEND", f"BD{c}", L=1.0, ANGLE=a, E1=0.02, E2=0.02, N_SLICES=8)
        lat.add("DRIF", f"D8{c}", L=1.0)
    return lat


def _lossy_fringe_quad():
    lat = Lattice()
    lat.add("MAXAMP", "AP", X_MAX=0.0012, Y_MAX=0.001, ELLIPTICAL=1)
    lat.add("KQUAD", "QF", L=0.5, K1=2.5, N_KICKS=8, EDGE1_EFFECTS=2, EDGE2_EFFECTS=3, **QUAD_FRINGE_INTEGRALS)
    return lat


ELEMENT_CASES = {
    "drif": single("DRIF", L=1.3),
    "drif_order1": single("DRIF", L=0.7, ORDER=1),
    "edrift": single("EDRIFT", L=2.1),
    "kquad": single("KQUAD", L=0.3, K1=1.2, N_KICKS=8),
    "kquad_order2": single("KQUAD", L=0.3, K1=-1.1, N_SLICES=5, INTEGRATION_ORDER=2),
    "kquad_order6": single("KQUAD", L=0.5, K1=0.8, N_SLICES=3, INTEGRATION_ORDER=6),
    "kquad_misaligned": single("KQUAD", L=0.3, K1=1.2, N_KICKS=8, DX=1e-4, DY=-2e-4, DZ=1e-3, TILT=0.01),
    "kquad_kicks_fse": single("KQUAD", L=0.4, K1=0.9, N_KICKS=12, HKICK=1e-5, VKICK=-2e-5, FSE=1e-3),
    "kquad_leff": single("KQUAD", L=0.4, K1=0.9, N_KICKS=4, LEFFECTIVE=0.35),
    "kquad_fringe_linear": single("KQUAD", L=0.3, K1=1.2, N_KICKS=8, EDGE1_EFFECTS=1, EDGE2_EFFECTS=1,
                                  **QUAD_FRINGE_INTEGRALS),
    "kquad_fringe_order2": single("KQUAD", L=0.3, K1=-1.4, N_KICKS=8, EDGE1_EFFECTS=2, EDGE2_EFFECTS=2,
                                  **QUAD_FRINGE_INTEGRALS),
    "kquad_fringe_order3": single("KQUAD", L=0.4, K1=2.0, N_KICKS=8, EDGE1_EFFECTS=3, EDGE2_EFFECTS=3,
                                  EDGE2_LINEAR=0, EDGE1_NONLINEAR_FACTOR=0.8, LEFFECTIVE=0.35, DX=1e-4,
                                  **QUAD_FRINGE_INTEGRALS),
    "kquad_fringe_lossy": _lossy_fringe_quad(),
    "kquad_expand": single("KQUAD", L=0.3, K1=1.2, N_KICKS=8, EXPAND_HAMILTONIAN=1),
    "ksext": single("KSEXT", L=0.2, K2=40.0, N_KICKS=4),
    "ksext_k1j1": single("KSEXT", L=0.2, K2=-30.0, K1=0.01, J1=0.02, N_SLICES=2, TILT=0.1),
    "koct": single("KOCT", L=0.2, K3=500.0),
    "csbend": single("CSBEND", L=1.0, ANGLE=2 * math.pi / 80, N_KICKS=16),
    "csbend_negative": single("CSBEND", L=1.0, ANGLE=-0.05, N_KICKS=8),
    "csbend_k1": single("CSBEND", L=1.0, ANGLE=2 * math.pi / 280, K1=-0.4, N_KICKS=32),
    "csbend_k1k2": single("CSBEND", L=0.8, ANGLE=0.03, K1=0.3, K2=5.0, N_SLICES=10),
    "csbend_edges": single("CSBEND", L=1.0, ANGLE=0.08, E1=0.04, E2=0.03, N_SLICES=8),
    "csbend_edges_fringe": single("CSBEND", L=1.0, ANGLE=0.08, E1=0.04, E2=0.03, HGAP=0.02, FINT=0.5, N_SLICES=8),
    "csbend_edge_order2": single("CSBEND", L=1.0, ANGLE=0.08, E1=0.04, E2=0.03, EDGE_ORDER=2, K1=0.2, N_SLICES=8),
    "csbend_edge3": single("CSBEND", L=1.0, ANGLE=0.08, E1=0.04, E2=0.03, EDGE1_EFFECTS=3, EDGE2_EFFECTS=3,
                           N_SLICES=8),
    "csbend_hwang": single("CSBEND", L=1.0, ANGLE=0.08, E1=0.04, E2=0.03, HGAP=0.02, FINT=0.5, H1=0.3, H2=-0.2,
                           EDGE1_EFFECTS=2, EDGE2_EFFECTS=2, N_SLICES=8),
    "csbend_hwang_order2": single("CSBEND", L=1.0, ANGLE=0.08, E1=0.04, E2=0.03, HGAP=0.02, FINT1=0.45, FINT2=0.55,
                                  H1=0.3, H2=-0.2, EDGE1_EFFECTS=2, EDGE2_EFFECTS=2, EDGE_ORDER=2, K1=0.2,
                                  N_SLICES=8),
    "csbend_hwang_lindberg": single("CSBEND", L=1.0, ANGLE=0.08, E1=0.04, E2=0.03, HGAP=0.025, FINT=0.5, H1=0.3,
                                    H2=-0.2, EDGE1_EFFECTS=4, EDGE2_EFFECTS=4, N_SLICES=8),
    "csbend_hwang_negative": single("CSBEND", L=1.0, ANGLE=-0.06, E1=0.02, E2=0.05, HGAP=0.02, FINT=0.6,
                                    EDGE1_EFFECTS=4, EDGE2_EFFECTS=2, N_SLICES=8),
    "csbend_curved": single("CSBEND", L=1.0, ANGLE=0.08, E1=0.04, E2=0.03, K1=0.2, EDGE1_EFFECTS=5,
                            EDGE2_EFFECTS=5, N_SLICES=8, **CURVED_FRINGE),
    "csbend_curved_order2": single("CSBEND", L=1.0, ANGLE=0.08, E1=0.04, E2=-0.03, K1=-0.3, EDGE1_EFFECTS=5,
                                   EDGE2_EFFECTS=5, EDGE_ORDER=2, N_SLICES=8, **CURVED_FRINGE),
    "csbend_curved_small_m": single("CSBEND", L=1.0, ANGLE=-0.06, E1=0.02, E2=0.05, K1=0.1, EDGE1_EFFECTS=5,
                                    EDGE2_EFFECTS=5, EDGE_ORDER=2, N_SLICES=8, FRINGE1K0=1.5e-3, FRINGE1K1=0.02,
                                    FRINGE1K2=0.03, FRINGE1K3=4e-6, FRINGE1K4=2e-6, FRINGE1K5=0.04, FRINGE1K6=-0.1,
                                    FRINGE2K0=-1e-3, FRINGE2K1=0.01, FRINGE2K2=0.02, FRINGE2K3=-3e-6,
                                    FRINGE2K4=1e-6, FRINGE2K5=0.06, FRINGE2K6=0.2),
    "csbend_curved_mixed": single("CSBEND", L=1.0, ANGLE=0.08, E1=0.04, E2=0.03, HGAP=0.02, FINT=0.5,
                                  EDGE1_EFFECTS=5, EDGE2_EFFECTS=2, N_SLICES=8, **CURVED_FRINGE),
    "csbend_rad_edges": single("CSBEND", L=1.0, ANGLE=-0.08, E1=0.04, E2=0.03, K1=0.1, SYNCH_RAD=1, N_SLICES=8),
    "csbend_expanded": single("CSBEND", L=1.0, ANGLE=0.08, E1=0.04, E2=0.03, K1=0.2, K2=3.0, EXPAND_HAMILTONIAN=1,
                              N_SLICES=8),
    "csbend_expanded_fringes": single("CSBEND", L=1.0, ANGLE=-0.07, E1=0.03, E2=0.05, HGAP=0.02, FINT=0.5,
                                      EDGE1_EFFECTS=5, EDGE2_EFFECTS=3, EXPAND_HAMILTONIAN=1, N_SLICES=8,
                                      INTEGRATION_ORDER=6, **CURVED_FRINGE),
    "csbend_expanded_hwang_rad": single("CSBEND", L=1.0, ANGLE=0.08, E1=0.04, E2=0.03, HGAP=0.02, FINT=0.5,
                                        EDGE1_EFFECTS=2, EDGE2_EFFECTS=4, K1=0.1, SYNCH_RAD=1, EXPAND_HAMILTONIAN=1,
                                        N_SLICES=8, INTEGRATION_ORDER=2),
    "csbend_xreference": single("CSBEND", L=1.0, ANGLE=0.06, XREFERENCE=0.02, F1=1e-3, F2=-2e-3, F3=5e-4, G1=4e-4,
                                G2=-1e-4, N_SLICES=8, EPITCH=1e-3, EYAW=-2e-3, XSTEERING=1, SQRT_ORDER=2,
                                FRINGE1K0=0.1, TRACKING_MATRIX=2),
    "kquad_inert_params": single("KQUAD", L=0.3, K1=1.2, N_KICKS=8, HSTEERING=1, VSTEERING=1, SQRT_ORDER=1,
                                 SYSTEMATIC_MULTIPOLE_FACTOR=2, MIN_NORMAL_ORDER=2, TRACKING_MATRIX=3),
    "csbend_misaligned": single("CSBEND", L=1.0, ANGLE=0.05, DX=1e-4, DY=2e-4, DZ=-1e-4, TILT=0.02, N_SLICES=8),
    "csbend_order6": single("CSBEND", L=1.0, ANGLE=0.05, N_SLICES=4, INTEGRATION_ORDER=6),
    "kquad_rad": single("KQUAD", L=0.3, K1=1.2, N_KICKS=8, SYNCH_RAD=1),
    "kquad_rad_kicks": single("KQUAD", L=0.4, K1=-0.9, N_KICKS=12, HKICK=2e-5, VKICK=-1e-5, SYNCH_RAD=1),
    "ksext_rad": single("KSEXT", L=0.2, K2=40.0, N_KICKS=4, SYNCH_RAD=1),
    "koct_rad": single("KOCT", L=0.2, K3=500.0, SYNCH_RAD=1),
    "csbend_rad": single("CSBEND", L=1.0, ANGLE=2 * math.pi / 80, N_KICKS=16, SYNCH_RAD=1),
    "csbend_k1_rad": single("CSBEND", L=1.0, ANGLE=2 * math.pi / 280, K1=-0.4, N_KICKS=32, SYNCH_RAD=1),
    "rfca_thin": single("RFCA", L=0.0, VOLT=4e6, FREQ=352e6, PHASE=170.0),
    "rfca_long": single("RFCA", L=0.5, VOLT=2e6, FREQ=500e6, PHASE=160.0, N_KICKS=5, END1_FOCUS=1, END2_FOCUS=1),
    "rfca_tref": single("RFCA", L=0.0, VOLT=1e6, FREQ=352e6, PHASE=90.0, T_REFERENCE=1e-12),
    "rfca_zero_volt": single("RFCA", L=0.3, VOLT=0.0),
    "rfca_lock_phase": single("RFCA", L=0.0, VOLT=2e6, FREQ=352e6, PHASE=160.0, LOCK_PHASE=1),
    "rfca_linearize": single("RFCA", L=0.3, VOLT=2e6, FREQ=352e6, PHASE=170.0, N_KICKS=1, LINEARIZE=1, END1_FOCUS=1,
                             END2_FOCUS=1),
    "rfca_change_p0": single("RFCA", L=0.2, VOLT=3e6, FREQ=352e6, PHASE=60.0, N_KICKS=2, CHANGE_P0=1),
    "rfca_lock_linearize": single("RFCA", L=0.2, VOLT=1e6, FREQ=500e6, PHASE=150.0, N_KICKS=1, LOCK_PHASE=1,
                                  LINEARIZE=1),
}
