"""Ring cases of the golden fixtures (shared by make_golden.py and the test)."""
from elegant_b200 import Lattice, configs
from tests.cases import fringe_ring


def ring_cases():
    lossy = Lattice()
    lossy.add("MAXAMP", "AP", X_MAX=0.004, Y_MAX=0.003, ELLIPTICAL=1)
    lossy.extend(configs.c1_lattice(cells=2))
    trw = configs.c1_lattice(cells=1)
    trw.add("CHARGE", "Q", TOTAL=2e-9)
    i = trw.add("TRWAKE", "TW", N_BINS=0)
    t, W = configs.resonator_wake(points=256, dt=2e-12, f_r=5e9)
    trw.set_wake(i, t, W * 1e3, W * 0.5e3)
    return {
        "ring_fodo": (configs.c1_lattice(cells=2), configs.gaussian_beam(64, seed=62), 2),
        "ring_rf_wake": (configs.c2_lattice(cells=2, n_bins=300), configs.gaussian_beam(200, seed=63), 2),
        "ring_lossy": (lossy, configs.gaussian_beam(100, seed=64, sigma_x=2e-3, sigma_xp=2e-4), 3),
        "ring_trwake": (trw, configs.gaussian_beam(100, seed=65), 2),
        "ring_fringes": (fringe_ring(), configs.gaussian_beam(100, seed=66), 3),
    }
