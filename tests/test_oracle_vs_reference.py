"""Pins the oracle (oracle/trk_oracle.c, the C restatement the GPU parity
tests check against) to elegant's own code: the reference's tracking sources
compiled unmodified into oracle/_ref/libref.so (oracle/ref/Makefile) and
driven through do_tracking's pass loop (oracle/ref/ref_driver.c).

Both are run on the same seeded beams, in the reference's own arithmetic
(glibc sin/cos/asin, Kahan and index-order sums) and in the arithmetic of the
CUDA parity build (correctly rounded sin/cos/asin/tan, double-double beam
sums).  Every coordinate, survivor, loss pass and loss element must agree
bit for bit.  Skipped where the reference sources were not there to build
libref.so.
"""
import numpy as np
import pytest

from elegant_b200 import TYPE_CODE, Lattice, configs
from oracle import pyoracle
from tests.cases import ELEMENT_CASES, fringe_ring

PC = configs.P_CENTRAL

pytestmark = pytest.mark.skipif(not pyoracle.ref_available(), reason="oracle/_ref/libref.so not built")

MODES = {"reference_arith": (False, False), "parity_arith": (True, True)}


def both(lat, beam, n_passes, mode, pass_offset=0):
    es, cr = MODES[mode]
    r = pyoracle.track_ref(lat, beam, n_passes, PC, pass_offset=pass_offset, exact_sums=es, cr_math=cr)
    with pyoracle.modes(exact_sums=es, cr_math=cr):
        o = pyoracle.track(lat, beam, n_passes, PC, pass_offset=pass_offset)
    return r, o


def assert_same(r, o):
    rr, rn, re = r
    orow, on, oe = o
    assert rn == on and re == oe, (rn, on, re, oe)
    diff = rr != orow
    both_nan = np.isnan(rr) & np.isnan(orow)
    bad = diff & ~both_nan
    assert not bad.any(), f"{bad.any(axis=1).sum()} rows differ; columns {bad.sum(axis=0)}"


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("name", sorted(ELEMENT_CASES))
def test_element_matches_reference(name, mode):
    beam = configs.gaussian_beam(400, seed=21)
    assert_same(*both(ELEMENT_CASES[name], beam, 2, mode))


@pytest.mark.parametrize("mode", sorted(MODES))
def test_fodo_ring_matches_reference(mode):
    beam = configs.gaussian_beam(300, seed=22)
    assert_same(*both(configs.c1_lattice(cells=4), beam, 3, mode))


@pytest.mark.parametrize("mode", sorted(MODES))
def test_fringe_ring_matches_reference(mode):
    beam = configs.gaussian_beam(600, seed=29)
    assert_same(*both(fringe_ring(cells=3), beam, 4, mode))


@pytest.mark.parametrize("mode", sorted(MODES))
def test_locked_rf_ring_matches_reference(mode):
    """LOCK_PHASE and LINEARIZE cavities take the beam's mean arrival time
    anew on every pass."""
    beam = configs.gaussian_beam(800, seed=30)
    lat = configs.c2_lattice(cells=2, n_bins=300)
    for el in lat.elements:
        if el[0] == "RFCA":
            el[2]["LOCK_PHASE"] = 1
    lat.add("RFCA", "RF2", L=0.0, VOLT=5e5, FREQ=500e6, PHASE=175.0, LINEARIZE=1)
    assert_same(*both(lat, beam, 4, mode))


@pytest.mark.parametrize("mode", sorted(MODES))
def test_change_p0_ring_matches_reference(mode):
    """RFCA and WAKE with CHANGE_P0: the central momentum follows the beam's
    mean after each (do_match_energy), and every later element sees it."""
    beam = configs.gaussian_beam(800, seed=32)
    lat = configs.c2_lattice(cells=2, n_bins=300)
    for el in lat.elements:
        if el[0] in ("RFCA", "WAKE"):
            el[2]["CHANGE_P0"] = 1
    r, o = both(lat, beam, 4, mode)
    assert_same(r, o)


@pytest.mark.parametrize("mode", sorted(MODES))
def test_rf_wake_ring_matches_reference(mode):
    beam = configs.gaussian_beam(1500, seed=23)
    lat = configs.c2_lattice(cells=2, n_bins=300)
    assert_same(*both(lat, beam, 3, mode))


@pytest.mark.parametrize("mode", sorted(MODES))
def test_losses_match_reference(mode):
    lat = Lattice()
    lat.add("MAXAMP", "AP", X_MAX=0.004, Y_MAX=0.003)
    lat.extend(configs.c1_lattice(cells=2))
    lat.add("MAXAMP", "AP2", X_MAX=0.005, Y_MAX=0.004, ELLIPTICAL=1)
    lat.extend(configs.c1_lattice(cells=2))
    beam = configs.gaussian_beam(800, seed=24, sigma_x=2e-3, sigma_xp=2e-4)
    r, o = both(lat, beam, 3, mode)
    assert r[1] < beam.shape[0]
    assert_same(r, o)


@pytest.mark.parametrize("mode", sorted(MODES))
def test_trwake_matches_reference(mode):
    lat = configs.c1_lattice(cells=2)
    lat.add("CHARGE", "Q", TOTAL=2e-9)
    i = lat.add("TRWAKE", "TW", N_BINS=0)
    t, W = configs.resonator_wake(points=512, dt=2e-12, f_r=5e9)
    lat.set_wake(i, t, W * 1e3, W * 0.5e3)
    beam = configs.gaussian_beam(600, seed=25)
    assert_same(*both(lat, beam, 2, mode))


@pytest.mark.parametrize("first", ["KQUAD", "KSEXT", "CSBEND", "DRIF", "RFCA"])
def test_nonfinite_and_limits_match_reference(first):
    """Non-finite coordinates and particles beyond the multipole coordinate
    and slope limits entering each element type (loss positions included)."""
    beam = configs.gaussian_beam(300, seed=26)
    beam[0, 0] = 30.0  # first particle processed
    beam[3, 0] = np.nan
    beam[7, 1] = np.inf
    beam[8, 3] = 2.0  # beyond the slope limit
    beam[11, 5] = np.nan
    beam[13, 0] = 20.0  # beyond the coordinate limit
    beam[14, 2] = -np.inf
    lat = Lattice()
    params = {"KQUAD": dict(L=0.3, K1=1.2, N_KICKS=8), "KSEXT": dict(L=0.2, K2=40.0, N_KICKS=4),
              "CSBEND": dict(L=1.0, ANGLE=0.0785, N_KICKS=16), "DRIF": dict(L=1.0),
              "RFCA": dict(L=0.2, VOLT=1e6, FREQ=352e6, PHASE=170.0, N_KICKS=4)}[first]
    lat.add(first, "E1", **params)
    lat.extend(configs.c1_lattice(cells=1))
    for mode in MODES:
        assert_same(*both(lat, beam, 1, mode))


def test_parameter_defaults_match_reference():
    """Every parameter of the library's tables has the reference's default
    (src/track_data.c *_param[]), read from the compiled reference tables."""
    lib = pyoracle.load_ref()
    for tname, code in TYPE_CODE.items():
        n = lib.trk_param_count(code)
        ours = np.array([lib.trk_param_default(code, i) for i in range(n)])
        ref = pyoracle.ref_param_defaults(code)
        names = [lib.trk_param_name(code, i).decode() for i in range(n)]
        bad = [(nm, a, b) for nm, a, b in zip(names, ours, ref) if not (a == b or (np.isnan(a) and np.isnan(b)))]
        assert not bad, (tname, bad)
