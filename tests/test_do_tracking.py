"""Pins the pass loop of the reference driver (oracle/ref/ref_driver.c,
which the oracle and the GPU library are checked against) to elegant's own
do_tracking() (src/do_tracking.c:144), compiled unmodified into
oracle/_ref/libref.so: the same element structures tracked by both loops
must give the same rows in the same order (survivors first), the same loss
pass for every lost row, the same survivor count and the same effort.
do_tracking records no loss element, so that column is not compared.

Both arithmetic modes of the reference build are used.  Skipped where the
reference sources were not there to build libref.so.
"""
import numpy as np
import pytest

from elegant_b200 import Lattice, configs
from oracle import pyoracle
from tests.cases import ELEMENT_CASES, fringe_ring

PC = configs.P_CENTRAL

pytestmark = pytest.mark.skipif(not pyoracle.ref_available(), reason="oracle/_ref/libref.so not built")

MODES = {"reference_arith": (False, False), "parity_arith": (True, True)}


def assert_same_loop(lat, beam, n_passes, mode, pass_offset=0):
    es, cr = MODES[mode]
    kw = dict(pass_offset=pass_offset, exact_sums=es, cr_math=cr)
    a, an, ae = pyoracle.track_ref(lat, beam, n_passes, PC, loop="driver", **kw)
    b, bn, be = pyoracle.track_ref(lat, beam, n_passes, PC, loop="do_tracking", **kw)
    assert an == bn and ae == be, (an, bn, ae, be)
    x, y = a[:, :8], b[:, :8]
    bad = (x != y) & ~(np.isnan(x) & np.isnan(y))
    assert not bad.any(), f"{bad.any(axis=1).sum()} rows differ; columns {bad.sum(axis=0)}"
    return an


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("name", sorted(ELEMENT_CASES))
def test_element_loop_is_do_tracking(name, mode):
    beam = configs.gaussian_beam(400, seed=21, sigma_x=1.5e-3, sigma_xp=1.5e-4)
    assert_same_loop(ELEMENT_CASES[name], beam, 2, mode)


@pytest.mark.parametrize("mode", sorted(MODES))
def test_rings_loop_is_do_tracking(mode):
    assert_same_loop(configs.c1_lattice(cells=4), configs.gaussian_beam(300, seed=22), 3, mode)
    assert_same_loop(configs.c2_lattice(cells=2, n_bins=300), configs.gaussian_beam(1500, seed=23), 3, mode)
    assert_same_loop(configs.c2_lattice(cells=2, n_bins=300), configs.gaussian_beam(500, seed=27), 2, mode,
                     pass_offset=5)
    assert_same_loop(fringe_ring(), configs.gaussian_beam(400, seed=28), 3, mode)


@pytest.mark.parametrize("mode", sorted(MODES))
def test_losses_loop_is_do_tracking(mode):
    lat = Lattice()
    lat.add("MAXAMP", "AP", X_MAX=0.004, Y_MAX=0.003)
    lat.extend(configs.c1_lattice(cells=2))
    lat.add("MAXAMP", "AP2", X_MAX=0.005, Y_MAX=0.004, ELLIPTICAL=1)
    lat.extend(configs.c1_lattice(cells=2))
    beam = configs.gaussian_beam(800, seed=24, sigma_x=2e-3, sigma_xp=2e-4)
    assert assert_same_loop(lat, beam, 3, mode) < beam.shape[0]


@pytest.mark.parametrize("mode", sorted(MODES))
def test_trwake_loop_is_do_tracking(mode):
    lat = configs.c1_lattice(cells=2)
    lat.add("CHARGE", "Q", TOTAL=2e-9)
    i = lat.add("TRWAKE", "TW", N_BINS=0)
    t, W = configs.resonator_wake(points=512, dt=2e-12, f_r=5e9)
    lat.set_wake(i, t, W * 1e3, W * 0.5e3)
    assert_same_loop(lat, configs.gaussian_beam(600, seed=25), 2, mode)


@pytest.mark.parametrize("first", ["KQUAD", "KSEXT", "CSBEND", "DRIF", "RFCA"])
def test_nonfinite_and_limits_loop_is_do_tracking(first):
    beam = configs.gaussian_beam(300, seed=26)
    beam[0, 0] = 30.0
    beam[3, 0] = np.nan
    beam[7, 1] = np.inf
    beam[8, 3] = 2.0
    beam[11, 5] = np.nan
    beam[13, 0] = 20.0
    beam[14, 2] = -np.inf
    lat = Lattice()
    params = {"KQUAD": dict(L=0.3, K1=1.2, N_KICKS=8), "KSEXT": dict(L=0.2, K2=40.0, N_KICKS=4),
              "CSBEND": dict(L=1.0, ANGLE=0.0785, N_KICKS=16), "DRIF": dict(L=1.0),
              "RFCA": dict(L=0.2, VOLT=1e6, FREQ=352e6, PHASE=170.0, N_KICKS=4)}[first]
    lat.add(first, "E1", **params)
    lat.extend(configs.c1_lattice(cells=1))
    for mode in MODES:
        assert_same_loop(lat, beam, 1, mode)
