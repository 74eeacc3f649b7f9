"""Error paths of the C ABI on the device, each made on the host (no GPU
fault is provoked): the reference's own physics check (a beam longer than the
wake, src/wake.c:134-140), a wake table too short to be one, element tables
the path does not take, and a device allocation refused by the library's
test hook (trk_test_fail_allocation).  Every failing call returns its error
code and leaves its context usable: the next run gives the same bits as a
fresh context."""
import numpy as np
import pytest

from elegant_b200 import Lattice, TrackingError, Tracker, configs, load_library

pytestmark = pytest.mark.gpu
PC = configs.P_CENTRAL
ERR_ARG, ERR_UNKNOWN_TYPE, ERR_UNKNOWN_PARAM, ERR_UNSUPPORTED, ERR_NOMEM, ERR_PHYSICS = -1, -2, -3, -4, -6, -8


def _reference_run(lat, beam, passes):
    with Tracker(0) as trk:
        trk.load(beam)
        trk.track(lat, passes, PC, fast=False)
        return trk.store(stride=7, with_loss=True)


def _same(a, b):
    assert a[0] == b[0]
    ia, ib = np.argsort(a[1][:, 6]), np.argsort(b[1][:, 6])
    assert np.array_equal(a[1][ia], b[1][ib], equal_nan=True)
    assert np.array_equal(a[2][ia], b[2][ib]) and np.array_equal(a[3][ia], b[3][ib])


def _long_beam_lattice():
    """A WAKE whose table spans 20 ps, shorter than the +-5 sigma of a 3 mm bunch."""
    lat = Lattice()
    lat.add("CHARGE", "Q", TOTAL=1e-9)
    lat.extend(configs.c1_lattice(cells=1))
    i = lat.add("WAKE", "W", N_BINS=400)
    t, W = configs.resonator_wake(points=401, dt=50e-15)
    lat.set_wake(i, t, W)
    return lat


def test_beam_longer_than_wake_is_a_physics_error_and_the_context_survives():
    beam = configs.gaussian_beam(3000, seed=71)
    good = configs.c2_lattice(cells=2, n_bins=300)
    want = _reference_run(good, beam, 2)
    with Tracker(0) as trk:
        trk.load(beam)
        with pytest.raises(TrackingError) as ei:
            trk.track(_long_beam_lattice(), 1, PC, fast=False)
        assert ei.value.code == ERR_PHYSICS and "longer than the" in str(ei.value)
        trk.load(beam)
        trk.track(good, 2, PC, fast=False)
        _same(trk.store(stride=7, with_loss=True), want)
    # ALLOW_LONG_BEAM=1 tracks the same beam (the reference's switch)
    lat = _long_beam_lattice()
    lat.elements[-1][2]["ALLOW_LONG_BEAM"] = 1
    with Tracker(0) as trk:
        trk.load(beam)
        trk.track(lat, 1, PC, fast=False)


def test_wake_table_too_short_is_rejected():
    lat = configs.c1_lattice(cells=1)
    lat.add("CHARGE", "Q", TOTAL=1e-9)
    i = lat.add("WAKE", "W", N_BINS=100)
    lat.set_wake(i, np.array([0.0]), np.array([1.0]))
    with Tracker(0) as trk:
        trk.load(configs.gaussian_beam(100, seed=72))
        with pytest.raises(TrackingError) as ei:
            trk.track(lat, 1, PC)
        assert ei.value.code in (ERR_ARG, ERR_PHYSICS)


def test_bad_element_tables_are_rejected_before_any_launch():
    lib = load_library()
    assert lib.trk_type_code(b"NOSUCHELEMENT") < 0
    lat = Lattice()
    lat.add("KQUAD", "Q", L=0.3, K1=1.0, NOSUCH=1.0)
    with Tracker(0) as trk:
        trk.load(configs.gaussian_beam(100, seed=73))
        with pytest.raises(TrackingError) as ei:
            trk.track(lat, 1, PC)
        assert ei.value.code == ERR_UNKNOWN_PARAM
        unsupported = Lattice()
        unsupported.add("KQUAD", "Q", L=0.3, K1=1.0, MALIGN_METHOD=2)
        with pytest.raises(TrackingError) as ei:
            trk.track(unsupported, 1, PC)
        assert ei.value.code == ERR_UNSUPPORTED
        # the context still tracks
        trk.track(configs.c1_lattice(cells=1), 1, PC)


@pytest.mark.parametrize("after", [0, 1, 2, 3])
def test_refused_allocation_leaves_the_context_usable(after):
    lib = load_library()
    lat = configs.c2_lattice(cells=2, n_bins=300)
    beam = configs.gaussian_beam(5000, seed=74)
    want = _reference_run(lat, beam, 2)
    with Tracker(0) as trk:
        trk.load(configs.gaussian_beam(10, seed=75))  # a small beam first: the load below must grow it
        lib.trk_test_fail_allocation(after)
        try:
            failed = False
            try:
                trk.load(beam)
                trk.track(lat, 2, PC, fast=False)
                trk.store(stride=7, with_loss=True)
            except TrackingError as e:
                failed = True
                assert e.code == ERR_NOMEM and "test hook" in str(e)
        finally:
            lib.trk_test_fail_allocation(-1)
        assert failed or after > 0
        trk.load(beam)
        trk.track(lat, 2, PC, fast=False)
        _same(trk.store(stride=7, with_loss=True), want)
