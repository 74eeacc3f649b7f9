"""Dynamic-aperture searches.  Line modes (trk_aperture_search_lines) against
elegant's do_aperture_search_line restated serially over the oracle
(oracle/pyoracle.py: one particle at a time, each sweep stopping at the first
loss), and its island clipping and area against elegant's own
trimApertureSearchResult (compiled from the reference sources).  Grid mode
(trk_aperture_search_grid) against do_aperture_search_grid restated over the
oracle, in (x, y), (delta, x) and (delta, y), one- and two-sided."""
import numpy as np
import pytest

from elegant_b200 import Lattice, configs
from oracle import pyoracle

PC = configs.P_CENTRAL


def _box_lattice():
    """A drift inside an elliptical 10 mm x 5 mm aperture: the aperture is
    the dynamic aperture."""
    lat = Lattice()
    lat.add("MAXAMP", "AP", X_MAX=0.01, Y_MAX=0.005, ELLIPTICAL=1)
    lat.add("DRIF", "D", L=1.0)
    return lat


def test_serial_restatement_on_a_known_aperture():
    r = pyoracle.aperture_search_lines(_box_lattice(), PC, 2, lines=5, nx=41, xmax=0.02, ymax=0.01, n_splits=3,
                                       split_fraction=0.5)
    assert r["origin_stable"]
    xl, yl = r["x_limit"], r["y_limit"]
    # every limit inside the ellipse, and within one final step of its edge
    assert np.all((xl / 0.01) ** 2 + (yl / 0.005) ** 2 <= 1 + 1e-12)
    step = 0.02 / 40 / 8
    r_lim = np.hypot(xl, yl)
    ang = np.arctan2(yl, xl)
    r_edge = 1 / np.sqrt((np.cos(ang) / 0.01) ** 2 + (np.sin(ang) / 0.005) ** 2)
    assert np.all(r_edge - r_lim < 2 * step * 1.5)


@pytest.mark.skipif(not pyoracle.ref_available(), reason="oracle/_ref/libref.so not built")
def test_reference_trimming_on_the_restatement():
    r = pyoracle.aperture_search_lines(_box_lattice(), PC, 2, lines=7, nx=21, xmax=0.02, ymax=0.01,
                                       area_fn=pyoracle.trim_aperture_ref)
    # the ellipse's upper half: pi a b / 2, resolved by the 7-line polygon
    assert 0.5 * np.pi * 0.01 * 0.005 * 0.6 < r["area"] < 0.5 * np.pi * 0.01 * 0.005


def _ring(seed=0):
    return configs.c3_variant(seed=seed)


@pytest.mark.gpu
@pytest.mark.skipif(not pyoracle.ref_available(), reason="oracle/_ref/libref.so not built")
@pytest.mark.parametrize("opts", [dict(lines=5, nx=11, n_splits=2, split_fraction=0.5),
                                  dict(lines=2, nx=9, n_splits=1, split_fraction=0.25),
                                  dict(lines=9, nx=8, n_splits=1, split_fraction=0.5, full_plane=1)])
def test_search_equals_serial_reference_restatement(tracker, opts):
    lat, passes = _ring(), 30
    kw = dict(xmax=0.03, ymax=0.015, **opts)
    g = tracker.aperture_search_lines(lat, PC, passes, fast=False, **kw)
    with pyoracle.modes(exact_sums=True, cr_math=True):
        r = pyoracle.aperture_search_lines(lat, PC, passes, area_fn=pyoracle.trim_aperture_ref, **kw)
    for k in ("x_limit", "y_limit", "x_lost", "y_lost", "s_lost", "x_clipped", "y_clipped"):
        assert np.array_equal(g[k][0], r[k]), (k, g[k][0], r[k])
    assert g["area"][0] == r["area"]
    assert np.any(r["x_lost"] < 1e300)  # the search reaches the dynamic aperture


@pytest.mark.gpu
def test_search_slope_mode(tracker):
    lat, passes = _ring(), 20
    kw = dict(lines=3, nx=9, xmax=0.0, ymax=0.0, xpmax=2e-3, ypmax=1e-3, slope_mode=1, n_splits=1)
    g = tracker.aperture_search_lines(lat, PC, passes, fast=False, **kw)
    with pyoracle.modes(exact_sums=True, cr_math=True):
        r = pyoracle.aperture_search_lines(lat, PC, passes, **kw)
    assert np.array_equal(g["x_limit"][0], r["x_limit"]) and np.array_equal(g["y_limit"][0], r["y_limit"])


@pytest.mark.gpu
@pytest.mark.parametrize("fast", [False, True])
def test_error_seed_batch_equals_separate_searches(tracker, fast):
    """Four error seeds in one batched search give each seed's own result."""
    lats = [_ring(seed=s) for s in range(4)]
    kw = dict(lines=7, nx=16, xmax=0.03, ymax=0.015, n_splits=2, split_fraction=0.5)
    g = tracker.aperture_search_lines(lats, PC, 40, fast=fast, **kw)
    for v, lat in enumerate(lats):
        one = tracker.aperture_search_lines(lat, PC, 40, fast=fast, **kw)
        for k in ("x_limit", "y_limit", "x_lost", "y_lost", "s_lost", "x_clipped", "y_clipped"):
            assert np.array_equal(g[k][v], one[k][0]), (v, k)
        assert g["area"][v] == one["area"][0]
    assert len(set(np.round(g["area"], 12))) > 1  # the seeds differ


def test_grid_restatement_on_a_known_aperture():
    """On the elliptical box, each column's limit is the last grid point
    inside the ellipse, and both sides agree by symmetry."""
    r = pyoracle.aperture_search_grid(_box_lattice(), PC, 1, nx=11, ny=9, xmin=-0.012, xmax=0.012, ymin=-0.006,
                                      ymax=0.006)
    u, v = r["u_limit"][0], r["v_limit"][0]
    dv = 0.006 / 8
    for k in range(11):
        inside = [j * dv for j in range(9) if (u[k] / 0.01) ** 2 + (j * dv / 0.005) ** 2 <= 1]
        assert v[k] == (max(inside) if inside else 0.0)
    assert np.array_equal(r["v_limit"][1], -r["v_limit"][0])
    assert r["area"] > 0


GRID_CASES = [dict(nx=9, ny=7, xmin=-0.03, xmax=0.03, ymin=0.0, ymax=0.015),
              dict(nx=8, ny=6, xmin=-0.03, xmax=0.025, ymin=-0.012, ymax=0.015),
              dict(delta_mode=1, ndelta=7, nx=8, deltamin=-0.02, deltamax=0.02, xmin=-0.03, xmax=0.03),
              dict(delta_mode=2, ndelta=6, ny=7, deltamin=-0.015, deltamax=0.02, ymin=0.0, ymax=0.015)]


@pytest.mark.gpu
@pytest.mark.parametrize("opts", GRID_CASES)
def test_grid_search_equals_reference_restatement(tracker, opts):
    lat, passes = _ring(), 30
    g = tracker.aperture_search_grid(lat, PC, passes, fast=False, **opts)
    with pyoracle.modes(exact_sums=True, cr_math=True):
        r = pyoracle.aperture_search_grid(lat, PC, passes, **opts)
    for k in ("u_limit", "v_limit", "x_lost", "y_lost", "s_lost", "delta_lost"):
        assert np.array_equal(g[k][0], r[k]), (k, g[k][0], r[k])
    assert g["area"][0] == r["area"]
    assert np.any(r["x_lost"] < 1e300) and np.any(r["v_limit"] != 0)


@pytest.mark.gpu
def test_grid_error_seed_batch_equals_separate_searches(tracker):
    lats = [_ring(seed=s) for s in range(3)]
    kw = GRID_CASES[1]
    g = tracker.aperture_search_grid(lats, PC, 30, fast=True, **kw)
    for v, lat in enumerate(lats):
        one = tracker.aperture_search_grid(lat, PC, 30, fast=True, **kw)
        for k in ("u_limit", "v_limit", "x_lost", "y_lost", "s_lost", "delta_lost"):
            assert np.array_equal(g[k][v], one[k][0]), (v, k)
        assert g["area"][v] == one["area"][0]


@pytest.mark.gpu
def test_grid_rejects_a_one_point_axis(tracker):
    with pytest.raises(Exception):
        tracker.aperture_search_grid(_box_lattice(), PC, 1, nx=1, ny=5, xmax=0.01, ymax=0.01)
