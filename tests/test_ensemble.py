"""Batched ensembles (trk_track_ensemble): many lattice variants of one
structure (error seeds) with uneven particle counts, tracked in one
graph-captured launch sequence.  Each variant's particles must come out
exactly as a separate run of that variant gives them, and the parity build's
ensemble exactly as the oracle."""
import numpy as np
import pytest

from elegant_b200 import Lattice, TrackingError, Tracker, configs
from oracle import pyoracle
from tests.helpers import compare

pytestmark = pytest.mark.gpu
PC = configs.P_CENTRAL


def _variants(counts, cells=3):
    lats = [configs.c3_variant(seed=v, cells=cells) for v in range(len(counts))]
    beams, first = [], 1
    for v, n in enumerate(counts):
        b = configs.da_grid(n, first_id=first) if v % 2 == 0 else \
            configs.gaussian_beam(n, seed=80 + v, sigma_x=4e-3, sigma_xp=3e-4, first_id=first)
        beams.append(b)
        first += n
    return lats, beams


def _by_id(rows):
    return rows[np.argsort(rows[:, 6])]


@pytest.mark.parametrize("fast", [True, False])
def test_ensemble_equals_separate_runs(fast):
    counts = [300, 0, 1000, 37, 513]
    lats, beams = _variants(counts)
    passes = 12
    with Tracker(0) as trk:
        trk.load(np.concatenate(beams))
        st = trk.track_ensemble(lats, counts, passes, PC, fast=fast)
        nl, ens, lp, le = trk.store(stride=7, with_loss=True)
        parts = []
        for lat, b in zip(lats, beams):
            if len(b) == 0:
                continue
            trk.load(b)
            trk.track(lat, passes, PC, fast=fast)
            parts.append(trk.store(stride=7, with_loss=True))
    sep = np.concatenate([p[1] for p in parts])
    sep_lp = np.concatenate([p[2] for p in parts])
    sep_le = np.concatenate([p[3] for p in parts])
    assert nl == sum(p[0] for p in parts) and st["n_left"] == nl
    assert st["variant"] in (1, 4, 7, 8)
    a, b = np.argsort(ens[:, 6]), np.argsort(sep[:, 6])
    same = (ens[a] == sep[b]) | (np.isnan(ens[a]) & np.isnan(sep[b]))
    assert same.all(), f"{(~same).any(axis=1).sum()} particles differ"
    assert np.array_equal(lp[a], sep_lp[b]) and np.array_equal(le[a], sep_le[b])
    assert 0 < nl < sum(counts)  # the grid reaches the dynamic aperture


def test_ensemble_parity_build_vs_oracle():
    counts = [200, 150, 90]
    lats, beams = _variants(counts, cells=2)
    passes = 6
    with Tracker(0) as trk:
        trk.load(np.concatenate(beams))
        trk.track_ensemble(lats, counts, passes, PC, fast=False)
        nl, ens, lp, le = trk.store(stride=7, with_loss=True)
    rows = []
    with pyoracle.modes(exact_sums=True, cr_math=True):
        for lat, b in zip(lats, beams):
            rows.append(pyoracle.track(lat, b, passes, PC)[0])
    rows = np.concatenate(rows)
    rows = rows[np.argsort(rows[:, 7] >= 0, kind="stable")]  # survivors first, as one run returns them
    nlo = int(np.sum(rows[:, 7] < 0))
    r = compare(ens, rows, nl, nlo)
    assert r["same_survivors"] and r["bit_exact"] and r["lost_equal"], r
    o = _by_id(rows)
    lost = o[:, 7] >= 0
    gi = np.argsort(ens[:, 6])
    assert np.array_equal(lp[gi][lost], o[lost, 7].astype(np.int64))
    assert np.array_equal(le[gi][lost], o[lost, 8].astype(np.int32))


def test_autotuner_choice_is_kept_and_overridable():
    counts = [400, 400]
    lats, beams = _variants(counts, cells=2)
    with Tracker(0) as trk:
        trk.load(np.concatenate(beams))
        v1 = trk.track_ensemble(lats, counts, 3, PC)["variant"]
        trk.load(np.concatenate(beams))
        v2 = trk.track_ensemble(lats, counts, 3, PC)["variant"]
        trk.load(np.concatenate(beams))
        v3 = trk.track_ensemble(lats, counts, 3, PC, variant=4)["variant"]
    assert v1 == v2 and v1 in (1, 4, 7, 8) and v3 == 4


def test_ensemble_rejects_mixed_structures_and_wakes():
    lats, beams = _variants([10, 10], cells=2)
    other = Lattice()
    other.add("DRIF", "D", L=1.0)
    with Tracker(0) as trk:
        trk.load(np.concatenate(beams))
        with pytest.raises(TrackingError):
            trk.track_ensemble([lats[0], other], [10, 10], 1, PC)
        with pytest.raises(TrackingError):
            trk.track_ensemble([configs.c2_lattice(cells=1, n_bins=50)] * 2, [10, 10], 1, PC)
        with pytest.raises(TrackingError):
            trk.track_ensemble(lats, [10, 5], 1, PC)


@pytest.mark.parametrize("fast", [True, False])
def test_compaction_changes_no_result(fast):
    """Survivor compaction (trk_run.compact_every) only changes which lanes
    track which particles: an ensemble and a fused multi-pass run give the
    same bits with compaction every 3 passes, every 64 (the default) and
    never."""
    counts = [400, 700, 0, 250]
    lats, beams = _variants(counts)
    beam = np.concatenate(beams)
    passes = 10
    outs = []
    with Tracker(0) as trk:
        for every in (0, 3, None):
            trk.load(beam)
            st = trk.track_ensemble(lats, counts, passes, PC, fast=fast, compact_every=every)
            outs.append((st, trk.store(stride=7, with_loss=True)))
        for every in (0, 3):
            trk.load(beams[0])
            st = trk.track(lats[0], passes, PC, fast=fast, compact_every=every)
            outs.append((st, trk.store(stride=7, with_loss=True)))
    for (st_a, a), (st_b, b) in [(outs[0], outs[1]), (outs[0], outs[2]), (outs[3], outs[4])]:
        assert a[0] == b[0] and st_a["particle_passes"] == st_b["particle_passes"]
        ia, ib = np.argsort(a[1][:, 6]), np.argsort(b[1][:, 6])
        same = (a[1][ia] == b[1][ib]) | (np.isnan(a[1][ia]) & np.isnan(b[1][ib]))
        assert same.all()
        assert np.array_equal(a[2][ia], b[2][ib]) and np.array_equal(a[3][ia], b[3][ib])
    assert 0 < outs[0][1][0] < sum(counts)
