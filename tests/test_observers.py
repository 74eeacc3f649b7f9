"""Beam observers and whole-beam steps between elements: compute_centroids,
accumulate_beam_sums, do_match_energy and the particle-ID sort.

CPU: the oracle restatement against elegant's own compute_centroids.c
(compiled from the reference sources) in both arithmetic modes.  GPU: the
library (trk_beam_centroids, trk_accumulate_beam_sums, trk_match_energy,
trk_sort_by_id) against the oracle with double-double sums (bit-exact where
the reference's sums are KahanPlus sums; the sigma sums are the reference's
in-line Kahan sums, which stay compensated sums in every mode, so they agree
to rounding), and elegant's own code driven through its GPU hooks against its
CPU build.
"""
import numpy as np
import pytest

from elegant_b200 import configs
from oracle import pyoracle

PC = configs.P_CENTRAL
SECOND = 0x8
FLAG_SETS = [SECOND, SECOND | 0x1, SECOND | 0x2, SECOND | 0x4, 0x0]


def _beam(n=3000, seed=61):
    b = configs.gaussian_beam(n, seed=seed, sigma_x=1e-3, sigma_xp=1e-4)
    b[:, 0] += 3e-4
    b[:, 5] += 2e-4
    return b


def _close(a, b, rel=1e-13):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    scale = np.maximum(np.abs(b), 1e-300)
    both_nan = np.isnan(a) & np.isnan(b)
    return bool(np.all(both_nan | (np.abs(a - b) <= rel * scale)))


def _same_sums(a, b, sigma_rel=None, second=True):
    """Equal sums; the BEAM_SUMS2 part only when it was kept."""
    da, db = pyoracle.sums_dict(a), pyoracle.sums_dict(b)
    assert np.array_equal(da["centroid"], db["centroid"]), (da["centroid"], db["centroid"])
    for k in ("n_part", "p0", "charge"):
        assert da[k] == db[k], (k, da[k], db[k])
    if not second:
        return
    for k in ("maxabs", "min", "max"):
        assert np.array_equal(da[k], db[k]), (k, da[k], db[k])
    for k in ("sigma", "sigman"):
        if sigma_rel is None:
            assert np.array_equal(da[k], db[k]), (k, da[k] - db[k])
        else:
            assert _close(da[k], db[k], sigma_rel), (k, da[k], db[k])


@pytest.mark.skipif(not pyoracle.ref_available(), reason="oracle/_ref/libref.so not built")
@pytest.mark.parametrize("exact", [False, True])
@pytest.mark.parametrize("flags", FLAG_SETS)
def test_oracle_observers_vs_reference(exact, flags):
    beam = _beam()
    c_ref, s_ref = pyoracle.observe_ref(beam, PC, mp_charge=1e-12, flags=flags, repeats=2, exact_sums=exact)
    with pyoracle.modes(exact_sums=exact, cr_math=False):
        c = pyoracle.beam_centroids(beam)
        s = pyoracle.zero_beam_sums()
        for _ in range(2):
            pyoracle.accumulate_beam_sums(beam, s, PC, 1e-12, flags=flags)
    assert np.array_equal(c, c_ref)
    _same_sums(s, s_ref, second=bool(flags & SECOND))


@pytest.mark.skipif(not pyoracle.ref_available(), reason="oracle/_ref/libref.so not built")
def test_oracle_selection_vs_reference():
    """ID window and time window of accumulate_beam_sums."""
    beam = _beam(2000, seed=62)
    t = beam[:, 4] * np.sqrt((PC * (1 + beam[:, 5])) ** 2 + 1) / (2.99792458e8 * PC * (1 + beam[:, 5]))
    t_lo, t_hi = np.quantile(t, [0.2, 0.9])
    for kw in ({"start_pid": 100, "end_pid": 900}, {"t_min": t_lo, "t_max": t_hi}):
        c_ref, s_ref = pyoracle.observe_ref(beam, PC, flags=SECOND, **kw)
        s = pyoracle.zero_beam_sums()
        pyoracle.accumulate_beam_sums(beam, s, PC, flags=SECOND, **kw)
        _same_sums(s, s_ref)
        assert 0 < s.n_part < len(beam)


def _gpu_sums(trk, beam, flags, repeats=2, **kw):
    from elegant_b200 import BeamSums
    s = BeamSums.zeroed()
    trk.load(beam)
    for _ in range(repeats):
        trk.accumulate_beam_sums(s, PC, mp_charge=1e-12, flags=flags, **kw)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("flags", FLAG_SETS)
def test_gpu_beam_sums_vs_oracle(tracker, flags):
    beam = _beam(50_000, seed=63)
    g = _gpu_sums(tracker, beam, flags)
    with pyoracle.modes(exact_sums=True, cr_math=False):
        s = pyoracle.zero_beam_sums()
        for _ in range(2):
            pyoracle.accumulate_beam_sums(beam, s, PC, 1e-12, flags=flags)
    _same_sums(g, s, sigma_rel=1e-13, second=bool(flags & SECOND))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 7, 1023, 1_000_003, 2_500_001])
def test_gpu_beam_sums_sizes(tracker, n):
    """Beams of one particle, ragged tiles and chunks, and sizes with
    several chunks per block (the chunk size follows the particle count);
    with an ID window so the ID column is staged too."""
    beam = _beam(n, seed=66)
    for kw in ({}, {"start_pid": n // 5, "end_pid": (4 * n) // 5 + 1}):
        g = _gpu_sums(tracker, beam, SECOND, repeats=1, **kw)
        with pyoracle.modes(exact_sums=True, cr_math=False):
            s = pyoracle.zero_beam_sums()
            pyoracle.accumulate_beam_sums(beam, s, PC, 1e-12, flags=SECOND, **kw)
        _same_sums(g, s, sigma_rel=1e-13)
    c, m = tracker.centroids()
    with pyoracle.modes(exact_sums=True, cr_math=False):
        assert np.array_equal(c, pyoracle.beam_centroids(beam)) and m == n


@pytest.mark.gpu
def test_gpu_observer_scratch_per_context():
    """Observer scratch belongs to its context: several contexts created,
    used side by side on beams of different sizes, and destroyed, give the
    oracle's sums every time and give their device memory back."""
    import torch
    from elegant_b200 import BeamSums, Tracker
    beams = [_beam(n, seed=67 + n % 5) for n in (30_000, 7_001, 120_000)]
    with pyoracle.modes(exact_sums=True, cr_math=False):
        want = []
        for b in beams:
            s = pyoracle.zero_beam_sums()
            pyoracle.accumulate_beam_sums(b, s, PC, 1e-12, flags=SECOND)
            want.append(s)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):
        trks = [Tracker(0) for _ in beams]
        try:
            for trk, b in zip(trks, beams):
                trk.load(b)
            for _ in range(2):
                for trk, w in zip(trks, want):
                    g = BeamSums.zeroed()
                    trk.accumulate_beam_sums(g, PC, mp_charge=1e-12, flags=SECOND)
                    _same_sums(g, w, sigma_rel=1e-13)
                    trk.sort_by_id()
        finally:
            for trk in trks:
                trk.close()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(0)[0]
    assert free0 - free1 < 64 << 20, (free0, free1)


@pytest.mark.gpu
def test_gpu_beam_sums_selection_and_losses(tracker):
    """ID and time windows; lost particles are left out."""
    beam = _beam(20_000, seed=64)
    lat = configs.c1_lattice(cells=1)
    lat.elements.insert(0, ["MAXAMP", "AP", {"X_MAX": 1.5e-3, "Y_MAX": 1.5e-3, "ELLIPTICAL": 1.0}, None])
    tracker.load(beam)
    tracker.track(lat, 1, PC, fast=False)
    n_left, rows = tracker.store()
    survivors = rows[:n_left]
    assert 0 < n_left < len(beam)
    t = survivors[:, 4] * np.sqrt((PC * (1 + survivors[:, 5])) ** 2 + 1) / (2.99792458e8 * PC * (1 + survivors[:, 5]))
    t_lo, t_hi = np.quantile(t, [0.1, 0.8])
    for kw in ({}, {"start_pid": 3000, "end_pid": 15000}, {"t_min": t_lo, "t_max": t_hi}):
        from elegant_b200 import BeamSums
        g = BeamSums.zeroed()
        tracker.accumulate_beam_sums(g, PC, flags=SECOND, **kw)
        with pyoracle.modes(exact_sums=True, cr_math=False):
            s = pyoracle.zero_beam_sums()
            pyoracle.accumulate_beam_sums(survivors, s, PC, flags=SECOND, **kw)
        _same_sums(g, s, sigma_rel=1e-13)
    c, n = tracker.centroids()
    with pyoracle.modes(exact_sums=True, cr_math=False):
        assert np.array_equal(c, pyoracle.beam_centroids(survivors)) and n == n_left


@pytest.mark.gpu
@pytest.mark.parametrize("change_beam", [0, 1])
def test_gpu_match_energy_vs_oracle(tracker, change_beam):
    beam = _beam(30_000, seed=65)
    tracker.load(beam)
    pc = tracker.match_energy(PC, change_beam)
    n, out = tracker.store()
    with pyoracle.modes(exact_sums=True, cr_math=False):
        ref, pc_ref = pyoracle.match_energy(beam, PC, change_beam)
    assert pc == pc_ref and (pc != PC) == (change_beam == 0)
    a, b = out[np.argsort(out[:, 6])], ref[np.argsort(ref[:, 6])]
    assert np.array_equal(a[:, :7], b[:, :7])


@pytest.mark.gpu
def test_gpu_sort_by_id(tracker):
    """Survivors in increasing ID, lost particles after them in their order."""
    rng = np.random.Generator(np.random.Philox(66))
    beam = _beam(10_000, seed=66)
    beam = beam[rng.permutation(len(beam))]
    lat = configs.c1_lattice(cells=1)
    lat.elements.insert(0, ["MAXAMP", "AP", {"X_MAX": 1.5e-3, "Y_MAX": 1.5e-3, "ELLIPTICAL": 1.0}, None])
    tracker.load(beam)
    tracker.track(lat, 1, PC, fast=False)
    n0, before, lp0, le0 = tracker.store(with_loss=True)
    tracker.sort_by_id()
    n1, after, lp1, le1 = tracker.store(with_loss=True)
    assert n0 == n1
    order = np.argsort(before[:n0, 6], kind="stable")
    assert np.array_equal(after[:n1], before[:n0][order])
    assert np.array_equal(after[n1:], before[n0:]) and np.array_equal(lp1[n1:], lp0[n0:])
    assert np.all(np.diff(after[:n1, 6]) > 0)


@pytest.mark.gpu
@pytest.mark.skipif(not pyoracle.ref_available(), reason="oracle/_ref/libref.so not built")
@pytest.mark.parametrize("flags", [SECOND, SECOND | 0x4, 0x0])
def test_hooks_observers_vs_reference_cpu(tracker, flags):
    """elegant's compute_centroids.c built with HAVE_GPU (its observers call
    gpu_compute_centroids / gpu_accumulate_beam_sums, i.e. the library) against
    the same file built for the CPU with double-double KahanPlus."""
    beam = _beam(5000, seed=67)
    c_gpu, s_gpu = pyoracle.observe_refgpu(beam, PC, mp_charge=1e-12, flags=flags, repeats=2)
    c_cpu, s_cpu = pyoracle.observe_ref(beam, PC, mp_charge=1e-12, flags=flags, repeats=2, exact_sums=True)
    assert np.array_equal(c_gpu, c_cpu)
    _same_sums(s_gpu, s_cpu, sigma_rel=1e-13, second=bool(flags & SECOND))
