"""Long-run parity of the CUDA tracking path against elegant's own tracking
code, through the C ABI, on the benchmark configurations as configured:

  - the plain FODO ring (40 cells), 1e4 particles, 1 and 100 turns;
  - the full 40-cell ring with RF and a 2000-bin wake, 4000 particles, 1 and
    10 turns.

The fixtures (tests/golden/long_tracks.npz, tests/golden/make_long_golden.py)
were written by the reference's element functions compiled from its sources,
in its own arithmetic (glibc libm) and in the parity build's (correctly
rounded libm, double-double beam sums).

Error metric per coordinate: |gpu - ref| / max(|ref|, sigma_c), sigma_c the
rms of that coordinate over the reference's survivors.  Bounds:
  parity build vs parity arithmetic   bit-exact, same survivors, same losses;
  parity build vs glibc arithmetic    <= 1e-8 (glibc misrounds sin/cos/asin
                                      on a few calls per million and the
                                      CSBEND drift amplifies each by ~rho0/x:
                                      the reference itself moves by 3.9e-9
                                      between the two libms, after 1 turn as
                                      after 100);
  fast build vs either arithmetic     <= 1.5e-8 (measured 4.9e-9 after 1 turn
                                      and 6.3e-9 after 100 on the FODO ring).
The CPU test checks the oracle itself against the fixtures on a sample.
"""
import os

import numpy as np
import pytest

from elegant_b200 import configs
from oracle import pyoracle
from tests.helpers import by_id, gpu_run

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "long_tracks.npz")
PC = configs.P_CENTRAL
C1_N, C1_SEED, C2_N, C2_SEED = 10_000, 1, 4000, 7


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _ref(gold, ring, turns, mode):
    k = f"{ring}/turns{turns}/{mode}"
    return gold[k + "/coords"], gold[k + "/loss"], gold[k + "/meta"]


def _lattice(ring):
    return configs.c1_lattice() if ring == "c1" else configs.c2_lattice()


def _beam(ring):
    return configs.gaussian_beam(C1_N, seed=C1_SEED) if ring == "c1" else configs.gaussian_beam(C2_N, seed=C2_SEED)


def errors(g_coords, g_lost_pass, r_coords, r_loss):
    """Scaled errors per coordinate over the reference's survivors."""
    g = by_id(g_coords)
    assert np.array_equal(g[:, 6], r_coords[:, 6])
    r_alive = r_loss[:, 0] < 0
    g_alive = g_lost_pass < 0
    sig = np.std(r_coords[r_alive, :6], axis=0)
    d = np.abs(g[r_alive, :6] - r_coords[r_alive, :6])
    scale = np.maximum(np.abs(r_coords[r_alive, :6]), sig)
    return {"same_survivors": bool(np.array_equal(g_alive, r_alive)),
            "bit_exact": bool(np.array_equal(g[r_alive, :6], r_coords[r_alive, :6])),
            "max_err": float(np.max(d / scale)) if r_alive.any() else 0.0,
            "n_diff": int(np.sum(np.any(g[r_alive, :6] != r_coords[r_alive, :6], axis=1)))}


def test_oracle_matches_long_fixtures_sample(gold):
    """The oracle restatement against the reference's 100-turn FODO fixture,
    bit for bit in both arithmetics (sampled: the FODO ring's particles are
    independent, so a subset tracks like the full beam)."""
    beam = _beam("c1")[:40]
    for mode, (es, cr) in {"reference_arith": (False, False), "parity_arith": (True, True)}.items():
        with pyoracle.modes(exact_sums=es, cr_math=cr):
            rows, n_left, _ = pyoracle.track(configs.c1_lattice(), beam, 100, PC)
        want, _, _ = _ref(gold, "c1", 100, mode)
        got = by_id(rows[:, :7])
        assert np.array_equal(got, want[:40]), mode


@pytest.mark.gpu
@pytest.mark.parametrize("ring,turns", [("c1", 1), ("c1", 100), ("c2", 1), ("c2", 10)])
def test_parity_build_long(tracker, gold, ring, turns):
    nl, g, lp, le, st = gpu_run(tracker, _lattice(ring), _beam(ring), turns, PC, fast=False)
    coords, loss, meta = _ref(gold, ring, turns, "parity_arith")
    r = errors(g, lp[np.argsort(g[:, 6], kind="stable")], coords, loss)
    assert r["same_survivors"] and r["bit_exact"], r
    assert nl == meta[0] and st["particle_passes"] == meta[1]
    gi = np.argsort(g[:, 6], kind="stable")
    lost = loss[:, 0] >= 0
    assert np.array_equal(lp[gi][lost], loss[lost, 0]) and np.array_equal(le[gi][lost], loss[lost, 1])
    coords_g, loss_g, _ = _ref(gold, ring, turns, "reference_arith")
    r = errors(g, lp[gi], coords_g, loss_g)
    assert r["same_survivors"], r
    assert r["max_err"] <= 1e-8, r


@pytest.mark.gpu
@pytest.mark.parametrize("ring,turns", [("c1", 1), ("c1", 100), ("c2", 1), ("c2", 10)])
def test_fast_build_long(tracker, gold, ring, turns):
    nl, g, lp, le, st = gpu_run(tracker, _lattice(ring), _beam(ring), turns, PC, fast=True)
    coords, loss, meta = _ref(gold, ring, turns, "parity_arith")
    r = errors(g, lp[np.argsort(g[:, 6], kind="stable")], coords, loss)
    assert r["same_survivors"], r
    assert r["max_err"] <= 1.5e-8, r
