"""The oracle against golden fixtures written by elegant's own tracking code
(tests/golden/make_golden.py over oracle/_ref/libref.so): bit for bit, in the
reference's arithmetic and in the parity build's.  Runs without the reference
sources."""
import os

import numpy as np
import pytest

from elegant_b200 import configs
from oracle import pyoracle
from tests.cases import ELEMENT_CASES
from tests.golden.golden_cases import ring_cases

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_tracks.npz")
MODES = {"reference_arith": (False, False), "parity_arith": (True, True)}


def _cases():
    c = {f"element_{k}": (lat, configs.gaussian_beam(24, seed=61), 2) for k, lat in ELEMENT_CASES.items()}
    c.update(ring_cases())
    return c


CASES = _cases()


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_golden(gold, name, mode):
    lat, beam, passes = CASES[name]
    es, cr = MODES[mode]
    with pyoracle.modes(exact_sums=es, cr_math=cr):
        rows, n_left, eff = pyoracle.track(lat, beam, passes, configs.P_CENTRAL)
    want = gold[f"{name}/{mode}/rows"]
    meta = gold[f"{name}/{mode}/meta"]
    assert n_left == meta[0] and eff == meta[1]
    same = (rows == want) | (np.isnan(rows) & np.isnan(want))
    assert same.all(), f"{(~same).any(axis=1).sum()} rows differ"
