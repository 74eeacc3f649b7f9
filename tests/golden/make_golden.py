"""Writes tests/golden/reference_tracks.npz: final coordinates, loss pass and
loss element of small seeded beams tracked by elegant's own tracking code
(oracle/_ref/libref.so, compiled from the reference sources by
oracle/ref/Makefile), in the reference's arithmetic and in the parity
build's (correctly rounded libm, double-double sums).

    make -C oracle/ref REF=<reference tree> && python tests/golden/make_golden.py

The fixtures let the oracle be checked against the reference where the
reference sources (and so libref.so) are not available."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from elegant_b200 import configs  # noqa: E402
from oracle import pyoracle  # noqa: E402
from tests.cases import ELEMENT_CASES  # noqa: E402
from tests.golden.golden_cases import ring_cases  # noqa: E402

MODES = {"reference_arith": (False, False), "parity_arith": (True, True)}


def main():
    out = {}
    cases = {f"element_{k}": (lat, configs.gaussian_beam(24, seed=61), 2) for k, lat in ELEMENT_CASES.items()}
    cases.update(ring_cases())
    for name, (lat, beam, passes) in sorted(cases.items()):
        for mode, (es, cr) in MODES.items():
            rows, n_left, eff = pyoracle.track_ref(lat, beam, passes, configs.P_CENTRAL, exact_sums=es, cr_math=cr)
            out[f"{name}/{mode}/rows"] = rows
            out[f"{name}/{mode}/meta"] = np.array([n_left, eff, passes], dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, "reference_tracks.npz"), **out)
    print(len(out) // 2, "tracks written")


if __name__ == "__main__":
    main()
