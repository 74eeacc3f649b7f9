"""Writes tests/golden/long_tracks.npz: long-run fixtures written by elegant's
own tracking code (oracle/_ref/libref.so, compiled from the reference
sources by oracle/ref/Makefile), in the reference's arithmetic (glibc libm)
and in the parity build's (correctly rounded libm, double-double sums):

  c1/turns1, c1/turns100   the plain FODO ring exactly as configured: 40
                           cells, 1e4 particles (Gaussian, seed 1), 1 and
                           100 turns;
  c2/turns1, c2/turns10    the full 40-cell ring with RF and a 2000-bin
                           wake, 4000 particles (seed 7), 1 and 10 turns.

Each entry holds the final coordinates (x, x', y, y', s, delta, id; rows
sorted by id), the loss pass and element (-1 for survivors) and
(n_left, particle_passes, turns).

    make -C oracle/ref REF=<reference tree> && python tests/golden/make_long_golden.py

The FODO ring has no collective element, so its particles are tracked in
independent shards on all host cores; the wake ring runs as one beam."""
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

MODES = {"reference_arith": (False, False), "parity_arith": (True, True)}
C1_PARTICLES, C1_SEED = 10_000, 1
C2_PARTICLES, C2_SEED = 4000, 7


def c1_beam():
    from elegant_b200 import configs
    return configs.gaussian_beam(C1_PARTICLES, seed=C1_SEED)


def c2_beam():
    from elegant_b200 import configs
    return configs.gaussian_beam(C2_PARTICLES, seed=C2_SEED)


def _job(args):
    ring, lo, hi, turns, mode = args
    sys.path.insert(0, ROOT)
    from elegant_b200 import configs
    from oracle import pyoracle
    es, cr = MODES[mode]
    if ring == "c1":
        lat, beam = configs.c1_lattice(), c1_beam()[lo:hi]
    else:
        lat, beam = configs.c2_lattice(), c2_beam()
    rows, n_left, eff = pyoracle.track_ref(lat, beam, turns, configs.P_CENTRAL, exact_sums=es, cr_math=cr)
    return args, rows, n_left, eff


def main():
    jobs = []
    shards = 16
    edges = np.linspace(0, C1_PARTICLES, shards + 1).astype(int)
    for mode in MODES:
        for turns in (1, 100):
            for k in range(shards):
                jobs.append(("c1", int(edges[k]), int(edges[k + 1]), turns, mode))
        for turns in (1, 10):
            jobs.append(("c2", 0, C2_PARTICLES, turns, mode))
    # longest first
    jobs.sort(key=lambda j: -(j[2] - j[1]) * j[3] * (3 if j[0] == "c2" else 1))
    with mp.get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        results = pool.map(_job, jobs, chunksize=1)
    parts = {}
    for (ring, lo, hi, turns, mode), rows, n_left, eff in results:
        parts.setdefault((ring, turns, mode), []).append((rows, n_left, eff))
    out = {}
    for (ring, turns, mode), lst in sorted(parts.items()):
        rows = np.concatenate([r for r, _, _ in lst])
        rows = rows[np.argsort(rows[:, 6], kind="stable")]
        key = f"{ring}/turns{turns}/{mode}"
        out[key + "/coords"] = rows[:, :7]
        out[key + "/loss"] = rows[:, 7:9].astype(np.int32)
        out[key + "/meta"] = np.array([sum(n for _, n, _ in lst), sum(e for _, _, e in lst), turns], dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, "long_tracks.npz"), **out)
    print(len(out) // 3, "long tracks written")


if __name__ == "__main__":
    main()
