"""Shared helpers for the parity tests: run the CUDA path and the oracle on
the same seeded beam and compare particle by particle (matched by id)."""
import numpy as np

from elegant_b200 import Lattice, Tracker  # noqa: F401
from oracle import pyoracle


def gpu_run(tracker, lattice, beam, n_passes, p_central, fast, pass_offset=0, variant=-1):
    tracker.load(beam)
    stats = tracker.track(lattice, n_passes, p_central, pass_offset=pass_offset, fast=fast, variant=variant)
    n_left, out, lp, le = tracker.store(stride=7, with_loss=True)
    return n_left, out, lp, le, stats


def by_id(rows):
    order = np.argsort(rows[:, 6], kind="stable")
    return rows[order]


def compare(gpu, oracle_rows, n_left_gpu, n_left_orc, sig=None):
    """Returns dict with survivor-set agreement and max scaled error over
    surviving particles: |gpu-ref| / max(|ref|, sigma_c)."""
    g_alive = set(gpu[:n_left_gpu, 6].tolist())
    o_alive = set(oracle_rows[:n_left_orc, 6].tolist())
    g = by_id(gpu[:, :7])
    o = by_id(oracle_rows[:, :7])
    assert np.array_equal(g[:, 6], o[:, 6])
    alive = np.array([i in o_alive for i in o[:, 6]])
    res = {"same_survivors": g_alive == o_alive, "n_alive": len(o_alive)}
    if sig is None:
        sig = np.maximum(np.std(o[alive, :6], axis=0), 1e-300) if alive.any() else np.ones(6)
    d = np.abs(g[alive, :6] - o[alive, :6])
    scale = np.maximum(np.abs(o[alive, :6]), sig)
    res["max_err"] = float(np.max(d / scale)) if alive.any() else 0.0
    res["bit_exact"] = bool(np.array_equal(g[alive, :6], o[alive, :6]))
    res["n_diff"] = int(np.sum(np.any(g[alive, :6] != o[alive, :6], axis=1)))
    lost = ~alive
    res["lost_equal"] = bool(np.array_equal(g[lost, :6], o[lost, :6], equal_nan=True))
    return res


def oracle_run(lattice, beam, n_passes, p_central, pass_offset=0):
    return pyoracle.track(lattice, beam, n_passes, p_central, pass_offset=pass_offset)
