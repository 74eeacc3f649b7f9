"""The sharded library path on one GPU: a one-rank NCCL communicator runs
every exchange of a sharded run (statistics all-gather and combine, histogram
all-reduce, particle-count all-reduce) and must leave the result exactly as
the unsharded path computes it.  (Runs with several ranks need one GPU per
rank; the decomposition itself is tested on CPU ranks in
test_sharded_cpu.py.)"""
import numpy as np
import pytest

import elegant_b200
from elegant_b200 import Tracker, configs
from tests.helpers import compare

pytestmark = pytest.mark.gpu
PC = configs.P_CENTRAL


def _run(lat, beam, passes, fast, comm):
    with Tracker(0) as trk:
        if comm:
            trk.set_comm(elegant_b200.nccl_unique_id(), 1, 0)
        trk.load(beam)
        st = trk.track(lat, passes, PC, fast=fast)
        nl, out, lp, le = trk.store(stride=7, with_loss=True)
    return nl, out, lp, le, st


@pytest.mark.parametrize("fast", [False, True])
def test_one_rank_comm_rf_wake(fast):
    lat = configs.c2_lattice(cells=4, n_bins=400)
    beam = configs.gaussian_beam(4000, seed=51)
    a = _run(lat, beam, 3, fast, False)
    b = _run(lat, beam, 3, fast, True)
    assert a[0] == b[0] and a[4]["particle_passes"] == b[4]["particle_passes"]
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])


def test_one_rank_comm_trwake():
    lat = configs.c1_lattice(cells=2)
    lat.add("CHARGE", "Q", TOTAL=2e-9)
    i = lat.add("TRWAKE", "TW", N_BINS=0)
    t, W = configs.resonator_wake(points=512, dt=2e-12, f_r=5e9)
    lat.set_wake(i, t, W * 1e3, W * 0.5e3)
    beam = configs.gaussian_beam(3000, seed=52)
    a = _run(lat, beam, 2, False, False)
    b = _run(lat, beam, 2, False, True)
    r = compare(b[1], np.concatenate([a[1], np.zeros((a[1].shape[0], 2))], axis=1), b[0], a[0])
    assert r["same_survivors"]
    # transverse histogram bins are FP64 atomic sums (order-dependent in the last bit)
    assert r["max_err"] < 1e-12, r
