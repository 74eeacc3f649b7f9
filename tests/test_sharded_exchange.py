"""The library's own sharded path at world size 2, with its exchanges run
through the host-exchange communicator (trk_context_set_exchange) backed by
gloo collectives on CPU tensors.

Two processes share one GPU, each driving its own context over its own block
of particle IDs; every exchange goes device -> host -> gloo -> host ->
device between kernel launches (no kernel waits on the other rank).  This
runs the rank-order combine of the gathered beam statistics
(stats_combine_kernel), the histogram sums and the particle-count sum with
two ranks, which the one-rank NCCL test cannot.  The sharded result must
equal the unsharded run bit for bit: every particle, survivor and loss
record, for an uneven split and for a split with an empty shard (TRWAKE,
whose transverse histogram is an FP64 atomic sum, to 1e-12).
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _lattice(ring):
    from elegant_b200 import configs
    lat = configs.c2_lattice(cells=3, n_bins=400)
    if ring == "trwake":
        i = lat.add("TRWAKE", "TW", N_BINS=0)
        t, W = configs.resonator_wake(points=512, dt=2e-12, f_r=5e9)
        lat.set_wake(i, t, W * 1e3, W * 0.5e3)
    return lat


def _beam(n):
    from elegant_b200 import configs
    return configs.gaussian_beam(n, seed=47, sigma_x=1.5e-3, sigma_xp=1.5e-4)


def _rank_main(rank, world, port, ring, n, split, passes, fast, out_dir):
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    from elegant_b200 import Tracker, configs
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        def sum_f64(a):
            t = torch.from_numpy(a)
            dist.all_reduce(t)

        def sum_i64(a):
            t = torch.from_numpy(a.view(np.int64))
            dist.all_reduce(t)

        def gather_f64(send, recv):
            t = torch.from_numpy(send.copy())
            parts = [torch.empty_like(t) for _ in range(world)]
            dist.all_gather(parts, t)
            recv[:] = torch.cat(parts).numpy()

        beam = _beam(n)
        lo, hi = (0, split) if rank == 0 else (split, n)
        with Tracker(0) as trk:
            trk.set_exchange(sum_f64, sum_i64, sum_i64, gather_f64, world, rank)
            trk.load(beam[lo:hi])
            st = trk.track(_lattice(ring), passes, configs.P_CENTRAL, fast=fast)
            nl, out, lp, le = trk.store(stride=7, with_loss=True)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), out=out, lp=lp, le=le, nl=nl,
                 eff=st["particle_passes"])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ring,split,fast", [("rf_wake", 1300, False), ("rf_wake", 3000, False),
                                             ("rf_wake", 1300, True), ("trwake", 1300, False)])
def test_two_rank_exchange_equals_unsharded(tmp_path, ring, split, fast):
    from elegant_b200 import Tracker, configs
    n, passes = 3000, 3
    mp.start_processes(_rank_main, args=(2, _free_port(), ring, n, split, passes, fast, str(tmp_path)), nprocs=2,
                       join=True, start_method="spawn")
    with Tracker(0) as trk:
        trk.load(_beam(n))
        st = trk.track(_lattice(ring), passes, configs.P_CENTRAL, fast=fast)
        nl, ref, rlp, rle = trk.store(stride=7, with_loss=True)
    parts = [np.load(os.path.join(tmp_path, f"rank{r}.npz")) for r in range(2)]
    out = np.concatenate([p["out"] for p in parts])
    lp = np.concatenate([p["lp"] for p in parts])
    le = np.concatenate([p["le"] for p in parts])
    assert sum(int(p["nl"]) for p in parts) == nl
    assert sum(int(p["eff"]) for p in parts) == st["particle_passes"]
    a, b = np.argsort(out[:, 6]), np.argsort(ref[:, 6])
    assert np.array_equal(lp[a], rlp[b]) and np.array_equal(le[a], rle[b])
    if ring == "trwake":
        # the transverse histogram is summed with FP64 atomics (order-dependent in the last bit):
        # |sharded - unsharded| / max(|unsharded|, sigma) per coordinate
        alive = rlp[b] < 0
        g, r = out[a][alive, :6], ref[b][alive, :6]
        sig = np.std(r, axis=0)
        assert np.max(np.abs(g - r) / np.maximum(np.abs(r), sig)) < 1e-12
    else:
        same = (out[a] == ref[b]) | (np.isnan(out[a]) & np.isnan(ref[b]))
        assert same.all(), f"{(~same).any(axis=1).sum()} particles differ"
