"""The multi-GPU decomposition, tested on CPU ranks (gloo, world size 2).

Each rank tracks its own contiguous block of particle IDs with the oracle,
exchanging only what the sharded library exchanges over NCCL: the beam time
statistics of WAKE/TRWAKE and of the first-pass RF fiducial (gathered and
combined in rank order), the wake histograms (summed) and the CHARGE
particle count (summed).  With double-double beam sums the sharded result
must equal the single-process result bit for bit, for every particle,
survivor and loss record, whatever the split -- including a rank whose shard
is empty.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _lattice(kind):
    from elegant_b200 import configs
    if kind == "rf_wake":
        return configs.c2_lattice(cells=2, n_bins=300)
    lat = configs.c1_lattice(cells=2)
    lat.add("CHARGE", "Q", TOTAL=2e-9)
    i = lat.add("TRWAKE", "TW", N_BINS=0)
    t, W = configs.resonator_wake(points=512, dt=2e-12, f_r=5e9)
    lat.set_wake(i, t, W * 1e3, W * 0.5e3)
    lat.add("WAKE", "LW", N_BINS=0, CHARGE=1e-9)
    lat.set_wake(len(lat.elements) - 1, t, W)
    return lat


def _beam(n):
    from elegant_b200 import configs
    b = configs.gaussian_beam(n, seed=41, sigma_x=1.5e-3, sigma_xp=1.5e-4)
    return b


def _rank_main(rank, world, port, kind, n, split, passes, out_dir):
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    from elegant_b200 import configs
    from oracle import pyoracle
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        def gather(send):
            t = torch.from_numpy(send)
            out = [torch.empty_like(t) for _ in range(world)]
            dist.all_gather(out, t)
            return torch.cat(out).numpy()

        def allsum(buf):
            t = torch.from_numpy(buf)
            dist.all_reduce(t)
            return t.numpy()

        beam = _beam(n)
        lo, hi = (0, split) if rank == 0 else (split, n)
        pyoracle.set_collective(world, gather, allsum)
        with pyoracle.modes(exact_sums=True, cr_math=True):
            rows, n_left, eff = pyoracle.track(_lattice(kind), beam[lo:hi], passes, configs.P_CENTRAL)
        pyoracle.set_collective(1)
        np.save(os.path.join(out_dir, f"rows{rank}.npy"), rows)
        np.save(os.path.join(out_dir, f"meta{rank}.npy"), np.array([n_left, eff]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind,split", [("rf_wake", 700), ("rf_wake", 0), ("trwake", 333)])
def test_sharded_equals_single_process(tmp_path, kind, split):
    from elegant_b200 import configs
    from oracle import pyoracle
    n, passes, world = 1200, 3, 2
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, port, kind, n, split, passes, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    rows = np.concatenate([np.load(tmp_path / f"rows{r}.npy") for r in range(world)])
    meta = sum(np.load(tmp_path / f"meta{r}.npy") for r in range(world))
    with pyoracle.modes(exact_sums=True, cr_math=True):
        ref, n_left, eff = pyoracle.track(_lattice(kind), _beam(n), passes, configs.P_CENTRAL)
    assert meta[0] == n_left and meta[1] == eff
    a = rows[np.argsort(rows[:, 6])]
    b = ref[np.argsort(ref[:, 6])]
    assert np.array_equal(a[:, 6:], b[:, 6:])  # ids, loss pass, loss element
    if kind == "trwake":
        # the transverse histograms hold FP64 sums of positions: per-rank
        # partial sums added in rank order round differently from one
        # sequential sum, so kicks agree to rounding only
        alive = b[:, 7] < 0
        sig = np.std(b[alive, :6], axis=0)
        err = np.abs(a[alive, :6] - b[alive, :6]) / np.maximum(np.abs(b[alive, :6]), sig)
        assert err.max() < 1e-12, err.max()
        return
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    assert same.all(), f"{(~same).any(axis=1).sum()} particles differ"
