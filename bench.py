"""Benchmark: FP64 particle-turns/s of elegant's tracking path on B200.

Workload: the ring with RF and longitudinal wake (40 FODO cells with KQUAD,
KSEXT, CSBEND, DRIF, one RFCA and one WAKE with a 4096-point resonator Green
function on 2000 bins, CHARGE 1 nC), 1e6 particles from a seeded Gaussian
beam.  One step is one pass (turn) of the whole beam.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--build both|parity|fast]

Two builds of one kernel source are timed in the same run:
  parity (the headline `value`): the reference's operation sequence without
        FMA contraction and with correctly rounded sin/cos/asin; bit-exact
        with elegant's own tracking code run with a correctly rounded libm;
  fast (`fast_build`): FMA contraction and transcendental-free CSBEND and
        multipole bodies; within a few 1e-8 of the reference after one turn.
Each carries `accuracy`: its measured error against elegant's own tracking
code on the benchmark rings as configured (committed fixtures written by the
reference: 1e4 particles x 1 and 100 turns of the FODO ring, 4000 particles x
1 and 10 turns of this ring).

value : particle-turns/s with the beam resident on the device; each step is
        timed with CUDA events on the tracking stream, the L2 is flushed
        (a 512 MiB write) between timed steps and outside their events.
e2e   : the same metric through the C ABI with host buffers: each step loads
        the beam from pinned host memory, tracks one turn and stores it back.
roofline: FP64 bound; achieved = algorithmic FP64 flops per particle-turn
        (counted on the reference formulation, oracle/flops.json) times
        particle-turns/s, against the FP64 peak measured in this run by a
        dependent-FMA kernel (MEASURED_PEAKS.json has no FP64 figure).
--impl reference: elegant's own tracking code compiled from the reference
        sources (oracle/_ref/libref.so; the oracle restatement where that
        was not built) on all host cores, process-parallel by particle
        shards.
--workload c5: the large ring (40 multi-bend-achromat cells of combined-
        function CSBENDs, KQUADs, KSEXTs and KOCTs, with RFCA, WAKE and
        TRWAKE on 4000 bins), 1e7 particles, same metric and keys.
Multi-GPU: one process per GPU; each rank tracks its own particle shard of
1e6 particles (weak scaling); the library's NCCL communicator exchanges the
beam time statistics (all-gather) and the wake histogram (all-reduce) at the
WAKE element of every turn, the RF fiducial statistics on the first pass.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_PARTICLES = 1_000_000
# DRAM bytes per particle of one tracking-kernel launch: 10.63 MB read + 1.8 KB
# written at 2e5 particles (ncu; the coordinate writes stay in L2 and are
# written back during later kernels)
TRACK_DRAM_BYTES_PER_PARTICLE = 10.628e6 / 2e5
# the same for the MBA ring: 110.67 MB read + 120.53 MB written at 2e6 particles (ncu)
TRACK_DRAM_BYTES_PER_PARTICLE_C5 = (110.67e6 + 120.53e6) / 2e6

WORKLOADS = {
    "c1": {"workload": "ring_fodo40_1e6", "particles": 1_000_000,
           "lattice": "40 FODO cells (KQUAD, CSBEND, DRIF)"},
    "c2": {"workload": "ring_rf_wake_fodo40_1e6", "particles": 1_000_000,
           "lattice": "40 FODO cells + KSEXT, RFCA, WAKE", "wake_bins": 2000, "wake_points": 4096,
           "wake_dt_s": 5e-14, "charge_c": 1e-9},
    "rad": {"workload": "ring_rf_wake_fodo40_radiation_1e6", "particles": 1_000_000,
            "lattice": "40 FODO cells + KSEXT, RFCA, WAKE; SYNCH_RAD=1 and ISR=1 on every KQUAD, KSEXT, CSBEND",
            "wake_bins": 2000, "wake_points": 4096, "wake_dt_s": 5e-14, "charge_c": 1e-9},
    "c5": {"workload": "mba_ring_rf_wake_trwake_1e7", "particles": 10_000_000,
           "lattice": "40 MBA cells (7 CSBEND K1 N_KICKS=32, 12 KQUAD, 6 KSEXT, 2 KOCT, 27 DRIF) + RFCA, WAKE, "
                      "TRWAKE", "wake_bins": 4000, "wake_points": 4096, "wake_dt_s": 2.5e-13, "charge_c": 1e-9,
           "sigma_x_m": 30e-6},
}


def workload_config(n_particles, workload="c2"):
    cfg = dict(WORKLOADS[workload])
    del cfg["particles"]
    cfg.update({"particles_per_gpu": n_particles, "p_central": 13700.0, "l2": "flushed between timed steps"})
    return cfg


def workload_lattice(workload):
    from elegant_b200 import configs
    if workload == "rad":
        lat = configs.c2_lattice()
        for e in lat.elements:
            if e[0] in ("KQUAD", "KSEXT", "CSBEND"):
                e[2]["SYNCH_RAD"] = 1.0
                e[2]["ISR"] = 1.0
        return lat
    return {"c1": configs.c1_lattice, "c2": configs.c2_lattice, "c5": configs.c5_lattice}[workload]()


def workload_beam(workload, n, seed=1, first_id=1):
    from elegant_b200 import configs
    if workload == "c5":
        return configs.c5_beam(n, seed=seed, first_id=first_id)
    return configs.gaussian_beam(n, seed=seed, first_id=first_id)


def load_flops():
    p = os.path.join(ROOT, "oracle", "flops.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            for k, n in enumerate(names):
                if len(s) > 4 + k and s[4 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def _cpu_tracker():
    """elegant's own tracking code (oracle/_ref/libref.so, built from the
    reference sources) when present, else the oracle restatement."""
    from oracle import pyoracle
    if pyoracle.ref_available():
        return pyoracle.track_ref, "reference"
    pyoracle.load()
    return pyoracle.track, "port"


def cpu_baseline(cores=None, sample_particles=6000, sample_turns=3, workload="c2"):
    """Time the CPU tracking path on the host: particle-turns/s on a bounded
    sample of the benchmark ring (same lattice, same beam distribution)."""
    if cores is None:
        cores = 1
    if cores == 1:
        note = ""
        if workload == "rad":
            # the reference's ISR deviates come from the SDDS toolkit's generator, which is not in the
            # reference tree: its compiled code stops at them, so the radiating ring is timed on the oracle
            # restatement, which draws the library's deviates
            from oracle import pyoracle
            pyoracle.load()
            pyoracle.set_isr_seed(20261203)
            track, kind = pyoracle.track, "port"
            note = " (the oracle restatement: the reference's ISR generator is not in its tree)"
        else:
            track, kind = _cpu_tracker()
        lat = workload_lattice(workload)
        beam = workload_beam(workload, sample_particles, seed=1)
        t0 = time.perf_counter()
        _, _, eff = track(lat, beam, sample_turns, 13700.0)
        dt = time.perf_counter() - t0
        return {"value": eff / dt, "unit": "particle-turns/s", "cores": 1, "kind": kind,
                "sample": f"{sample_particles} particles x {sample_turns} turns of the same lattice, 1 core" + note}
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    per = sample_particles
    with ctx.Pool(cores) as pool:
        args = [(per, sample_turns, 1 + k, workload) for k in range(cores)]
        kinds = pool.map(_oracle_shard, [(10, 1, 99, workload)] * cores)  # warm the workers
        res = pool.map(_oracle_shard, args)
        dt = max(r[2] for r in res)
    return {"value": sum(r[0] for r in res) / dt, "unit": "particle-turns/s", "cores": cores, "kind": kinds[0][1],
            "sample": f"{cores} processes x {per} particles x {sample_turns} turns (particle shards; wake "
                      "histograms per shard)"}


def _oracle_shard(args):
    """One shard of the CPU leg: builds its lattice and beam, then times the
    tracking call alone.  Returns (particle-turns, kind, seconds)."""
    n, turns, seed, workload = args
    sys.path.insert(0, ROOT)
    track, kind = _cpu_tracker()
    lat = workload_lattice(workload)
    beam = workload_beam(workload, n, seed=seed)
    t0 = time.perf_counter()
    _, _, eff = track(lat, beam, turns, 13700.0)
    return eff, kind, time.perf_counter() - t0


def run_reference(args, rank, world):
    """The reference arm: the CPU tracking path on all host cores (one
    process per core, particle shards), each step a bounded sample of the
    benchmark ring; rank 0 only.  Each shard times its own tracking call
    (lattice and beam set-up outside the timed region); a step's time is the
    slowest shard's.  Shards run elegant's serial build, which bins and
    convolves its own wake histogram (Pelegant would sum the shards'
    histograms with one MPI_Allreduce per wake, src/wake.c:226-233; the
    work per shard is the same)."""
    if rank != 0:
        return 0
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    workload = args.workload if args.workload in ("c1", "c5") else "c2"
    per, turns = (100 if workload == "c5" else 1000), 1
    steps = []
    with mp.get_context("spawn").Pool(cores) as pool:
        kind = pool.map(_oracle_shard, [(10, 1, 99, workload)] * cores)[0][1]
        for k in range(args.warmup + args.steps):
            res = pool.map(_oracle_shard, [(per, turns, 1 + c, workload) for c in range(cores)])
            dt = max(r[2] for r in res)
            if k >= args.warmup:
                steps.append(sum(r[0] for r in res) / dt)
    v = float(np.mean(steps))
    sample = (f"{cores} processes x {per} particles x {turns} turn of the same ring per step (particle shards; "
              "wake histograms per shard); tracking calls timed, set-up excluded")
    line = {"metric": "particle-turns/s", "value": v, "unit": "particle-turns/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Gaussian beam)",
            "config": workload_config(WORKLOADS[workload]["particles"], workload), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "particle-turns/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": v, "unit": "particle-turns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--particles", type=int, default=None,
                    help="particles per GPU (1e6 for c1/c2, 1e7 for c5, 1e5 for c4)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--exact", action="store_true", help="the parity build alone (same as --build parity)")
    ap.add_argument("--build", default="both", choices=["both", "parity", "fast"],
                    help="both: the parity build (bit-exact with the reference's arithmetic under a correctly "
                         "rounded libm) is the headline value and the fast build is reported beside it")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5", "c5grad", "rad", "observe",
                                                       "da"],
                    help="c2: ring with RF and wake (the benchmark); c1: plain FODO ring (profiling); "
                         "c5: large MBA ring with RF, WAKE and TRWAKE, 1e7 particles; c5grad: batched "
                         "adjoint over 32 error seeds of the MBA ring against finite differences; rad: c2 with "
                         "SYNCH_RAD and ISR on every magnet; observe: beam sums of 1e7 particles (HBM); da: "
                         "dynamic-aperture line search over 256 error seeds; "
                         "c3: batched error-seed ensemble on dynamic-aperture grids; c4: adjoint gradient "
                         "against finite differences")
    ap.add_argument("--variants", type=int, default=256, help="c3: lattice variants")
    ap.add_argument("--turns", type=int, default=None, help="c3: 1024, c4: 64, c5grad: 8 unless given")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "c3":
        return run_ensemble(args, rank)
    if args.workload == "c4":
        return run_gradient(args, rank)
    if args.workload == "c5grad":
        return run_gradient_ensemble(args, rank)
    if args.workload == "observe":
        return run_observe(args, rank)
    if args.workload == "da":
        return run_da(args, rank)
    return run_gpu(args, rank, world, local)


def _ensemble_cpu_shard(args):
    """One variant of the ensemble on the CPU (reference code): a sample of
    its dynamic-aperture grid, tracked `turns` turns; the tracking call
    alone is timed.  Returns (particle-turns, kind, seconds)."""
    v, n, turns = args
    sys.path.insert(0, ROOT)
    from elegant_b200 import configs
    track, kind = _cpu_tracker()
    lat = configs.c3_variant(seed=v)
    beam = configs.da_grid(n)
    t0 = time.perf_counter()
    _, _, eff = track(lat, beam, turns, configs.P_CENTRAL)
    return eff, kind, time.perf_counter() - t0


def ensemble_cpu_baseline(variants=16, per_variant=256, turns=8):
    """The ensemble's CPU baseline: `variants` error seeds, each a sample of
    `per_variant` points of its grid tracked `turns` turns by the
    reference's code, one process per variant on the host cores; the
    slowest process's tracking time is the step time."""
    import multiprocessing as mp
    cores = min(os.cpu_count() or 1, variants)
    with mp.get_context("spawn").Pool(cores) as pool:
        pool.map(_ensemble_cpu_shard, [(0, 8, 1)] * cores)  # warm the workers
        res = pool.map(_ensemble_cpu_shard, [(v, per_variant, turns) for v in range(variants)])
    # variants run `variants / cores` rounds deep on `cores` processes: the
    # time is the summed work over the cores
    dt = sum(r[2] for r in res) / cores
    return {"value": sum(r[0] for r in res) / dt, "unit": "particle-turns/s", "cores": cores, "kind": res[0][1],
            "sample": f"{variants} error seeds x {per_variant} grid points x {turns} turns of the same ring "
                      f"(one process per seed on {cores} cores)"}


def run_ensemble(args, rank):
    """Batched ensemble: `variants` error seeds of the FODO+sextupole ring
    (rms dK1/K1 = 1e-3, dK2/K2 = 2e-3, 25 mm circular aperture), each with a
    dynamic-aperture grid of U{1000..65536} particles (x in +-20 mm, y in
    0..10 mm, delta = 0), all turns in one trk_track_ensemble call
    (graph-captured, autotuned launch shape, survivors compacted every 64
    passes).  Metric: particle-turns/s of the whole ensemble."""
    import torch
    from elegant_b200 import Tracker, configs
    if rank != 0:
        return 0
    torch.cuda.set_device(0)
    turns = args.turns or 1024
    rng = np.random.Generator(np.random.Philox(3))
    counts = rng.integers(1000, 65537, args.variants)
    lats = [configs.c3_variant(seed=v) for v in range(args.variants)]
    first, beams = 1, []
    for n in counts:
        beams.append(configs.da_grid(int(n), first_id=first))
        first += int(n)
    beam = np.concatenate(beams)
    fast = args.build != "parity" and not args.exact  # the fast build unless the parity build is asked for
    with Tracker(0) as trk:
        trk.load(beam)
        trk.track_ensemble(lats, counts, 4, configs.P_CENTRAL, fast=fast)  # autotunes
        trk.load(beam)
        torch.cuda.synchronize()
        with ClockSampler(0) as clocks:
            t0 = time.perf_counter()
            st = trk.track_ensemble(lats, counts, turns, configs.P_CENTRAL, fast=fast)
            wall = time.perf_counter() - t0
    value = st["particle_passes"] / (st["device_ms"] / 1e3)
    flops = load_flops()
    roof = None
    if flops:
        per = flops["per_particle"]
        fpt = flops["flops_per_particle_turn"]["c2"] - per["RFCA_L0"]["total"] - per["WAKE"]["total"]
        peak = measure_fp64_peak(0)
        achieved = fpt * value / 1e12
        roof = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if peak else None, "traffic": None, "flops_per_particle_turn": fpt,
                "kernel": "track_kernel (ensemble graph, compaction kernels included in the time)",
                "peak_source": "FP64 FMA peak measured in this run (independent dependent-FMA chains)"}
    cpu = None if args.no_cpu_baseline else ensemble_cpu_baseline()
    line = {"metric": "particle-turns/s", "value": value, "unit": "particle-turns/s", "n_gpus": 1, "steps": turns,
            "warmup": 4, "ms_per_step": st["device_ms"] / turns, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded error seeds, dynamic-aperture grids)",
            "config": {"workload": "ensemble_c3", "variants": args.variants, "particles": int(counts.sum()),
                       "turns": turns, "aperture_m": 0.025, "survivors": st["n_left"], "compact_every": 64},
            "build": "fast" if fast else "parity", "wall_s": wall, "launch_shape": st["variant"],
            "tuned_by": "autotuner", "gpu_launches": st["kernel_launches"], "roofline": roof, "cpu_baseline": cpu,
            "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)
    return 0


def _ref_fd_shard(args):
    """Central differences of the loss by elegant's own tracking code for a
    few parameters of the reduced gradient problem; returns (parameter
    indices, derivatives, seconds spent tracking)."""
    pidx, n, turns, w = args
    sys.path.insert(0, ROOT)
    from elegant_b200 import configs
    from elegant_b200.adjoint import fd_step, get_parameters, parameter_list, set_parameters
    track, _ = _cpu_tracker()
    lat = configs.c2_lattice(with_rf=False, with_wake=False)
    beam = configs.gaussian_beam(n, seed=5)
    k0 = get_parameters(lat)
    names = [nm for _, nm in parameter_list(lat)]
    out, dt = [], 0.0
    for p in pidx:
        # 1e-5 relative: the reference's CSBEND drift (X = rho0 (f - 1) + f X)
        # turns each rounding of cos() into ~rho0 2^-53 of x, noise that swamps
        # a 1e-7 step in its loss; the truncation error at 1e-5 is ~1e-10
        h = fd_step(names[p], k0[p], rel=1e-5)
        vals = []
        for sgn in (1, -1):
            k = k0.copy()
            k[p] += sgn * h
            set_parameters(lat, k)
            t0 = time.perf_counter()
            rows, n_left, _ = track(lat, beam, turns, configs.P_CENTRAL)
            dt += time.perf_counter() - t0
            alive = rows[:, 7] < 0
            x, y = rows[alive, 0], rows[alive, 2]
            vals.append(np.mean(x * x + y * y) + w * (np.mean(x) ** 2 + np.mean(y) ** 2))
        out.append((vals[0] - vals[1]) / (2 * h))
    return list(pidx), out, dt


def run_gradient(args, rank):
    """Gradient of mean(x^2 + y^2) + (mean x)^2 + (mean y)^2 after `turns`
    turns of 1e5 particles (the FODO configuration's Gaussian beam) on the
    FODO+sextupole ring (RF and wake off) with respect to every KQUAD K1,
    KSEXT K2 and CSBEND K1 and K2 (80 + 80 + 2 x 80: 160 K1 and 160 K2): the
    reverse-mode adjoint against central finite differences (h = 1e-7
    relative, 1e-7 x 1 m^-2 / 10 m^-3 absolute for the bends' zero K1, K2)
    with the same GPU tracking.  Metric: finite-difference time over adjoint
    time.  Also: the same gradient on a reduced problem (1e3 particles, 8
    turns) against central differences of elegant's own tracking code for
    16 sampled parameters, timed on the host cores."""
    import torch
    from elegant_b200 import Tracker, configs
    from elegant_b200.adjoint import fd_step, get_parameters, parameter_list, set_parameters
    if rank != 0:
        return 0
    torch.cuda.set_device(0)
    turns = args.turns or 64
    n = min(args.particles or 100_000, 100_000)
    lat = configs.c2_lattice(with_rf=False, with_wake=False)
    beam = configs.gaussian_beam(n, seed=5)  # the FODO configuration's beam (x, y 100 um; x', y' 10 urad)
    w = 1.0
    k0 = get_parameters(lat)
    names = [nm for _, nm in parameter_list(lat)]
    with Tracker(0) as trk:
        for _ in range(max(args.warmup, 1)):
            trk.load(beam)
            trk.adjoint(lat, turns, configs.P_CENTRAL, w)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        trk.load(beam)
        loss, grad = trk.adjoint(lat, turns, configs.P_CENTRAL, w)
        torch.cuda.synchronize()
        t_adj = time.perf_counter() - t0
        fd = np.zeros_like(k0)
        t0 = time.perf_counter()
        for p in range(len(k0)):
            h = fd_step(names[p], k0[p])
            vals = []
            for sgn in (1, -1):
                k = k0.copy()
                k[p] += sgn * h
                set_parameters(lat, k)
                trk.load(beam)
                trk.track(lat, turns, configs.P_CENTRAL)
                vals.append(trk.objective(w))
            fd[p] = (vals[0] - vals[1]) / (2 * h)
        torch.cuda.synchronize()
        t_fd = time.perf_counter() - t0
        set_parameters(lat, k0)
        # the reduced problem for the comparison with the reference's own differences
        rn, rturns = 1000, 8
        small = configs.gaussian_beam(rn, seed=5)
        trk.load(small)
        _, grad_small = trk.adjoint(lat, rturns, configs.P_CENTRAL, w)
    # the gradient error: max |adjoint - FD| over max |FD| (the relative error
    # of the gradient vector in the max norm); component-wise with a floor at
    # 1e-3 of the largest component for information
    err = float(np.max(np.abs(grad - fd)) / np.max(np.abs(fd)))
    scale = np.maximum(np.abs(fd), 1e-3 * np.max(np.abs(fd)))
    err_c = float(np.max(np.abs(grad - fd) / scale))
    is_k1 = np.array([nm == "K1" for nm in names])
    ref = None
    if not args.no_cpu_baseline:
        import multiprocessing as mp
        sample = np.unique(np.linspace(0, len(k0) - 1, 16).astype(int))
        cores = min(os.cpu_count() or 1, len(sample))
        chunks = [sample[c::cores] for c in range(cores)]
        t0 = time.perf_counter()
        with mp.get_context("spawn").Pool(cores) as pool:
            res = pool.map(_ref_fd_shard, [(list(ch), rn, rturns, w) for ch in chunks])
        wall = time.perf_counter() - t0
        ref_fd = np.zeros(len(sample))
        pos = {p: j for j, p in enumerate(sample)}
        for pidx, vals, _ in res:
            for p, v in zip(pidx, vals):
                ref_fd[pos[p]] = v
        g = grad_small[sample]
        track_s = sum(r[2] for r in res)
        ref = {"parameters": int(len(sample)), "particles": rn, "turns": rturns, "cores": cores,
               "tracking_s_summed": track_s, "wall_s": wall,
               "relative_gradient_error_vs_reference_fd": float(np.max(np.abs(g - ref_fd)) / np.max(np.abs(ref_fd))),
               "reference_fd_s_full_problem_estimate": track_s * (2 * len(k0) * n * turns) /
                                                        (2 * len(sample) * rn * rturns) / cores,
               "note": "central differences of elegant's own tracking code on the host cores; the full-problem "
                       "estimate scales the summed tracking time by particle-turns and divides by the cores"}
    line = {"metric": "adjoint gradient speed-up over GPU finite differences", "value": t_fd / t_adj,
            "unit": "x", "n_gpus": 1, "steps": 1, "warmup": max(args.warmup, 1), "ms_per_step": t_adj * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Gaussian beam)",
            "config": {"workload": "gradient_c4", "particles": n, "turns": turns, "parameters": int(len(k0)),
                       "parameters_k1": int(is_k1.sum()), "parameters_k2": int((~is_k1).sum()),
                       "centroid_weight": w, "fd_step_relative": 1e-7},
            "adjoint_s": t_adj, "finite_difference_s": t_fd, "loss": loss,
            "relative_gradient_error_vs_fd": err, "gradient_error_metric": "max_p |g_adj - g_FD| / max_p |g_FD|",
            "max_componentwise_relative_error_vs_fd": err_c, "reference_fd": ref, "build": "fast"}
    print(json.dumps(line), flush=True)
    return 0


def run_gradient_ensemble(args, rank):
    """Batched gradients on the large ring: 32 error seeds of the MBA ring
    (RF and wakes off; seeded rms dK1/K1 = 1e-3 on every KQUAD, dK2/K2 =
    2e-3 on every KSEXT), 1e5 particles split over the seeds, `turns` turns
    (8 by default: over more turns a few particles of this seeded ring,
    near the edge of its momentum acceptance, grow their sensitivities
    exponentially, so the loss gradient is dominated by them and central
    differences no longer resolve it); per seed the gradient of
    mean(x^2 + y^2) + (mean x)^2 + (mean y)^2 with respect to its 480 KQUAD
    K1, 240 KSEXT K2, 280 CSBEND K1 and 280 CSBEND K2, all seeds in one
    trk_adjoint_ensemble call.  Finite differences (h from fd_step: 1e-7
    relative, with a floor for zero strengths; every seed perturbed at once, one trk_track_ensemble
    run per sign, parameters updated in place with trk_lattice_set) are run
    for a sample of the parameters and their time scaled to all 720 by the
    parameter count (the cost is the same per parameter).  Metric: that
    finite-difference time over the adjoint time; the gradient error is
    max_p |g_adj - g_FD| / max_p |g_FD| over the sampled parameters."""
    import ctypes

    import torch
    from elegant_b200 import Tracker, configs
    from elegant_b200 import _Run, _Stats, _check
    from elegant_b200.adjoint import fd_step, get_parameters, parameter_list
    if rank != 0:
        return 0
    torch.cuda.set_device(0)
    turns = args.turns or 8
    seeds = 32
    n = args.particles or 100_000
    counts = np.full(seeds, n // seeds, dtype=np.int64)
    counts[: n % seeds] += 1
    lats, beams, first = [], [], 1
    for v in range(seeds):
        rng = np.random.Generator(np.random.Philox(1000 + v))
        lats.append(configs.c5_lattice(with_rf=False, with_wake=False, kq_errors=rng.normal(0, 1e-3, (40, 12)),
                                       k2_errors=rng.normal(0, 2e-3, (40, 6))))
        beams.append(configs.c5_beam(int(counts[v]), seed=2000 + v, first_id=first))
        first += int(counts[v])
    beam = np.concatenate(beams)
    bounds = np.concatenate([[0], np.cumsum(counts)])
    offs = bounds.astype(np.int64)
    w = 1.0
    k0 = [get_parameters(lat) for lat in lats]
    plist = parameter_list(lats[0])
    n_par = len(k0[0])
    sample = np.unique(np.linspace(0, n_par - 1, 24).astype(int))

    def losses_from_store(trk):
        nl, out, lp, le = trk.store(stride=7, with_loss=True)
        ids = out[:, 6].astype(np.int64) - 1
        alive = lp < 0
        res = np.zeros(seeds)
        for v in range(seeds):
            m = alive & (ids >= bounds[v]) & (ids < bounds[v + 1])
            x, y = out[m, 0], out[m, 2]
            res[v] = np.mean(x * x + y * y) + w * (np.mean(x) ** 2 + np.mean(y) ** 2)
        return res

    with Tracker(0) as trk:
        for _ in range(max(args.warmup, 1)):
            trk.load(beam)
            trk.adjoint_ensemble(lats, counts, turns, configs.P_CENTRAL, w)
        torch.cuda.synchronize()
        with ClockSampler(0) as clocks:
            t0 = time.perf_counter()
            trk.load(beam)
            loss, grad = trk.adjoint_ensemble(lats, counts, turns, configs.P_CENTRAL, w)
            torch.cuda.synchronize()
            t_adj = time.perf_counter() - t0
        # finite differences through the C ABI: native lattices built once,
        # the perturbed parameter set in place
        lib = trk.lib
        nats = [trk.native(lat) for lat in lats]
        arr = (ctypes.c_void_p * seeds)(*[nt.ptr.value for nt in nats])
        run = _Run()
        lib.trk_run_defaults(ctypes.byref(run))
        run.p_central = configs.P_CENTRAL
        run.n_passes = turns
        st = _Stats()
        fd = np.zeros((seeds, len(sample)))
        dev_ms = 0.0
        t0 = time.perf_counter()
        for j, p in enumerate(sample):
            e, pname = plist[p]
            name = pname.encode()
            h = [fd_step(pname, k0[v][p]) for v in range(seeds)]
            vals = []
            for sgn in (1, -1):
                for v in range(seeds):
                    _check(lib, lib.trk_lattice_set(nats[v].ptr, e, name, k0[v][p] + sgn * h[v]))
                trk.load(beam)
                _check(lib, lib.trk_track_ensemble(trk.ctx, arr, seeds,
                                                   offs.ctypes.data_as(ctypes.POINTER(ctypes.c_long)),
                                                   ctypes.byref(run), ctypes.byref(st)))
                dev_ms += st.device_ms
                vals.append(losses_from_store(trk))
            for v in range(seeds):
                _check(lib, lib.trk_lattice_set(nats[v].ptr, e, name, k0[v][p]))
                fd[v, j] = (vals[0][v] - vals[1][v]) / (2 * h[v])
        torch.cuda.synchronize()
        t_fd_sample = time.perf_counter() - t0
    scale = n_par / len(sample)
    t_fd = t_fd_sample * scale
    g = grad[:, sample]
    err = float(np.max(np.abs(g - fd)) / np.max(np.abs(fd)))
    line = {"metric": "adjoint gradient speed-up over GPU finite differences", "value": t_fd / t_adj,
            "unit": "x", "n_gpus": 1, "steps": 1, "warmup": max(args.warmup, 1), "ms_per_step": t_adj * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded error seeds, seeded Gaussian beam)",
            "config": {"workload": "gradient_ensemble_c5", "seeds": seeds, "particles": int(n), "turns": turns,
                       "parameters_per_seed": n_par, "centroid_weight": w, "fd_step_relative": 1e-7,
                       "fd_parameters_timed": int(len(sample))},
            "adjoint_s": t_adj, "finite_difference_s": t_fd,
            "finite_difference_device_s": dev_ms / 1e3 * scale,
            "finite_difference_s_note": f"{len(sample)} parameters timed ({t_fd_sample:.2f} s wall), scaled by "
                                        f"{n_par}/{len(sample)}; the device figure is the tracking kernels' time "
                                        "alone",
            "loss_mean": float(np.mean(loss)),
            "relative_gradient_error_vs_fd": err, "gradient_error_metric": "max_p |g_adj - g_FD| / max_p |g_FD|",
            "clocks": clocks.summary(), "build": "fast"}
    print(json.dumps(line), flush=True)
    return 0


def _measured_hbm_gbs():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            v = json.load(f).get("hbm_gbs")
            if v:
                return float(v), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback (earlier measurement on this pool)"


def run_observe(args, rank):
    """Beam observers on the device beam: trk_accumulate_beam_sums (centroids,
    7x7 second moments, extremes; elegant's accumulate_beam_sums) on 1e7
    particles of the MBA ring's beam.  HBM-bound: two passes over x, x', y,
    y', s, delta and the loss word (the ID column only with an ID window),
    52 B per particle each.  Metric: particles summed per second; roofline in
    GB/s against the measured HBM copy bandwidth."""
    import torch
    from elegant_b200 import BeamSums, SUMS_SECOND_ORDER, Tracker, configs
    if rank != 0:
        return 0
    torch.cuda.set_device(0)
    n = args.particles or 10_000_000
    beam = configs.c5_beam(n, seed=1)
    with Tracker(0) as trk:
        trk.load(beam)
        stream = torch.cuda.ExternalStream(trk.stream(), device="cuda:0")
        for _ in range(max(args.warmup, 3)):
            trk.accumulate_beam_sums(BeamSums.zeroed(), configs.P_CENTRAL, flags=SUMS_SECOND_ORDER)
        ms = []
        with ClockSampler(0) as clocks:
            for _ in range(args.steps):
                s = BeamSums.zeroed()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                trk.accumulate_beam_sums(s, configs.P_CENTRAL, flags=SUMS_SECOND_ORDER)
                e1.record(stream)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
        c_ms = []
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            trk.centroids()
            e1.record(stream)
            e1.synchronize()
            c_ms.append(e0.elapsed_time(e1))
    t = float(np.median(ms)) / 1e3
    tc = float(np.median(c_ms)) / 1e3
    peak, src = _measured_hbm_gbs()
    algo = 2 * 52.0 * n
    line = {"metric": "beam sums (accumulate_beam_sums) particles/s", "value": n / t, "unit": "particles/s",
            "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Gaussian beam)",
            "config": {"workload": "observe_beam_sums_1e7", "particles": n, "second_order": True,
                       "l2": "beam columns larger than L2 (no flush needed)"},
            "roofline": {"bound": "hbm", "achieved": algo / t / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": algo / t / 1e9 / peak, "traffic": None, "peak_source": src,
                         "bytes_per_particle": 104},
            "centroids_ms": tc * 1e3, "centroids_gbs": 52.0 * n / tc / 1e9, "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)
    return 0


def run_da(args, rank):
    """Dynamic-aperture line search over error seeds (trk_aperture_search_lines):
    256 seeds of the FODO+sextupole ring with its 25 mm aperture, 11 lines of
    41 points to 20 mm x 10 mm, two refinement sweeps, `turns` turns.  Metric:
    particle-turns/s of the whole search (every tracked point x turns over the
    search's wall time, host logic included)."""
    import torch
    from elegant_b200 import Tracker, configs
    if rank != 0:
        return 0
    torch.cuda.set_device(0)
    turns = args.turns or 1024
    seeds = min(args.variants, 256)
    lats = [configs.c3_variant(seed=v) for v in range(seeds)]
    kw = dict(lines=11, nx=41, xmax=0.02, ymax=0.01, n_splits=2, split_fraction=0.5)
    points = seeds * kw["lines"] * (kw["nx"] + 2 * max(1, int(1 / kw["split_fraction"] - 0.5)))
    with Tracker(0) as trk:
        trk.aperture_search_lines(lats, configs.P_CENTRAL, 4, **kw)  # autotune, warm
        torch.cuda.synchronize()
        with ClockSampler(0) as clocks:
            t0 = time.perf_counter()
            r = trk.aperture_search_lines(lats, configs.P_CENTRAL, turns, **kw)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
    line = {"metric": "aperture-search particle-turns/s", "value": points * turns / wall, "unit": "particle-turns/s",
            "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": wall * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded error seeds)",
            "config": {"workload": "da_search_256x11_lines", "seeds": seeds, "turns": turns, **kw,
                       "points_tracked": points},
            "search_s": wall, "mean_area_m2": float(np.mean(r["area"])), "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)
    return 0


def _timed_turns(trk, lat, fast, steps, warmup, pass_index, flush, stream, world, local):
    """Warm-up turns, then `steps` timed turns of the resident beam (CUDA
    events on the tracking stream, L2 flushed between steps outside the
    events).  Returns the measurements and the next pass index."""
    import torch
    from elegant_b200 import configs
    for _ in range(max(warmup, 3)):
        trk.track(lat, 1, configs.P_CENTRAL, pass_offset=pass_index, fast=fast)
        pass_index += 1
    step_ms, effort, launches, track_ms, track_launches = [], 0, 0, 0.0, 0
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        t_wall = time.perf_counter()
        for k in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))
            st = trk.track(lat, 1, configs.P_CENTRAL, pass_offset=pass_index, fast=fast, time_kernels=True)
            pass_index += 1
            step_ms.append(st["device_ms"])
            effort += st["particle_passes"]
            launches += st["kernel_launches"]
            track_ms += st["track_ms"]
            track_launches += st["track_launches"]
        torch.cuda.synchronize()
        wall = time.perf_counter() - t_wall
    dev_s = sum(step_ms) / 1e3
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([dev_s, float(effort)], dtype=torch.float64, device=f"cuda:{local}")
        dmax = t[:1].clone()
        dist.all_reduce(dmax, op=dist.ReduceOp.MAX)
        dsum = t[1:].clone()
        dist.all_reduce(dsum, op=dist.ReduceOp.SUM)
        dev_s = float(dmax.item())
        effort = float(dsum.item())
    return {"value": effort / dev_s, "dev_s": dev_s, "effort": effort, "launches": launches, "track_ms": track_ms,
            "track_launches": track_launches, "wall": wall, "clocks": clocks.summary()}, pass_index


def _e2e(trk, lat, fast, beam, steps, world):
    """The same metric through the C ABI with host buffers: each step loads
    the beam from pinned host memory, tracks one turn and stores it back."""
    import torch
    from elegant_b200 import configs
    pinned = torch.from_numpy(beam).pin_memory().numpy()
    pinned_out = torch.empty(beam.shape, dtype=torch.float64).pin_memory().numpy()
    e2e_ms, eff = [], 0
    for _ in range(max(3, steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        trk.load(pinned)
        st = trk.track(lat, 1, configs.P_CENTRAL, fast=fast)
        trk.store(stride=7, out=pinned_out)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        eff = st["particle_passes"]
    n = beam.shape[0]
    return {"value": eff / (np.median(e2e_ms) / 1e3) * world, "unit": "particle-turns/s",
            "h2d_bytes_per_step": int(n * 7 * 8), "d2h_bytes_per_step": int(n * 7 * 8)}


def _roofline(m, workload, world, peak, flops):
    """FP64 roofline of the fused tracking kernel: algorithmic flops of the
    elements it runs (reference formulation, oracle/flops.json) per launch
    over its CUDA-event launch time."""
    if not flops or not m["track_launches"]:
        return None
    # the radiating ring is counted as the plain one (the radiation's own flops are not counted)
    fpt = flops["flops_per_particle_turn"]["c2" if workload == "rad" else workload]
    # the wakes' per-particle work runs in the wake kernels
    fpt -= {"c1": 0, "c2": 1, "rad": 1, "c5": 2}[workload] * flops["per_particle"]["WAKE"]["total"]
    per_launch_flops = fpt * (m["effort"] / world) / m["track_launches"]
    avg_launch_s = m["track_ms"] / m["track_launches"] / 1e3
    achieved = per_launch_flops / avg_launch_s / 1e12
    traffic = {"c2": TRACK_DRAM_BYTES_PER_PARTICLE, "c5": TRACK_DRAM_BYTES_PER_PARTICLE_C5}.get(workload)
    return {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if peak else None,
            "traffic": traffic * (m["effort"] / world) / m["track_launches"] if traffic else None,
            "flops_per_particle_turn": fpt, "kernel": "track_kernel", "launches": m["track_launches"],
            "avg_launch_ms": avg_launch_s * 1e3,
            "peak_source": "FP64 FMA peak measured in this run (independent dependent-FMA chains); "
                           "MEASURED_PEAKS.json has no FP64 figure",
            "traffic_source": (None if not traffic else
                               "ncu dram__bytes_read.sum + dram__bytes_write.sum of one fast-build launch at "
                               + ("2e5" if workload == "c2" else "2e6") + " particles, scaled by particles")}


LONG_FIXTURES = os.path.join(ROOT, "tests", "golden", "long_tracks.npz")


def accuracy(local, fast):
    """Error of one build against elegant's own tracking code on the
    benchmark rings as configured, from the committed fixtures the
    reference wrote (tests/golden/long_tracks.npz): the FODO ring with 1e4
    particles after 1 and 100 turns, the RF + wake ring (2000 bins) with
    4000 particles after 1 and 10 turns.  Per coordinate |gpu - ref| /
    max(|ref|, sigma_c) over the reference's survivors, against the
    reference in the parity arithmetic (correctly rounded libm) and in its
    own (glibc libm); plus whether the survivor sets are identical."""
    from elegant_b200 import Tracker, configs
    if not os.path.exists(LONG_FIXTURES):
        return None
    gold = np.load(LONG_FIXTURES)
    cases = {"fodo40_1e4": ("c1", configs.c1_lattice, lambda: configs.gaussian_beam(10_000, seed=1), (1, 100)),
             "ring_rf_wake_4e3": ("c2", configs.c2_lattice, lambda: configs.gaussian_beam(4000, seed=7), (1, 10))}
    out = {}
    with Tracker(local) as trk:  # no communicator: a one-GPU run on every rank that asks
        for name, (ring, mk_lat, mk_beam, turn_list) in cases.items():
            lat, beam = mk_lat(), mk_beam()
            for turns in turn_list:
                trk.load(beam)
                trk.track(lat, turns, configs.P_CENTRAL, fast=fast)
                n_left, g, lp, le = trk.store(stride=7, with_loss=True)
                order = np.argsort(g[:, 6], kind="stable")
                g, lp = g[order], lp[order]
                res = {}
                for mode in ("parity_arith", "reference_arith"):
                    key = f"{ring}/turns{turns}/{mode}"
                    ref, loss = gold[key + "/coords"], gold[key + "/loss"]
                    alive = loss[:, 0] < 0
                    sig = np.std(ref[alive, :6], axis=0)
                    d = np.abs(g[alive, :6] - ref[alive, :6]) / np.maximum(np.abs(ref[alive, :6]), sig)
                    res[mode] = {"max_err": float(d.max()), "bit_exact": bool(np.array_equal(g[alive, :6],
                                                                                              ref[alive, :6])),
                                 "same_survivors": bool(np.array_equal(lp < 0, alive))}
                out[f"{name}_{turns}turn" + ("s" if turns > 1 else "")] = res
    return out


def run_gpu(args, rank, world, local):
    import torch
    from elegant_b200 import Tracker, configs
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    n = args.particles or WORKLOADS[args.workload]["particles"]
    lat = workload_lattice(args.workload)
    beam = workload_beam(args.workload, n, seed=1 + rank, first_id=1 + rank * n)
    builds = {"parity": ["parity"], "fast": ["fast"], "both": ["parity", "fast"]}[
        "parity" if args.exact else args.build]
    flops = load_flops()
    res = {}
    with Tracker(local) as trk:
        if world > 1:
            # the library's own NCCL communicator for the wake/RF exchanges
            import elegant_b200
            import torch.distributed as dist
            uid = elegant_b200.nccl_unique_id() if rank == 0 else bytes(128)
            t = torch.tensor(list(uid), dtype=torch.uint8, device=f"cuda:{local}")
            dist.broadcast(t, 0)
            trk.set_comm(bytes(t.cpu().tolist()), world, rank)
        flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
        stream = torch.cuda.ExternalStream(trk.stream(), device=f"cuda:{local}")
        for b in builds:
            fast = b == "fast"
            trk.load(beam)
            m, _ = _timed_turns(trk, lat, fast, args.steps, args.warmup, 0, flush, stream, world, local)
            m["e2e"] = _e2e(trk, lat, fast, beam, args.steps // 2, world)
            res[b] = m
        del flush
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    peak = measure_fp64_peak(local)
    acc = {b: accuracy(local, b == "fast") for b in builds} if world == 1 else None
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        if args.workload == "c5":
            cpu = cpu_baseline(cores=1, sample_particles=1500, sample_turns=2, workload="c5")
        elif args.workload == "rad":
            cpu = cpu_baseline(cores=1, sample_particles=3000, sample_turns=3, workload="rad")
        else:
            cpu = cpu_baseline(cores=1, workload=args.workload)
    head = builds[0]
    m = res[head]
    line = {"metric": "particle-turns/s", "value": m["value"], "unit": "particle-turns/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": m["dev_s"] * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Gaussian beam, seeded resonator wake)",
            "config": workload_config(n, args.workload), "build": head, "wall_s": m["wall"], "e2e": m["e2e"],
            "gpu_launches": m["launches"], "roofline": _roofline(m, args.workload, world, peak, flops),
            "cpu_baseline": cpu, "clocks": m["clocks"]}
    if acc and acc.get(head):
        line["accuracy"] = acc[head]
        line["accuracy_metric"] = ("max over surviving particles and coordinates of |gpu - ref| / max(|ref|, "
                                   "sigma_c) against elegant's own tracking code (fixtures written by it): "
                                   "parity_arith = with a correctly rounded libm, reference_arith = with glibc's")
    for b in builds[1:]:
        mb = res[b]
        line[f"{b}_build"] = {"value": mb["value"], "ms_per_step": mb["dev_s"] * 1e3 / args.steps,
                              "e2e": mb["e2e"], "gpu_launches": mb["launches"],
                              "roofline": _roofline(mb, args.workload, world, peak, flops),
                              "accuracy": acc.get(b) if acc else None, "clocks": mb["clocks"]}
    print(json.dumps(line), flush=True)
    return 0


_PEAK_SRC = r"""
extern "C" __global__ void fma_peak(double *out, int iters) {
  double a0 = threadIdx.x * 1e-9, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  const double b = 0.999999999, c = 1e-9;
  for (int i = 0; i < iters; i++) {
    a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
    a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}
"""


def measure_fp64_peak(device):
    """FP64 FMA peak (TFLOP/s, FMA = 2 flops) from a kernel of independent
    dependent-FMA chains, compiled with the runtime compiler."""
    try:
        import torch
        from cuda.bindings import nvrtc
    except Exception:
        try:
            from cuda import nvrtc  # noqa: F401
        except Exception:
            return None
    try:
        import ctypes
        import torch
        from cuda.bindings import nvrtc, driver
        prog = nvrtc.nvrtcCreateProgram(_PEAK_SRC.encode(), b"peak.cu", 0, [], [])[1]
        opts = [b"-arch=sm_100a"]
        nvrtc.nvrtcCompileProgram(prog, len(opts), opts)
        size = nvrtc.nvrtcGetCUBINSize(prog)[1]
        cubin = b" " * size
        nvrtc.nvrtcGetCUBIN(prog, cubin)
        torch.cuda.set_device(device)
        torch.cuda.synchronize()
        err, mod = driver.cuModuleLoadData(cubin)
        err, fn = driver.cuModuleGetFunction(mod, b"fma_peak")
        blocks, threads, iters = 148 * 16, 256, 20000
        out = torch.empty(blocks * threads, dtype=torch.float64, device=f"cuda:{device}")
        arg_ptr = ctypes.c_void_p(out.data_ptr())
        arg_it = ctypes.c_int(iters)
        params = (ctypes.c_void_p * 2)(ctypes.addressof(arg_ptr), ctypes.addressof(arg_it))
        stream = torch.cuda.current_stream().cuda_stream
        for rep in range(2):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            driver.cuLaunchKernel(fn, blocks, 1, 1, threads, 1, 1, 0, stream, ctypes.addressof(params), 0)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
        flops = 2.0 * 8 * iters * blocks * threads
        return flops / (ms / 1e3) / 1e12
    except Exception:
        return None


if __name__ == "__main__":
    sys.exit(main())
