"""The large ring (C5): multi-bend-achromat cells of combined-function CSBENDs
(K1 field expansion, N_KICKS=32), strong KQUADs, KSEXTs and KOCTs, with
RFCA, WAKE and TRWAKE on the broadband resonator wakes.

CPU: the seeded strength search is deterministic and gives a linearly stable
cell; the oracle restatement equals elegant's own compiled tracking code bit
for bit on a two-cell ring of this kind.  GPU: the parity build against the
oracle (TRWAKE bins are FP64 sums whose last bit depends on the atomic
order, hence a rounding-level bound), against the reference's own code, and
the fast build against the oracle.
"""
import numpy as np
import pytest

from elegant_b200 import configs
from oracle import pyoracle
from tests.helpers import compare, gpu_run, oracle_run

PC = configs.P_CENTRAL


def _ring(with_wake=True):
    return configs.c5_lattice(cells=2, n_bins=400, with_wake=with_wake)


def test_mba_strengths_deterministic_and_stable():
    a = configs.mba_strengths()
    b = configs.mba_strengths()
    assert a["seed"] == b["seed"]
    for k in ("kq", "kb", "k2", "k3"):
        assert np.array_equal(a[k], b[k])
    assert np.all(np.abs(a["kq"]) <= 6) and np.all(np.abs(a["kb"]) <= 0.5) and np.all(np.abs(a["k2"]) <= 300)
    for d in (-5e-3, 0.0, 5e-3):
        cx, cy, beta_max, eta_max = configs.mba_cell_optics(a["kq"], a["kb"], d)
        assert abs(cx) < 1 and abs(cy) < 1 and beta_max is not None
    lat = configs.c5_lattice()
    kinds = [e[0] for e in lat.elements]
    assert kinds.count("CSBEND") == 280 and kinds.count("KQUAD") == 480 and kinds.count("KSEXT") == 240
    assert kinds.count("KOCT") == 80 and kinds.count("TRWAKE") == 1 and kinds.count("WAKE") == 1
    bends = [e[2] for e in lat.elements if e[0] == "CSBEND"]
    assert abs(sum(p["ANGLE"] for p in bends) - 2 * np.pi) < 1e-12


@pytest.mark.skipif(not pyoracle.ref_available(), reason="oracle/_ref/libref.so not built")
@pytest.mark.parametrize("exact", [False, True])
def test_oracle_vs_reference_c5_cells(exact):
    lat = _ring()
    beam = configs.c5_beam(300, seed=51)
    rows, nl, eff = pyoracle.track_ref(lat, beam, 2, PC, exact_sums=exact, cr_math=exact)
    with pyoracle.modes(exact_sums=exact, cr_math=exact):
        o, nlo, effo = oracle_run(lat, beam, 2, PC)
    assert nl == nlo and eff == effo
    r = compare(o, rows, nlo, nl)
    assert r["same_survivors"] and r["bit_exact"] and r["lost_equal"], r


@pytest.mark.gpu
def test_c5_cells_parity_build(tracker):
    lat = _ring()
    beam = configs.c5_beam(3000, seed=52)
    nl, g, lp, le, st = gpu_run(tracker, lat, beam, 2, PC, fast=False)
    with pyoracle.modes(exact_sums=True, cr_math=True):
        rows, nlo, eff = oracle_run(lat, beam, 2, PC)
    assert st["particle_passes"] == eff
    r = compare(g, rows, nl, nlo)
    assert r["same_survivors"]
    assert r["max_err"] < 1e-12, r


@pytest.mark.gpu
def test_c5_cells_no_trwake_bit_exact(tracker):
    """Without the wakes every operation is order-independent: bit-exact."""
    lat = _ring(with_wake=False)
    beam = configs.c5_beam(3000, seed=53)
    nl, g, lp, le, _ = gpu_run(tracker, lat, beam, 2, PC, fast=False)
    with pyoracle.modes(exact_sums=True, cr_math=True):
        rows, nlo, _ = oracle_run(lat, beam, 2, PC)
    r = compare(g, rows, nl, nlo)
    assert r["same_survivors"] and r["bit_exact"] and r["lost_equal"], r


@pytest.mark.gpu
@pytest.mark.skipif(not pyoracle.ref_available(), reason="oracle/_ref/libref.so not built")
def test_c5_cells_parity_build_vs_reference_code(tracker):
    lat = _ring(with_wake=False)
    beam = configs.c5_beam(2000, seed=54)
    nl, g, lp, le, _ = gpu_run(tracker, lat, beam, 2, PC, fast=False)
    rows, nlr, _ = pyoracle.track_ref(lat, beam, 2, PC, exact_sums=True, cr_math=True)
    r = compare(g, rows, nl, nlr)
    assert r["same_survivors"] and r["bit_exact"] and r["lost_equal"], r


@pytest.mark.gpu
def test_c5_full_ring_fast_one_turn(tracker):
    """The whole 40-cell ring, one turn, fast build against the oracle."""
    lat = configs.c5_lattice()
    beam = configs.c5_beam(400, seed=55)
    nl, g, lp, le, _ = gpu_run(tracker, lat, beam, 1, PC, fast=True)
    with pyoracle.modes(exact_sums=True, cr_math=True):
        rows, nlo, _ = oracle_run(lat, beam, 1, PC)
    r = compare(g, rows, nl, nlo)
    assert r["same_survivors"]
    assert r["max_err"] < 5e-8, r
