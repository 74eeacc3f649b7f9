"""Incoherent synchrotron radiation (ISR=1) in KQUAD/KSEXT/KOCT and CSBEND.

The reference draws its deviates from the SDDS toolkit's generator, which is
not in the reference tree, so its ISR cannot be reproduced number for number.
The library draws truncated normal deviates from a counter-based generator
keyed by (seed, particle ID, pass, element, kick) (elegant_b200/csrc/
trk_philox.h); the oracle restates the reference's ISR formulas with the same
deviates.  Checked: the GPU against the oracle particle by particle (to the
rounding of log, cos and pow, which differ between CUDA and glibc); the
energy spread ISR adds against the reference's own formula for its variance
(isrConstant^2 F^3/2 ds per kick, src/csbend.c:1649-1653); repeatability and
independence from the launch shape.
"""
import math

import numpy as np
import pytest

from elegant_b200 import configs
from oracle import pyoracle
from tests.cases import single
from tests.helpers import compare

PC = configs.P_CENTRAL
SEED = 20261203

ISR_CASES = {
    "kquad_isr": single("KQUAD", L=0.3, K1=1.2, N_KICKS=8, ISR=1, SYNCH_RAD=1),
    "ksext_isr": single("KSEXT", L=0.2, K2=40.0, N_KICKS=4, ISR=1),
    "koct_isr": single("KOCT", L=0.2, K3=500.0, ISR=1, SYNCH_RAD=1),
    "csbend_isr": single("CSBEND", L=1.0, ANGLE=2 * math.pi / 80, N_KICKS=16, ISR=1, SYNCH_RAD=1),
    "csbend_k1_isr": single("CSBEND", L=1.0, ANGLE=2 * math.pi / 280, K1=-0.4, N_KICKS=32, ISR=1),
}


def _truncated_normal_variance(limit=3.0):
    phi = math.exp(-limit * limit / 2) / math.sqrt(2 * math.pi)
    return 1 - 2 * limit * phi / math.erf(limit / math.sqrt(2))


def _dipole_isr_prediction(L, angle, n_kicks):
    """std of delta after one pure dipole for an on-axis beam: sum over the
    kicks of (isrConstant^2 F^3/2 dsISR) with F = 1, times the variance of the
    deviate truncated at 3 (src/csbend.c:961-964, :1649-1653)."""
    rho = L / angle
    re = 2.8179403262e-15
    isr = re * math.sqrt(55.0 / (24 * math.sqrt(3.0)) * PC ** 5 * 137.0359895 / abs(rho) ** 3)
    n_slices = math.ceil(n_kicks / 4)
    ds_isr = (L / n_slices) / 3
    kicks = n_slices * 3
    return math.sqrt(kicks * isr ** 2 * ds_isr * _truncated_normal_variance())


def _on_axis(n):
    b = np.zeros((n, 7))
    b[:, 6] = np.arange(1, n + 1)
    return b


def test_oracle_isr_spread_matches_reference_formula():
    L, angle, nk = 1.0, 2 * math.pi / 80, 16
    lat = single("CSBEND", L=L, ANGLE=angle, N_KICKS=nk, ISR=1)
    pyoracle.set_isr_seed(SEED)
    rows, n_left, _ = pyoracle.track(lat, _on_axis(20000), 1, PC)
    pyoracle.set_isr_seed(0)
    d = rows[:n_left, 5]
    want = _dipole_isr_prediction(L, angle, nk)
    assert abs(np.std(d) / want - 1) < 0.02, (np.std(d), want)
    assert abs(np.mean(d)) < 4 * want / math.sqrt(len(d))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(ISR_CASES))
@pytest.mark.parametrize("fast", [False, True])
def test_isr_gpu_vs_oracle(tracker, name, fast):
    lat = ISR_CASES[name]
    beam = configs.gaussian_beam(4000, seed=81)
    tracker.load(beam)
    tracker.track(lat, 2, PC, fast=fast, isr_seed=SEED)
    nl, g = tracker.store()
    pyoracle.set_isr_seed(SEED)
    with pyoracle.modes(exact_sums=True, cr_math=True):
        rows, nlo, _ = pyoracle.track(lat, beam, 2, PC)
    pyoracle.set_isr_seed(0)
    r = compare(g, rows, nl, nlo)
    assert r["same_survivors"]
    assert r["max_err"] < (1e-12 if not fast else 5e-9), r
    # the deviates act: another seed gives other momenta
    pyoracle.set_isr_seed(SEED + 1)
    with pyoracle.modes(exact_sums=True, cr_math=True):
        other, _, _ = pyoracle.track(lat, beam, 2, PC)
    pyoracle.set_isr_seed(0)
    assert not np.array_equal(np.sort(other[:, 5]), np.sort(rows[:, 5]))


@pytest.mark.gpu
def test_isr_spread_matches_reference_formula(tracker):
    L, angle, nk = 1.0, 2 * math.pi / 80, 16
    lat = single("CSBEND", L=L, ANGLE=angle, N_KICKS=nk, ISR=1)
    tracker.load(_on_axis(400_000))
    tracker.track(lat, 1, PC, isr_seed=SEED)
    n, out = tracker.store()
    want = _dipole_isr_prediction(L, angle, nk)
    assert abs(np.std(out[:n, 5]) / want - 1) < 0.005, (np.std(out[:n, 5]), want)


@pytest.mark.gpu
def test_isr_repeatable_and_independent_of_launch_shape(tracker):
    lat = configs.c1_lattice(cells=2)
    for e in lat.elements:
        if e[0] in ("KQUAD", "CSBEND"):
            e[2]["ISR"] = 1.0
    beam = configs.gaussian_beam(3000, seed=82)
    outs = []
    for seed, variant in ((SEED, -1), (SEED, 4), (SEED + 1, -1)):
        tracker.load(beam)
        tracker.track(lat, 3, PC, isr_seed=seed, variant=variant)
        outs.append(tracker.store()[1])
    assert np.array_equal(outs[0], outs[1])
    assert not np.array_equal(outs[0], outs[2])


@pytest.mark.gpu
@pytest.mark.parametrize("isr1part", [0, 1])
def test_isr1part_single_particle(tracker, isr1part):
    """ISR1PART (src/multipole.c:758, src/csbend.c:963): with 0, a beam of
    one particle gets no quantum excitation (classical radiation stays on);
    with 1 it does.  The library decides on the beam it was handed (the
    reference on the particles entering the element, which differ only once
    all but one have been lost)."""
    beam = configs.gaussian_beam(1, seed=83)
    outs = {}
    for isr in (0, 1):
        lat = single("CSBEND", L=1.0, ANGLE=2 * math.pi / 80, N_KICKS=16, SYNCH_RAD=1, ISR=isr,
                     ISR1PART=isr1part)
        tracker.load(beam)
        tracker.track(lat, 2, PC, isr_seed=SEED, fast=False)
        outs[isr] = tracker.store()[1]
    if isr1part == 0:
        assert np.array_equal(outs[0], outs[1])
    else:
        assert not np.array_equal(outs[0], outs[1])
