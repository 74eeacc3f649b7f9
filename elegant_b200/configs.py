"""Lattices and seeded beams of the benchmark workloads.

C1  FODO ring, 40 cells (QF KQUAD L=0.3 K1=+1.2 N_KICKS=8, drift 1 m,
    CSBEND L=1 ANGLE=2pi/80 N_KICKS=16, drift, QD K1=-1.2, drift, CSBEND,
    drift), p_central = 13700, Gaussian beam, 100 turns.
C2  C1 plus a KSEXT (L=0.2, K2=+/-40, N_KICKS=4) after each quad, one RFCA
    (4 MV, h*f_rev near 352 MHz, PHASE=180) and a WAKE (4096-point seeded
    resonator Green function, R/Q=1 kOhm, Q=5, 20 GHz, 2000 bins), CHARGE
    1 nC; 1e6 particles, 1000 turns.
C3  256 error-seed variants of C2's lattice without RF and wake, dynamic
    aperture grids of 1000..65536 particles, 1024 turns, 25 mm circular MAXAMP.
C4  Gradient of mean(x^2+y^2) (+ centroid penalty) after 64 turns, C2 lattice
    without RF and wake, 1e5 particles.
C5  40 multi-bend-achromat cells (7 combined-function CSBENDs ANGLE=2pi/280,
    12 KQUAD, 6 KSEXT, 2 KOCT), RFCA, WAKE and TRWAKE, 1e7 particles.

All inputs are synthetic and seeded (numpy Philox); there is no dataset.
"""
import math

import numpy as np

from . import Lattice

C_MKS = 2.99792458e8
P_CENTRAL = 13700.0


def _beta(p):
    return p / math.sqrt(p * p + 1)


def fodo_cell(lat, sext=False, k2=40.0, kq=1.2, kq_errors=None, k2_errors=None, cell=0):
    """One FODO cell; error arrays give relative strength errors per cell."""
    dq = kq_errors[cell] if kq_errors is not None else (0.0, 0.0)
    ds = k2_errors[cell] if k2_errors is not None else (0.0, 0.0)
    lat.add("KQUAD", "QF", L=0.3, K1=kq * (1 + dq[0]), N_KICKS=8)
    if sext:
        lat.add("KSEXT", "SF", L=0.2, K2=k2 * (1 + ds[0]), N_KICKS=4)
    lat.add("DRIF", "D", L=1.0)
    lat.add("CSBEND", "B", L=1.0, ANGLE=2 * math.pi / 80, N_KICKS=16)
    lat.add("DRIF", "D", L=1.0)
    lat.add("KQUAD", "QD", L=0.3, K1=-kq * (1 + dq[1]), N_KICKS=8)
    if sext:
        lat.add("KSEXT", "SD", L=0.2, K2=-k2 * (1 + ds[1]), N_KICKS=4)
    lat.add("DRIF", "D", L=1.0)
    lat.add("CSBEND", "B", L=1.0, ANGLE=2 * math.pi / 80, N_KICKS=16)
    lat.add("DRIF", "D", L=1.0)


def c1_lattice(cells=40):
    lat = Lattice()
    for c in range(cells):
        fodo_cell(lat, cell=c)
    return lat


def resonator_wake(points=4096, dt=1e-12, f_r=20e9, r_over_q=1e3, q=5.0, seed=2, perturb=1e-3):
    """Broadband resonator Green function W(t) = 2k e^{-a t} (cos w t - (a/w) sin w t)
    with k = w (R/Q) / 2, a = w / (2Q), sampled at t = i*dt, times a seeded
    (1 +/- perturb) factor per sample."""
    w = 2 * math.pi * f_r
    a = w / (2 * q)
    k = w * r_over_q / 2
    t = np.arange(points, dtype=np.float64) * dt
    W = 2 * k * np.exp(-a * t) * (np.cos(w * t) - (a / w) * np.sin(w * t))
    rng = np.random.Generator(np.random.Philox(seed))
    W *= 1 + perturb * rng.uniform(-1.0, 1.0, points)
    return t, W


def c2_lattice(cells=40, with_rf=True, with_wake=True, n_bins=2000, wake_dt=50e-15, charge=1e-9, harmonic=329,
               kq_errors=None, k2_errors=None):
    lat = Lattice()
    if with_wake:
        lat.add("CHARGE", "Q", TOTAL=charge)
    for c in range(cells):
        fodo_cell(lat, sext=True, kq_errors=kq_errors, k2_errors=k2_errors, cell=c)
    if with_rf:
        circumference = lat.total_length()
        f_rev = _beta(P_CENTRAL) * C_MKS / circumference
        lat.add("RFCA", "RF", L=0.0, VOLT=4e6, FREQ=harmonic * f_rev, PHASE=180.0)
    if with_wake:
        i = lat.add("WAKE", "W", N_BINS=n_bins, ALLOW_LONG_BEAM=1)
        t, W = resonator_wake(dt=wake_dt)
        lat.set_wake(i, t, W)
    return lat


def c3_variant(seed, cells=40):
    """C2's lattice without RF and wake, with seeded Gaussian quad (rms 1e-3)
    and sextupole (rms 2e-3) relative errors, and a 25 mm circular MAXAMP."""
    rng = np.random.Generator(np.random.Philox(2 + seed))
    kq = rng.normal(0.0, 1e-3, (cells, 2))
    k2 = rng.normal(0.0, 2e-3, (cells, 2))
    lat = Lattice()
    lat.add("MAXAMP", "AP", X_MAX=0.025, Y_MAX=0.025, ELLIPTICAL=1)
    for c in range(cells):
        fodo_cell(lat, sext=True, kq_errors=kq, k2_errors=k2, cell=c)
    return lat


def gaussian_beam(n, seed=1, sigma_x=100e-6, sigma_xp=10e-6, sigma_s=3e-3, sigma_dp=1e-3, first_id=1):
    """(n, 7) beam: x, x', y, y', s, delta, id with Philox-seeded Gaussians."""
    rng = np.random.Generator(np.random.Philox(seed))
    b = np.empty((n, 7), dtype=np.float64)
    b[:, 0] = rng.normal(0.0, sigma_x, n)
    b[:, 1] = rng.normal(0.0, sigma_xp, n)
    b[:, 2] = rng.normal(0.0, sigma_x, n)
    b[:, 3] = rng.normal(0.0, sigma_xp, n)
    b[:, 4] = rng.normal(0.0, sigma_s, n)
    b[:, 5] = rng.normal(0.0, sigma_dp, n)
    b[:, 6] = np.arange(first_id, first_id + n, dtype=np.float64)
    return b


def da_grid(n, seed=0, first_id=1):
    """Dynamic-aperture grid: x in [-20, 20] mm, y in [0, 10] mm, delta = 0."""
    nx = max(1, int(round(math.sqrt(2 * n))))
    ny = max(1, (n + nx - 1) // nx)
    xs = np.linspace(-0.02, 0.02, nx)
    ys = np.linspace(0.0, 0.01, ny)
    X, Y = np.meshgrid(xs, ys)
    b = np.zeros((n, 7), dtype=np.float64)
    b[:, 0] = X.ravel()[:n]
    b[:, 2] = Y.ravel()[:n]
    b[:, 6] = np.arange(first_id, first_id + n, dtype=np.float64)
    return b
