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


def transverse_resonator_wake(points=4096, dt=50e-15, f_r=20e9, r_shunt=1e6, q=1.0, seed=3, perturb=1e-3):
    """Transverse resonator Green function W(t) = (w R_s / (Q wb)) e^{-a t} sin(wb t)
    [V/C/m] with a = w / (2Q), wb = sqrt(w^2 - a^2), sampled at t = i*dt,
    times a seeded (1 +/- perturb) factor per sample."""
    w = 2 * math.pi * f_r
    a = w / (2 * q)
    wb = math.sqrt(w * w - a * a)
    t = np.arange(points, dtype=np.float64) * dt
    W = (w * r_shunt / (q * wb)) * np.exp(-a * t) * np.sin(wb * t)
    rng = np.random.Generator(np.random.Philox(seed))
    W *= 1 + perturb * rng.uniform(-1.0, 1.0, points)
    return t, W


# C5 cell: 27 magnets, each followed by a 0.2 m drift.  Q = KQUAD (L=0.25,
# N_KICKS=8), B = combined-function CSBEND (L=0.8, ANGLE=2pi/280, N_KICKS=32),
# S = KSEXT (L=0.2, N_KICKS=4), O = KOCT (L=0.1, N_KICKS=4).
MBA_CELL = "Q Q O B Q S B Q S B Q S B S Q B S Q B S Q B Q Q O Q Q".split()
MBA_L = {"Q": 0.25, "B": 0.8, "S": 0.2, "O": 0.1}
MBA_DRIFT = 0.2
MBA_ANGLE = 2 * math.pi / 280


def _thick(K, L, h=0.0):
    """3x3 (x, x', delta) transfer matrix of a thick lens of focusing
    strength K over L; h = 1/rho adds the dispersion terms of a sector bend."""
    m = np.eye(3)
    if abs(K) < 1e-12:
        m[0, 1] = L
        m[0, 2], m[1, 2] = h * L * L / 2, h * L
        return m
    k = math.sqrt(abs(K))
    if K > 0:
        c, sn, d = math.cos(k * L), math.sin(k * L) / k, -k * math.sin(k * L)
    else:
        c, sn, d = math.cosh(k * L), math.sinh(k * L) / k, k * math.sinh(k * L)
    m[:2, :2] = [[c, sn], [d, c]]
    m[0, 2], m[1, 2] = h * (1 - c) / K, h * sn
    return m


def mba_cell_optics(kq, kb, delta=0.0):
    """Linear optics of the C5 cell at relative momentum offset delta: the
    half-traces (cos mu) of x and y, and when both are inside (-1, 1) the
    maximum beta function (either plane) and maximum |dispersion| at element
    boundaries; None for those when the cell is unstable."""
    elems = []
    iq = ib = 0
    for e in MBA_CELL:
        L = MBA_L[e]
        if e == "Q":
            k = kq[iq] / (1 + delta)
            ex, ey = _thick(k, L), _thick(-k, L)
            iq += 1
        elif e == "B":
            h = MBA_ANGLE / L
            k = kb[ib] / (1 + delta)
            ex, ey = _thick(k + h * h, L, h), _thick(-k, L)
            ib += 1
        else:
            ex = ey = _thick(0.0, L)
        elems += [(ex, ey[:2, :2]), (_thick(0.0, MBA_DRIFT), _thick(0.0, MBA_DRIFT)[:2, :2])]
    mx, my = np.eye(3), np.eye(2)
    for ex, ey in elems:
        mx, my = ex @ mx, ey @ my
    cx, cy = np.trace(mx[:2, :2]) / 2, np.trace(my) / 2
    if abs(cx) >= 1 or abs(cy) >= 1:
        return cx, cy, None, None
    eta = np.linalg.solve(np.eye(2) - mx[:2, :2], mx[:2, 2])
    twiss = []
    for m in (mx[:2, :2], my):
        sin_mu = math.copysign(math.sqrt(1 - (np.trace(m) / 2) ** 2), m[0, 1])
        beta, alpha = m[0, 1] / sin_mu, (m[0, 0] - m[1, 1]) / (2 * sin_mu)
        twiss.append(np.array([[beta, -alpha], [-alpha, (1 + alpha * alpha) / beta]]))
    tx, ty = twiss
    v = np.array([eta[0], eta[1], 1.0])
    beta_max, eta_max = max(tx[0, 0], ty[0, 0]), abs(v[0])
    for ex, ey in elems:
        tx, ty, v = ex[:2, :2] @ tx @ ex[:2, :2].T, ey @ ty @ ey.T, ex @ v
        beta_max, eta_max = max(beta_max, tx[0, 0], ty[0, 0]), max(eta_max, abs(v[0]))
    return cx, cy, beta_max, eta_max


def mba_strengths(seed=5, margin=0.9, beta_limit=25.0, eta_limit=0.3, delta_range=8e-3):
    """Seeded C5 magnet strengths: quads alternating in sign with |K1| in
    [1, 6], dipole K1 in [-0.5, 0.5], sextupoles alternating with |K2| in
    [100, 300], octupoles K3 in [-1000, 1000].  Draws continue from `seed`
    upwards until the cell is linearly stable in both planes, with both
    half-traces inside +/-margin, over delta in +/-delta_range, and has
    beta <= beta_limit and |dispersion| <= eta_limit on momentum (a ring
    whose random sextupoles do not lose the 1e-3 momentum spread).  The seed
    used is returned with the strengths."""
    sign = np.array([1.0 if i % 2 == 0 else -1.0 for i in range(12)])
    for s in range(seed, seed + 100000):
        rng = np.random.Generator(np.random.Philox(s))
        kq = sign * rng.uniform(1.0, 6.0, 12)
        kb = rng.uniform(-0.5, 0.5, 7)
        k2 = sign[:6] * rng.uniform(100.0, 300.0, 6)
        k3 = rng.uniform(-1000.0, 1000.0, 2)
        _, _, beta_max, eta_max = mba_cell_optics(kq, kb)
        if beta_max is None or beta_max > beta_limit or eta_max > eta_limit:
            continue
        ok = True
        for d in np.linspace(-delta_range, delta_range, 9):
            cx, cy, _, _ = mba_cell_optics(kq, kb, d)
            if abs(cx) > margin or abs(cy) > margin:
                ok = False
                break
        if ok:
            return {"seed": s, "kq": kq, "kb": kb, "k2": k2, "k3": k3}
    raise RuntimeError("no stable C5 cell found")


def c5_lattice(cells=40, with_rf=True, with_wake=True, n_bins=4000, wake_dt=0.25e-12, charge=1e-9, seed=5,
               kq_errors=None, k2_errors=None):
    """C5: `cells` identical multi-bend-achromat cells (MBA_CELL), then RFCA,
    WAKE and TRWAKE (seeded broadband resonators, Q=1 at 20 GHz, 4096 points
    every 0.25 ps: a 1 ns span, longer than the bunch once the mismatched
    Gaussian has rotated in the bucket; `n_bins` bins) behind a CHARGE
    element.  Error arrays (cells x 12 quads,
    cells x 6 sextupoles) give relative strength errors per magnet."""
    st = mba_strengths(seed)
    lat = Lattice()
    if with_wake:
        lat.add("CHARGE", "Q", TOTAL=charge)
    for c in range(cells):
        iq = ib = i2 = i3 = 0
        for e in MBA_CELL:
            L = MBA_L[e]
            if e == "Q":
                err = kq_errors[c][iq] if kq_errors is not None else 0.0
                lat.add("KQUAD", f"Q{iq + 1}", L=L, K1=st["kq"][iq] * (1 + err), N_KICKS=8)
                iq += 1
            elif e == "B":
                lat.add("CSBEND", f"B{ib + 1}", L=L, ANGLE=MBA_ANGLE, K1=st["kb"][ib], N_KICKS=32)
                ib += 1
            elif e == "S":
                err = k2_errors[c][i2] if k2_errors is not None else 0.0
                lat.add("KSEXT", f"S{i2 + 1}", L=L, K2=st["k2"][i2] * (1 + err), N_KICKS=4)
                i2 += 1
            else:
                lat.add("KOCT", f"O{i3 + 1}", L=L, K3=st["k3"][i3], N_KICKS=4)
                i3 += 1
            lat.add("DRIF", "D", L=MBA_DRIFT)
    if with_rf:
        f_rev = _beta(P_CENTRAL) * C_MKS / lat.total_length()
        lat.add("RFCA", "RF", L=0.0, VOLT=4e6, FREQ=round(352e6 / f_rev) * f_rev, PHASE=180.0)
    if with_wake:
        i = lat.add("WAKE", "W", N_BINS=n_bins, ALLOW_LONG_BEAM=1)
        t, W = resonator_wake(dt=wake_dt, q=1.0, seed=4)
        lat.set_wake(i, t, W)
        i = lat.add("TRWAKE", "TW", N_BINS=n_bins)
        t, Wx = transverse_resonator_wake(dt=wake_dt, seed=6)
        _, Wy = transverse_resonator_wake(dt=wake_dt, seed=7)
        lat.set_wake(i, t, Wx, Wy)
    return lat


def gaussian_beam(n, seed=1, sigma_x=100e-6, sigma_xp=10e-6, sigma_s=3e-3, sigma_dp=1e-3, first_id=1, sigma_y=None):
    """(n, 7) beam: x, x', y, y', s, delta, id with Philox-seeded Gaussians
    (sigma_y defaults to sigma_x)."""
    rng = np.random.Generator(np.random.Philox(seed))
    b = np.empty((n, 7), dtype=np.float64)
    b[:, 0] = rng.normal(0.0, sigma_x, n)
    b[:, 1] = rng.normal(0.0, sigma_xp, n)
    b[:, 2] = rng.normal(0.0, sigma_x if sigma_y is None else sigma_y, n)
    b[:, 3] = rng.normal(0.0, sigma_xp, n)
    b[:, 4] = rng.normal(0.0, sigma_s, n)
    b[:, 5] = rng.normal(0.0, sigma_dp, n)
    b[:, 6] = np.arange(first_id, first_id + n, dtype=np.float64)
    return b


def c5_beam(n, seed=1, first_id=1):
    """C5 beam: the C1 Gaussian with sigma_x = 30 um (sigma_y stays 100 um)."""
    return gaussian_beam(n, seed=seed, sigma_x=30e-6, sigma_y=100e-6, first_id=first_id)


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
