"""Reverse-mode gradients (trk_adjoint) of the tracked-beam objective
mean(x^2+y^2) + w (mean(x)^2 + mean(y)^2) with respect to every KQUAD K1,
KSEXT K2 and CSBEND K1 and K2, against central finite differences (h = 1e-7
relative; 1e-7 m^-2 and 1e-6 m^-3 absolute for a bend's zero K1 and K2) of
the GPU tracking and of elegant's own compiled tracking code; relative
gradient error <= 1e-6."""
import numpy as np
import pytest

from elegant_b200 import Tracker, configs
from elegant_b200.adjoint import fd_step, get_parameters, make_autograd, parameter_list, set_parameters
from oracle import pyoracle

pytestmark = pytest.mark.gpu
PC = configs.P_CENTRAL
W = 0.7


def _lattice(cells=2):
    return configs.c2_lattice(cells=cells, with_rf=False, with_wake=False)


def _beam(n=2000, seed=91):
    b = configs.gaussian_beam(n, seed=seed, sigma_x=1e-3, sigma_xp=5e-5)
    b[:, 0] += 2e-4  # an offset centroid so the centroid term matters
    return b


def _objective_rows(rows, w):
    alive = rows[:, 7] < 0
    x, y = rows[alive, 0], rows[alive, 2]
    return np.mean(x * x + y * y) + w * (np.mean(x) ** 2 + np.mean(y) ** 2)


def _rel_err(g, ref):
    scale = np.maximum(np.abs(ref), 1e-3 * np.max(np.abs(ref)))
    return np.max(np.abs(g - ref) / scale)


def test_adjoint_matches_gpu_finite_differences():
    lat, beam, passes = _lattice(), _beam(), 6
    with Tracker(0) as trk:
        trk.load(beam)
        loss, grad = trk.adjoint(lat, passes, PC, W)
        trk.load(beam)
        trk.track(lat, passes, PC)
        assert abs(trk.objective(W) - loss) <= 1e-14 * abs(loss)
        fd = _gpu_fd(trk, lat, beam, passes, W)
    # 4 KQUAD K1, 4 KSEXT K2, 4 CSBEND (K1, K2)
    names = [n for _, n in parameter_list(lat)]
    assert len(grad) == 16 and names.count("K1") == 8 and np.all(np.isfinite(grad))
    assert _rel_err(grad, fd) < 1e-6, (grad, fd)


@pytest.mark.skipif(not pyoracle.ref_available(), reason="oracle/_ref/libref.so not built")
def test_adjoint_matches_reference_code_finite_differences():
    """Central differences of elegant's own tracking (compiled from the
    reference sources, CPU) on a smaller beam; three parameters sampled.
    The step is 1e-5 relative here: the reference's CSBEND drift forms
    X = rho0 (f - 1) + f X, which turns each rounding of cos() into ~rho0 *
    2^-53 of x, so its loss function carries noise that swamps a 1e-7 step
    (the GPU formulation has no such cancellation and takes h = 1e-7)."""
    lat, beam, passes = _lattice(cells=1), _beam(n=300, seed=92), 4
    k0 = get_parameters(lat)
    plist = parameter_list(lat)
    bend = [i for i, (e, _) in enumerate(plist) if lat.elements[e][0] == "CSBEND"]
    with Tracker(0) as trk:
        trk.load(beam)
        _, grad = trk.adjoint(lat, passes, PC, W)
    for p in (0, 1, bend[0], bend[1]):
        h = fd_step(plist[p][1], k0[p], rel=1e-5)
        vals = []
        for sgn in (1, -1):
            k = k0.copy()
            k[p] += sgn * h
            set_parameters(lat, k)
            rows, _, _ = pyoracle.track_ref(lat, beam, passes, PC)
            vals.append(_objective_rows(rows, W))
        set_parameters(lat, k0)
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(grad[p] - fd) <= 1e-6 * max(abs(fd), 1e-3 * np.max(np.abs(grad))), (p, grad[p], fd)


def test_torch_autograd_wrapper():
    import torch
    lat, beam, passes = _lattice(cells=1), _beam(n=500, seed=93), 3
    fn, trk = make_autograd(lat, beam, passes, PC, W)
    try:
        k = torch.tensor(get_parameters(lat), dtype=torch.float64, requires_grad=True)
        loss = fn.apply(k)
        loss.backward()
        trk.load(beam)
        l2, g2 = trk.adjoint(lat, passes, PC, W)
    finally:
        trk.close()
    # sums over particles and parameter sensitivities use atomic adds: equal to rounding
    assert abs(loss.item() - l2) <= 1e-13 * abs(l2)
    assert np.allclose(k.grad.numpy(), g2, rtol=1e-11, atol=1e-11 * np.max(np.abs(g2)))


def test_losses_are_left_out_and_elements_checked():
    lat = _lattice(cells=1)
    lat.add("MAXAMP", "AP", X_MAX=0.002, Y_MAX=0.002)
    lat.elements.insert(0, lat.elements.pop())
    beam = _beam(n=1000, seed=94)
    with Tracker(0) as trk:
        trk.load(beam)
        loss, grad = trk.adjoint(lat, 3, PC, W)
        assert trk.count() < 1000 and np.all(np.isfinite(grad))
        rf = configs.c2_lattice(cells=1, with_wake=False)
        trk.load(beam)
        with pytest.raises(Exception):
            trk.adjoint(rf, 2, PC, W)


def _gpu_fd(trk, lat, beam, passes, w, params=None, rel=1e-7):
    k0 = get_parameters(lat)
    names = [n for _, n in parameter_list(lat)]
    fd = np.zeros_like(k0)
    for p in (range(len(k0)) if params is None else params):
        h = fd_step(names[p], k0[p], rel)
        vals = []
        for sgn in (1, -1):
            k = k0.copy()
            k[p] += sgn * h
            set_parameters(lat, k)
            trk.load(beam)
            trk.track(lat, passes, PC)
            vals.append(trk.objective(w))
        fd[p] = (vals[0] - vals[1]) / (2 * h)
    set_parameters(lat, k0)
    return fd


def _mba(cells=1, **kw):
    return configs.c5_lattice(cells=cells, with_rf=False, with_wake=False, **kw)


def test_adjoint_through_combined_function_bends():
    """The MBA cell: combined-function CSBENDs (K1 field expansion), strong
    quadrupoles, sextupoles and octupoles; gradient w.r.t. its 12 KQUAD K1,
    6 KSEXT K2 and 7 CSBEND (K1, K2) against GPU central differences."""
    lat, passes = _mba(), 6
    beam = configs.c5_beam(3000, seed=93)
    beam[:, 0] += 5e-5
    with Tracker(0) as trk:
        trk.load(beam)
        loss, grad = trk.adjoint(lat, passes, PC, W)
        trk.load(beam)
        trk.track(lat, passes, PC)
        assert abs(trk.objective(W) - loss) <= 1e-14 * abs(loss)
        fd = _gpu_fd(trk, lat, beam, passes, W)
    assert len(grad) == 32 and np.all(np.isfinite(grad))
    assert np.linalg.norm(grad - fd) / np.linalg.norm(fd) < 1e-6, (grad, fd)
    assert _rel_err(grad, fd) < 1e-5, (grad, fd)


def test_adjoint_ensemble_equals_separate_adjoints():
    """Four error seeds of the MBA cell with uneven particle counts in one
    batched call: each variant's loss and gradient equal its own adjoint run
    (to the order of the atomic sums)."""
    counts = [700, 1300, 64, 950]
    rng = np.random.Generator(np.random.Philox(94))
    lats, beams, first = [], [], 1
    for v, n in enumerate(counts):
        kq = rng.normal(0, 1e-3, (1, 12))
        k2 = rng.normal(0, 2e-3, (1, 6))
        lats.append(_mba(kq_errors=kq, k2_errors=k2))
        b = configs.c5_beam(n, seed=95 + v, first_id=first)
        b[:, 0] += 5e-5
        beams.append(b)
        first += n
    passes = 5
    with Tracker(0) as trk:
        trk.load(np.concatenate(beams))
        losses, grads = trk.adjoint_ensemble(lats, counts, passes, PC, W)
        for v, (lat, b) in enumerate(zip(lats, beams)):
            trk.load(b)
            loss, grad = trk.adjoint(lat, passes, PC, W)
            assert abs(losses[v] - loss) <= 1e-13 * abs(loss), (v, losses[v], loss)
            assert np.max(np.abs(grads[v] - grad)) <= 1e-10 * np.max(np.abs(grad)), v
    assert grads.shape == (4, 32)
    assert np.max(np.abs(grads[0] - grads[1])) > 0  # the variants differ


def test_adjoint_ensemble_vs_finite_differences():
    """The batched gradient of one variant against central differences of
    that variant tracked alone."""
    counts = [800, 1200]
    lats = [_mba(kq_errors=np.full((1, 12), 1e-3 * s), k2_errors=np.full((1, 6), -2e-3 * s)) for s in (1, -1)]
    beams = [configs.c5_beam(800, seed=96), configs.c5_beam(1200, seed=97, first_id=801)]
    passes = 4
    with Tracker(0) as trk:
        trk.load(np.concatenate(beams))
        _, grads = trk.adjoint_ensemble(lats, counts, passes, PC, W)
        fd = _gpu_fd(trk, lats[1], beams[1], passes, W)
    assert np.linalg.norm(grads[1] - fd) / np.linalg.norm(fd) < 1e-6, (grads[1], fd)


def test_adjoint_rejects_misaligned_bend():
    lat = _mba()
    i = next(k for k, e in enumerate(lat.elements) if e[0] == "CSBEND")
    lat.elements[i][2]["DX"] = 1e-4
    with Tracker(0) as trk:
        trk.load(configs.c5_beam(100, seed=98))
        with pytest.raises(RuntimeError):
            trk.adjoint(lat, 2, PC, W)
