"""Gradients of tracked-beam objectives through the C ABI's reverse-mode
adjoint (trk_adjoint), with a torch.autograd.Function wrapper.

The parameters are, in lattice order, the K1 of every KQUAD, the K2 of every
KSEXT and the K1 and K2 of every CSBEND; the objective is
    mean(x^2 + y^2) + w (mean(x)^2 + mean(y)^2)
over the particles that survive n_passes passes.
"""
import numpy as np

from . import Tracker

PARAM_NAMES = {"KQUAD": ("K1",), "KSEXT": ("K2",), "CSBEND": ("K1", "K2")}
# finite-difference step scale of each name where the value itself is zero
PARAM_SCALE = {"K1": 1.0, "K2": 10.0}


def parameter_list(lattice):
    """(element index, parameter name) of every gradient entry, in order."""
    return [(i, n) for i, (t, _, _, _) in enumerate(lattice.elements) for n in PARAM_NAMES.get(t, ())]


def parameter_elements(lattice):
    """Element index of every gradient entry (a CSBEND appears twice)."""
    return [i for i, _ in parameter_list(lattice)]


def get_parameters(lattice):
    return np.array([lattice.elements[i][2].get(n, 0.0) for i, n in parameter_list(lattice)])


def set_parameters(lattice, values):
    plist = parameter_list(lattice)
    if len(plist) != len(values):
        raise ValueError(f"{len(values)} values for {len(plist)} parameters")
    for (i, n), v in zip(plist, values):
        lattice.elements[i][2][n] = float(v)


def fd_step(name, value, rel=1e-7):
    """Central-difference step: rel x |value|, or rel x the name's scale for a zero value."""
    return rel * (abs(value) if value != 0 else PARAM_SCALE.get(name, 1.0))


def loss_and_grad(tracker, lattice, beam, n_passes, p_central, centroid_weight=0.0):
    tracker.load(beam)
    return tracker.adjoint(lattice, n_passes, p_central, centroid_weight)


def make_autograd(lattice, beam, n_passes, p_central, centroid_weight=0.0, device=0, tracker=None):
    """A torch.autograd.Function whose forward maps the parameter vector to
    the objective (tracking on the GPU) and whose backward returns the
    adjoint gradient, and the Tracker it tracks with.  Pass `tracker` to
    track with one of your own; otherwise a new Tracker is created, and the
    caller owns it: close it (tracker.close(), or use it in a with block)
    when the function is no longer needed."""
    import torch

    if tracker is None:
        tracker = Tracker(device)

    class TrackedLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, params):
            set_parameters(lattice, params.detach().cpu().numpy().astype(np.float64))
            loss, grad = loss_and_grad(tracker, lattice, beam, n_passes, p_central, centroid_weight)
            ctx.save_for_backward(torch.as_tensor(grad, dtype=params.dtype))
            return params.new_tensor(loss)

        @staticmethod
        def backward(ctx, grad_out):
            (grad,) = ctx.saved_tensors
            return grad_out * grad

    return TrackedLoss, tracker
