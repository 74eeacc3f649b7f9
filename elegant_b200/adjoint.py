"""Gradients of tracked-beam objectives through the C ABI's reverse-mode
adjoint (trk_adjoint), with a torch.autograd.Function wrapper.

The parameters are the K1 of every KQUAD and the K2 of every KSEXT of a
lattice, in lattice order; the objective is
    mean(x^2 + y^2) + w (mean(x)^2 + mean(y)^2)
over the particles that survive n_passes passes.
"""
import numpy as np

from . import Tracker

PARAM_NAME = {"KQUAD": "K1", "KSEXT": "K2"}


def parameter_elements(lattice):
    """Element indices of the gradient parameters, in gradient order."""
    return [i for i, (t, _, _, _) in enumerate(lattice.elements) if t in PARAM_NAME]


def get_parameters(lattice):
    return np.array([lattice.elements[i][2].get(PARAM_NAME[lattice.elements[i][0]], 0.0)
                     for i in parameter_elements(lattice)])


def set_parameters(lattice, values):
    idx = parameter_elements(lattice)
    if len(idx) != len(values):
        raise ValueError(f"{len(values)} values for {len(idx)} parameters")
    for i, v in zip(idx, values):
        lattice.elements[i][2][PARAM_NAME[lattice.elements[i][0]]] = float(v)


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
