"""Differentiable TOR projector.

* ``TorProject``: forward = TOR projection A x of one axis group (image in the kernel
  layout), backward = the plain adjoint A^T g (``srf_tor_backproject_adjoint``).
* ``TorBackproject``: forward = A^T v, backward = A g. Together they make any
  composition of projections and back-projections differentiable, including the
  reference's back-projection A^T(1/Ax) written as ``TorBackproject(1 / TorProject(x))``.
* ``project(model, image, data)``: all three dominant-axis groups of a SplitLoRsModel,
  differentiable w.r.t. the [nx, ny, nz] image (the axis transposes are torch ops).
* ``poisson_nll``: list-mode Poisson negative log-likelihood
  sum_j s_j x_j - sum_i log((A x)_i) (s = sensitivity), and the per-event form
  sum_i ((A x)_i - log (A x)_i); ``quadratic_penalty``: beta/2 sum over 6-neighbour
  pairs of (x_j - x_k)^2.
* ``unrolled_osem``: K differentiable OSEM (MLEM) iterations
  x <- x * effinv * A^T(1/(A x)), each under ``torch.utils.checkpoint`` so only the
  iterates are stored.

There is no counterpart in the reference (its TF ops have no registered gradients).
"""

import torch
import torch.utils.checkpoint as cp

from . import ops
from .data import Image
from .physics import SplitLoRsModel


class TorProject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, image_k, lors, geom, model):
        g, c, s = geom
        out = ops.tor_projection(lors, image_k.contiguous(), g, c, s, model.kernel_width,
                                 model.geo_sigma2_flag, model.tof_bin, model.tof_sigma2,
                                 layout="nc")
        ctx.save_for_backward(lors)
        ctx.geom, ctx.model = geom, model
        return out

    @staticmethod
    def backward(ctx, grad_out):
        (lors,) = ctx.saved_tensors
        g, c, s = ctx.geom
        m = ctx.model
        grad = ops.tor_backproject_adjoint(grad_out.contiguous(), lors, g, c, s, m.kernel_width,
                                           m.geo_sigma2_flag, m.tof_bin, m.tof_sigma2,
                                           layout="nc")
        return grad, None, None, None


class TorBackproject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, lors, geom, model):
        g, c, s = geom
        out = ops.tor_backproject_adjoint(values.contiguous(), lors, g, c, s, model.kernel_width,
                                          model.geo_sigma2_flag, model.tof_bin,
                                          model.tof_sigma2, layout="nc")
        ctx.save_for_backward(lors)
        ctx.geom, ctx.model = geom, model
        return out

    @staticmethod
    def backward(ctx, grad_img):
        (lors,) = ctx.saved_tensors
        g, c, s = ctx.geom
        m = ctx.model
        grad = ops.tor_projection(lors, grad_img.contiguous(), g, c, s, m.kernel_width,
                                  m.geo_sigma2_flag, m.tof_bin, m.tof_sigma2, layout="nc")
        return grad, None, None, None


class Projector:
    """Differentiable A and A^T for one SplitLoRsModel, LOR set and image geometry."""

    def __init__(self, model, data, grid, center, size):
        if not isinstance(model, SplitLoRsModel):
            raise TypeError("the differentiable projector runs the TOR model")
        self.model = model
        self.lors = {a: data[a].lors for a in model.AXIS}
        probe = Image(torch.empty(grid, device=next(iter(self.lors.values())).device), center,
                      size)
        self.geom = {a: model.kernel_geometry(probe, a)[1:] for a in model.AXIS}
        self.grid = list(grid)

    def forward(self, x):
        """{'x','y','z'}: projections of the [nx, ny, nz] image x (differentiable)."""
        m = self.model
        return {a: TorProject.apply(x.permute(*m.perm(a)), self.lors[a], self.geom[a], m)
                for a in m.AXIS if self.lors[a].shape[0] > 0}

    def adjoint(self, values):
        """A^T values as an [nx, ny, nz] image (differentiable in the values)."""
        m = self.model
        out = None
        for a, v in values.items():
            b = TorBackproject.apply(v, self.lors[a], self.geom[a], m).permute(*m.perm_back(a))
            out = b if out is None else out + b
        return out

    def reference_backprojection(self, x):
        """A^T(1/(A x)) — the reference's back-projection of its own projection, with
        its 1e-7 threshold — differentiable w.r.t. x."""
        p = self.forward(x)
        inv = {a: torch.where(v > 1e-7, 1.0 / torch.clamp(v, min=1e-30), torch.zeros_like(v))
               for a, v in p.items()}
        return self.adjoint(inv)


def poisson_nll(proj, x=None, sensitivity=None, per_event=False):
    """List-mode Poisson NLL: sum_j s_j x_j - sum_i log p_i, or with ``per_event`` the
    form sum_i (p_i - log p_i). ``proj`` is a dict of projections."""
    p = torch.cat([v for v in proj.values()])
    logp = torch.log(torch.clamp(p, min=1e-30))
    if per_event:
        return (p - logp).sum()
    if sensitivity is None or x is None:
        raise ValueError("the list-mode NLL needs the image and its sensitivity")
    return (sensitivity * x).sum() - logp.sum()


def quadratic_penalty(x, beta=0.01):
    """beta/2 * sum over 6-neighbour pairs (each pair once) of (x_j - x_k)^2."""
    d0 = x[1:, :, :] - x[:-1, :, :]
    d1 = x[:, 1:, :] - x[:, :-1, :]
    d2 = x[:, :, 1:] - x[:, :, :-1]
    return 0.5 * beta * ((d0 * d0).sum() + (d1 * d1).sum() + (d2 * d2).sum())


def unrolled_osem(projector, x0, effinv, n_iterations=5, checkpoint=True):
    """K differentiable MLEM iterations x <- x * effinv * A^T(1/(A x)); with
    ``checkpoint`` each iteration is recomputed in the backward pass instead of storing
    its intermediates."""
    def one(x):
        return x * effinv * projector.reference_backprojection(x)

    x = x0
    for _ in range(n_iterations):
        x = cp.checkpoint(one, x, use_reentrant=False) if checkpoint else one(x)
    return x
