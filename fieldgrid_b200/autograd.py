"""torch.autograd wrapper of the flux-objective adjoint: J(eps_r, sigma) over a design box, with
its gradient from the engine's discrete adjoint (one forward run and one backward sweep on the
device). Torch only carries the parameters and the gradient here; the solve is the engine's."""
from __future__ import annotations

import numpy as np
import torch

from . import fdtd


class FluxObjective(torch.autograd.Function):
    """J = FluxObjective.apply(eps_r, sigma, gpu, scene, spec, driven).

    `scene(eps_r, sigma)` builds the Scene with the design block set to the given arrays (shaped
    like the block); `spec` is the FluxSpec. The forward runs the adjoint whenever an input needs
    a gradient, so backward only scales the stored gradient."""

    @staticmethod
    def forward(ctx, eps, sigma, gpu, scene, spec: fdtd.FluxSpec, driven: int = 0):
        sc = scene(eps.detach().cpu().numpy().astype(np.float32), sigma.detach().cpu().numpy().astype(np.float32))
        sim = fdtd.Sim.try_new(*sc.args())
        want = eps.requires_grad or sigma.requires_grad
        r = fdtd.flux_gradient(gpu, sim, driven, sc.pulse, spec, grad=want)
        if want:
            ctx.save_for_backward(torch.from_numpy(r.grad_eps).to(eps.dtype), torch.from_numpy(r.grad_sigma).to(sigma.dtype))
        ctx.info = r
        return torch.tensor(r.objective, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        ge, gs = ctx.saved_tensors
        g = grad_out.to(ge.dtype)
        return g * ge, g * gs, None, None, None, None
