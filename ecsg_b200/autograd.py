"""torch.autograd.Function over the device misfit gradient (ecsg_misfit_gradient).

    loss = MisfitGradient.apply(sim_case, observed, ckpt_every, precision, b0, c0_0, ..., c0_20, b1, ...)

takes the medium of every grid as tensors (node buoyancy, then the 21 stiffness
slots of ecsg_set_medium_cij21, per grid), runs the forward from rest and the
checkpointed adjoint on the device, and returns the misfit
1/2 sum (receiver samples - observed)^2; backward hands back the device
gradients.  The tensors only carry values across the boundary: the
computation is the library's.
"""
import copy

import numpy as np
import torch

from . import Simulation

__all__ = ["MisfitGradient", "misfit"]


class MisfitGradient(torch.autograd.Function):
    @staticmethod
    def forward(ctx, case, observed, ckpt_every, precision, *medium):
        ng = len(case.grids)
        c = copy.copy(case)
        c.medium = "gen21"
        c.media = []
        for g in range(ng):
            t = medium[22 * g: 22 * (g + 1)]
            c.media.append({"buoy": t[0].detach().cpu().double().numpy(),
                            "c21": [x.detach().cpu().double().numpy() for x in t[1:]]})
        obs = observed.detach().cpu().float().numpy() if torch.is_tensor(observed) else np.asarray(observed, np.float32)
        with Simulation(c, precision=precision) as sim:
            loss = sim.misfit_gradient(obs, ckpt_every=ckpt_every)
            grads = [torch.from_numpy(sim.gradient(g, w)).to(medium[22 * g + w].dtype)
                     for g in range(ng) for w in range(22)]
        ctx.save_for_backward(*grads)
        return torch.tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_loss):
        grads = ctx.saved_tensors
        return (None, None, None, None) + tuple(grad_loss.to(g.dtype) * g for g in grads)


def misfit(case, observed, medium, ckpt_every=50, precision="f64"):
    """medium: list over grids of [buoyancy, c0, ..., c20] tensors."""
    flat = [t for grid in medium for t in grid]
    return MisfitGradient.apply(case, observed, ckpt_every, precision, *flat)
