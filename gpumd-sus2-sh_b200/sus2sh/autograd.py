"""torch.autograd.Function over the engine's forward/backward C-ABI pair
(sus2sh_forward / sus2sh_backward).  The engine keeps the state of the last
forward, so each forward must be followed by its backward before the next
forward on the same handle."""
from __future__ import annotations

import torch

from .potential import SUS2_SH, Box


class SiteEnergy(torch.autograd.Function):
    """E_i(positions) with d(sum_i w_i E_i)/d positions from the engine's
    explicit adjoint."""

    @staticmethod
    def forward(ctx, position, engine: SUS2_SH, box: Box, types):
        pe = torch.empty(types.numel(), dtype=torch.float64, device=position.device)
        engine.forward(box, types, position.detach().contiguous(), pe)
        ctx.engine = engine
        ctx.shape = position.shape
        return pe

    @staticmethod
    def backward(ctx, grad_pe):
        grad_pos = torch.empty(ctx.shape, dtype=torch.float64, device=grad_pe.device)
        ctx.engine.backward(grad_pe.contiguous().to(torch.float64), grad_pos)
        return grad_pos, None, None, None


def site_energy(engine: SUS2_SH, box: Box, types, position):
    return SiteEnergy.apply(position, engine, box, types)
