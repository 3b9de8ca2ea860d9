"""torch.autograd binding of the discrete adjoint (a thin test binding).

`DragFn.apply(s, sim, box, nsteps, window)` returns the time-averaged drag J
of `nsteps` steps of lattice `sim` from its current state, with the solid
fraction `s` (a [z][y][x] tensor over `box`) applied by partial bounce-back.
Its backward calls wt_adjoint through the C ABI from the same starting state
(saved with wt_get_state), so autograd sees the hand-written discrete adjoint
of the fused CUDA step; nothing is differentiated by torch itself.
"""
from __future__ import annotations

import numpy as np
import torch

from .lbm import LBM


class DragFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, s: torch.Tensor, sim: LBM, box, nsteps: int, window: int,
                component: int = 0, checkpoint: int = 0, keep: bool = False):
        sv = s.detach().to("cpu", torch.float64).numpy()
        sim.set_solid_fraction(box, sv)
        start = sim.get_state()
        f = sim.step_forces(int(nsteps))
        J = float(f[-int(window):, component].mean())
        ctx.sim, ctx.box, ctx.start, ctx.sv = sim, box, start, sv
        ctx.cfg = (int(nsteps), int(window), int(component), int(checkpoint), bool(keep))
        ctx.s_meta = (s.dtype, s.device)
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ: torch.Tensor):
        sim = ctx.sim
        end = sim.get_state()
        sim.set_state(ctx.start)
        sim.set_solid_fraction(ctx.box, ctx.sv)
        _, g, _ = sim.adjoint(*ctx.cfg)
        sim.set_state(end)   # the lattice stays where the forward pass left it
        dtype, device = ctx.s_meta
        grad = torch.from_numpy(np.ascontiguousarray(g)).to(device=device, dtype=dtype)
        return gJ.to(dtype) * grad, None, None, None, None, None, None, None


def drag(s: torch.Tensor, sim: LBM, box, nsteps: int, window: int, component: int = 0,
         checkpoint: int = 0, keep: bool = False) -> torch.Tensor:
    """Time-averaged force component with the discrete adjoint as its gradient.
    keep: the backward pass leaves its device memory in `sim` for the next
    backward (an optimisation loop over the same lattice)."""
    return DragFn.apply(s, sim, box, nsteps, window, component, checkpoint, keep)
