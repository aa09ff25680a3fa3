"""torch.autograd.Function over the C ABI's adjoint gradient (check harness only).

J(amplitudes) runs lee_adjoint_gradient, which returns the objective and its gradient with
respect to the distributed source's lattice amplitudes; backward scales that gradient.
"""
from __future__ import annotations

import copy

import numpy as np
import torch

from camille_b200 import api


class LeeObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, amps, lib, case, dt, checkpoint_every: int = 5):
        c = copy.deepcopy(case)
        c.distributed.amplitudes = np.ascontiguousarray(amps.detach().cpu().numpy(), np.float64)
        s = api.Solver(lib, c)
        J, g, mism = s.adjoint_gradient(c.nsteps, dt, checkpoint_every=checkpoint_every, recompute=True)
        s.close()
        if mism:
            raise RuntimeError(f"checkpoint replay differs in {mism} trace values")
        ctx.save_for_backward(torch.from_numpy(g).to(amps))
        return amps.new_tensor(J)

    @staticmethod
    def backward(ctx, gout):
        (g,) = ctx.saved_tensors
        return gout * g, None, None, None, None
