"""torch.autograd view of the library's adjoint gradient (used by the gradient tests only).

StirrerLoss.apply(theta, run, inp, nsteps, mask, checkpoint_every) runs the forward of a TDRun
from the seeded start state with the first len(theta) user parameters set to theta and returns
the loss L = sum_r |Delta(r, T)|^2 mask(r) dV as a 0-d float64 tensor.  The forward is the
library's recorded forward (wtd_adjoint_forward: checkpoints every checkpoint_every steps);
the backward is its reverse sweep (wtd_adjoint_backward: segment recompute, adjoint ABM steps)
and returns grad_output * dL/dtheta, so the loss composes with any torch expression.  The run
must not be used between the two.
"""
import numpy as np
import torch


class StirrerLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, run, inp, nsteps, mask, checkpoint_every):
        params = np.array(inp["params"], dtype=np.float64)
        th = theta.detach().cpu().numpy().astype(np.float64)
        params[: th.size] = th
        run.setup(inp["states"], inp["pots"], inp["occ"], params, inp["extra"])
        if ctx.needs_input_grad[0]:
            loss = run.adjoint_forward(nsteps, mask=mask, checkpoint_every=checkpoint_every)
        else:
            loss, _ = run.adjoint(nsteps, mask=mask)
        ctx.run, ctx.nparam, ctx.dtype = run, th.size, theta.dtype
        return torch.tensor(loss, dtype=theta.dtype)

    @staticmethod
    def backward(ctx, grad_output):
        g = torch.from_numpy(ctx.run.adjoint_backward(ctx.nparam)).to(ctx.dtype)
        return grad_output * g, None, None, None, None, None
