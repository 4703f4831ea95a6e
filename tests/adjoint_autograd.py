"""torch.autograd view of the library's adjoint gradient (used by the gradient tests only).

StirrerLoss.apply(theta, run, inp, nsteps, mask, checkpoint_every) runs the forward of a TDRun
from the seeded start state with the first len(theta) user parameters set to theta and returns
the loss L = sum_r |Delta(r, T)|^2 mask(r) dV as a 0-d float64 tensor.  Its backward returns
grad_output * dL/dtheta from the library's reverse sweep (wtd_adjoint: checkpointed forward,
segment recompute, adjoint ABM steps), so the loss composes with any torch expression.
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
        need = ctx.needs_input_grad[0]
        loss, grad = run.adjoint(nsteps, nparam=th.size if need else 0, mask=mask, checkpoint_every=checkpoint_every)
        if need:
            ctx.save_for_backward(torch.from_numpy(grad).to(theta.dtype))
        return torch.tensor(loss, dtype=theta.dtype)

    @staticmethod
    def backward(ctx, grad_output):
        (g,) = ctx.saved_tensors
        return grad_output * g, None, None, None, None, None
