"""A torch.autograd.Function over the differentiated Z4c evolution: a thin
harness that lets torch code take gradients through the hand-written adjoint
(z4c_adj_gradient, include/z4c_b200.h).

    J = Z4cObjective.apply(u0, ctx, dt, nsteps)   # u0: float64 tensor, the
    J.backward()                                  # state in the register layout
    u0.grad                                        # dJ/du0 from the adjoint run

J is the H-norm objective of the context (volume times the sum over the
history cells of H^2) after nsteps RK4 steps, plus w_step times its sum over
the steps.  The forward pass runs the evolution on the device and keeps the
initial state; the backward pass runs the revolve-checkpointed adjoint from
it (nsnap snapshots) and scales the gradient by the incoming grad_output.
Tensors cross the boundary through host memory (upload / download): the
harness is for checks and small drivers, not the hot loop.
"""
import numpy as np
import torch

from . import REG_ADJ, REG_U


class Z4cObjective(torch.autograd.Function):
    @staticmethod
    def forward(fctx, u0, z4c, dt, nsteps, nsnap=8, w_final=1.0, w_step=0.0):
        state = u0.detach().to("cpu", torch.float64).contiguous().numpy()
        z4c.upload(REG_U, state)
        J = 0.0
        for _ in range(nsteps):
            z4c.evolve(dt, 1)
            if w_step:
                J += w_step * z4c.objective(REG_U)[0]
        J += w_final * z4c.objective(REG_U)[0]
        fctx.save_for_backward(u0)
        fctx.z4c, fctx.args = z4c, (dt, nsteps, nsnap, w_final, w_step)
        return torch.tensor(J, dtype=torch.float64, device=u0.device)

    @staticmethod
    def backward(fctx, grad_output):
        (u0,) = fctx.saved_tensors
        z4c = fctx.z4c
        dt, nsteps, nsnap, w_final, w_step = fctx.args
        z4c.upload(REG_U, u0.detach().to("cpu", torch.float64).contiguous().numpy())
        z4c.gradient(dt, nsteps, nsnap, w_final, w_step)
        g = torch.from_numpy(np.ascontiguousarray(z4c.download(REG_ADJ))).to(u0.device)
        return grad_output * g, None, None, None, None, None, None
