"""torch.autograd view of the discrete adjoint (dsem_adjoint), for checking.

``objective(jq0, inv_re, case)`` returns J, the sum of eps * dt over the last
``case.window`` of ``case.nsteps`` steps started from ``jq0`` (the enstrophy
dissipation eps that dsem_diag reports after each step), as a 0-d float64
tensor.  Its backward pass returns dJ/djq0 and dJ/d(1/Re) computed by the
library's hand-written adjoint, so ``J.backward()`` (or torch.autograd.grad)
exposes the adjoint to torch code and to torch's own checking tools.

The context's Reynolds number is fixed when it is created: ``inv_re`` must
equal 1/Re of ``case``'s solver and is an input only so that torch tracks the
derivative.  ``jq0`` is in the solver's upload layout [ngrid][5][ldx]^3.
"""
import numpy as np
import torch

from .solver import Solver


class AdjointCase:
    """A solver and the run whose objective is differentiated."""

    def __init__(self, desc, re, dt, nsteps, window, snapshots=0, **phys):
        self.re = float(re)
        self.dt, self.nsteps, self.window, self.snapshots = float(dt), int(nsteps), int(window), int(snapshots)
        self.solver = Solver(desc, re=self.re, **phys)

    def close(self):
        self.solver.close()


class DsemObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, jq0, inv_re, case):
        if abs(float(inv_re) - 1.0 / case.re) > 1e-14 / case.re:
            raise ValueError("inv_re must equal 1/Re of the case's solver")
        s = case.solver
        s.upload(jq0.detach().to("cpu", torch.float64).numpy())
        J, g, lr, _ = s.adjoint(case.dt, case.nsteps, case.window, case.snapshots, want_grad=True)
        ctx.save_for_backward(torch.from_numpy(np.ascontiguousarray(g)).to(jq0.device),
                              torch.tensor(lr, dtype=torch.float64, device=inv_re.device))
        return torch.tensor(J, dtype=torch.float64, device=jq0.device)

    @staticmethod
    def backward(ctx, gJ):
        g, lr = ctx.saved_tensors
        return gJ * g, gJ * lr, None


def objective(jq0, inv_re, case):
    """J(jq0, 1/Re) with the library's adjoint as its backward pass."""
    return DsemObjective.apply(jq0, inv_re, case)
