"""x = D(theta)^{-1} b as a torch.autograd.Function over the C ABI.

Forward: U = exp(i theta) is loaded into an AMGContext, the hierarchy is set up and the
sources are solved (amg_solve_dev).  Backward, for an upstream gradient g = dL/dx (PyTorch's
convention for complex tensors, dL = Re(g^dagger dx)):

    lambda  = D^{-dagger} g          (amg_solve_adjoint_dev: gamma5 D^{-1} gamma5 on the same hierarchy)
    dL/db   = lambda
    dL/dtheta_mu(n) = -Re(lambda^dagger dD/dtheta_mu(n) x)   (amg_force_dev)

The reference has no adjoint; the operator it differentiates is D_phi
(src/dirac_operator.cpp:3-27).  All tensors live on the context's GPU; the library runs on
its own stream and returns after its work is complete, so the caller's stream is
synchronised before each call.
"""
from __future__ import annotations

import torch

from . import AMGContext


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


class DiracSolve(torch.autograd.Function):
    """x = D(theta)^{-1} b.

    theta: float64 [N][2] link angles (U_mu(n) = exp(i theta_mu(n)), mu = 0 time, 1 space);
    b: complex128 [N][2] or [nrhs][N][2]; solver: an AMGContext of the same lattice.
    """

    @staticmethod
    def forward(fctx, theta: torch.Tensor, b: torch.Tensor, solver: AMGContext):
        dev = torch.device("cuda", solver.device)
        U = torch.polar(torch.ones_like(theta, dtype=torch.float64), theta.to(torch.float64))
        solver.set_gauge(U.detach().cpu().numpy())
        solver.setup()
        bd = b.detach().to(device=dev, dtype=torch.complex128).contiguous()
        nrhs = 1 if bd.dim() == 2 else bd.shape[0]
        x = torch.empty_like(bd)
        torch.cuda.current_stream(dev).synchronize()
        infos = solver.solve_dev(_ptr(bd), _ptr(x), nrhs)
        fctx.solver = solver
        fctx.nrhs = nrhs
        fctx.infos = infos
        fctx.theta_shape = theta.shape
        fctx.theta_device = theta.device
        fctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(fctx, gx: torch.Tensor):
        (x,) = fctx.saved_tensors
        solver = fctx.solver
        g = gx.to(device=x.device, dtype=torch.complex128).contiguous()
        lam = torch.empty_like(g)
        F = torch.empty((solver.N, 2), dtype=torch.float64, device=x.device)
        torch.cuda.current_stream(x.device).synchronize()
        solver.solve_adjoint_dev(_ptr(g), _ptr(lam), fctx.nrhs)
        solver.force_dev(_ptr(lam), _ptr(x), fctx.nrhs, _ptr(F))
        return F.reshape(fctx.theta_shape).to(fctx.theta_device), lam, None


def dirac_solve(theta: torch.Tensor, b: torch.Tensor, solver: AMGContext) -> torch.Tensor:
    """Differentiable x = D(theta)^{-1} b (see DiracSolve)."""
    return DiracSolve.apply(theta, b, solver)
