"""Test-harness-only torch.autograd.Function around the adjoint entry points
of the monolis C API: forward assembles A(kappa) = sum_e kappa_e K_ref and
solves A x = b (monolis_solve_R); backward solves A^T lambda = dL/dx
(monolis_b200_solve_transpose_R) and reduces -lambda_e^T K_ref x_e per element
(monolis_b200_element_gradient_R). The library itself has no torch types."""
import numpy as np
import torch

from monolis_b200 import api
from monolis_b200 import problems as P


class DiffusionSystem:
    """The scalar Q1 diffusion system of the adjoint workload on an n^3 node
    grid (x = 0 face clamped, b = 1) in one library (product or oracle)."""

    def __init__(self, lib, n, tol=1e-12, precision=0):
        self.lib, self.n, self.tol, self.precision = lib, n, tol, precision
        self.elem = P.hex_elements(n)
        self.kref = P.hex8_diffusion_ke(1.0 / (n - 1))
        self.fixed = P.face_x0_fixed(n, 1)

    def assemble(self, kappa):
        m = api.Monolis(self.lib)
        b, _, _, _ = P.diffusion_kappa(m, n=self.n, kappa=np.ascontiguousarray(kappa, dtype=np.float64))
        m.quiet()
        m.set_error_abort(False)
        m.set_method(api.ITER_CG)
        m.set_precond(api.PREC_DIAG)
        m.set_tolerance(self.tol)
        m.set_maxiter(20000)
        if self.lib.is_product:
            m.set_precision(self.precision)
        return m, b

    def forward(self, kappa):
        m, b = self.assemble(kappa)
        x = np.zeros_like(b)
        m.solve(b, x)
        assert m.get_error_tag() == 0
        return m, x

    def loss(self, kappa, target):
        _, x = self.forward(kappa)
        return 0.5 * float(np.dot(x - target, x - target))


class SolveFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, kappa, system):
        m, x = system.forward(kappa.detach().cpu().numpy())
        ctx.m, ctx.x, ctx.system = m, x, system
        return torch.from_numpy(x.copy())

    @staticmethod
    def backward(ctx, grad_x):
        s, m, x = ctx.system, ctx.m, ctx.x
        lam = np.zeros_like(x)
        rc = m.solve_transpose(np.ascontiguousarray(grad_x.detach().cpu().numpy(), dtype=np.float64), lam)
        assert rc == 0
        g = m.element_gradient(s.elem, 8, s.kref.reshape(-1), 0, lam, x, fixed=s.fixed, scale=-1.0)
        return torch.from_numpy(g), None


def loss_and_grad(system, kappa, target):
    k = torch.tensor(kappa, dtype=torch.float64, requires_grad=True)
    x = SolveFn.apply(k, system)
    L = 0.5 * torch.sum((x - torch.from_numpy(target)) ** 2)
    L.backward()
    return float(L.detach()), k.grad.numpy().copy()
