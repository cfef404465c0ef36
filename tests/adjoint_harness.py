"""Gradient test harness: a torch.autograd.Function over the C ABI.

J(log kappa) = 1/2 ||u(kappa) - u_obs||^2 where u solves the assembled
Poisson system with the per-element coefficient kappa; forward runs the
device assembly + FP64 PCG, backward returns the adjoint gradient
(phgGpuAdjointGradient).  Used only by the tests.
"""
import numpy as np
import torch


class MisfitProblem:
    def __init__(self, pb, order, verts, elems, e2l, bdry, f, u_obs, rtol=1e-10):
        self.s = pb.Solver(0)
        self.s.set_mesh(verts, elems)
        self.s.set_dof_map(order, e2l, bdry)
        self.f, self.u_obs, self.rtol = f, u_obs, rtol

    def solve(self, kappa, rtol=None):
        self.s.build_linear_system(kappa=kappa, f=self.f)
        u, nits, _ = self.s.solve_pcg(rtol=self.rtol if rtol is None else rtol, btol=0.0, atol=0.0,
                                      maxit=200000)
        return u

    def misfit(self, kappa, rtol=None):
        u = self.solve(kappa, rtol)
        return 0.5 * float(np.sum((u - self.u_obs) ** 2))


class LogKappaMisfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, logk, problem):
        kappa = np.exp(logk.detach().cpu().numpy().astype(np.float64))
        u = problem.solve(kappa)
        grad, J, _ = problem.s.adjoint_gradient(u, problem.u_obs, rtol=problem.rtol)
        ctx.save_for_backward(torch.from_numpy(grad).to(logk.device, logk.dtype))
        return torch.tensor(J, dtype=logk.dtype, device=logk.device)

    @staticmethod
    def backward(ctx, gJ):
        (grad,) = ctx.saved_tensors
        return gJ * grad, None
