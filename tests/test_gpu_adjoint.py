"""Adjoint gradient dJ/dlog kappa_e (phgGpuAdjointGradient) through a
torch.autograd.Function harness, checked against central finite differences
of the device solves and against finite differences of the CPU oracle's
solves.  Tolerance: 1e-5 relative (to the gradient's largest entry on the
checked elements)."""
import numpy as np
import pytest
import torch

from adjoint_harness import LogKappaMisfit, MisfitProblem

pytestmark = pytest.mark.gpu


def make_problem(pb, p, m, seed):
    v, e = pb.kuhn_cube(m)
    e2l, bdry, nodes = pb.lagrange_dofs(v, e, p)
    f = pb.sine_source(nodes)
    rng = np.random.default_rng(seed)
    logk = rng.standard_normal(len(e))
    kappa_obs = np.exp(rng.standard_normal(len(e)))
    prob = MisfitProblem(pb, p, v, e, e2l, bdry, f, np.zeros(len(bdry)))
    u_obs = prob.solve(kappa_obs, rtol=1e-12) + 0.01 * rng.standard_normal(len(bdry))
    u_obs[bdry.astype(bool)] = 0.0
    prob.u_obs = u_obs
    return prob, logk, (v, e, e2l, bdry, f, u_obs)


@pytest.mark.parametrize("p,m", [(1, 6), (2, 3)])
def test_adjoint_matches_central_differences(gpu, p, m):
    prob, logk, _ = make_problem(gpu, p, m, 42)
    lk = torch.tensor(logk, requires_grad=True)
    J = LogKappaMisfit.apply(lk, prob)
    (g,) = torch.autograd.grad(J, lk)
    g = g.numpy()
    rng = np.random.default_rng(1)
    els = rng.choice(len(logk), 16, replace=False)
    h = 1e-6
    fd = []
    for e in els:
        kp, km = np.exp(logk.copy()), np.exp(logk.copy())
        kp[e] = np.exp(logk[e] + h)
        km[e] = np.exp(logk[e] - h)
        fd.append((prob.misfit(kp, rtol=1e-13) - prob.misfit(km, rtol=1e-13)) / (2 * h))
    fd = np.array(fd)
    scale = np.max(np.abs(g[els]))
    err = np.max(np.abs(fd - g[els])) / scale
    print("p=%d m=%d: max rel FD error %.2e (scale %.3e)" % (p, m, err, scale))
    assert err < 1e-5


def test_adjoint_matches_cpu_oracle_differences(gpu, oracle):
    """Reference gradient from the repo's own CPU solves (oracle assembly +
    oracle PCG), by central differences on a few elements."""
    prob, logk, (v, e, e2l, bdry, f, u_obs) = make_problem(gpu, 1, 5, 7)
    u = prob.solve(np.exp(logk))
    g, J, _ = prob.s.adjoint_gradient(u, u_obs, rtol=1e-12)

    def cpu_misfit(kappa):
        o = oracle.assemble(1, v, e, e2l, bdry, f, None, kappa)
        x, _, _, _ = oracle.pcg(o["ptr"], o["cols"], o["vals"], o["diag"], o["rhs"], rtol=1e-13,
                                btol=0.0, atol=0.0, maxit=100000)
        return 0.5 * np.sum((x - u_obs) ** 2)

    assert abs(cpu_misfit(np.exp(logk)) - J) <= 1e-9 * abs(J)
    h = 1e-6
    els = np.random.default_rng(3).choice(len(e), 6, replace=False)
    for el in els:
        kp, km = np.exp(logk), np.exp(logk)
        kp[el] = np.exp(logk[el] + h)
        km[el] = np.exp(logk[el] - h)
        fd = (cpu_misfit(kp) - cpu_misfit(km)) / (2 * h)
        assert abs(fd - g[el]) <= 1e-5 * np.max(np.abs(g)), (el, fd, g[el])


def test_adjoint_zero_at_perfect_data(gpu):
    """u_obs = u gives J = 0 and a zero gradient."""
    prob, logk, (v, e, e2l, bdry, f, u_obs) = make_problem(gpu, 2, 3, 5)
    u = prob.solve(np.exp(logk))
    g, J, nits = prob.s.adjoint_gradient(u, u, rtol=1e-10)
    assert J == 0.0 and nits == 0 and not g.any()
