"""Restarted right-preconditioned Jacobi-GMRES on the device
(phgGpuSolverGMRES) against the oracle's restatement of solver_GMRES_r
(solver-phg.c:1050-1260), which is pinned bit for bit against the reference
on the golden cases.

The device's dot products sum in a different order than the reference's
loops, so iterates differ by rounding: iteration counts are compared within
a few iterations, solutions by relative L2 distance (1e3 * rtol), and the
true residual of the device solution is recomputed in FP64."""
import numpy as np
import pytest
import scipy.sparse as sp

from test_gpu_bicgstab import convection_diffusion, resid

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,pe,restart", [(7, 0.5, 10), (20, 3.0, 10), (20, 3.0, 30), (48, 10.0, 10)])
def test_nonsymmetric_vs_oracle(gpu, oracle, m, pe, restart):
    ptr, cols, vals, b = convection_diffusion(m, pe, seed=m)
    diag = np.asarray(sp.csr_matrix((vals, cols, ptr)).diagonal())
    xo, no, ro = oracle.gmres(ptr, cols, vals, diag, b, restart=restart, rtol=1e-10, btol=0.0, atol=0.0)
    with gpu.Solver(0) as s:
        s.set_matrix(ptr, cols, vals, b)
        x, nits, res = s.solve_gmres(restart=restart, rtol=1e-10, btol=0.0, atol=0.0)
    assert abs(nits - no) <= max(2, no // 20)
    assert np.linalg.norm(x - xo) <= 1e3 * 1e-10 * np.linalg.norm(xo)
    assert res <= 1e-10 * np.linalg.norm(b)
    assert resid(oracle, ptr, cols, vals, b, x) <= 10 * 1e-10 * np.linalg.norm(b)


def test_assembled_p2_vs_pcg(gpu, oracle):
    v, e = gpu.kuhn_cube(24)
    e2l, bdry, nodes = gpu.lagrange_dofs(v, e, 2)
    with gpu.Solver(0) as s:
        s.set_mesh(v, e)
        s.set_dof_map(2, e2l, bdry)
        s.build_linear_system(f=gpu.sine_source(nodes))
        ptr, cols, vals = s.get_matrix()
        rhs = s.get_rhs()
        diag = s.get_diagonal()
        xg, ng, rg = s.solve_gmres(restart=20, rtol=1e-10, btol=0.0, atol=0.0)
        xp, npcg, rp = s.solve_pcg(rtol=1e-10, btol=0.0, atol=0.0)
    xo, no, ro = oracle.gmres(ptr, cols, vals, diag, rhs, restart=20, rtol=1e-10, btol=0.0, atol=0.0)
    assert abs(ng - no) <= max(2, no // 20)
    assert np.linalg.norm(xg - xp) <= 1e-6 * np.linalg.norm(xp)
    assert resid(oracle, ptr, cols, vals, rhs, xg) <= 10 * 1e-10 * np.linalg.norm(rhs)


def test_happy_breakdown(gpu, oracle):
    """b = 4 e_0 and a power-of-two diagonal: the first Arnoldi vector is
    mapped onto itself, h_21 = 0 exactly, and the reference's happy-breakdown
    branch (solver-phg.c:1149-1153) drops the step; x += z / diag then gives
    the exact solution and the next cycle stops with residual 0."""
    n = 64
    d = 2.0 ** np.random.default_rng(1).integers(-2, 4, n)
    ptr = np.arange(n + 1, dtype=np.int64)
    cols = np.arange(n, dtype=np.int32)
    b = np.zeros(n)
    b[0] = 4.0
    xo, no, ro = oracle.gmres(ptr, cols, d, d, b, restart=10, rtol=1e-12, btol=0.0, atol=0.0)
    assert no == 1 and ro == 0.0 and np.array_equal(xo, b / d)
    with gpu.Solver(0) as s:
        s.set_matrix(ptr, cols, d, b)
        x, nits, res = s.solve_gmres(restart=10, rtol=1e-12, btol=0.0, atol=0.0)
    assert nits == 1 and res == 0.0 and np.array_equal(x, b / d)


def test_maxit_zero_rhs_restart_limit(gpu, oracle):
    ptr, cols, vals, b = convection_diffusion(9, 1.0, seed=4)
    diag = np.asarray(sp.csr_matrix((vals, cols, ptr)).diagonal())
    with gpu.Solver(0) as s:
        s.set_matrix(ptr, cols, vals, b)
        # maxit ends the solve: the reference reports ||r0|| (solver-phg.c:1090, 1254)
        x, nits, res = s.solve_gmres(restart=5, rtol=1e-14, btol=0.0, atol=0.0, maxit=7)
        xo, no, ro = oracle.gmres(ptr, cols, vals, diag, b, restart=5, maxit=7, rtol=1e-14, btol=0.0, atol=0.0)
        assert nits == no == 7
        assert res == pytest.approx(np.linalg.norm(b), rel=1e-12) and ro == pytest.approx(res, rel=1e-12)
        assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)
        x0 = np.linspace(-1, 1, len(b))
        x, nits, res = s.solve_gmres(x0=x0, restart=10, rtol=1e-10, btol=0.0, atol=0.0)
        xo, no, _ = oracle.gmres(ptr, cols, vals, diag, b, x0=x0, restart=10, rtol=1e-10, btol=0.0, atol=0.0)
        assert abs(nits - no) <= 2
        assert np.linalg.norm(x - xo) <= 1e-7 * np.linalg.norm(xo)
        with pytest.raises(gpu.PhgGpuError) as ei:
            s.solve_gmres(restart=65)
        assert ei.value.code == -4
        s.set_matrix(ptr, cols, vals, np.zeros_like(b))
        x, nits, res = s.solve_gmres(x0=x0, rtol=1e-10)
        assert nits == 0 and res == 0.0 and not x.any()
