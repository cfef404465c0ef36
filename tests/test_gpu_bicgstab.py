"""Jacobi-BiCGstab on the device (phgGpuSolverBiCGstab) against the oracle's
restatement of solver_BiCGstab (solver-phg.c:606-781), which is pinned bit
for bit against the reference on the golden cases.

The device sums its dot products in a different order than the reference's
sequential loops, so the iterates differ by rounding: iteration counts are
compared within a few iterations, solutions by relative L2 distance
(1e3 * rtol), and every residual is recomputed independently in FP64."""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def convection_diffusion(m, peclet, seed):
    """Upwind convection-diffusion on an m^3 grid (7-point stencil, Dirichlet
    rows eliminated): a non-symmetric M-matrix, CSR with int64 row pointers."""
    rng = np.random.default_rng(seed)
    n = m ** 3
    idx = np.arange(n).reshape(m, m, m)
    rows, cols, vals = [], [], []
    diag = np.full(n, 6.0)
    for ax in range(3):
        w = peclet * (0.5 + rng.random(3))[ax]
        for sgn in (-1, 1):
            a = np.take(idx, range(1, m), axis=ax) if sgn < 0 else np.take(idx, range(m - 1), axis=ax)
            b = np.take(idx, range(m - 1), axis=ax) if sgn < 0 else np.take(idx, range(1, m), axis=ax)
            c = -1.0 - (w if sgn < 0 else 0.0)    # upwind: the upstream neighbour is stronger
            rows.append(a.ravel()); cols.append(b.ravel()); vals.append(np.full(a.size, c))
        diag += w
    rows.append(np.arange(n)); cols.append(np.arange(n)); vals.append(diag)
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    A.sort_indices()
    b = rng.standard_normal(n)
    return A.indptr.astype(np.int64), A.indices.astype(np.int32), A.data.astype(np.float64), b


def resid(oracle, ptr, cols, vals, b, x):
    return np.linalg.norm(b - oracle.spmv(ptr, cols, vals, x))


@pytest.mark.parametrize("m,pe", [(7, 0.5), (20, 3.0), (48, 10.0)])
def test_nonsymmetric_vs_oracle(gpu, oracle, m, pe):
    ptr, cols, vals, b = convection_diffusion(m, pe, seed=m)
    diag = np.asarray(sp.csr_matrix((vals, cols, ptr)).diagonal())
    xo, no, ro, _, st = oracle.bicgstab(ptr, cols, vals, diag, b, rtol=1e-10, btol=0.0, atol=0.0)
    assert st == 0
    with gpu.Solver(0) as s:
        s.set_matrix(ptr, cols, vals, b)
        x, nits, res, hist = s.solve_bicgstab(rtol=1e-10, btol=0.0, atol=0.0, history=True)
    assert abs(nits - no) <= max(2, no // 10)
    assert np.linalg.norm(x - xo) <= 1e3 * 1e-10 * np.linalg.norm(xo)
    assert res <= 1e-10 * hist[0]
    # the recurrence residual tracks the true residual
    assert resid(oracle, ptr, cols, vals, b, x) <= 10 * 1e-10 * np.linalg.norm(b)


def test_assembled_p2_vs_pcg(gpu, oracle):
    """On an assembled SPD system BiCGstab and PCG reach the same solution."""
    v, e = gpu.kuhn_cube(24)
    e2l, bdry, nodes = gpu.lagrange_dofs(v, e, 2)
    with gpu.Solver(0) as s:
        s.set_mesh(v, e)
        s.set_dof_map(2, e2l, bdry)
        s.build_linear_system(f=gpu.sine_source(nodes))
        ptr, cols, vals = s.get_matrix()
        rhs = s.get_rhs()
        xb, nb, rb = s.solve_bicgstab(rtol=1e-10, btol=0.0, atol=0.0)
        xp, npcg, rp = s.solve_pcg(rtol=1e-10, btol=0.0, atol=0.0)
    assert np.linalg.norm(xb - xp) <= 1e-7 * np.linalg.norm(xp)
    assert resid(oracle, ptr, cols, vals, rhs, xb) <= 10 * 1e-10 * np.linalg.norm(rhs)
    assert nb < npcg   # two SpMVs per iteration


def test_small_s_path(gpu, oracle):
    """A diagonal matrix of powers of two: the Jacobi-preconditioned first
    step is exact (v = D (r / D) = r, alpha = 1, s = 0), and the reference's
    ||s|| <= 1e-60 branch corrects x and recomputes the residual from b - A x
    (solver-phg.c:717-729).  Integer right-hand side: every dot product is
    exact in any summation order, so the device takes the branch as well."""
    n = 1001
    d = 2.0 ** np.random.default_rng(2).integers(-2, 4, n)
    ptr = np.arange(n + 1, dtype=np.int64)
    cols = np.arange(n, dtype=np.int32)
    b = np.random.default_rng(3).integers(-8, 9, n).astype(np.float64)
    b[0] = 1.0
    xo, no, ro, _, st = oracle.bicgstab(ptr, cols, d, d, b, rtol=1e-12, btol=0.0, atol=0.0)
    assert st == 2 and no == 1
    with gpu.Solver(0) as s:
        s.set_matrix(ptr, cols, d, b)
        x, nits, res = s.solve_bicgstab(rtol=1e-12, btol=0.0, atol=0.0)
    assert nits == 1
    assert np.array_equal(x, b / d) and np.array_equal(xo, b / d)
    assert res == ro == 0.0


def test_maxit_zero_rhs_and_initial_guess(gpu, oracle):
    ptr, cols, vals, b = convection_diffusion(9, 1.0, seed=4)
    diag = np.asarray(sp.csr_matrix((vals, cols, ptr)).diagonal())
    with gpu.Solver(0) as s:
        s.set_matrix(ptr, cols, vals, b)
        _, nits, _ = s.solve_bicgstab(rtol=1e-14, btol=0.0, atol=0.0, maxit=3)
        assert nits == 3
        x0 = np.linspace(-1, 1, len(b))
        x, nits, res = s.solve_bicgstab(x0=x0, rtol=1e-10, btol=0.0, atol=0.0)
        xo, no, _, _, _ = oracle.bicgstab(ptr, cols, vals, diag, b, x0=x0, rtol=1e-10, btol=0.0, atol=0.0)
        assert abs(nits - no) <= 2
        assert np.linalg.norm(x - xo) <= 1e-7 * np.linalg.norm(xo)
        s.set_matrix(ptr, cols, vals, np.zeros_like(b))
        x, nits, res = s.solve_bicgstab(x0=x0, rtol=1e-10)
        assert nits == 0 and res == 0.0 and not x.any()
