"""Block PCG over many right-hand sides (phgGpuSolverBlockPCG): every column
must match the single-vector PCG of the CPU oracle (iteration count within 2,
solution within relative L2 distance 1e3 * rtol, residual recomputed in FP64
by the oracle), in FP64 and in the mixed FP32/FP64 mode."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def assembled(pb, p, m):
    v, e = pb.kuhn_cube(m)
    e2l, bdry, nodes = pb.lagrange_dofs(v, e, p)
    s = pb.Solver(0)
    s.set_mesh(v, e)
    s.set_dof_map(p, e2l, bdry)
    s.build_linear_system(f=pb.sine_source(nodes))
    return s, bdry


def rhs_block(bdry, nrhs, seed):
    B = np.random.default_rng(seed).standard_normal((len(bdry), nrhs))
    B[bdry.astype(bool)] = 0.0
    return np.ascontiguousarray(B)


@pytest.mark.parametrize("nrhs,mixed", [(1, False), (3, False), (16, False), (64, False),
                                        (5, True), (64, True)])
def test_block_columns_match_oracle(gpu, oracle, nrhs, mixed):
    s, bdry = assembled(gpu, 2, 6)
    ptr, cols, vals = s.get_matrix()
    diag = s.get_diagonal()
    B = rhs_block(bdry, nrhs, 11 + nrhs)
    rtol = 1e-8
    X, nits, res = s.solve_block_pcg(B, rtol=rtol, mixed=mixed)
    for k in range(nrhs):
        xo, no, _, _ = oracle.pcg(ptr, cols, vals, diag, B[:, k], rtol=rtol, btol=0.0, atol=0.0)
        r = B[:, k] - oracle.spmv(ptr, cols, vals, X[:, k])
        assert np.linalg.norm(r) <= rtol * np.linalg.norm(B[:, k]) * (1 + 1e-9), k
        assert abs(res[k] - np.linalg.norm(r)) <= 1e-6 * np.linalg.norm(r) + 1e-300
        if not mixed:
            assert abs(int(nits[k]) - no) <= 2, (k, nits[k], no)
        else:
            assert int(nits[k]) <= 1.5 * no + 5
        assert np.linalg.norm(X[:, k] - xo) <= 1e3 * rtol * np.linalg.norm(xo)
    tile, times = s.block_tile()
    assert tile in (8, 16, 32, 64)
    s.close()


def test_block_zero_columns_and_limit(gpu):
    s, bdry = assembled(gpu, 1, 6)
    B = rhs_block(bdry, 4, 3)
    B[:, 2] = 0.0
    X, nits, res = s.solve_block_pcg(B, rtol=1e-10)
    assert nits[2] == 0 and not X[:, 2].any()
    with pytest.raises(gpu.PhgGpuError) as ei:
        s.solve_block_pcg(np.zeros((len(bdry), 65)))
    assert ei.value.code == -4
    s.close()
