"""phgGpuSolverPCGNoAlloc: the Jacobi-PCG entry point that allocates no
memory, for callers that cannot allocate device memory (an application whose
own pool has reserved the GPU, a plugin in a process whose device memory
another runtime owns).  It keeps its working vectors in a fixed array inside
the library.

Checked through the C ABI against the regular entry point (phgGpuSetMatrix +
phgGpuSolverPCG) on the same CSR, on two calls in a row -- the second call
reuses the array the first one left behind, on a different matrix size --
with the tolerance the other parity tests use.  Named to be collected last.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

TOL = 1e3   # relative L2 distance <= TOL * rtol, as in test_gpu_parity


def regular(pb, G, rtol):
    with pb.Solver(0) as s:
        s.set_matrix(G["rows_ptr"], G["rows_cols"], G["rows_vals"], G["rhs"])
        x, nits, res = s.solve_pcg(rtol=rtol, btol=0.0, atol=0.0)
    return x, nits


def no_alloc(G, rtol):
    import torch
    from phg_b200.core import solve_pcg_no_alloc
    dev = {k: torch.from_numpy(np.ascontiguousarray(G[k])).cuda()
           for k in ("rows_ptr", "rows_cols", "rows_vals", "rhs")}
    x = torch.zeros(len(G["rhs"]), dtype=torch.float64, device="cuda")
    nits, res = solve_pcg_no_alloc(dev["rows_ptr"], dev["rows_cols"], dev["rows_vals"], dev["rhs"], x,
                                   rtol=rtol, btol=0.0, atol=0.0)
    torch.cuda.synchronize()
    return x.cpu().numpy(), nits


def test_two_calls_match_regular_entry_point(gpu):
    for name in ("p2_m6_sine", "p3_m3_kappa"):
        G = load_golden(name)
        rtol = float(G["rtol"])
        xr, nr = regular(gpu, G, rtol)
        xn, nn = no_alloc(G, rtol)
        assert nn == nr
        assert np.linalg.norm(xn - xr) <= TOL * rtol * np.linalg.norm(xr)
        assert np.linalg.norm(xn - G["x"]) <= TOL * rtol * np.linalg.norm(G["x"])


def test_rejects_sizes_beyond_the_limit(gpu):
    import torch
    from phg_b200.core import NOALLOC_MAX_ROWS, solve_pcg_no_alloc
    n = NOALLOC_MAX_ROWS + 1
    ptr = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    cols = torch.zeros(1, dtype=torch.int32, device="cuda")
    vals = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(gpu.PhgGpuError) as ei:
        solve_pcg_no_alloc(ptr, cols, vals, torch.zeros(n, dtype=torch.float64, device="cuda"),
                           torch.zeros(n, dtype=torch.float64, device="cuda"))
    assert ei.value.code == -4
    assert "limit" in str(ei.value)
