"""SpMV layouts and the mixed-precision (FP32 inner / FP64 refinement) PCG."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def system(pb, p, m, kappa_seed=None):
    v, e = pb.kuhn_cube(m)
    e2l, bdry, nodes = pb.lagrange_dofs(v, e, p)
    f = pb.sine_source(nodes)
    kappa = None
    if kappa_seed is not None:
        kappa = np.exp(0.5 * np.random.default_rng(kappa_seed).standard_normal(len(e)))
    s = pb.Solver(0)
    s.set_mesh(v, e)
    s.set_dof_map(p, e2l, bdry)
    s.build_linear_system(kappa=kappa, f=f)
    return s


@pytest.mark.parametrize("layout,param", [("csr", 4), ("csr", 8), ("csr", 16), ("csr", 32),
                                          ("sell", 2), ("sell", 4), ("sell", 8), ("q16", 1)])
def test_every_spmv_layout_matches_oracle(gpu, oracle, layout, param):
    for name in ("p2_m6_sine", "p3_m3_kappa", "p1_m5_kappa"):
        G = load_golden(name)
        s = gpu.Solver(0)
        s.set_matrix(G["rows_ptr"], G["rows_cols"], G["rows_vals"], G["rhs"])
        s.set_spmv_plan(layout, param)
        x = np.random.default_rng(3).standard_normal(len(G["rhs"]))
        y = s.mat_vec(x)
        yo = oracle.spmv(G["rows_ptr"], G["rows_cols"], G["rows_vals"], x)
        assert np.allclose(y, yo, rtol=1e-13, atol=1e-13 * np.abs(yo).max()), (name, layout, param)
        # PCG through the same layout
        xs, nits, _ = s.solve_pcg(rtol=float(G["rtol"]), btol=0.0, atol=0.0)
        assert abs(nits - int(G["nits"])) <= 2
        assert np.linalg.norm(xs - G["x"]) <= 1e3 * float(G["rtol"]) * np.linalg.norm(G["x"])
        s.close()


def test_autotuner_reports_a_choice(gpu):
    s = system(gpu, 2, 8)
    s.solve_pcg(rtol=1e-8, btol=0.0, atol=0.0)
    layout, param, times = s.spmv_plan()
    assert (layout, param) in gpu.Solver.SPMV_LAYOUTS
    assert all(times[k] > 0 for k in ("csr4", "csr8", "csr16", "csr32", "sell_u2", "sell_u4", "sell_u8"))
    s.close()


@pytest.mark.parametrize("p,m,seed", [(1, 32, None), (2, 12, None), (2, 10, 7), (3, 6, 9)])
def test_mixed_precision_reaches_fp64_tolerance(gpu, oracle, p, m, seed):
    """Tolerances: the FP64 residual ||b - A x|| (recomputed here by the oracle
    in FP64) meets the reference's stopping rule; the solution is as close to
    the tightly converged FP64 solution as the FP64 PCG result at the same
    rtol is, within a factor of 10 (+ 1e-12 relative)."""
    rtol = 1e-8
    s = system(gpu, p, m, seed)
    ptr, cols, vals = s.get_matrix()
    rhs, diag = s.get_rhs(), s.get_diagonal()
    x64, n64, _ = s.solve_pcg(rtol=rtol, btol=0.0, atol=0.0)
    xm, nm, res, nupd = s.solve_pcg_mixed(rtol=rtol, btol=0.0, atol=0.0)
    r = rhs - oracle.spmv(ptr, cols, vals, xm)
    assert np.linalg.norm(r) <= rtol * np.linalg.norm(rhs) * (1 + 1e-9)
    assert abs(res - np.linalg.norm(r)) <= 1e-6 * res + 1e-300
    xt, _, _, _ = oracle.pcg(ptr, cols, vals, diag, rhs, rtol=1e-13, btol=0.0, atol=0.0)
    e64 = np.linalg.norm(x64 - xt) / np.linalg.norm(xt)
    em = np.linalg.norm(xm - xt) / np.linalg.norm(xt)
    print("p=%d m=%d: fp64 %d its err %.2e, mixed %d its (%d updates) err %.2e"
          % (p, m, n64, e64, nm, nupd, em))
    assert em <= 10 * e64 + 1e-12
    assert nm <= 1.5 * n64 + 5
    s.close()


def test_mixed_zero_rhs_and_breakdown(gpu):
    G = load_golden("p2_m3_sine")
    s = gpu.Solver(0)
    s.set_matrix(G["rows_ptr"], G["rows_cols"], G["rows_vals"], np.zeros_like(G["rhs"]))
    x, nits, res, _ = s.solve_pcg_mixed(x0=np.ones(len(G["rhs"])))
    assert nits == 0 and not x.any()
    s.close()
    # a breakdown stops the iteration as the FP64 PCG does: count returned,
    # the warning set, the FP64 residual of the iterate reported
    s = gpu.Solver(0)
    s.set_matrix(np.array([0, 1, 2]), np.array([0, 1], np.int32), np.array([1.0, -1.0]), np.array([1.0, 1.0]))
    x, nits, res, _ = s.solve_pcg_mixed(rtol=1e-10)
    assert nits == 1 and "not be SPD" in gpu.last_warning()
    assert res == np.linalg.norm(np.array([1.0, 1.0]) - np.array([1.0, -1.0]) * x)
    s.close()


def far_coupled_spd(n, offsets, seed):
    """Symmetric, diagonally dominant matrix coupling row i with i +- 1 and
    i +- o (mod n) for each o in offsets: the rows' columns lie in clusters
    far apart."""
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    i = np.arange(n)
    rows, cols = [i], [i]
    vals = [np.full(n, 2.0 + 3 * (1 + len(offsets)))]   # > the largest off-diagonal row sum
    for o in (1,) + tuple(offsets):
        w = -0.5 - rng.random(n)
        rows += [i, (i + o) % n]
        cols += [(i + o) % n, i]
        vals += [w, w]
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    return A.indptr.astype(np.int64), A.indices.astype(np.int32), A.data, rng.standard_normal(n)


LAYOUTS32 = [("sell", 4), ("sell", 8), ("sell", 16), ("pair", 2), ("pair", 4), ("pair", 8), ("q16", 1),
             ("q16", 2)]


@pytest.mark.parametrize("case", ["p2_m16", "p3_m6", "far_coupled"])
def test_every_fp32_layout_in_mixed_pcg(gpu, oracle, case):
    """The mixed solver with each FP32 product layout forced: the FP64
    residual (recomputed by the oracle) meets the stopping rule and the
    iteration counts agree within a few iterations (the layouts differ only
    in the FP32 summation order).  "far_coupled" is a matrix given through
    phgGpuSetMatrix whose rows couple columns far apart; P3 rows (up to 175
    entries) take several rounds of the warp that builds the q16 layout."""
    if case in ("p2_m16", "p3_m6"):
        s = system(gpu, 2, 16) if case == "p2_m16" else system(gpu, 3, 6)
        ptr, cols, vals = s.get_matrix()
        rhs = s.get_rhs()
    else:
        ptr, cols, vals, rhs = far_coupled_spd(200003, (70001, 140003), seed=5)
        s = gpu.Solver(0)
        s.set_matrix(ptr, cols, vals, rhs)
    its = {}
    for layout, u in LAYOUTS32:
        if layout == "q16" and case == "far_coupled":
            # rows span three 65536-column windows: the layout is refused
            with pytest.raises(gpu.PhgGpuError):
                s.set_spmv_plan32(layout, u)
            continue
        s.set_spmv_plan32(layout, u)
        x, nits, res, nupd = s.solve_pcg_mixed(rtol=1e-8)
        r = rhs - oracle.spmv(ptr, cols, vals, x)
        assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(rhs) * (1 + 1e-9), (layout, u)
        its[(layout, u)] = nits
        assert s.spmv_plan()[2]["fp32_layout"] == layout
    s.close()
    assert max(its.values()) - min(its.values()) <= max(3, min(its.values()) // 20), its


def test_q16_layout_follows_the_matrix(gpu, oracle):
    """The autotuner offers q16 only for matrices whose rows fit two column
    windows; a matrix of the same shape that does not fit makes a q16 choice
    fall back to a new tuning, and a new matrix that fits gets its own q16
    arrays (the residual is recomputed by the oracle each time)."""
    n = 200003
    s = gpu.Solver(0)
    # banded first: every row fits one window
    ptr, cols, vals, rhs = far_coupled_spd(n, (3, 7), seed=1)
    s.set_matrix(ptr, cols, vals, rhs)
    s.set_spmv_plan32("q16", 1)
    x, nits, res, _ = s.solve_pcg_mixed(rtol=1e-8)
    assert np.linalg.norm(rhs - oracle.spmv(ptr, cols, vals, x)) <= 1e-8 * np.linalg.norm(rhs) * (1 + 1e-9)
    assert s.spmv_plan()[2]["fp32_layout"] == "q16"
    # same shape (n, nnz), rows spanning three windows
    ptr2, cols2, vals2, rhs2 = far_coupled_spd(n, (70001, 140003), seed=2)
    assert len(cols2) == len(cols)
    s.set_matrix(ptr2, cols2, vals2, rhs2)
    x, nits, res, _ = s.solve_pcg_mixed(rtol=1e-8)
    assert np.linalg.norm(rhs2 - oracle.spmv(ptr2, cols2, vals2, x)) <= 1e-8 * np.linalg.norm(rhs2) * (1 + 1e-9)
    info = s.spmv_plan()[2]
    assert info["fp32_layout"] != "q16"
    assert info["fp32_q16_u1"] == 0.0 and info["fp32_q16_u2"] == 0.0
    # back to a matrix that fits: new values, same pattern as the first
    s.set_matrix(ptr, cols, vals * 2.0, rhs)
    s.set_spmv_plan32("q16", 2)
    x, nits, res, _ = s.solve_pcg_mixed(rtol=1e-8)
    assert np.linalg.norm(rhs - oracle.spmv(ptr, cols, vals * 2.0, x)) <= 1e-8 * np.linalg.norm(rhs) * (1 + 1e-9)
    s.close()


@pytest.mark.parametrize("layout,param", [("csr", 8), ("sell", 4), ("q16", 1)])
def test_krylov_solvers_on_each_fp64_layout(gpu, oracle, layout, param):
    """PCG, BiCGstab and GMRES_r (their products with epilogues) on each FP64
    layout forced for a P2 system with variable kappa: the FP64 residual,
    recomputed by the oracle, meets the stopping rule, and the iteration
    counts agree with the CSR layout's within a few iterations (the layouts
    differ only in the summation order)."""
    s = system(gpu, 2, 12, kappa_seed=4)
    ptr, cols, vals = s.get_matrix()
    rhs = s.get_rhs()
    nb = np.linalg.norm(rhs)
    its = {}
    for lay, par in (("csr", 8), (layout, param)):
        s.set_spmv_plan(lay, par)
        x, n_pcg, _ = s.solve_pcg(rtol=1e-9, btol=0.0, atol=0.0)
        assert np.linalg.norm(rhs - oracle.spmv(ptr, cols, vals, x)) <= 1e-9 * nb * 1.01, lay
        x, n_bicg, _ = s.solve_bicgstab(rtol=1e-9, btol=0.0, atol=0.0)
        assert np.linalg.norm(rhs - oracle.spmv(ptr, cols, vals, x)) <= 1e-8 * nb, lay
        x, n_gm, _ = s.solve_gmres(restart=30, rtol=1e-9, btol=0.0, atol=0.0)
        assert np.linalg.norm(rhs - oracle.spmv(ptr, cols, vals, x)) <= 1e-8 * nb, lay
        its[lay] = (n_pcg, n_bicg, n_gm)
        assert s.spmv_plan()[0] == lay
    s.close()
    for a, b in zip(its["csr"], its[layout]):
        assert abs(a - b) <= max(3, a // 20), its


def test_plain_graphs_same_solves(gpu, monkeypatch):
    """$PHG_GPU_PLAIN_GRAPHS=1 builds the solver graphs without conditional
    nodes (for profilers) and relaunches them from the host: the same kernels
    in the same order, so the same iterations and the same bits."""
    G = load_golden("p2_m6_sine")
    args = (G["rows_ptr"], G["rows_cols"], G["rows_vals"], G["rhs"])
    out = []
    for plain in ("0", "1"):
        monkeypatch.setenv("PHG_GPU_PLAIN_GRAPHS", plain)
        s = gpu.Solver(0)
        s.set_matrix(*args)
        s.set_spmv_plan("q16", 1)      # the tuner chooses by timing: fix the layouts
        s.set_spmv_plan32("q16", 2)
        x64, n64, r64 = s.solve_pcg(rtol=1e-10, btol=0.0, atol=0.0)
        xm, nm, rm, nu = s.solve_pcg_mixed(rtol=1e-10, btol=0.0, atol=0.0)
        out.append((x64, n64, r64, xm, nm, rm, nu))
        s.close()
    a, b = out
    assert a[1] == b[1] and a[2] == b[2] and np.array_equal(a[0], b[0])
    assert a[4] == b[4] and a[5] == b[5] and a[6] == b[6] and np.array_equal(a[3], b[3])


def test_mixed_maxit_stops_with_fp64_residual(gpu, oracle):
    """maxit ends the mixed solve after exactly maxit steps (the reliable
    update that follows makes the last FP64 residual test), and the residual
    it reports is the FP64 ||b - A x|| of the iterate it returns."""
    G = load_golden("p2_m6_sine")
    s = gpu.Solver(0)
    s.set_matrix(G["rows_ptr"], G["rows_cols"], G["rows_vals"], G["rhs"])
    x, nits, res, nupd = s.solve_pcg_mixed(rtol=1e-12, btol=0.0, atol=0.0, maxit=10)
    assert nits == 10 and nupd >= 1
    r = G["rhs"] - oracle.spmv(G["rows_ptr"], G["rows_cols"], G["rows_vals"], x)
    assert abs(res - np.linalg.norm(r)) <= 1e-10 * np.linalg.norm(G["rhs"])
    assert res > 1e-12 * np.linalg.norm(G["rhs"])
    s.close()
