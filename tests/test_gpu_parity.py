"""Parity of the CUDA path (through the C ABI) with the reference.

* Golden cases (tests/golden/, outputs of the unmodified reference): matrix
  rows, saved boundary columns, RHS and Jacobi diagonal must match BIT FOR BIT
  -- the element kernel repeats the reference's floating-point operations and
  the row walk adds contributions in the reference's element order.
* Larger meshes: the same, against the CPU oracle on identical inputs.
* PCG: the device reductions sum in a different order than the reference's
  sequential loops, so iterates differ by rounding.  Tolerances: iteration
  count within 2 of the reference; relative L2 distance of the solution to
  the reference's at most 1e-6 * rtol^(1/2)... written per test below.
"""
import numpy as np
import pytest

from conftest import golden_cases, load_golden

pytestmark = pytest.mark.gpu


def build(pb, order, verts, elems, e2l, bdry, f, g=None, kappa=None, mass=0.0, geom=None):
    s = pb.Solver(0)
    s.set_mesh(verts, elems)
    if geom is not None:
        s.set_geometry(geom)
    s.set_dof_map(order, e2l, bdry)
    s.build_linear_system(kappa=kappa, f=f, g=g, mass=mass)
    return s


def phg_geometry(name, G):
    """PHG's stored geometry for meshes it refined by bisection (interpolated
    from the parents, geom.c:460-565); None (the coordinates') otherwise."""
    return G["geom"] if "refined" in name else None


def solution_tol(rtol):
    # two PCG runs to relative residual rtol that differ only in rounding
    return 1e3 * rtol


@pytest.mark.parametrize("name", golden_cases())
def test_golden_assembly_bitexact(gpu, name):
    G = load_golden(name)
    s = build(gpu, int(G["order"]), G["verts"], G["elems"], G["e2l"], G["bdry"], G["f"], G["g"],
              G.get("kappa"), float(G.get("mass", 0.0)), phg_geometry(name, G))
    ptr, cols, vals = s.get_matrix()
    assert np.array_equal(ptr, G["rows_ptr"])
    assert np.array_equal(cols, G["rows_cols"])
    assert np.array_equal(vals, G["rows_vals"])
    bptr, bcols, bvals = s.get_bdry_columns()
    assert np.array_equal(bptr, G["bdry_rows_ptr"])
    assert np.array_equal(bcols, G["bdry_rows_cols"])
    assert np.array_equal(bvals, G["bdry_rows_vals"])
    assert np.array_equal(s.get_rhs(), G["rhs"])
    assert np.array_equal(s.get_diagonal(), G["diag"])
    s.close()


@pytest.mark.parametrize("name", golden_cases())
def test_golden_solve(gpu, name):
    """The reference's solver of each golden case (PCG, BiCGstab, GMRES_r or
    PHG's default GMRES, FLGMRES_r)."""
    G = load_golden(name)
    s = build(gpu, int(G["order"]), G["verts"], G["elems"], G["e2l"], G["bdry"], G["f"], G["g"],
              G.get("kappa"), float(G.get("mass", 0.0)), phg_geometry(name, G))
    rtol = float(G["rtol"])
    solver = str(G["solver"]) if "solver" in G else "pcg"
    if solver in ("gmres_r", "flgmres_r"):
        if solver == "gmres_r":
            x, nits, res = s.solve_gmres(restart=int(G["restart"]), rtol=rtol, btol=0.0, atol=0.0)
        else:
            x, nits, res = s.solve_flgmres(restart=int(G["restart"]), augk=2, rtol=rtol, btol=0.0, atol=0.0)
        assert abs(nits - int(G["nits"])) <= 2
        ref = G["x"]
        assert np.linalg.norm(x - ref) <= solution_tol(rtol) * np.linalg.norm(ref)
        s.close()
        return
    solve = s.solve_bicgstab if solver == "bicgstab" else s.solve_pcg
    x, nits, res, hist = solve(rtol=rtol, btol=0.0, atol=0.0, history=True)
    assert abs(nits - int(G["nits"])) <= 2
    ref = G["x"]
    assert np.linalg.norm(x - ref) <= solution_tol(rtol) * np.linalg.norm(ref)
    assert res <= rtol * hist[0]
    assert len(hist) == nits + 1
    s.close()


@pytest.mark.parametrize("p,m", [(1, 32), (2, 12), (3, 6)])
def test_larger_meshes_vs_oracle(gpu, oracle, p, m):
    v, e = gpu.kuhn_cube(m)
    e2l, bdry, nodes = gpu.lagrange_dofs(v, e, p)
    f = gpu.sine_source(nodes)
    kappa = np.exp(0.5 * np.random.default_rng(p * 100 + m).standard_normal(len(e)))
    o = oracle.assemble(p, v, e, e2l, bdry, f, None, kappa)
    s = build(gpu, p, v, e, e2l, bdry, f, None, kappa)
    ptr, cols, vals = s.get_matrix()
    assert np.array_equal(ptr, o["ptr"])
    assert np.array_equal(cols, o["cols"])
    assert np.array_equal(vals, o["vals"])
    assert np.array_equal(s.get_rhs(), o["rhs"])
    assert np.array_equal(s.get_diagonal(), o["diag"])
    rtol = 1e-10
    xo, no, ro, _ = oracle.pcg(o["ptr"], o["cols"], o["vals"], o["diag"], o["rhs"], rtol=rtol,
                               btol=0.0, atol=0.0)
    x, nits, res = s.solve_pcg(rtol=rtol, btol=0.0, atol=0.0)
    assert abs(nits - no) <= 2
    assert np.linalg.norm(x - xo) <= solution_tol(rtol) * np.linalg.norm(xo)
    # the GPU's own residual, recomputed independently in FP64 by the oracle
    r = o["rhs"] - oracle.spmv(o["ptr"], o["cols"], o["vals"], x)
    assert np.linalg.norm(r) <= 2 * rtol * np.linalg.norm(o["rhs"])
    s.close()


@pytest.mark.parametrize("p,m,mass", [(1, 24, 1e3), (2, 10, 0.7), (3, 5, 42.0)])
def test_mass_term_vs_oracle(gpu, oracle, p, m, mass):
    """-div(kappa grad u) + c u = f: element matrices stiffness + c * mass
    (examples/simplest.c:68-72), bit for bit against the oracle on meshes
    larger than the golden cases; the mass term makes the system better
    conditioned, so PCG needs fewer iterations than without it."""
    v, e = gpu.kuhn_cube(m)
    e2l, bdry, nodes = gpu.lagrange_dofs(v, e, p)
    f = gpu.sine_source(nodes)
    kappa = np.exp(0.5 * np.random.default_rng(p * 1000 + m).standard_normal(len(e)))
    o = oracle.assemble(p, v, e, e2l, bdry, f, None, kappa, mass)
    s = build(gpu, p, v, e, e2l, bdry, f, None, kappa, mass)
    ptr, cols, vals = s.get_matrix()
    assert np.array_equal(ptr, o["ptr"])
    assert np.array_equal(cols, o["cols"])
    assert np.array_equal(vals, o["vals"])
    bptr, bcols, bvals = s.get_bdry_columns()
    assert np.array_equal(bcols, o["bcols"]) and np.array_equal(bvals, o["bvals"])
    assert np.array_equal(s.get_rhs(), o["rhs"])
    assert np.array_equal(s.get_diagonal(), o["diag"])
    xo, no, _, _ = oracle.pcg(o["ptr"], o["cols"], o["vals"], o["diag"], o["rhs"], rtol=1e-10,
                              btol=0.0, atol=0.0)
    x, nits, _ = s.solve_pcg(rtol=1e-10, btol=0.0, atol=0.0)
    assert abs(nits - no) <= 2
    assert np.linalg.norm(x - xo) <= solution_tol(1e-10) * np.linalg.norm(xo)
    # the adjoint differentiates kappa-scaled stiffness only: a mass term is refused
    with pytest.raises(gpu.PhgGpuError) as ei:
        s.adjoint_gradient(x, x, rtol=1e-8)
    assert ei.value.code == -3
    s.build_linear_system(kappa=kappa, f=f)
    _, n0, _ = s.solve_pcg(rtol=1e-10, btol=0.0, atol=0.0)
    assert nits <= n0
    s.close()


def test_matvec_vs_oracle(gpu, oracle):
    G = load_golden("p2_m6_sine")
    s = build(gpu, 2, G["verts"], G["elems"], G["e2l"], G["bdry"], G["f"], G["g"])
    x = np.random.default_rng(5).standard_normal(len(G["bdry"]))
    y = s.mat_vec(x)
    yo = oracle.spmv(G["rows_ptr"], G["rows_cols"], G["rows_vals"], x)
    assert np.allclose(y, yo, rtol=1e-13, atol=1e-13 * np.abs(yo).max())
    s.close()


def test_set_matrix_path(gpu):
    """The OEM-solver entry: a CSR assembled elsewhere (the reference's rows)."""
    G = load_golden("p3_m3_kappa")
    s = gpu.Solver(0)
    s.set_matrix(G["rows_ptr"], G["rows_cols"], G["rows_vals"], G["rhs"])
    assert np.array_equal(s.get_diagonal(), G["diag"])
    x, nits, res = s.solve_pcg(rtol=float(G["rtol"]), btol=0.0, atol=0.0)
    assert abs(nits - int(G["nits"])) <= 2
    assert np.linalg.norm(x - G["x"]) <= solution_tol(float(G["rtol"])) * np.linalg.norm(G["x"])
    s.close()


def test_device_tensors_in_place(gpu):
    import torch
    G = load_golden("p2_m5_kappa")
    dev = {k: torch.from_numpy(np.ascontiguousarray(G[k])).cuda()
           for k in ("verts", "elems", "e2l", "bdry", "f", "g", "kappa")}
    s = build(gpu, 2, dev["verts"], dev["elems"], dev["e2l"], dev["bdry"], dev["f"], dev["g"], dev["kappa"])
    ptr, cols, vals = s.get_matrix()
    assert np.array_equal(vals, G["rows_vals"])
    x = torch.zeros(len(G["bdry"]), dtype=torch.float64, device="cuda")
    _, nits, res = s.solve_pcg(rtol=float(G["rtol"]), btol=0.0, atol=0.0, out=x)
    assert abs(nits - int(G["nits"])) <= 2
    xr = G["x"]
    assert np.linalg.norm(x.cpu().numpy() - xr) <= solution_tol(float(G["rtol"])) * np.linalg.norm(xr)
    s.close()


def test_maxit_stops(gpu):
    G = load_golden("p2_m6_sine")
    s = build(gpu, 2, G["verts"], G["elems"], G["e2l"], G["bdry"], G["f"], G["g"])
    x, nits, res = s.solve_pcg(rtol=1e-14, btol=0.0, atol=0.0, maxit=5)
    assert nits == 5
    s.close()


def test_nonzero_initial_guess(gpu, oracle):
    G = load_golden("p1_m5_kappa")
    s = build(gpu, 1, G["verts"], G["elems"], G["e2l"], G["bdry"], G["f"], G["g"], G["kappa"])
    x0 = np.linspace(0, 1, len(G["bdry"]))
    xo, no, _, _ = oracle.pcg(G["rows_ptr"], G["rows_cols"], G["rows_vals"], G["diag"], G["rhs"],
                              x0=x0, rtol=1e-10, btol=0.0, atol=0.0)
    x, nits, _ = s.solve_pcg(x0=x0, rtol=1e-10, btol=0.0, atol=0.0)
    assert abs(nits - no) <= 2
    assert np.linalg.norm(x - xo) <= 1e-7 * np.linalg.norm(xo)
    s.close()


def test_breakdown_reported(gpu, oracle):
    """p.Ap == 0 stops PCG as the reference does (solver-phg.c:561-571): the
    iteration count comes back with x as it is, and the warning the
    reference prints ("the matrix may not be SPD") is readable."""
    ptr, cols, vals = np.array([0, 1, 2]), np.array([0, 1], np.int32), np.array([1.0, -1.0])
    b = np.array([1.0, 1.0])
    s = gpu.Solver(0)
    s.set_matrix(ptr, cols, vals, b)
    x, nits, res = s.solve_pcg(rtol=1e-10)
    xo, no, ro, _ = oracle.pcg(ptr, cols, vals, vals, b, rtol=1e-10)
    assert nits == no == 1
    assert np.array_equal(x, xo) and res == ro
    assert "not be SPD" in gpu.last_warning()
    # the next solver call clears the warning
    s.set_matrix(ptr, cols, np.array([1.0, 2.0]), b)
    x, nits, _ = s.solve_pcg(rtol=1e-10)
    assert gpu.last_warning() == "" and nits >= 1
    s.close()


def test_nonfinite_input_reported(gpu):
    """A NaN or infinite kappa, f, g or coordinate is PHG_GPU_ERR_NAN at
    build time (the system stays usable); so is a non-finite right-hand
    side handed to phgGpuSetRHS."""
    G = load_golden("p2_m3_sine")
    s = gpu.Solver(0)
    s.set_mesh(G["verts"], G["elems"])
    s.set_dof_map(2, G["e2l"], G["bdry"])
    nel, nd = len(G["elems"]), len(G["bdry"])
    cases = []
    k = np.ones(nel); k[5] = np.nan; cases.append(dict(kappa=k, f=G["f"]))
    k = np.ones(nel); k[0] = np.inf; cases.append(dict(kappa=k, f=G["f"]))
    f = G["f"].copy(); f[7] = np.nan; cases.append(dict(f=f))
    g = np.zeros(nd); g[np.flatnonzero(G["bdry"])[3]] = -np.inf; cases.append(dict(f=G["f"], g=g))
    for kw in cases:
        with pytest.raises(gpu.PhgGpuError) as ei:
            s.build_linear_system(**kw)
        assert ei.value.code == -6, kw.keys()
    v = G["verts"].copy(); v[2, 1] = np.nan
    s.set_mesh(v, G["elems"])
    s.set_dof_map(2, G["e2l"], G["bdry"])
    with pytest.raises(gpu.PhgGpuError) as ei:
        s.build_linear_system(f=G["f"])
    assert ei.value.code == -6
    s.set_mesh(G["verts"], G["elems"])
    s.set_dof_map(2, G["e2l"], G["bdry"])
    s.build_linear_system(f=G["f"])
    assert np.array_equal(s.get_rhs(), G["rhs"])
    r = G["rhs"].copy(); r[1] = np.nan
    with pytest.raises(gpu.PhgGpuError) as ei:
        s.set_rhs(r)
    assert ei.value.code == -6
    s.close()


def test_set_rhs_new_solve(gpu, oracle):
    """phgGpuSetRHS keeps the matrix and solves a new right-hand side, as a
    second phgSolverVecSolve on the same matrix does."""
    G = load_golden("p2_m5_kappa")
    s = build(gpu, 2, G["verts"], G["elems"], G["e2l"], G["bdry"], G["f"], G["g"], G["kappa"])
    b2 = np.random.default_rng(3).standard_normal(len(G["rhs"]))
    b2[G["bdry"] != 0] = 0.0
    s.set_rhs(b2)
    assert np.array_equal(s.get_rhs(), b2)
    x, nits, _ = s.solve_pcg(rtol=1e-10, btol=0.0, atol=0.0)
    xo, no, _, _ = oracle.pcg(G["rows_ptr"], G["rows_cols"], G["rows_vals"], G["diag"], b2,
                              rtol=1e-10, btol=0.0, atol=0.0)
    assert abs(nits - no) <= 2
    assert np.linalg.norm(x - xo) <= 1e-7 * np.linalg.norm(xo)
    s.close()


def test_bad_index_reported(gpu):
    G = load_golden("p1_m4_sine")
    s = gpu.Solver(0)
    s.set_mesh(G["verts"], G["elems"])
    e2l = G["e2l"].copy()
    e2l[3, 2] = len(G["bdry"]) + 7
    with pytest.raises(gpu.PhgGpuError) as ei:
        s.set_dof_map(1, e2l, G["bdry"])
    assert ei.value.code == -1
    # the system stays usable
    s.set_dof_map(1, G["e2l"], G["bdry"])
    s.build_linear_system(f=G["f"], g=G["g"])
    assert np.array_equal(s.get_rhs(), G["rhs"])
    s.close()


def test_zero_rhs_gives_zero(gpu):
    G = load_golden("p2_m3_sine")
    s = build(gpu, 2, G["verts"], G["elems"], G["e2l"], G["bdry"], np.zeros_like(G["f"]))
    x, nits, res = s.solve_pcg(x0=np.ones(len(G["bdry"])))
    assert nits == 0 and not x.any()
    s.close()


def test_rebuild_on_recorded_pattern(gpu, oracle):
    """Repeated builds on one mesh and DOF map: the second records the
    pattern, later ones add the contributions at their recorded places (the
    value walk).  Every build is bit for bit the oracle's, including a kappa
    with zeros (whole element matrices vanish: the pattern changes and the
    build walks the rows again) and the return to the old pattern; solves on
    the refreshed layouts match the oracle's."""
    import phg_b200 as pb
    v, e = pb.kuhn_cube(7)
    e2l, bdry, nodes = pb.lagrange_dofs(v, e, 2)
    f = pb.sine_source(nodes)
    rng = np.random.default_rng(5)
    kappas = [np.exp(rng.standard_normal(len(e))) for _ in range(4)]
    kz = kappas[3].copy()
    kz[rng.choice(len(e), 40, replace=False)] = 0.0
    seq = [kappas[0], kappas[1], kappas[2], kz, kappas[3], kappas[0]]
    with gpu.Solver(0) as s:
        s.set_mesh(v, e)
        s.set_dof_map(2, e2l, bdry)
        for i, k in enumerate(seq):
            s.build_linear_system(kappa=k, f=f)
            o = oracle.assemble(2, v, e, e2l, bdry, f, kappa=k)
            ptr, cols, vals = s.get_matrix()
            assert np.array_equal(ptr, o["ptr"]) and np.array_equal(cols, o["cols"]), i
            assert np.array_equal(vals, o["vals"]), i
            bp, bc, bv = s.get_bdry_columns()
            assert np.array_equal(bc, o["bcols"]) and np.array_equal(bv, o["bvals"]), i
            assert np.array_equal(s.get_rhs(), o["rhs"]) and np.array_equal(s.get_diagonal(), o["diag"]), i
            if i in (2, 5):   # solves on the layouts refreshed in place
                x, nits, _ = s.solve_pcg(rtol=1e-10, btol=0.0, atol=0.0)
                xm, nm, rm, _ = s.solve_pcg_mixed(rtol=1e-10)
                xo, no, _, _ = oracle.pcg(o["ptr"], o["cols"], o["vals"], o["diag"], o["rhs"], rtol=1e-10,
                                          btol=0.0, atol=0.0)
                assert abs(nits - no) <= 2
                assert np.linalg.norm(x - xo) <= 1e-7 * np.linalg.norm(xo)
                assert rm <= 1e-10 * np.linalg.norm(o["rhs"]) * (1 + 1e-9)


@pytest.mark.parametrize("name", ["p2_m5_kappa", "p3_m3_mass"])
def test_given_geometry_on_unrefined_mesh(gpu, name):
    """On a mesh PHG did not refine, its stored geometry is the one the GPU
    computes from the coordinates: the rows are the same bit for bit either
    way, and a non-finite geometry is refused."""
    G = load_golden(name)
    args = (gpu, int(G["order"]), G["verts"], G["elems"], G["e2l"], G["bdry"], G["f"], G["g"],
            G.get("kappa"), float(G.get("mass", 0.0)))
    a, b = build(*args), build(*args, geom=G["geom"])
    for x, y in zip(a.get_matrix() + (a.get_rhs(),), b.get_matrix() + (b.get_rhs(),)):
        assert np.array_equal(x, y)
    bad = G["geom"].copy()
    bad[3, 16] = np.nan
    with pytest.raises(gpu.PhgGpuError):
        b.set_geometry(bad)
    with pytest.raises(gpu.PhgGpuError):
        b.set_geometry(G["geom"][:-1])
    a.close()
    b.close()


@pytest.mark.parametrize("name", ["p2_corner_refined", "p3_corner_refined", "p1_corner_refined", "p3_m3_mass"])
def test_rebuild_on_recorded_pattern_refined(gpu, name):
    """Builds two and three on one mesh and DOF map (the second records the
    pattern and its contribution lists, the third gathers over them) give the
    first build's rows bit for bit, on PHG-refined meshes whose rows reach
    past the walk's table (P3: 281 entries) and past the gather's staging
    (high-valence vertices), with the reference's golden rows."""
    G = load_golden(name)
    args = (gpu, int(G["order"]), G["verts"], G["elems"], G["e2l"], G["bdry"], G["f"], G["g"],
            G.get("kappa"), float(G.get("mass", 0.0)), phg_geometry(name, G))
    s = build(*args)
    for _ in range(2):
        s.build_linear_system(kappa=G.get("kappa"), f=G["f"], g=G["g"], mass=float(G.get("mass", 0.0)))
        ptr, cols, vals = s.get_matrix()
        assert np.array_equal(ptr, G["rows_ptr"]) and np.array_equal(cols, G["rows_cols"])
        assert np.array_equal(vals, G["rows_vals"])
        bptr, bcols, bvals = s.get_bdry_columns()
        assert np.array_equal(bcols, G["bdry_rows_cols"]) and np.array_equal(bvals, G["bdry_rows_vals"])
        assert np.array_equal(s.get_rhs(), G["rhs"]) and np.array_equal(s.get_diagonal(), G["diag"])
    s.close()


@pytest.mark.parametrize("p,k", [(1, 3), (2, 1), (2, 5), (3, 2)])
def test_ragged_element_counts(gpu, oracle, p, k):
    """Element counts that leave the element kernels' warps part-filled (P1
    takes 8 elements a warp, P2 6, P3 one; every Kuhn cube has 6 m^3): the
    4^3 cube without its last k elements.  The first build, rebuilds on the
    recorded pattern with new kappas and one with a mass term are bit for bit
    the oracle's, and the PCG solve matches the oracle's."""
    v, e = gpu.kuhn_cube(4)
    e = np.ascontiguousarray(e[:-k])
    e2l, bdry, nodes = gpu.lagrange_dofs(v, e, p)
    f = gpu.sine_source(nodes)
    rng = np.random.default_rng(10 * p + k)
    cases = [(None, 0.0), (np.exp(rng.standard_normal(len(e))), 0.0),
             (np.exp(rng.standard_normal(len(e))), 0.0), (None, 2.5)]
    with gpu.Solver(0) as s:
        s.set_mesh(v, e)
        s.set_dof_map(p, e2l, bdry)
        for i, (kappa, mass) in enumerate(cases):
            s.build_linear_system(kappa=kappa, f=f, mass=mass)
            o = oracle.assemble(p, v, e, e2l, bdry, f, kappa=kappa, mass=mass)
            ptr, cols, vals = s.get_matrix()
            assert np.array_equal(ptr, o["ptr"]) and np.array_equal(cols, o["cols"]), i
            assert np.array_equal(vals, o["vals"]), i
            bp, bc, bv = s.get_bdry_columns()
            assert np.array_equal(bc, o["bcols"]) and np.array_equal(bv, o["bvals"]), i
            assert np.array_equal(s.get_rhs(), o["rhs"]) and np.array_equal(s.get_diagonal(), o["diag"]), i
            if i == 1:
                x, nits, _ = s.solve_pcg(rtol=1e-10, btol=0.0, atol=0.0)
                xo, no, _, _ = oracle.pcg(o["ptr"], o["cols"], o["vals"], o["diag"], o["rhs"], rtol=1e-10,
                                          btol=0.0, atol=0.0)
                assert abs(nits - no) <= 2
                assert np.linalg.norm(x - xo) <= solution_tol(1e-10) * np.linalg.norm(xo)
