"""The per-call shim (phg_b200/shim/libphg_quad_shim.so) preloaded into an
unmodified PHG user program: oracle/ref_driver/phg_dump.c linked against a
shared build of the reference (oracle/_ref/phg_dump_dyn).  The program's own
element loop calls phgQuadGradBasAGradBas / phgQuadDofTimesBas; the shim
answers them from the element table the GPU computes, PHG assembles and
solves as usual, and everything it dumps -- rows, right-hand side, solution,
iteration count -- is bit for bit the reference's own run (the golden
fixtures).  The mass term of the mass cases (phgQuadBasDotBas) comes from
the GPU's mass table too."""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, load_golden

pytestmark = pytest.mark.gpu

DUMP = os.path.join(ROOT, "oracle", "_ref", "phg_dump_dyn")
SHIM = os.path.join(ROOT, "phg_b200", "shim", "libphg_quad_shim.so")
MAT_SHIM = os.path.join(ROOT, "phg_b200", "shim", "libphg_mat_shim.so")
sys.path.insert(0, GOLDEN)
from make_golden import CASES, GMRES_RESTART, mesh_args  # noqa: E402


def run(name, shim, mat_shim=False):
    m, P, case, kseed, rtol, *rest = CASES[name]
    mass = rest[0] if rest else 0.0
    solver = rest[1] if len(rest) > 1 else "pcg"
    from phg_b200.mesh import kuhn_cube
    with tempfile.TemporaryDirectory() as d:
        e = kuhn_cube(m)[1]
        args = [DUMP, *mesh_args(name, d), "-dof_type", "P%d" % P,
                "-solver", "gmres" if solver == "gmres_r" else solver, "-pcg_pc_type", "jacobi",
                "-solver_rtol", repr(rtol), "-solver_btol", "0", "-solver_atol", "0",
                "-solver_maxit", "10000", "-map_reorder", "no", "-dump_dir", d, "-rhs_case", case]
        if mass != 0.0:
            args += ["-mass_coef", repr(mass)]
        if solver == "gmres_r":
            args += ["-gmres_type", "gmres_r", "-gmres_pc_type", "jacobi",
                     "-gmres_restart", str(GMRES_RESTART)]
        if kseed is not None:
            np.exp(np.random.default_rng(kseed).standard_normal(len(e))).tofile(os.path.join(d, "kappa.in"))
            args += ["-kappa_file", os.path.join(d, "kappa.in")]
        env = dict(os.environ)
        pre = ([SHIM] if shim else []) + ([MAT_SHIM] if mat_shim else [])
        if pre:
            env["LD_PRELOAD"] = " ".join(pre)
            env["PHG_QUAD_SHIM_STATS"] = "1"
            env["PHG_MAT_SHIM_STATS"] = "1"
        p = subprocess.run(args, env=env, capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stderr[-2000:]
        meta = dict(l.split() for l in open(os.path.join(d, "meta.txt")))

        def L(n, t):
            return np.fromfile(os.path.join(d, n), t)
        out = {"nits": int(meta["nits"]), "residual": float(meta["residual"]),
               "rhs": L("rhs.f64", np.float64), "x": L("x.f64", np.float64)}
        for pre in ("rows", "bdry_rows"):
            out[pre + "_ptr"] = L(pre + "_ptr.i64", np.int64)
            out[pre + "_cols"] = L(pre + "_cols.i32", np.int32)
            out[pre + "_vals"] = L(pre + "_vals.f64", np.float64)
        stats = [l for l in p.stderr.splitlines() if l.startswith("phg_quad_shim:")]
        if mat_shim:
            return out, stats, [l for l in p.stderr.splitlines() if l.startswith("phg_mat_shim:")]
        return out, stats


@pytest.mark.parametrize("name", ["p1_m4_sine", "p2_m5_kappa", "p3_m3_linear", "p2_m4_kappa_mass",
                                  "p1_m5_mass", "p3_m3_mass", "p2_m5_kappa_bicgstab", "p2_corner_refined"])
def test_unmodified_program_with_shim_matches_reference(name):
    G = load_golden(name)
    out, stats = run(name, shim=True)
    assert len(stats) == 1, stats
    served = [int(t) for t in stats[0].replace(",", " ").split() if t.isdigit()]
    nelem, N = G["e2l"].shape
    # the driver's loop asks for N (N + 1) / 2 stiffness pairs per element
    # (PHG itself asks for a few more), one RHS entry per non-Dirichlet basis
    # and, with a mass term, N (N + 1) / 2 mass pairs; none is forwarded
    assert served[0] >= nelem * N * (N + 1) // 2
    assert served[1] > 0 and served[3] == 0
    if float(G.get("mass", 0.0)) != 0.0:
        assert served[2] >= nelem * N * (N + 1) // 2
    else:
        assert served[2] == 0
    for k in ("rows_ptr", "rows_cols", "rows_vals", "bdry_rows_ptr", "bdry_rows_cols", "bdry_rows_vals",
              "rhs", "x"):
        assert np.array_equal(out[k], G[k]), k
    assert out["nits"] == int(G["nits"]) and out["residual"] == float(G["residual"])


@pytest.mark.parametrize("name", ["p1_m4_sine", "p2_m5_kappa", "p3_m3_linear", "p2_m4_kappa_mass",
                                  "p2_m5_kappa_bicgstab", "p2_corner_refined", "p3_corner_refined"])
def test_unmodified_program_with_quad_and_mat_shims(name):
    """Both shims preloaded: the element integrals come from the GPU tables
    and the row insertion (phgSolverAddMatrixEntries -> phgMatAddEntries_) is
    recorded and assembled on the GPU at phgMatAssemble (phgGpuAssembleRows);
    PHG's own phgMatAssemble, boundary elimination and solver follow.  Rows
    after elimination, saved boundary columns, RHS, solution and iteration
    count are bit for bit the reference's own run.  p3_corner_refined has
    rows beyond 256 entries (the record walk's second pass)."""
    G = load_golden(name)
    out, qstats, mstats = run(name, shim=True, mat_shim=True)
    assert len(mstats) == 1, mstats
    nums = [int(t) for t in mstats[0].replace(",", " ").split() if t.isdigit()]
    recorded, assembled, replayed, forwarded = nums
    nelem, N = G["e2l"].shape
    # every element row was recorded and the matrix assembled on the GPU
    # (PHG's own later calls, if any, are forwarded and counted apart)
    assert recorded >= nelem * N and assembled == 1 and replayed == 0, mstats
    for k in ("rows_ptr", "rows_cols", "rows_vals", "bdry_rows_ptr", "bdry_rows_cols", "bdry_rows_vals",
              "rhs", "x"):
        assert np.array_equal(out[k], G[k]), k
    assert out["nits"] == int(G["nits"]) and out["residual"] == float(G["residual"])


def test_assemble_rows_first_touch_semantics(gpu):
    """phgGpuAssembleRows on hand-made segments: zeros and negative columns
    dropped, first appearance fixes the place, later ones add (in segment
    order), an empty first segment does not count as the row's first; a
    column repeated inside a row's first segment is refused."""
    s = gpu.Solver(0)
    segs = [(0, [3, 1, 0], [1.0, 2.0, 0.0]), (2, [2], [5.0]), (0, [1, -1, 4], [0.5, 9.0, 0.0]),
            (1, [0, 1], [0.0, 0.0]), (1, [2, 0], [1.5, -2.0]), (0, [4, 3], [7.0, 0.25])]
    rows = np.array([r for r, _, _ in segs], np.int32)
    ptr = np.concatenate([[0], np.cumsum([len(c) for _, c, _ in segs])]).astype(np.int64)
    cols = np.concatenate([c for _, c, _ in segs]).astype(np.int32)
    vals = np.concatenate([v for _, _, v in segs]).astype(np.float64)
    s.assemble_rows(5, rows, ptr, cols, vals)
    p, c, v = s.get_matrix()
    assert p.tolist() == [0, 3, 5, 6, 6, 6]
    assert c.tolist() == [3, 1, 4, 2, 0, 2]
    assert v.tolist() == [1.0 + 0.25, 2.0 + 0.5, 7.0, 1.5, -2.0, 5.0]
    bad = np.array([0, 0], np.int32)
    with pytest.raises(gpu.PhgGpuError) as ei:
        s.assemble_rows(2, bad[:1], np.array([0, 2], np.int64), bad, np.array([1.0, 2.0]))
    assert ei.value.code == -1
    s.close()
