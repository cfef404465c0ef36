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
sys.path.insert(0, GOLDEN)
from make_golden import CASES, GMRES_RESTART, mesh_args  # noqa: E402


def run(name, shim):
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
        if shim:
            env["LD_PRELOAD"] = SHIM
            env["PHG_QUAD_SHIM_STATS"] = "1"
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
    if float(G["mass"]) != 0.0:
        assert served[2] >= nelem * N * (N + 1) // 2
    else:
        assert served[2] == 0
    for k in ("rows_ptr", "rows_cols", "rows_vals", "bdry_rows_ptr", "bdry_rows_cols", "bdry_rows_vals",
              "rhs", "x"):
        assert np.array_equal(out[k], G[k]), k
    assert out["nits"] == int(G["nits"]) and out["residual"] == float(G["residual"])
