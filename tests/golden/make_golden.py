"""Generates the parity fixtures in tests/golden/ from the UNMODIFIED
reference (PHG 0.9.7) built from its own sources by `make -C oracle ref`.

For every case it writes the mesh as Medit, runs oracle/_ref/phg_dump (the
reference's element loop + phgSolverAssemble + phgSolverUpdateRHS +
phgSolverSolve with -solver pcg, bicgstab or gmres (gmres_r or PHG's default
flgmres_r), see oracle/ref_driver/phg_dump.c) and stores
the reference's own inputs (coordinates, element vertices and element->DOF
maps as PHG numbered them, PHG's element geometry (Jacobian and volume), f
and g at the DOF nodes, Dirichlet flags, kappa)
and outputs (matrix rows before and after boundary elimination, saved
boundary columns, RHS before/after update_rhs, Jacobi diagonal, solution,
iteration count, residual) in one compressed .npz per case, plus the
reference's quadrature rules (quad_rules.npz).  Cases with a mass
coefficient c assemble -div(kappa grad u) + c u = f: each element matrix is
stiffness + c * phgQuadBasDotBas, as in examples/simplest.c:68-72.

Run here, where the reference is available:  python tests/golden/make_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from phg_b200.mesh import kuhn_cube, write_medit  # noqa: E402

DUMP = os.path.join(ROOT, "oracle", "_ref", "phg_dump")
QDUMP = os.path.join(ROOT, "oracle", "_ref", "quad_dump")

# name: (m, P, rhs case, kappa seed or None, rtol[, mass coefficient[, solver]])
CASES = {
    "p1_m4_sine": (4, 1, "sine", None, 1e-10),
    "p1_m5_kappa": (5, 1, "sine", 11, 1e-10),
    "p2_m3_sine": (3, 2, "sine", None, 1e-10),
    "p2_m5_kappa": (5, 2, "sine", 12, 1e-8),
    "p2_m6_sine": (6, 2, "sine", None, 1e-8),
    "p3_m2_sine": (2, 3, "sine", None, 1e-10),
    "p3_m3_linear": (3, 3, "linear", None, 1e-10),
    "p3_m3_kappa": (3, 3, "sine", 13, 1e-10),
    "p1_m5_mass": (5, 1, "sine", None, 1e-10, 3.7),
    "p2_m4_kappa_mass": (4, 2, "sine", 14, 1e-10, 0.3),
    "p3_m3_mass": (3, 3, "linear", None, 1e-10, 25.0),
    "p1_m6_bicgstab": (6, 1, "sine", None, 1e-10, 0.0, "bicgstab"),
    "p2_m5_kappa_bicgstab": (5, 2, "sine", 12, 1e-10, 0.0, "bicgstab"),
    "p3_m3_mass_bicgstab": (3, 3, "linear", None, 1e-12, 25.0, "bicgstab"),
    "p1_m6_gmres": (6, 1, "sine", None, 1e-10, 0.0, "gmres_r"),
    "p2_m5_kappa_gmres": (5, 2, "sine", 12, 1e-10, 0.0, "gmres_r"),
    "p3_m3_mass_gmres": (3, 3, "linear", None, 1e-12, 25.0, "gmres_r"),
    # PHG's default GMRES (FLGMRES_r: restart 10, two augmenting corrections)
    "p1_m6_flgmres": (6, 1, "sine", None, 1e-10, 0.0, "flgmres_r"),
    "p2_m5_kappa_flgmres": (5, 2, "sine", 12, 1e-10, 0.0, "flgmres_r"),
    "p3_m3_mass_flgmres": (3, 3, "linear", None, 1e-12, 25.0, "flgmres_r"),
    # meshes PHG refined itself (the element and DOF numbering are PHG's):
    # the reference's test/cube.dat bisected uniformly, and a Kuhn cube
    # refined locally around the corner (0,0,0)
    "p2_cubedat_refined": (1, 2, "sine", None, 1e-10, 0.0, "pcg", dict(mesh="cube.dat", refine=9)),
    "p1_corner_refined": (2, 1, "linear", None, 1e-10, 0.0, "pcg", dict(refine=3, refine_corner=8)),
    "p2_corner_refined": (2, 2, "sine", None, 1e-10, 0.0, "pcg", dict(refine=3, refine_corner=9)),
    "p3_corner_refined": (2, 3, "linear", None, 1e-10, 0.0, "pcg", dict(refine=2, refine_corner=5)),
}
GMRES_RESTART = 10   # the reference's default (-gmres_restart)
LGMRES_AUGK = 2      # the reference's default (-lgmres_augk)


def input_mesh(name):
    """Text of a case's input mesh file that is not generated here: the
    reference's test/cube.dat, read from the reference tree when generating
    and kept in the case's fixture (key input_mesh) for runs without it."""
    fx = os.path.join(HERE, name + ".npz")
    if os.path.exists(fx):
        with np.load(fx) as z:
            if "input_mesh" in z.files:
                return str(z["input_mesh"])
    ref = os.environ.get("PHG_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")
    with open(os.path.join(ref, "test", "cube.dat")) as src:
        return src.read()


def mesh_args(name, d):
    """Writes the case's input mesh into directory d and returns the driver
    arguments that read (and, for the refined cases, refine) it."""
    m = CASES[name][0]
    opts = CASES[name][7] if len(CASES[name]) > 7 else {}
    path = os.path.join(d, "m.mesh")
    if opts.get("mesh") == "cube.dat":
        path = os.path.join(d, "cube.dat")   # ALBERT format, recognised by its name
        with open(path, "w") as dst:
            dst.write(input_mesh(name))
    else:
        v, e = kuhn_cube(m)
        write_medit(path, v, e)
    args = ["-mesh_file", path]
    if opts.get("refine"):
        args += ["-refine", str(opts["refine"])]
    if opts.get("refine_corner"):
        args += ["-refine_corner", str(opts["refine_corner"])]
    return args


def run_case(name, m, P, case, kseed, rtol, mass=0.0, solver="pcg", opts=None):
    with tempfile.TemporaryDirectory() as d:
        e = kuhn_cube(m)[1]
        args = [DUMP, *mesh_args(name, d), "-dof_type", "P%d" % P,
                "-solver", "gmres" if solver in ("gmres_r", "flgmres_r") else solver, "-pcg_pc_type", "jacobi",
                "-solver_rtol", repr(rtol),
                "-solver_btol", "0", "-solver_atol", "0", "-solver_maxit", "10000",
                "-map_reorder", "no", "-dump_dir", d, "-rhs_case", case]
        if mass != 0.0:
            args += ["-mass_coef", repr(mass)]
        if solver in ("gmres_r", "flgmres_r"):
            args += ["-gmres_type", solver, "-gmres_pc_type", "jacobi",
                     "-gmres_restart", str(GMRES_RESTART), "-lgmres_augk", str(LGMRES_AUGK)]
        kappa = None
        if kseed is not None:
            kappa = np.exp(np.random.default_rng(kseed).standard_normal(len(e)))
            kappa.tofile(os.path.join(d, "kappa.in"))
            args += ["-kappa_file", os.path.join(d, "kappa.in")]
        subprocess.run(args, check=True, capture_output=True)
        meta = dict(l.split() for l in open(os.path.join(d, "meta.txt")))

        def L(n, t):
            return np.fromfile(os.path.join(d, n), t)
        N = int(meta["nbas"])
        out = dict(
            order=P, m=m, rtol=rtol, nits=int(meta["nits"]), mass=float(meta["mass_coef"]), solver=solver,
            restart=GMRES_RESTART,
            residual=float(meta["residual"]),
            verts=L("verts.f64", np.float64).reshape(-1, 3),
            elems=L("elems.i32", np.int32).reshape(-1, 4),
            e2l=L("e2l.i32", np.int32).reshape(-1, N),
            bdry=L("bdry.u8", np.uint8), f=L("f.f64", np.float64), g=L("g.f64", np.float64),
            rhs_raw=L("rhs_raw.f64", np.float64), rhs=L("rhs.f64", np.float64),
            diag=L("diag.f64", np.float64), x=L("x.f64", np.float64),
            geom=L("geom.f64", np.float64).reshape(-1, 17))
        if kappa is not None:
            out["kappa"] = L("kappa.f64", np.float64)
        if (opts or {}).get("mesh") == "cube.dat":
            out["input_mesh"] = np.array(input_mesh(name))
        for pre in ("rows_raw", "rows", "bdry_rows"):
            out[pre + "_ptr"] = L(pre + "_ptr.i64", np.int64)
            out[pre + "_cols"] = L(pre + "_cols.i32", np.int32)
            out[pre + "_vals"] = L(pre + "_vals.f64", np.float64)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "ndof", len(out["bdry"]), "nnz", len(out["rows_cols"]), "nits", out["nits"])


def quad_rules():
    txt = subprocess.run([QDUMP], check=True, capture_output=True, text=True).stdout
    rules = {}
    cur = None
    for line in txt.splitlines():
        if line.startswith("order"):
            cur = int(line.split()[1])
            rules[cur] = []
        elif cur is not None and line.strip():
            rules[cur].append([float.fromhex(t) for t in line.split()])
    np.savez_compressed(os.path.join(HERE, "quad_rules.npz"),
                        **{"order%d" % k: np.array(v) for k, v in rules.items()})
    print("quad rules:", {k: len(v) for k, v in rules.items()})


if __name__ == "__main__":
    quad_rules()
    only = sys.argv[1:]
    for name, args in CASES.items():
        if not only or name in only:
            run_case(name, *args)
