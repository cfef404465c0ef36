"""The GPU solvers as PHG OEM solvers (phg_b200/shim/libphg_gpu_solver.so):
the reference's own program (oracle/ref_driver/phg_dump.c, linked against a
shared build of the reference as oracle/_ref/phg_dump_gpu) assembles with
PHG and passes &phgSolverGpuPCG_ (or the mixed, BiCGstab, GMRES twin) to
phgSolverCreate (-gpu_solver).  PHG packs its rows and phgSolverSolve runs
on the GPU; the dumped solution and iteration count are compared with the
reference's own run (the golden fixtures): iterations within 2, solution
within 1e3 * rtol (relative L2; device dot products sum in another order)."""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden_cases, load_golden

pytestmark = pytest.mark.gpu

DUMP = os.path.join(ROOT, "oracle", "_ref", "phg_dump_gpu")
sys.path.insert(0, GOLDEN)
from make_golden import CASES, GMRES_RESTART, mesh_args  # noqa: E402


def run(name, gpu_solver, extra=()):
    m, P, case, kseed, rtol, *rest = CASES[name]
    mass = rest[0] if rest else 0.0
    solver = rest[1] if len(rest) > 1 else "pcg"
    from phg_b200.mesh import kuhn_cube
    with tempfile.TemporaryDirectory() as d:
        e = kuhn_cube(m)[1]
        args = [DUMP, *mesh_args(name, d), "-dof_type", "P%d" % P,
                "-solver_rtol", repr(rtol), "-solver_btol", "0", "-solver_atol", "0",
                "-solver_maxit", "10000", "-map_reorder", "no", "-dump_dir", d, "-rhs_case", case,
                "-gpu_solver", gpu_solver, "-gmres_restart", str(GMRES_RESTART), *extra]
        if mass != 0.0:
            args += ["-mass_coef", repr(mass)]
        if kseed is not None:
            np.exp(np.random.default_rng(kseed).standard_normal(len(e))).tofile(os.path.join(d, "kappa.in"))
            args += ["-kappa_file", os.path.join(d, "kappa.in")]
        p = subprocess.run(args, capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, (p.stdout[-2000:], p.stderr[-2000:])
        meta = dict(l.split() for l in open(os.path.join(d, "meta.txt")))
        x = np.fromfile(os.path.join(d, "x.f64"), np.float64)
        rhs = np.fromfile(os.path.join(d, "rhs.f64"), np.float64)
        return {"nits": int(meta["nits"]), "residual": float(meta["residual"]), "x": x, "rhs": rhs,
                "stdout": p.stdout}


PLUGIN_OF = {"pcg": "pcg", "bicgstab": "bicgstab", "gmres_r": "gmres", "flgmres_r": "gmres"}


def solver_of(name):
    rest = CASES[name][5:]
    return rest[1] if len(rest) > 1 else "pcg"


@pytest.mark.parametrize("name", golden_cases())
def test_reference_program_through_gpu_oem_solver(name):
    G = load_golden(name)
    solver = solver_of(name)
    extra = ("-gmres_type", solver) if solver in ("gmres_r", "flgmres_r") else ()
    out = run(name, PLUGIN_OF[solver], extra)
    rtol = float(G["rtol"])
    assert np.array_equal(out["rhs"], G["rhs"])   # PHG's own assembly, unchanged
    assert abs(out["nits"] - int(G["nits"])) <= 2, (out["nits"], int(G["nits"]))
    assert np.linalg.norm(out["x"] - G["x"]) <= 1e3 * rtol * np.linalg.norm(G["x"])


@pytest.mark.parametrize("name", [n for n in golden_cases() if solver_of(n) == "pcg"])
def test_reference_program_through_mixed_oem_solver(name):
    """The mixed-precision OEM solver meets the same FP64 stopping rule."""
    G = load_golden(name)
    out = run(name, "pcg_mixed")
    rtol = float(G["rtol"])
    assert out["residual"] <= rtol * np.linalg.norm(G["rhs"]) * (1 + 1e-9)
    assert np.linalg.norm(out["x"] - G["x"]) <= 1e3 * rtol * np.linalg.norm(G["x"])
