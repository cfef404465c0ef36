"""The C-ABI library loads and exports every entry point include/*.h
declares (no GPU needed: nothing here calls into CUDA)."""
import glob
import os
import re
import subprocess

from conftest import ROOT


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(phgGpu\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    assert {"phgGpuCreate", "phgGpuBuildLinearSystem", "phgGpuSolverPCG", "phgGpuMatVec"} <= names


def test_library_exports_all_declared_symbols():
    import phg_b200
    path = phg_b200.LIB_PATH
    assert os.path.exists(path), "library not built"
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    missing = declared_functions() - exported
    assert not missing, missing


def test_python_binding_covers_header():
    import phg_b200
    from phg_b200.core import SIGNATURES
    lib = phg_b200.load_library()
    assert set(SIGNATURES) == declared_functions()
    for name in SIGNATURES:
        assert getattr(lib, name) is not None
    assert lib.phgGpuVersion() >= 100
