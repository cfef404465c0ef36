"""ctypes binding of libphg_b200.so (include/phg_gpu.h).

`Solver` mirrors the reference's objects for this path: a GRID (set_mesh), a
DOF layout (set_dof_map), the user element loop plus phgSolverAssemble
(build_linear_system), phgMatVec (mat_vec) and phgSolverSolve with the PCG
solver (solve_pcg).  Arrays may be numpy arrays (host memory) or torch CUDA
tensors (device memory, used in place).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libphg_b200.so")

ERRORS = {-1: "PHG_GPU_ERR_ARG", -2: "PHG_GPU_ERR_CUDA", -3: "PHG_GPU_ERR_STATE",
          -4: "PHG_GPU_ERR_LIMIT", -5: "PHG_GPU_ERR_BREAKDOWN", -6: "PHG_GPU_ERR_NAN"}

# name -> (restype, argtypes) of every entry point declared in phg_gpu.h
_P = C.c_void_p
_I64 = C.c_int64
SIGNATURES = {
    "phgGpuLastError": (C.c_char_p, []),
    "phgGpuLastWarning": (C.c_char_p, []),
    "phgGpuVersion": (C.c_int, []),
    "phgGpuCreate": (C.c_int, [C.c_int, _P, C.POINTER(_P)]),
    "phgGpuDestroy": (C.c_int, [_P]),
    "phgGpuSetStream": (C.c_int, [_P, _P]),
    "phgGpuSetMesh": (C.c_int, [_P, _I64, _P, _I64, _P]),
    "phgGpuSetGeometry": (C.c_int, [_P, _I64, _P]),
    "phgGpuSetDofMap": (C.c_int, [_P, C.c_int, _I64, _P, _P]),
    "phgGpuBuildLinearSystem": (C.c_int, [_P, _P, _P, _P]),
    "phgGpuBuildLinearSystemMass": (C.c_int, [_P, _P, C.c_double, _P, _P]),
    "phgGpuSetMatrix": (C.c_int, [_P, _I64, _P, _P, _P, _P]),
    "phgGpuSetRHS": (C.c_int, [_P, _P]),
    "phgGpuAssembleRows": (C.c_int, [_P, _I64, _I64, _P, _P, _P, _P]),
    "phgGpuGetSizes": (C.c_int, [_P, C.POINTER(_I64), C.POINTER(_I64), C.POINTER(_I64)]),
    "phgGpuGetMatrix": (C.c_int, [_P, _P, _P, _P]),
    "phgGpuGetBdryColumns": (C.c_int, [_P, _P, _P, _P]),
    "phgGpuGetRHS": (C.c_int, [_P, _P]),
    "phgGpuGetDiagonal": (C.c_int, [_P, _P]),
    "phgGpuMatVec": (C.c_int, [_P, _P, _P]),
    "phgGpuSolverPCG": (C.c_int, [_P, C.c_double, C.c_double, C.c_double, C.c_int, _P,
                                  C.POINTER(C.c_double), _P]),
    "phgGpuSolverBiCGstab": (C.c_int, [_P, C.c_double, C.c_double, C.c_double, C.c_int, _P,
                                       C.POINTER(C.c_double), _P]),
    "phgGpuSolverGMRES": (C.c_int, [_P, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, _P,
                                    C.POINTER(C.c_double)]),
    "phgGpuSolverFLGMRES": (C.c_int, [_P, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                      _P, C.POINTER(C.c_double)]),
    "phgGpuSetSpMVPlan32": (C.c_int, [_P, C.c_int, C.c_int]),
    "phgGpuElementMatrices": (C.c_int, [_P, _P, C.c_double, _P, _P, _P]),
    "phgGpuGetLaunchCount": (C.c_int, [_P, C.POINTER(_I64)]),
    "phgGpuGetSpMVPlan": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), _P]),
    "phgGpuSetSpMVPlan": (C.c_int, [_P, C.c_int, C.c_int]),
    "phgGpuSolverBlockPCG": (C.c_int, [_P, C.c_int, _P, _P, C.c_double, C.c_int, C.c_int, _P, _P]),
    "phgGpuGetBlockTile": (C.c_int, [_P, C.POINTER(C.c_int), _P]),
    "phgGpuAdjointGradient": (C.c_int, [_P, _P, _P, C.c_double, C.c_int, _P, C.POINTER(C.c_double),
                                        C.POINTER(C.c_int)]),
    "phgGpuTimeSpMV": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "phgGpuSpMVBytes": (C.c_int, [_P, C.c_int, C.POINTER(_I64)]),
    "phgGpuSolverPCGMixed": (C.c_int, [_P, C.c_double, C.c_double, C.c_double, C.c_int, _P,
                                       C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "phgGpuSolverPCGNoAlloc": (C.c_int, [_I64, _P, _P, _P, _P, _P, C.c_double, C.c_double,
                                         C.c_double, C.c_int, _P, C.POINTER(C.c_double)]),
}

NOALLOC_MAX_ROWS = 262144

_LIB = None


class PhgGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "error"), code, msg))
        self.code = code


def load_library(path=LIB_PATH):
    """Loads the library without touching the GPU (no CUDA calls)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(path):
            raise RuntimeError("libphg_b200.so is not built (run __graft_entry__.build())")
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def lib():
    return load_library()


def _check(rc):
    if rc < 0:
        raise PhgGpuError(rc, lib().phgGpuLastError().decode())
    return rc


def last_warning():
    """Warning text of the calling thread's last solver call ("" if none):
    e.g. a PCG breakdown, which the reference reports as "the matrix may not
    be SPD" and survives (solver-phg.c:547-571)."""
    return lib().phgGpuLastWarning().decode()


def _ptr(a):
    """Raw pointer of a numpy array or a torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return a.data_ptr()
    raise TypeError("expected a numpy array or a torch tensor, got %r" % type(a))


def _np(a, dtype):
    if a is None or hasattr(a, "data_ptr"):
        return a
    return np.ascontiguousarray(a, dtype=dtype)


# FP64 product layouts (solvers, mat_vec) and FP32 product layouts of the
# mixed solver, by their C-ABI codes
LAYOUTS64 = ("csr", "sell", "q16")
LAYOUTS32 = ("sell", "pair", "q16")


class Solver:
    """One assembled linear system on one GPU (a phgGpuSystem)."""

    def __init__(self, device=0, stream=None):
        self._h = C.c_void_p()
        _check(lib().phgGpuCreate(int(device), stream, C.byref(self._h)))
        self._keep = []

    def close(self):
        if self._h:
            lib().phgGpuDestroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream):
        _check(lib().phgGpuSetStream(self._h, stream))

    def set_mesh(self, verts, elems):
        verts, elems = _np(verts, np.float64), _np(elems, np.int32)
        self.nelem = len(elems)
        _check(lib().phgGpuSetMesh(self._h, len(verts), _ptr(verts), len(elems), _ptr(elems)))

    def set_geometry(self, geo):
        """PHG's stored element geometry (nelem x 17: Jacobian, volume), used
        instead of the coordinates' until the next set_mesh; on elements PHG
        made by bisection it is interpolated from the parent."""
        geo = _np(geo, np.float64)
        if geo.ndim != 2 or geo.shape[1] != 17:
            raise ValueError("geometry must be nelem x 17")
        _check(lib().phgGpuSetGeometry(self._h, len(geo), _ptr(geo)))

    def set_dof_map(self, order, e2l, bdry):
        e2l, bdry = _np(e2l, np.int32), _np(bdry, np.uint8)
        self.nbas = {1: 4, 2: 10, 3: 20}.get(int(order), 0)
        _check(lib().phgGpuSetDofMap(self._h, int(order), len(bdry), _ptr(e2l), _ptr(bdry)))

    def build_linear_system(self, kappa=None, f=None, g=None, mass=0.0):
        """Element loop + assembly; mass != 0 adds mass * (element mass
        matrix) to every element matrix (-div(kappa grad u) + mass u = f)."""
        kappa, f, g = _np(kappa, np.float64), _np(f, np.float64), _np(g, np.float64)
        if mass != 0.0:
            _check(lib().phgGpuBuildLinearSystemMass(self._h, _ptr(kappa), float(mass), _ptr(f), _ptr(g)))
        else:
            _check(lib().phgGpuBuildLinearSystem(self._h, _ptr(kappa), _ptr(f), _ptr(g)))

    def element_matrices(self, kappa=None, f=None, mass=0.0):
        """Element matrices (nelem, N, N) and right-hand sides (nelem, N)."""
        n_el = self.nelem
        N = self.nbas
        kappa, f = _np(kappa, np.float64), _np(f, np.float64)
        Ke = np.empty((n_el, N, N))
        Re = np.empty((n_el, N))
        _check(lib().phgGpuElementMatrices(self._h, _ptr(kappa), float(mass), _ptr(f), _ptr(Ke), _ptr(Re)))
        return Ke, Re

    def set_matrix(self, ptr, cols, vals, rhs):
        ptr, cols = _np(ptr, np.int64), _np(cols, np.int32)
        vals, rhs = _np(vals, np.float64), _np(rhs, np.float64)
        _check(lib().phgGpuSetMatrix(self._h, len(ptr) - 1, _ptr(ptr), _ptr(cols), _ptr(vals), _ptr(rhs)))

    def assemble_rows(self, n, rec_row, rec_ptr, rec_cols, rec_vals):
        """Rows from row segments in call order, as phgMatAddEntries_ builds
        them (zeros dropped, first-touch column order)."""
        rec_row, rec_ptr = _np(rec_row, np.int32), _np(rec_ptr, np.int64)
        rec_cols, rec_vals = _np(rec_cols, np.int32), _np(rec_vals, np.float64)
        _check(lib().phgGpuAssembleRows(self._h, int(n), len(rec_row), _ptr(rec_row), _ptr(rec_ptr),
                                        _ptr(rec_cols), _ptr(rec_vals)))

    def set_rhs(self, rhs):
        """Replaces the right-hand side of the assembled system (after
        boundary elimination), keeping the matrix."""
        rhs = _np(rhs, np.float64)
        _check(lib().phgGpuSetRHS(self._h, _ptr(rhs)))

    def sizes(self):
        n, nnz, bnnz = _I64(), _I64(), _I64()
        _check(lib().phgGpuGetSizes(self._h, C.byref(n), C.byref(nnz), C.byref(bnnz)))
        return n.value, nnz.value, bnnz.value

    def get_matrix(self):
        n, nnz, _ = self.sizes()
        ptr, cols, vals = np.empty(n + 1, np.int64), np.empty(nnz, np.int32), np.empty(nnz)
        _check(lib().phgGpuGetMatrix(self._h, _ptr(ptr), _ptr(cols), _ptr(vals)))
        return ptr, cols, vals

    def get_bdry_columns(self):
        n, _, bnnz = self.sizes()
        ptr, cols, vals = np.empty(n + 1, np.int64), np.empty(bnnz, np.int32), np.empty(bnnz)
        _check(lib().phgGpuGetBdryColumns(self._h, _ptr(ptr), _ptr(cols), _ptr(vals)))
        return ptr, cols, vals

    def get_rhs(self):
        out = np.empty(self.sizes()[0])
        _check(lib().phgGpuGetRHS(self._h, _ptr(out)))
        return out

    def get_diagonal(self):
        out = np.empty(self.sizes()[0])
        _check(lib().phgGpuGetDiagonal(self._h, _ptr(out)))
        return out

    def mat_vec(self, x, y=None):
        x = _np(x, np.float64)
        if y is None:
            y = np.empty(self.sizes()[0])
        _check(lib().phgGpuMatVec(self._h, _ptr(x), _ptr(y)))
        return y

    def solve_pcg_mixed(self, x0=None, rtol=1e-8, btol=0.0, atol=0.0, maxit=10000, out=None):
        """FP32-inner / FP64-refinement Jacobi-PCG.  Returns
        (x, nits, residual, reliable_updates); residual = ||b - A x|| in FP64."""
        n = self.sizes()[0]
        if out is not None:
            x = out
        else:
            x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
        res, nupd = C.c_double(), C.c_int()
        nits = _check(lib().phgGpuSolverPCGMixed(self._h, rtol, btol, atol, int(maxit), _ptr(x),
                                                 C.byref(res), C.byref(nupd)))
        return x, nits, res.value, nupd.value

    SPMV_LAYOUTS = (("csr", 4), ("csr", 8), ("csr", 16), ("csr", 32),
                    ("sell", 2), ("sell", 4), ("sell", 8), ("q16", 1))

    def time_spmv(self, fp32=False, reps=50):
        """Average ms of one SpMV launch (chosen layout; FP32 values if fp32)."""
        ms = C.c_double()
        _check(lib().phgGpuTimeSpMV(self._h, 1 if fp32 else 0, int(reps), C.byref(ms)))
        return ms.value

    def spmv_bytes(self, fp32=False):
        """Bytes one product moves in the layout in use (values, indices,
        metadata as stored, x read once, y written once)."""
        b = _I64()
        _check(lib().phgGpuSpMVBytes(self._h, 1 if fp32 else 0, C.byref(b)))
        return b.value

    def set_spmv_plan(self, layout, param):
        _check(lib().phgGpuSetSpMVPlan(self._h, LAYOUTS64.index(layout), int(param)))

    def set_spmv_plan32(self, layout, unroll):
        """Forces the mixed solver's FP32 product: layout "sell", "pair" or
        "q16" (16-bit column offsets; only for matrices whose rows fit two
        65536-column windows) with the given unroll."""
        _check(lib().phgGpuSetSpMVPlan32(self._h, LAYOUTS32.index(layout), int(unroll)))

    def solve_block_pcg(self, B, rtol=1e-8, maxit=10000, mixed=False, out=None):
        """Block PCG on the columns of B (n x nrhs).  Returns (X, nits[nrhs],
        residuals[nrhs])."""
        B = _np(B, np.float64)
        n, nrhs = B.shape
        X = np.empty((n, nrhs)) if out is None else out
        nits = np.zeros(nrhs, np.int32)
        res = np.zeros(nrhs)
        _check(lib().phgGpuSolverBlockPCG(self._h, nrhs, _ptr(B), _ptr(X), rtol, int(maxit),
                                          1 if mixed else 0, _ptr(nits), _ptr(res)))
        return X, nits, res

    def block_tile(self):
        t = C.c_int()
        times = np.zeros(4)
        _check(lib().phgGpuGetBlockTile(self._h, C.byref(t), _ptr(times)))
        return t.value, dict(zip((8, 16, 32, 64), times.tolist()))

    def adjoint_gradient(self, u, u_obs, rtol=1e-10, maxit=100000, out=None):
        """dJ/dlog kappa_e for J = 1/2 ||u - u_obs||^2, u the solution of the
        last built system.  Returns (grad, J, adjoint iterations)."""
        u, u_obs = _np(u, np.float64), _np(u_obs, np.float64)
        if out is None:
            out = np.empty(self.nelem)
        J, nits = C.c_double(), C.c_int()
        _check(lib().phgGpuAdjointGradient(self._h, _ptr(u), _ptr(u_obs), rtol, int(maxit), _ptr(out),
                                           C.byref(J), C.byref(nits)))
        return out, J.value, nits.value

    def spmv_plan(self):
        """(layout, parameter, {candidate: ms}) chosen by the SpMV autotuner."""
        kind, param = C.c_int(), C.c_int()
        times = np.zeros(24)
        nc = _check(lib().phgGpuGetSpMVPlan(self._h, C.byref(kind), C.byref(param), _ptr(times)))
        names = ["csr4", "csr8", "csr16", "csr32", "sell_u2", "sell_u4", "sell_u8", "q16"][:nc]
        info = dict(zip(names, times[:nc].tolist()))
        names32 = ("fp32_sell_u4", "fp32_sell_u8", "fp32_sell_u16", "fp32_pair_u2", "fp32_pair_u4",
                   "fp32_pair_u8", "fp32_q16_u1", "fp32_q16_u2")
        for i, name in enumerate(names32):
            info[name] = float(times[nc + i])
        k = nc + len(names32)
        info["fp32_unroll"] = int(times[k])
        info["fp32_layout"] = LAYOUTS32[int(times[k + 1])]
        return LAYOUTS64[kind.value], param.value, info

    def launch_count(self):
        c = _I64()
        _check(lib().phgGpuGetLaunchCount(self._h, C.byref(c)))
        return c.value

    def solve_pcg(self, x0=None, rtol=1e-10, btol=1e-10, atol=0.0, maxit=10000, history=False, out=None):
        """phgSolverSolve with -solver pcg -pcg_pc_type jacobi.  Returns
        (x, nits, residual) or (x, nits, residual, history)."""
        n = self.sizes()[0]
        if out is not None:
            x = out
        else:
            x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
        hist = np.empty(maxit + 1) if history else None
        res = C.c_double()
        nits = _check(lib().phgGpuSolverPCG(self._h, rtol, btol, atol, int(maxit), _ptr(x),
                                            C.byref(res), _ptr(hist)))
        if history:
            return x, nits, res.value, hist[:nits + 1]
        return x, nits, res.value

    def solve_bicgstab(self, x0=None, rtol=1e-10, btol=1e-10, atol=0.0, maxit=10000, history=False, out=None):
        """phgSolverSolve with -solver bicgstab -pcg_pc_type jacobi.  Returns
        (x, nits, residual) or (x, nits, residual, history)."""
        n = self.sizes()[0]
        if out is not None:
            x = out
        else:
            x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
        hist = np.empty(maxit + 1) if history else None
        res = C.c_double()
        nits = _check(lib().phgGpuSolverBiCGstab(self._h, rtol, btol, atol, int(maxit), _ptr(x),
                                                 C.byref(res), _ptr(hist)))
        if history:
            return x, nits, res.value, hist[:nits + 1]
        return x, nits, res.value


    def solve_gmres(self, x0=None, restart=10, rtol=1e-10, btol=1e-10, atol=0.0, maxit=10000, out=None):
        """phgSolverSolve with -solver gmres -gmres_type gmres_r
        -gmres_pc_type jacobi -gmres_restart `restart`.  Returns
        (x, nits, residual)."""
        n = self.sizes()[0]
        if out is not None:
            x = out
        else:
            x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
        res = C.c_double()
        nits = _check(lib().phgGpuSolverGMRES(self._h, int(restart), rtol, btol, atol, int(maxit), _ptr(x),
                                              C.byref(res)))
        return x, nits, res.value

    def solve_flgmres(self, x0=None, restart=10, augk=2, rtol=1e-10, btol=1e-10, atol=0.0, maxit=10000,
                      out=None):
        """phgSolverSolve with -solver gmres (PHG's default -gmres_type
        flgmres_r) -gmres_pc_type jacobi -gmres_restart `restart`
        -lgmres_augk `augk`.  Returns (x, nits, residual)."""
        n = self.sizes()[0]
        if out is not None:
            x = out
        else:
            x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
        res = C.c_double()
        nits = _check(lib().phgGpuSolverFLGMRES(self._h, int(restart), int(augk), rtol, btol, atol, int(maxit),
                                                _ptr(x), C.byref(res)))
        return x, nits, res.value


def solve_pcg_no_alloc(ptr, cols, vals, rhs, x, rtol=1e-10, btol=1e-10, atol=0.0, maxit=10000,
                       stream=None):
    """phgGpuSolverPCGNoAlloc: Jacobi-PCG on a CSR matrix held in device
    memory (torch CUDA tensors: ptr int64, cols int32, vals/rhs/x float64),
    without allocating any memory -- for callers that cannot allocate.  x is
    the initial guess and receives the solution.  Returns (nits, residual)."""
    res = C.c_double()
    nits = _check(lib().phgGpuSolverPCGNoAlloc(len(ptr) - 1, _ptr(ptr), _ptr(cols), _ptr(vals),
                                               _ptr(rhs), _ptr(x), rtol, btol, atol, int(maxit),
                                               stream, C.byref(res)))
    return nits, res.value
