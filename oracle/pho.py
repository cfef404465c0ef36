"""ctypes binding of the CPU restatement in oracle/phg_oracle.c.

TEST INFRASTRUCTURE ONLY: the oracle that tests/, smoke() and bench.py's
CPU-baseline leg compare with; the product never imports it.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libphg_oracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle restatement`")
        L = C.CDLL(path)
        P = C.c_void_p
        L.pho_jacobian.argtypes = [P, P]
        L.pho_volume.argtypes = [P]
        L.pho_volume.restype = C.c_double
        L.pho_quad_rule.argtypes = [C.c_int, C.POINTER(P), C.POINTER(P)]
        L.pho_quad_rule.restype = C.c_int
        L.pho_elem_stiffness.argtypes = [C.c_int, P, C.c_double, P]
        L.pho_elem_mass.argtypes = [C.c_int, P, P]
        L.pho_elem_rhs.argtypes = [C.c_int, P, P, P]
        L.pho_assemble.argtypes = [C.c_int, C.c_int64, P, C.c_int64, P, P,
                                   C.c_int64, P, P, P, P, C.c_double, P, P]
        L.pho_assemble.restype = C.c_int
        L.pho_system_free.argtypes = [P]
        L.pho_spmv.argtypes = [C.c_int64, P, P, P, P, P]
        L.pho_pcg.argtypes = [C.c_int64, P, P, P, P, P, P, C.c_int,
                              C.c_double, C.c_double, C.c_double,
                              C.POINTER(C.c_double), P]
        L.pho_pcg.restype = C.c_int
        L.pho_bicgstab.argtypes = [C.c_int64, P, P, P, P, P, P, C.c_int,
                                   C.c_double, C.c_double, C.c_double,
                                   C.POINTER(C.c_double), P, C.POINTER(C.c_int)]
        L.pho_bicgstab.restype = C.c_int
        L.pho_gmres.argtypes = [C.c_int64, P, P, P, P, P, P, C.c_int, C.c_int,
                                C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double)]
        L.pho_gmres.restype = C.c_int
        L.pho_flgmres.argtypes = [C.c_int64, P, P, P, P, P, P, C.c_int, C.c_int, C.c_int,
                                  C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double)]
        L.pho_flgmres.restype = C.c_int
        _LIB = L
    return _LIB


class _System(C.Structure):
    _fields_ = [("n", C.c_int64)] + [
        (name, C.c_void_p) for name in (
            "raw_ptr", "raw_cols", "raw_vals", "ptr", "cols", "vals",
            "bptr", "bcols", "bvals", "rhs_raw", "rhs", "diag")]


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _arr(p, dtype, n):
    if n == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(
        C.cast(p, C.POINTER(np.ctypeslib.as_ctypes_type(dtype))),
        shape=(n,)).copy()


def quad_rule(order):
    pts, wts = C.c_void_p(), C.c_void_p()
    n = lib().pho_quad_rule(order, C.byref(pts), C.byref(wts))
    return (_arr(pts.value, np.float64, 4 * n).reshape(n, 4),
            _arr(wts.value, np.float64, n))


def jacobian(x):
    x = np.ascontiguousarray(x, np.float64)
    J = np.zeros(16)
    lib().pho_jacobian(_ptr(x), _ptr(J))
    return J.reshape(4, 4)


def volume(x):
    return lib().pho_volume(_ptr(np.ascontiguousarray(x, np.float64)))


def elem_stiffness(p, x, kappa=None):
    n = {1: 4, 2: 10, 3: 20}[p]
    A = np.zeros((n, n))
    lib().pho_elem_stiffness(p, _ptr(np.ascontiguousarray(x, np.float64)),
                             -1.0 if kappa is None else float(kappa), _ptr(A))
    return A


def elem_mass(p, x):
    n = {1: 4, 2: 10, 3: 20}[p]
    M = np.zeros((n, n))
    lib().pho_elem_mass(p, _ptr(np.ascontiguousarray(x, np.float64)), _ptr(M))
    return M


def assemble(p, verts, elems, e2l, bdry, f, g=None, kappa=None, mass=0.0, geom=None):
    """Returns a dict of numpy arrays (see pho_system in phg_oracle.h).
    mass != 0 adds mass * (element mass matrix) to each element matrix.
    geom (nelem x 17: Jacobian, volume) is the element geometry PHG stores;
    None computes it from the coordinates (what PHG does on elements it did
    not make by bisection)."""
    verts = np.ascontiguousarray(verts, np.float64)
    elems = np.ascontiguousarray(elems, np.int32)
    e2l = np.ascontiguousarray(e2l, np.int32)
    bdry = np.ascontiguousarray(bdry, np.uint8)
    f = np.ascontiguousarray(f, np.float64)
    g = None if g is None else np.ascontiguousarray(g, np.float64)
    kappa = None if kappa is None else np.ascontiguousarray(kappa, np.float64)
    geom = None if geom is None else np.ascontiguousarray(geom, np.float64)
    ndof = len(bdry)
    S = _System()
    rc = lib().pho_assemble(p, len(verts), _ptr(verts), len(elems),
                            _ptr(elems), _ptr(e2l), ndof, _ptr(bdry), _ptr(f),
                            _ptr(g), _ptr(kappa), C.c_double(mass), _ptr(geom), C.byref(S))
    if rc != 0:
        raise ValueError("pho_assemble failed: %d" % rc)
    n = S.n
    out = {}
    for pre in ("raw_", "", "b"):
        ptr = _arr(getattr(S, pre + "ptr"), np.int64, n + 1)
        nnz = int(ptr[-1])
        out[pre + "ptr"] = ptr
        out[pre + "cols"] = _arr(getattr(S, pre + "cols"), np.int32, nnz)
        out[pre + "vals"] = _arr(getattr(S, pre + "vals"), np.float64, nnz)
    for k in ("rhs_raw", "rhs", "diag"):
        out[k] = _arr(getattr(S, k), np.float64, n)
    lib().pho_system_free(C.byref(S))
    return out


def spmv(ptr, cols, vals, x):
    n = len(ptr) - 1
    y = np.zeros(n)
    lib().pho_spmv(n, _ptr(np.ascontiguousarray(ptr, np.int64)),
                   _ptr(np.ascontiguousarray(cols, np.int32)),
                   _ptr(np.ascontiguousarray(vals, np.float64)),
                   _ptr(np.ascontiguousarray(x, np.float64)), _ptr(y))
    return y


def pcg(ptr, cols, vals, diag, b, x0=None, maxit=10000, rtol=1e-10, btol=0.0,
        atol=0.0):
    """Returns (x, nits, residual, history)."""
    n = len(ptr) - 1
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    hist = np.zeros(maxit + 1)
    res = C.c_double()
    nits = lib().pho_pcg(n, _ptr(np.ascontiguousarray(ptr, np.int64)),
                         _ptr(np.ascontiguousarray(cols, np.int32)),
                         _ptr(np.ascontiguousarray(vals, np.float64)),
                         _ptr(np.ascontiguousarray(diag, np.float64)),
                         _ptr(np.ascontiguousarray(b, np.float64)), _ptr(x),
                         maxit, rtol, btol, atol, C.byref(res), _ptr(hist))
    return x, nits, res.value, hist[:nits + 1]


def bicgstab(ptr, cols, vals, diag, b, x0=None, maxit=10000, rtol=1e-10, btol=0.0,
             atol=0.0):
    """Jacobi-BiCGstab.  Returns (x, nits, residual, history, status)."""
    n = len(ptr) - 1
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    hist = np.zeros(maxit + 1)
    res = C.c_double()
    st = C.c_int()
    nits = lib().pho_bicgstab(n, _ptr(np.ascontiguousarray(ptr, np.int64)),
                              _ptr(np.ascontiguousarray(cols, np.int32)),
                              _ptr(np.ascontiguousarray(vals, np.float64)),
                              _ptr(np.ascontiguousarray(diag, np.float64)),
                              _ptr(np.ascontiguousarray(b, np.float64)), _ptr(x),
                              maxit, rtol, btol, atol, C.byref(res), _ptr(hist), C.byref(st))
    return x, nits, res.value, hist[:nits + 1], st.value


def gmres(ptr, cols, vals, diag, b, x0=None, restart=10, maxit=10000, rtol=1e-10, btol=0.0,
          atol=0.0):
    """Restarted right-preconditioned Jacobi-GMRES.  Returns (x, nits, residual)."""
    n = len(ptr) - 1
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    res = C.c_double()
    nits = lib().pho_gmres(n, _ptr(np.ascontiguousarray(ptr, np.int64)),
                           _ptr(np.ascontiguousarray(cols, np.int32)),
                           _ptr(np.ascontiguousarray(vals, np.float64)),
                           _ptr(np.ascontiguousarray(diag, np.float64)),
                           _ptr(np.ascontiguousarray(b, np.float64)), _ptr(x),
                           restart, maxit, rtol, btol, atol, C.byref(res))
    return x, nits, res.value


def flgmres(ptr, cols, vals, diag, b, x0=None, restart=10, augk=2, maxit=10000, rtol=1e-10, btol=0.0,
            atol=0.0):
    """PHG's default GMRES (FLGMRES_r), Jacobi PC.  Returns (x, nits, residual)."""
    n = len(ptr) - 1
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    res = C.c_double()
    nits = lib().pho_flgmres(n, _ptr(np.ascontiguousarray(ptr, np.int64)),
                             _ptr(np.ascontiguousarray(cols, np.int32)),
                             _ptr(np.ascontiguousarray(vals, np.float64)),
                             _ptr(np.ascontiguousarray(diag, np.float64)),
                             _ptr(np.ascontiguousarray(b, np.float64)), _ptr(x),
                             restart, augk, maxit, rtol, btol, atol, C.byref(res))
    return x, nits, res.value
