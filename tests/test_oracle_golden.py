"""Pins the CPU oracle (oracle/phg_oracle.c) against outputs of the
unmodified reference built from its sources (tests/golden/, generated by
tests/golden/make_golden.py).  Everything is compared bit for bit."""
import numpy as np
import pytest

from conftest import golden_cases, load_golden, GOLDEN


def test_quadrature_rules_bitexact(oracle):
    z = np.load(GOLDEN + "/quad_rules.npz")
    for order in range(7):
        ref = z["order%d" % order]
        pts, wts = oracle.quad_rule(order)
        assert np.array_equal(pts, ref[:, :4]), order
        assert np.array_equal(wts, ref[:, 4]), order


def refined(name):
    """Meshes PHG refined by bisection: their elements' Jacobians and volumes
    are interpolated from the parents (geom.c:460-565), not computed from
    the coordinates, so the assembly takes PHG's stored geometry."""
    return "refined" in name


@pytest.mark.parametrize("name", golden_cases())
def test_assembly_bitexact(oracle, name):
    G = load_golden(name)
    o = oracle.assemble(int(G["order"]), G["verts"], G["elems"], G["e2l"], G["bdry"], G["f"],
                        G["g"], G.get("kappa"), float(G.get("mass", 0.0)),
                        geom=G["geom"] if refined(name) else None)
    for pre, op in (("rows_raw", "raw_"), ("rows", ""), ("bdry_rows", "b")):
        assert np.array_equal(G[pre + "_ptr"], o[op + "ptr"]), pre
        assert np.array_equal(G[pre + "_cols"], o[op + "cols"]), pre
        assert np.array_equal(G[pre + "_vals"], o[op + "vals"]), pre
    for k in ("rhs_raw", "rhs", "diag"):
        assert np.array_equal(G[k], o[k]), k


@pytest.mark.parametrize("name", [n for n in golden_cases() if not refined(n)])
def test_coordinate_geometry_is_phgs(oracle, name):
    """On meshes PHG imported (no bisection) the geometry computed from the
    coordinates (compute_jacobian, geom.c:103-169) is PHG's stored one, so
    assembling with PHG's dumped geometry changes nothing."""
    G = load_golden(name)
    args = (int(G["order"]), G["verts"], G["elems"], G["e2l"], G["bdry"], G["f"], G["g"], G.get("kappa"),
            float(G.get("mass", 0.0)))
    a, b = oracle.assemble(*args), oracle.assemble(*args, geom=G["geom"])
    for k in ("raw_ptr", "raw_cols", "raw_vals", "vals", "rhs"):
        assert np.array_equal(a[k], b[k]), k


def test_refined_geometry_differs_from_coordinates(oracle):
    """On a bisected mesh PHG's interpolated Jacobians differ from the ones
    the coordinates give in the last bits, and the assembled rows keep
    entries the coordinates would turn into round-off (or the reverse)."""
    G = load_golden("p1_corner_refined")
    args = (1, G["verts"], G["elems"], G["e2l"], G["bdry"], G["f"], G["g"], G.get("kappa"))
    a, b = oracle.assemble(*args), oracle.assemble(*args, geom=G["geom"])
    assert not np.array_equal(a["raw_cols"], b["raw_cols"])
    assert np.array_equal(b["raw_cols"], G["rows_raw_cols"])


def solver_of(G):
    return str(G["solver"]) if "solver" in G else "pcg"


@pytest.mark.parametrize("name", golden_cases())
def test_solver_bitexact(oracle, name):
    """Iteration count, final residual and solution of the reference's
    solve_pcg, solver_BiCGstab, solver_GMRES_r or solver_FLGMRES_r, bit for
    bit."""
    G = load_golden(name)
    args = (G["rows_ptr"], G["rows_cols"], G["rows_vals"], G["diag"], G["rhs"])
    if solver_of(G) == "bicgstab":
        x, nits, res, hist, status = oracle.bicgstab(*args, rtol=float(G["rtol"]), btol=0.0, atol=0.0)
        assert status == 0
    elif solver_of(G) == "gmres_r":
        x, nits, res = oracle.gmres(*args, restart=int(G["restart"]), rtol=float(G["rtol"]), btol=0.0,
                                    atol=0.0)
        hist = None
    elif solver_of(G) == "flgmres_r":
        x, nits, res = oracle.flgmres(*args, restart=int(G["restart"]), augk=2, rtol=float(G["rtol"]),
                                      btol=0.0, atol=0.0)
        hist = None
    else:
        x, nits, res, hist = oracle.pcg(*args, rtol=float(G["rtol"]), btol=0.0, atol=0.0)
    assert nits == int(G["nits"])
    assert res == float(G["residual"])
    assert np.array_equal(x, G["x"])
    if hist is not None:
        assert hist[-1] == res and len(hist) == nits + 1


def test_linear_solution_reproduced():
    """u = x + y + z lies in every P_k space (examples/functions.h:34-42,
    TEST_CASE 1): the reference's discrete solution equals it at the nodes up
    to the solver tolerance."""
    import phg_b200 as pb
    G = load_golden("p3_m3_linear")
    e2l, bdry, nodes = pb.lagrange_dofs(G["verts"], G["elems"], 3)
    perm = np.empty(len(bdry), np.int64)
    perm[G["e2l"].ravel()] = e2l.ravel()
    u = nodes[perm].sum(axis=1)
    assert np.max(np.abs(G["x"] - u)) < 1e-7
    b = G["bdry"].astype(bool)
    assert np.allclose(G["g"][b], u[b], rtol=0, atol=1e-15)


def test_zero_drop_pattern_is_value_dependent():
    """With non-dyadic coordinates (m = 5) rounding leaves tiny non-zero
    element entries that the reference keeps: the P1 pattern is wider than
    the exact-arithmetic 7-point stencil, so a pattern built from exact
    arithmetic would not match."""
    G = load_golden("p1_m5_kappa")
    ptr = G["rows_ptr"]
    interior = np.flatnonzero(G["bdry"] == 0)
    lens = ptr[interior + 1] - ptr[interior]
    assert lens.max() > 7
