"""Host-side mesh and DOF numbering (no GPU)."""
import numpy as np
import pytest

import phg_b200 as pb
from conftest import load_golden


@pytest.mark.parametrize("m", [1, 2, 3])
def test_kuhn_counts(m):
    v, e = pb.kuhn_cube(m)
    assert v.shape == ((m + 1) ** 3, 3)
    assert e.shape == (6 * m ** 3, 4)
    # positive volumes, all equal to 1 / (6 m^3)
    x = v[e]
    d = np.linalg.det(x[:, 1:] - x[:, :1])
    assert np.allclose(np.abs(d) / 6, 1 / (6 * m ** 3))


@pytest.mark.parametrize("p,ndof", [(1, 125), (2, 729), (3, 2197)])
def test_lagrange_counts(p, ndof):
    v, e = pb.kuhn_cube(4)
    e2l, bdry, nodes = pb.lagrange_dofs(v, e, p)
    assert len(bdry) == ndof == (4 * p + 1) ** 3
    # boundary DOFs are exactly the nodes on the cube's surface
    on = np.any((np.abs(nodes) < 1e-12) | (np.abs(nodes - 1) < 1e-12), axis=1)
    assert np.array_equal(on, bdry.astype(bool))
    # every DOF is used, element maps have distinct entries
    assert len(np.unique(e2l)) == ndof
    assert all(len(set(r)) == e2l.shape[1] for r in e2l[:50])


@pytest.mark.parametrize("name", ["p2_m3_sine", "p3_m3_kappa", "p3_m3_linear"])
def test_numbering_matches_reference_up_to_permutation(oracle, name):
    """Our DOF numbering, applied to the reference's elements (with the
    reference's vertex order inside each element, which its refinement setup
    chooses), yields the reference's element->DOF map up to a permutation of
    the DOFs, and the same assembled rows entry for entry."""
    G = load_golden(name)
    p = int(G["order"])
    v, e = G["verts"], G["elems"]
    e2l, bdry, nodes = pb.lagrange_dofs(v, e, p)
    n = len(bdry)
    perm = np.full(n, -1)
    perm[G["e2l"].ravel()] = e2l.ravel()
    # a consistent bijection: every reference DOF maps to one of ours
    assert (perm >= 0).all() and len(np.unique(perm)) == n
    assert np.array_equal(perm[G["e2l"]], e2l)
    assert np.array_equal(bdry[perm], G["bdry"])
    o = oracle.assemble(p, v, e, e2l, bdry, G["f"][np.argsort(perm)], G["g"][np.argsort(perm)],
                        G.get("kappa"))
    ptr, cols, vals = G["rows_ptr"], G["rows_cols"], G["rows_vals"]
    assert len(o["cols"]) == len(cols)
    for i in range(n):
        j = perm[i]
        ref = sorted(zip(perm[cols[ptr[i]:ptr[i + 1]]], vals[ptr[i]:ptr[i + 1]]))
        got = sorted(zip(o["cols"][o["ptr"][j]:o["ptr"][j + 1]], o["vals"][o["ptr"][j]:o["ptr"][j + 1]]))
        assert ref == got
    assert np.array_equal(o["rhs"][perm], G["rhs"])
