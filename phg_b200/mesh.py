"""Host-side mesh utilities for the synthetic unit-cube meshes.

The meshes are the Kuhn (Freudenthal) subdivision of an m x m x m grid of
subcubes into 6 tetrahedra each, all sharing the subcube's main diagonal --
the same 6-tetrahedron pattern as the reference's ``test/cube.dat`` fixture
(test/cube.dat:1-40), repeated over the grid.  Mesh generation stays on the
host (as PHG's own mesh import and refinement do); these helpers only build
the vertex/element arrays and write them in the Medit text format that PHG's
``phgImportMedit`` (src/medit.c:203) reads.
"""
import numpy as np

# The 6 axis permutations; tetrahedron p of a subcube walks from the subcube's
# low corner along axes PERMS[p][0], PERMS[p][1], PERMS[p][2].
PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


def kuhn_cube(m):
    """Returns (verts float64[(m+1)^3, 3], elems int32[6 m^3, 4]).

    Vertex (i, j, k) has index i + (m+1) (j + (m+1) k) and coordinates
    (i/m, j/m, k/m).  Subcubes are visited with i fastest; each contributes
    6 tetrahedra in PERMS order.  A tetrahedron walking w0 -> w1 -> w2 -> w3
    from the subcube's low corner to its high corner is stored as
    (w0, w3, w2, w1): the main diagonal first, which is the vertex order the
    reference's refinement setup gives these elements after import (it keeps
    this order unchanged), so the element Jacobians -- and the exact zeros of
    the element matrices -- are the reference's.
    """
    m = int(m)
    n1 = m + 1
    ii, jj, kk = np.meshgrid(np.arange(n1), np.arange(n1), np.arange(n1),
                             indexing="ij")
    ii, jj, kk = (a.transpose(2, 1, 0).reshape(-1) for a in (ii, jj, kk))
    verts = np.stack([ii / m, jj / m, kk / m], axis=1).astype(np.float64)

    ci, cj, ck = np.meshgrid(np.arange(m), np.arange(m), np.arange(m),
                             indexing="ij")
    ci, cj, ck = (a.transpose(2, 1, 0).reshape(-1) for a in (ci, cj, ck))
    corner = np.stack([ci, cj, ck], axis=1)
    stride = np.array([1, n1, n1 * n1])
    elems = np.empty((corner.shape[0], 6, 4), dtype=np.int64)
    for p, perm in enumerate(PERMS):
        pos = corner.copy()
        elems[:, p, 0] = pos @ stride
        for s in range(3):
            pos[:, perm[s]] += 1
            elems[:, p, s + 1] = pos @ stride
    return verts, elems[:, :, [0, 3, 2, 1]].reshape(-1, 4).astype(np.int32)


def write_medit(path, verts, elems):
    """Writes a Medit mesh (Vertices + Tetrahedra, 1-based) with coordinates
    printed to 17 significant digits so they read back bit-exactly."""
    with open(path, "w") as fp:
        fp.write("MeshVersionFormatted 1\nDimension 3\n")
        fp.write("Vertices\n%d\n" % len(verts))
        np.savetxt(fp, np.concatenate([verts, np.zeros((len(verts), 1))], 1),
                   fmt=["%.17g", "%.17g", "%.17g", "%d"])
        fp.write("Tetrahedra\n%d\n" % len(elems))
        np.savetxt(fp, np.concatenate(
            [elems.astype(np.int64) + 1,
             np.ones((len(elems), 1), dtype=np.int64)], 1), fmt="%d")
        fp.write("End\n")


# local edge k of a tetrahedron joins local vertices EDGES[k]; local face k is
# opposite local vertex k (the reference's conventions, lagrange.c P2/P3 bases)
EDGES = ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))
FACES = ((1, 2, 3), (0, 2, 3), (0, 1, 3), (0, 1, 2))


def lagrange_dofs(verts, elems, p):
    """Numbers the DOFs of a continuous Lagrange P`p` space (p = 1, 2, 3) the
    way PHG lays out a DOF object: vertex DOFs first (by vertex index), then
    edge DOFs (p - 1 per edge), then face DOFs (one per face for P3).

    Returns (e2l int32 [nelem, N], bdry uint8 [ndof], nodes float64 [ndof, 3]):
    the vector index of each element basis function (local order: vertices,
    edges -- for P3 the node nearer the edge's first local vertex first --,
    faces), the Dirichlet flag (DOF on a boundary face, i.e. a face that
    belongs to one element), and the Lagrange node of each DOF.  On an edge
    with two DOFs, slot 0 is the node nearer the lower-numbered vertex.
    """
    verts = np.asarray(verts, np.float64)
    elems = np.asarray(elems, np.int64)
    ne, nv = len(elems), len(verts)
    N = {1: 4, 2: 10, 3: 20}[p]
    e2l = np.empty((ne, N), np.int64)
    e2l[:, :4] = elems
    ndof = nv

    # boundary faces: faces owned by exactly one element
    fv = elems[:, FACES].reshape(-1, 3)
    lo, hi = fv.min(axis=1), fv.max(axis=1)
    mid = fv.sum(axis=1) - lo - hi
    fkey = (lo * nv + mid) * nv + hi
    del fv, lo, hi, mid
    fu, finv, fcnt = np.unique(fkey, return_inverse=True, return_counts=True)
    bface = (fcnt == 1)[finv].reshape(ne, 4)

    bdry_v = np.zeros(nv, bool)
    for k in range(4):
        for v in FACES[k]:
            bdry_v[elems[bface[:, k], v]] = True
    nodes = [verts]
    bflags = [bdry_v]

    if p >= 2:
        ev = elems[:, EDGES]                           # ne x 6 x 2
        lo, hi = ev.min(axis=2), ev.max(axis=2)
        ekey = lo * nv + hi
        eu, einv = np.unique(ekey.reshape(-1), return_inverse=True)
        einv = einv.reshape(ne, 6)
        nedge = len(eu)
        elo, ehi = eu // nv, eu % nv
        # an edge is on the boundary iff it lies in a boundary face
        bedge = np.zeros(nedge, bool)
        for k in range(4):
            f = FACES[k]
            for a, b in ((f[0], f[1]), (f[0], f[2]), (f[1], f[2])):
                j = EDGES.index((a, b))
                bedge[einv[bface[:, k], j]] = True
        if p == 2:
            e2l[:, 4:10] = ndof + einv
            nodes.append(0.5 * (verts[elo] + verts[ehi]))
            bflags.append(bedge)
            ndof += nedge
        else:
            first_is_low = ev[:, :, 0] < ev[:, :, 1]       # local first vertex is the lower one
            slot_a = np.where(first_is_low, 0, 1)
            e2l[:, 4:16:2] = ndof + 2 * einv + slot_a
            e2l[:, 5:16:2] = ndof + 2 * einv + (1 - slot_a)
            enodes = np.empty((2 * nedge, 3))
            enodes[0::2] = (2.0 * verts[elo] + verts[ehi]) / 3.0
            enodes[1::2] = (verts[elo] + 2.0 * verts[ehi]) / 3.0
            nodes.append(enodes)
            bflags.append(np.repeat(bedge, 2))
            ndof += 2 * nedge
    if p == 3:
        e2l[:, 16:20] = ndof + finv.reshape(ne, 4)
        fa, fb, fc = fu // (nv * nv), (fu // nv) % nv, fu % nv
        nodes.append((verts[fa] + verts[fb] + verts[fc]) / 3.0)
        bflags.append(fcnt == 1)
        ndof += len(fu)
    return (e2l.astype(np.int32), np.concatenate(bflags).astype(np.uint8),
            np.concatenate(nodes))


def sine_source(nodes):
    """f = 3 pi^2 sin(pi x) sin(pi y) sin(pi z) at the given nodes; the exact
    solution of -Laplace u = f with u = 0 on the unit cube's boundary is
    sin(pi x) sin(pi y) sin(pi z)."""
    x, y, z = nodes[:, 0], nodes[:, 1], nodes[:, 2]
    return 3.0 * np.pi ** 2 * np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)
