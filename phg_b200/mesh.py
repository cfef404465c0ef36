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
    6 tetrahedra in PERMS order, vertices ordered along the walk.
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
    return verts, elems.reshape(-1, 4).astype(np.int32)


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
