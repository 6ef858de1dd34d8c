"""The oracle's own mesh generator (oracle/mesh.c) against the product's.

The oracle restates the benchmark mesh recipe (Kuhn tets, Morton hex order,
sorted cell vertices, MT19937-64 jitter, first-touch CG numbering) without
the product library, so the CPU baseline and the checker never take their
mesh from the code they check.  Both generators must agree bit for bit,
which also pins the product's generator to the recipe.  Host only.
"""
import numpy as np
import pytest

import oracle as orc
import simplexfem as sf

CASES = [((5, 4, 3), 0.1, 0), ((7, 9, 6), 0.2, 12345), ((3, 3, 3), 0.0, 0), ((1, 1, 1), 0.1, 4),
         ((16, 16, 16), 0.1, 0), ((32, 32, 32), 0.1, 0), ((2, 11, 5), 0.1, 2**63 + 17)]


@pytest.mark.parametrize("shape,jitter,seed", CASES)
def test_oracle_mesh_equals_product_mesh(shape, jitter, seed):
    a = sf.Mesh(shape, jitter=jitter, seed=seed)
    b = orc.KuhnMesh(shape, jitter=jitter, seed=seed)
    assert a.n_cells == b.n_cells and a.n_vertices == b.n_vertices
    assert np.array_equal(a.vertices(), b.vertices())
    assert np.array_equal(a.cells(), b.cells())
    for u, v in zip(a.neighbors(), b.neighbors()):
        assert np.array_equal(u, v)
    assert (a.n_interior_faces, a.n_boundary_faces) == (b.n_interior_faces, b.n_boundary_faces)
    if a.n_cells <= 6 * 16**3:
        for p in (1, 2, 3):
            cd, cm = a.cg_dofs(p)
            cd2, cm2 = b.cg_dofs(p)
            assert np.array_equal(cd, cd2) and np.array_equal(cm, cm2), p


def test_oracle_mesh_recipe():
    """Properties the recipe fixes: jittered interior only, within 0.1h, the
    Kuhn count of faces, and positive volumes."""
    m = orc.KuhnMesh(6, jitter=0.1, seed=0)
    x = m.vertices()
    lat = np.stack(np.meshgrid(np.arange(7), np.arange(7), np.arange(7), indexing="ij"), -1)
    lat = lat.transpose(2, 1, 0, 3).reshape(-1, 3) / 6.0   # x fastest
    d = np.abs(x - lat)
    boundary = np.any((lat == 0) | (lat == 1), axis=1)
    assert d[boundary].max() < 1e-15 and 0 < d[~boundary].max() <= 0.1 / 6
    c = m.cells()
    assert np.all(np.diff(c, axis=1) > 0)
    J = x[c[:, 1:]] - x[c[:, :1]]
    assert np.all(np.abs(np.linalg.det(J)) > 0)
    assert m.n_boundary_faces == 2 * 6 * 6 * 6 and m.n_interior_faces == (4 * m.n_cells - 432) // 2
    cd, cm = m.cg_dofs(2)
    assert len(cm) == 13**3 and cm.sum() == 13**3 - 11**3
