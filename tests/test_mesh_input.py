"""Unstructured meshes from arrays and from legacy VTK files (host only).

The reference reads its meshes with GridIn::read_vtk and reorders them with
SparsityTools::reorder_hierarchical (CG/cells_batched/application.cc:
1696-1757).  fem_mesh_create_from_arrays / fem_mesh_read_vtk take any tet
mesh, sort every cell's vertices, put the cells in Morton order of their
centroids and rebuild the face adjacency.  Checked here against the Kuhn
generator's own mesh after relabelling vertices, permuting each cell's
vertices and shuffling the cells.
"""
import numpy as np
import pytest

import simplexfem as sf


def write_vtk(path, x, cells, cell_type=10):
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 3.0\ntest mesh\nASCII\nDATASET UNSTRUCTURED_GRID\n")
        f.write(f"POINTS {len(x)} double\n")
        for p in x:
            f.write(" ".join(f"{float(v):.17g}" for v in p) + "\n")
        f.write(f"CELLS {len(cells)} {5 * len(cells)}\n")
        for c in cells:
            f.write("4 " + " ".join(str(int(v)) for v in c) + "\n")
        f.write(f"CELL_TYPES {len(cells)}\n")
        f.write("\n".join(str(cell_type) for _ in cells) + "\n")
        f.write(f"CELL_DATA {len(cells)}\nSCALARS material int 1\nLOOKUP_TABLE default\n")
        f.write("\n".join("0" for _ in cells) + "\n")


def scrambled(mesh, seed=0):
    """The mesh with vertices relabelled, cells shuffled and each cell's
    vertices permuted; returns (x, cells, cell permutation)."""
    rng = np.random.default_rng(seed)
    x, cells = mesh.vertices(), mesh.cells()
    relabel = rng.permutation(len(x))            # old vertex -> new vertex
    x2 = np.empty_like(x)
    x2[relabel] = x
    perm = rng.permutation(len(cells))           # new cell i = old cell perm[i]
    c2 = relabel[cells[perm]]
    for row in c2:
        rng.shuffle(row)
    return x2, c2.astype(np.int32), perm


def cell_keys(x, cells):
    """Cells as sorted tuples of rounded vertex coordinates (label-free)."""
    pts = np.round(x[cells], 12)
    return sorted(tuple(sorted(map(tuple, p))) for p in pts)


@pytest.mark.parametrize("reorder", [True, False])
def test_mesh_from_arrays_equals_the_same_mesh(reorder):
    m0 = sf.Mesh((5, 4, 6), jitter=0.1, seed=3)
    x2, c2, perm = scrambled(m0)
    m = sf.Mesh.from_arrays(x2, c2, reorder=reorder)
    assert (m.n_cells, m.n_vertices) == (m0.n_cells, m0.n_vertices)
    assert (m.n_interior_faces, m.n_boundary_faces) == (m0.n_interior_faces, m0.n_boundary_faces)
    cells = m.cells()
    assert np.all(np.diff(cells, axis=1) > 0)
    assert cell_keys(m.vertices(), cells) == cell_keys(m0.vertices(), m0.cells())
    inp = m.input_cells()
    assert np.array_equal(np.sort(cells, axis=1), np.sort(c2[inp], axis=1))
    if not reorder:
        assert np.array_equal(inp, np.arange(m.n_cells))
    # neighbours are symmetric and share three vertices
    nb, nbf = m.neighbors()
    for c in range(m.n_cells):
        for f in range(4):
            o = nb[c, f]
            if o >= 0:
                assert nb[o, nbf[c, f]] == c
                assert len(set(cells[c]) & set(cells[o])) == 3


def test_morton_reorder_gives_locality():
    """After the hierarchical reorder consecutive cells are close: the mean
    centroid distance of neighbours in the cell order is a small multiple of
    the mesh size, unlike the shuffled input order."""
    m0 = sf.Mesh(8, jitter=0.1, seed=1)
    x2, c2, _ = scrambled(m0, seed=2)
    m = sf.Mesh.from_arrays(x2, c2, reorder=True)
    cen = m.vertices()[m.cells()].mean(axis=1)
    d_reordered = np.linalg.norm(np.diff(cen, axis=0), axis=1).mean()
    cen_in = x2[c2].mean(axis=1)
    d_input = np.linalg.norm(np.diff(cen_in, axis=0), axis=1).mean()
    assert d_reordered < 0.25 * d_input and d_reordered < 2.0 / 8


def test_read_vtk(tmp_path):
    m0 = sf.Mesh((4, 3, 5), jitter=0.1, seed=7)
    x2, c2, _ = scrambled(m0, seed=5)
    p = tmp_path / "mesh.vtk"
    write_vtk(p, x2, c2)
    m = sf.Mesh.read_vtk(p)
    assert cell_keys(m.vertices(), m.cells()) == cell_keys(m0.vertices(), m0.cells())
    assert (m.n_interior_faces, m.n_boundary_faces) == (m0.n_interior_faces, m0.n_boundary_faces)


def test_bad_meshes_are_rejected(tmp_path):
    x = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1], [0.3, 0.3, -1.0]], float)
    with pytest.raises(sf.FemError) as e:
        sf.Mesh.from_arrays(x, [[0, 1, 2, 9]])
    assert e.value.code == sf.FEM_ERR_ARG
    with pytest.raises(sf.FemError):
        sf.Mesh.from_arrays(x, [[0, 1, 2, 2]])
    with pytest.raises(sf.FemError):  # flat cell
        sf.Mesh.from_arrays(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], float), [[0, 1, 2, 3]])
    with pytest.raises(sf.FemError):  # three cells on face (0,1,2)
        sf.Mesh.from_arrays(np.vstack([x, [[0.2, 0.2, 2.0]]]), [[0, 1, 2, 3], [0, 1, 2, 5], [0, 1, 2, 6]])
    p = tmp_path / "hex.vtk"
    write_vtk(p, x, [[0, 1, 2, 3]], cell_type=12)
    with pytest.raises(sf.FemError):
        sf.Mesh.read_vtk(p)
    with pytest.raises(sf.FemError):
        sf.Mesh.read_vtk(tmp_path / "missing.vtk")
