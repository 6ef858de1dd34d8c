"""The C ABI library loads, exports every declared symbol, and its host-only
entry points behave (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

import simplexfem as sf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"^\s*(?:int|const char\*|int64_t|void)\s+(fem_\w+)\s*\(", txt, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = sf.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    bound = {p[0] for p in sf._PROTOS}
    assert set(declared_symbols()) <= bound | {"fem_vector_alloc", "fem_vector_free"}


def test_version_and_errors():
    lib = sf.lib()
    a, b = ctypes.c_int32(), ctypes.c_int32()
    assert lib.fem_version(ctypes.byref(a), ctypes.byref(b)) == 0
    assert lib.fem_version(None, None) == sf.FEM_OK + 1  # FEM_ERR_ARG
    assert b"NULL" in lib.fem_last_error_string()


def test_bad_mesh_rejected():
    with pytest.raises(sf.FemError) as e:
        sf.Mesh(0)
    assert e.value.code == 1


def test_bad_degree_rejected_before_device_work():
    m = sf.Mesh(2)
    with pytest.raises(sf.FemError) as e:
        sf.Operator(m, 4, "cg")
    assert e.value.code == 1


@pytest.mark.parametrize("n", [1, 2, 5])
def test_mesh_counts(n):
    m = sf.Mesh(n, jitter=0.1, seed=0)
    assert m.n_cells == 6 * n ** 3
    assert m.n_vertices == (n + 1) ** 3
    assert m.n_boundary_faces == 12 * n * n
    assert 2 * m.n_interior_faces + m.n_boundary_faces == 4 * m.n_cells
    cells = m.cells()
    assert np.all(np.diff(cells, axis=1) > 0)  # sorted local vertices


def test_config_sizes():
    """Exact DoF counts of the benchmark meshes (Kuhn 6 tets per hex)."""
    m16 = sf.Mesh(16)
    _, cm = m16.cg_dofs(2)
    assert len(cm) == 35937
    assert m16.n_cells == 24576
    m32 = sf.Mesh(32)
    assert m32.n_cells == 196608 and 20 * m32.n_cells == 3932160
    assert m32.n_interior_faces == 387072 and m32.n_boundary_faces == 12288


def test_neighbors_symmetric():
    m = sf.Mesh(3, jitter=0.1, seed=1)
    nb, nbf = m.neighbors()
    for c in range(m.n_cells):
        for f in range(4):
            if nb[c, f] >= 0:
                assert nb[nb[c, f], nbf[c, f]] == c
                assert nbf[nb[c, f], nbf[c, f]] == f


def test_jitter_is_seeded_and_bounded():
    a = sf.Mesh(4, jitter=0.1, seed=0).vertices()
    b = sf.Mesh(4, jitter=0.1, seed=0).vertices()
    c = sf.Mesh(4, jitter=0.1, seed=1).vertices()
    z = sf.Mesh(4).vertices()
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.abs(a - z).max() <= 0.1 * 0.25 + 1e-15
