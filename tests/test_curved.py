"""Curvilinear meshes (fem_mesh_curve) on the host and in the oracle.

The reference keeps per-quadrature-point Jacobians for non-affine cells
(CG/cells_batched/application.cc:1361-1376).  fem_mesh_curve moves the mesh
by a smooth bump that keeps the box boundary and gives every cell a
quadratic geometry; the checks here pin that map and the oracle's curved
cell integrals (no GPU).
"""
import numpy as np
import pytest

import oracle as orc
import simplexfem as sf


def bump(x, a):
    return x + a * np.prod(np.sin(np.pi * x), axis=-1, keepdims=True)


def test_curve_moves_vertices_and_edge_nodes():
    m = sf.Mesh((4, 5, 3), jitter=0.1, seed=2)
    x0, cells = m.vertices().copy(), m.cells()
    m.curve(0.08)
    assert np.allclose(m.vertices(), bump(x0, 0.08), atol=1e-15, rtol=0)
    edges = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    mid = np.stack([0.5 * (x0[cells[:, a]] + x0[cells[:, b]]) for a, b in edges], axis=1)
    assert np.allclose(m.edge_nodes(), bump(mid, 0.08), atol=1e-15, rtol=0)
    with pytest.raises(sf.FemError):
        m.curve(0.08)  # already curved
    with pytest.raises(sf.FemError):
        sf.Mesh(2).curve(0.9)


def test_curved_meshes_reject_what_needs_affine_cells():
    m = sf.Mesh(2).curve(0.05)
    with pytest.raises(sf.FemError):
        sf.Partition(m, 2, "cg", 2, 0)


def _curved_oracle(m, p, quad_points):
    cd, cm = m.cg_dofs(p)
    o = orc.Oracle(m.vertices(), m.cells(), p, orc.CG, cell_dofs=cd, constrained=cm, quad_points=quad_points)
    o.set_p2_geometry(m.edge_nodes())
    return o, cm.astype(bool)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_oracle_curved_cells(p):
    """Straight edge nodes give the affine operator; on curved cells the
    operator stays symmetric and annihilates constants away from the
    boundary."""
    m = sf.Mesh(3, jitter=0.1, seed=5)
    flat = sf.Mesh(3, jitter=0.1, seed=5).curve(0.0)
    o_aff = orc.for_mesh(m, p, orc.CG, quad_points=p + 1)
    o_flat, cm = _curved_oracle(flat, p, p + 1)
    x = np.random.default_rng(2).uniform(-1, 1, o_aff.n)
    x[cm] = 0
    y_aff = o_aff.vmult(x)
    assert np.linalg.norm(o_flat.vmult(x) - y_aff) <= 1e-13 * np.linalg.norm(y_aff)
    mc = sf.Mesh(4, jitter=0.1, seed=5).curve(0.1)
    oc, cm = _curved_oracle(mc, p, p + 1)
    A = np.stack([oc.vmult(e) for e in np.eye(oc.n)], axis=1)
    assert np.abs(A - A.T).max() <= 1e-13 * np.abs(A).max()
    flat4 = orc.for_mesh(sf.Mesh(4, jitter=0.1, seed=5), p, orc.CG, quad_points=p + 1)
    assert np.linalg.norm(A - np.stack([flat4.vmult(e) for e in np.eye(oc.n)], axis=1)) > 1e-3 * np.abs(A).max()
    cd, _ = mc.cg_dofs(p)
    near = np.zeros(oc.n, bool)
    near[np.unique(cd[np.any(cm[cd], axis=1)])] = True
    inner = ~near
    assert np.abs((A @ np.ones(oc.n))[inner]).max() <= 1e-12 * np.abs(A).max()
