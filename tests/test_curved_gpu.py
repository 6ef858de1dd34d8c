"""Curved-cell CG operator (per-quadrature-point metric) against the oracle.

On curved cells the integrand is not a polynomial, so the quadrature is part
of the operator: the GPU operator and the oracle both use the collapsed
Gauss-Legendre rule with p + 1 points per direction.  Tolerances as the other
parity tests: relative l2 <= 1e-12 (FP64), <= 2e-6 (FP32).  With straight
edge nodes the curved path must reproduce the affine operator.
"""
import numpy as np
import pytest

import oracle as orc
import simplexfem as sf
from util import rel_l2, seeded_src

pytestmark = pytest.mark.gpu


def run(op, x):
    import torch
    y = op.initialize_dof_vector()
    op.vmult(y, torch.tensor(x, dtype=op.dtype, device="cuda"))
    torch.cuda.synchronize()
    return y.double().cpu().numpy()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_curved_cg_operator(cuda, p, precision):
    import torch
    mesh = sf.Mesh((6, 5, 7), jitter=0.1, seed=4).curve(0.12)
    op = sf.Operator(mesh, p, "cg", precision)
    cd, cm = mesh.cg_dofs(p)
    o = orc.Oracle(mesh.vertices(), mesh.cells(), p, orc.CG, cell_dofs=cd, constrained=cm, quad_points=p + 1)
    o.set_p2_geometry(mesh.edge_nodes())
    x = seeded_src(op.m(), 3, cm)
    xr = x.astype(np.float32).astype(np.float64) if precision == "fp32" else x
    tol = 1e-12 if precision == "fp64" else 2e-6
    assert rel_l2(run(op, x), o.vmult(xr)) <= tol
    d = op.initialize_dof_vector()
    op.compute_diagonal(d)
    torch.cuda.synchronize()
    assert rel_l2(d.double().cpu().numpy(), o.diagonal()) <= tol


@pytest.mark.parametrize("p", [1, 2, 3])
def test_straight_edge_nodes_give_the_affine_operator(cuda, p):
    flat = sf.Mesh((5, 4, 6), jitter=0.1, seed=8).curve(0.0)
    aff = sf.Mesh((5, 4, 6), jitter=0.1, seed=8)
    a, b = sf.Operator(flat, p, "cg"), sf.Operator(aff, p, "cg")
    x = seeded_src(a.m(), 5, a.constrained())
    assert rel_l2(run(a, x), run(b, x)) <= 1e-13


def test_curved_meshes_need_cg(cuda):
    m = sf.Mesh(2).curve(0.05)
    with pytest.raises(sf.FemError):
        sf.Operator(m, 2, "dg")
    with pytest.raises(sf.FemError):
        sf.Multigrid(sf.Operator(m, 2, "cg"))
