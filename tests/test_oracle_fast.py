"""The optimized CPU restatement (oracle/fast.cpp) against the scalar oracle.

fast.cpp restates the reference's hand-optimised vmult (SIMD cell batches,
batched dense shape-matrix products, face groups by local face numbers,
thread partitions with shared-entry buffers) and is timed as the CPU
baseline.  It must give the scalar oracle's operator to rounding, for every
kind and degree, for any number of threads (the shared-DoF and shared-cell
buffers at partition boundaries), on the mesh both build from
oracle.KuhnMesh.  Host only.
"""
import numpy as np
import pytest

import fast
import oracle as orc
from util import rel_l2

CASES = [(orc.CG, 1, 1), (orc.CG, 2, 1), (orc.CG, 3, 1), (orc.DG, 1, 1), (orc.DG, 2, 1), (orc.DG, 3, 1),
         (orc.HELMHOLTZ, 1, 3), (orc.HELMHOLTZ, 2, 3), (orc.HELMHOLTZ, 2, 1)]


@pytest.mark.parametrize("threads", [1, 3, 8])
@pytest.mark.parametrize("kind,p,nc", CASES)
def test_fast_port_equals_oracle(kind, p, nc, threads):
    mesh = orc.KuhnMesh((6, 5, 7), jitter=0.1, seed=3)
    o = orc.for_mesh(mesh, p, kind, n_components=nc)
    f = fast.FastOperator(mesh, p, kind, n_components=nc, n_threads=threads)
    assert f.n == o.n and f.threads == threads
    x = np.random.default_rng(5).uniform(-1, 1, o.n)
    if kind == orc.CG:
        cm = mesh.cg_dofs(p)[1].astype(bool)
        x[cm] = 0.0
    y = f.vmult(x)
    assert rel_l2(y, o.vmult(x)) <= 1e-13
    if kind == orc.CG:
        assert np.array_equal(y[cm], x[cm])


def test_fast_port_penalty_square_and_repeat():
    mesh = orc.KuhnMesh(4, jitter=0.1, seed=0)
    o = orc.for_mesh(mesh, 3, orc.DG, penalty=1)
    f = fast.FastOperator(mesh, 3, orc.DG, penalty=1)
    x = np.random.default_rng(1).uniform(-1, 1, o.n)
    y1 = f.vmult(x)
    y2 = f.vmult(x, np.full(f.n, np.nan))
    assert np.array_equal(y1, y2)
    assert rel_l2(y1, o.vmult(x)) <= 1e-13


def test_fast_port_rules_are_small():
    """The quadrature the port runs is no larger than the reference's
    QGaussSimplex(p+1): 14 cell and 12 face points for DG P3."""
    f = fast.FastOperator(orc.KuhnMesh(2), 3, orc.DG)
    assert (f.n_cell_points, f.n_face_points, f.lanes) == (14, 12, 8)


@pytest.mark.parametrize("p", [2, 3])
def test_fast_multigrid_equals_assembled_oracle(p):
    """The matrix-free CPU multigrid (oracle/fast_mg.py, the timed CPU solve
    baseline) gives the same V-cycle as the assembled restatement
    (mg_oracle.MGOracle) and the same MG-CG iteration count to 1e-8."""
    import torch
    import fast_mg
    import mg_oracle
    mg = fast_mg.FastMG(8, p)
    mo = mg_oracle.MGOracle(lambda k: orc.KuhnMesh(k), 8, p)
    L = mg.levels[-1]
    b = np.random.default_rng(5).uniform(-1, 1, L.n)
    b[L.constrained.numpy()] = 0.0
    z = mg.vcycle(torch.from_numpy(b.copy())).numpy()
    assert rel_l2(z, mo.vcycle(b)) <= 1e-12
    _, its = mg.solve(torch.from_numpy(b.copy()), rtol=1e-8)
    A = mo.levels[-1].A
    _, its_ref = mg_oracle.pcg(lambda v: A @ v, b, mo.vcycle, 1e-8, 100)
    assert its == its_ref
