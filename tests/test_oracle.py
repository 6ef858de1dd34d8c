"""Pins of the CPU oracle (no GPU): golden element matrices and known answers."""
import json
import os

import numpy as np
import pytest

import oracle as orc
import simplexfem as sf
from util import dg_interpolate

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "element_matrices.json")


def single_tet_oracle(verts, p, kind, mass=0.0):
    x = np.array(verts, np.float64)
    cells = np.array([[0, 1, 2, 3]], np.int32)
    K = (p + 1) * (p + 2) * (p + 3) // 6
    if kind == orc.CG:
        return orc.Oracle(x, cells, p, orc.CG, cell_dofs=np.arange(K, dtype=np.int32)[None, :],
                          constrained=np.zeros(K, np.uint8))
    return orc.Oracle(x, cells, p, kind, mass=mass)


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("tet", ["reference", "skewed"])
def test_golden_stiffness(p, tet):
    g = json.load(open(GOLDEN))
    ref = np.array(g["matrices"][f"{tet}/P{p}"]["stiffness"])
    o = single_tet_oracle(g["tets"][tet], p, orc.CG)
    M = o.cell_matrix(0)
    assert np.abs(M - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("tet", ["reference", "skewed"])
def test_golden_mass(p, tet):
    g = json.load(open(GOLDEN))
    ref = np.array(g["matrices"][f"{tet}/P{p}"]["mass"])
    a = single_tet_oracle(g["tets"][tet], p, orc.HELMHOLTZ, mass=3.0).cell_matrix(0)
    b = single_tet_oracle(g["tets"][tet], p, orc.HELMHOLTZ, mass=0.0).cell_matrix(0)
    M = (a - b)[: len(ref), : len(ref)] / 3.0
    assert np.abs(M - ref).max() <= 1e-13 * np.abs(ref).max()


def test_kuhn_p1_stencil_is_seven_point():
    """P1 on the unjittered Kuhn mesh: h * (6, -1 x 6 axis neighbours, 0 elsewhere)."""
    n, h = 4, 0.25
    m = sf.Mesh(n)
    o = orc.for_mesh(m, 1, orc.CG)
    cd, cm = m.cg_dofs(1)
    pos = np.zeros((len(cm), 3))
    xv, cells = m.vertices(), m.cells()
    for c in range(m.n_cells):
        pos[cd[c]] = xv[cells[c]]
    v = int(np.argmin(((pos - 0.5) ** 2).sum(1)))
    e = np.zeros(len(cm))
    e[v] = 1
    y = o.vmult(e)
    offs = np.round((pos - pos[v]) / h).astype(int)
    for i in range(len(cm)):
        d = tuple(offs[i])
        if d == (0, 0, 0):
            want = 6 * h
        elif sorted(map(abs, d)) == [0, 0, 1]:
            want = -h
        else:
            want = 0.0
        assert abs(y[i] - want) < 1e-13, (d, y[i])


@pytest.mark.parametrize("p", [1, 2, 3])
def test_cg_numbering_consistent(p):
    m = sf.Mesh((3, 4, 2), jitter=0.1, seed=5)
    assert orc.for_mesh(m, p, orc.CG).check_cg_numbering(m.lo, m.hi) == 0


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("kind", [orc.CG, orc.DG, orc.HELMHOLTZ])
def test_two_quadrature_rules_agree(p, kind):
    m = sf.Mesh(3, jitter=0.1, seed=0)
    kw = dict(n_components=3 if kind == orc.HELMHOLTZ else 1)
    a = orc.for_mesh(m, p, kind, quad_points=p + 2, **kw)
    b = orc.for_mesh(m, p, kind, quad_points=p + 4, **kw)
    x = np.random.default_rng(1).uniform(-1, 1, a.n)
    ya, yb = a.vmult(x), b.vmult(x)
    assert np.linalg.norm(ya - yb) <= 1e-13 * np.linalg.norm(yb)


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("kind", [orc.CG, orc.DG, orc.HELMHOLTZ])
def test_symmetric_positive(p, kind):
    m = sf.Mesh(3, jitter=0.1, seed=0)
    o = orc.for_mesh(m, p, kind, n_components=3 if kind == orc.HELMHOLTZ else 1)
    rng = np.random.default_rng(2)
    x, y = rng.uniform(-1, 1, o.n), rng.uniform(-1, 1, o.n)
    ax, ay = o.vmult(x), o.vmult(y)
    assert abs(y @ ax - x @ ay) <= 1e-12 * abs(y @ ax)
    assert x @ ax > 0


@pytest.mark.parametrize("p", [1, 2, 3])
def test_dg_annihilates_linears_inside(p):
    m = sf.Mesh(4, jitter=0.1, seed=0)
    o = orc.for_mesh(m, p, orc.DG)
    u = dg_interpolate(m, p, lambda X: 1.0 + 2 * X[:, 0] - 3 * X[:, 1] + 0.5 * X[:, 2])
    y = o.vmult(u).reshape(m.n_cells, -1)
    nb, _ = m.neighbors()
    inner = np.all(nb >= 0, axis=1)
    assert np.abs(y[inner]).max() < 1e-12 * np.abs(y).max()


def test_cg_diagonal_matches_unit_vectors():
    m = sf.Mesh(2, jitter=0.1, seed=3)
    o = orc.for_mesh(m, 2, orc.CG)
    d = o.diagonal()
    for i in range(0, o.n, 7):
        e = np.zeros(o.n)
        e[i] = 1
        assert abs(o.vmult(e)[i] - d[i]) < 1e-13 * max(1.0, abs(d[i]))


@pytest.mark.parametrize("p,order", [(2, "ph"), (3, "hp")])
def test_mg_oracle_converges_mesh_independently(p, order):
    """The CPU multigrid oracle itself: few PCG iterations, independent of h."""
    import mg_oracle as mgo
    its = []
    for n in (4, 8):
        M = mgo.MGOracle(lambda k: sf.Mesh(k), n, p, order=order, coarse_n=2)
        top = M.levels[-1]
        b = np.random.default_rng(3).uniform(-1, 1, top.n)
        b[top.cm.astype(bool)] = 0
        x, it = mgo.pcg(lambda v: top.A @ v, b, M.vcycle, 1e-8, 100)
        assert np.linalg.norm(b - top.A @ x) <= 1e-8 * np.linalg.norm(b)
        its.append(it)
    assert max(its) <= 12 and abs(its[0] - its[1]) <= 2, its


def test_dg_mg_oracle_levels_and_convergence():
    """The probed DG level matrix equals the oracle's DG vmult and is symmetric;
    the DG p/c/h multigrid oracle (phc) converges far faster than Jacobi."""
    import mg_oracle as mgo
    mesh = sf.Mesh(3, jitter=0.1, seed=1)
    L = mgo.DGLevel(mesh, 2)
    o = orc.for_mesh(mesh, 2, orc.DG)
    x = np.random.default_rng(0).uniform(-1, 1, L.n)
    assert np.linalg.norm(L.A @ x - o.vmult(x)) <= 1e-13 * np.linalg.norm(o.vmult(x))
    assert abs(L.A - L.A.T).max() <= 1e-13 * abs(L.A).max()
    M = mgo.DGMGOracle(lambda k: sf.Mesh(k), 4, 2, c_transfer=0, coarse_n=2)
    assert [type(l).__name__ for l in M.levels] == ["Level", "Level", "DGLevel", "DGLevel"]
    top = M.levels[-1]
    b = np.random.default_rng(5).uniform(-1, 1, top.n)
    _, its_mg = mgo.pcg(lambda v: top.A @ v, b, M.vcycle, 1e-8, 100)
    _, its_j = mgo.pcg(lambda v: top.A @ v, b, lambda r: top.invd * r, 1e-8, 2000)
    assert its_mg < 30 and its_mg * 5 < its_j, (its_mg, its_j)
