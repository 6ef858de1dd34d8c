"""The generated reference tables agree with the oracle's independent basis."""
import numpy as np
import pytest

import gen_tables
import oracle as orc


@pytest.fixture(scope="module")
def tables():
    return gen_tables.build()


@pytest.mark.parametrize("p", [1, 2, 3])
def test_gradient_matrix(tables, p):
    d = tables[p]
    qnodes = [np.array([0.25, 0.25, 0.25])] if p == 1 else [
        np.array([float(x) for x in gen_tables.node_pos(a, p - 1)]) for a in gen_tables.nodes(p - 1)]
    D = np.array([[[float(x) for x in row] for row in Da] for Da in d["D"]])
    for m, xq in enumerate(qnodes):
        _, g = orc.basis(p, xq)
        for a in range(3):
            assert np.allclose(D[a, m], g[:, a], atol=1e-13)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_nodes_are_lagrange(tables, p):
    for i, x in enumerate(tables[p]["NODES"]):
        v, _ = orc.basis(p, np.array([float(c) for c in x]))
        e = np.zeros(len(v))
        e[i] = 1
        assert np.allclose(v, e, atol=1e-13)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_mass_matrices(tables, p):
    """MP equals the oracle-quadrature mass matrix on the reference tet."""
    x = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float64)
    a = orc.Oracle(x, np.array([[0, 1, 2, 3]], np.int32), p, orc.HELMHOLTZ, mass=1.0, n_components=1)
    b = orc.Oracle(x, np.array([[0, 1, 2, 3]], np.int32), p, orc.HELMHOLTZ, mass=0.0, n_components=1)
    M = a.cell_matrix(0) - b.cell_matrix(0)
    MP = np.array([[float(v) for v in r] for r in tables[p]["MP"]])
    assert np.allclose(M, MP, atol=1e-14)


@pytest.mark.parametrize("p", [2, 3])
def test_embedding_reproduces_coarse_basis(tables, p):
    EMB = np.array([[float(v) for v in r] for r in tables[p]["EMB"]])
    rng = np.random.default_rng(0)
    coarse = rng.uniform(-1, 1, EMB.shape[1])
    fine = EMB @ coarse
    for x in rng.uniform(0, 0.3, (5, 3)):
        vc, _ = orc.basis(p - 1, x)
        vf, _ = orc.basis(p, x)
        assert abs(vc @ coarse - vf @ fine) < 1e-13


@pytest.mark.parametrize("p", [2, 3])
def test_gradient_matrices_are_vertex_permutations_of_one(tables, p):
    """D_a[m][i] = D_0[q(m)][p(i)]: swapping reference vertices 1 and a+1
    (barycentric lattice components 1 and a+1) maps the x_0 derivative onto
    the x_a derivative, and permutes the P_p and P_{p-1} nodes (p, q).  This
    is the symmetry a per-direction split of the cell term relies on."""
    d, dq = tables[p], tables[p - 1]
    lat, latq = [tuple(x) for x in d["LATTICE"]], [tuple(x) for x in dq["LATTICE"]]
    D = [[[float(x) for x in row] for row in Da] for Da in d["D"]]

    def swap(t, a):
        t = list(t)
        t[1], t[a + 1] = t[a + 1], t[1]
        return tuple(t)

    for a in (1, 2):
        perm = [lat.index(swap(x, a)) for x in lat]
        permq = [latq.index(swap(x, a)) for x in latq]
        for m in range(d["KQ"]):
            for i in range(d["K"]):
                assert D[a][m][i] == D[0][permq[m]][perm[i]]


@pytest.mark.parametrize("p", [1, 2, 3])
def test_face_node_lists_lie_on_faces(tables, p):
    lat = tables[p]["LATTICE"]
    for f in range(4):
        for n in tables[p]["FN"][f]:
            assert lat[n][f] == 0
        assert len(tables[p]["FN"][f]) == (p + 1) * (p + 2) // 2


def test_mlp_oracle_gradient_is_the_derivative():
    """Pin of the MLP oracle: its gradient matches central finite differences."""
    import mlp_oracle
    rng = np.random.default_rng(0)
    w = (rng.standard_normal(mlp_oracle.NPARAM) * 0.2).astype(np.float32)
    w = mlp_oracle.bf16_round(w)  # exactly representable, so rounding is the identity
    X = rng.standard_normal((8, 29))
    Y = rng.standard_normal((8, 20))
    _, g = mlp_oracle.loss_and_grad(w, X, Y)
    for i in rng.choice(mlp_oracle.NPARAM, 12, replace=False):
        # step of one bf16 ulp pair around w[i] keeps the rounded weights exact
        wp, wm = w.copy(), w.copy()
        h = max(abs(float(w[i])), 1e-3) * 2 ** -7
        wp[i] = mlp_oracle.bf16_round(np.array([w[i] + h], np.float32))[0]
        wm[i] = mlp_oracle.bf16_round(np.array([w[i] - h], np.float32))[0]
        lp, _ = mlp_oracle.loss_and_grad(wp, X, Y)
        lm, _ = mlp_oracle.loss_and_grad(wm, X, Y)
        fd = (lp - lm) / (float(wp[i]) - float(wm[i]))
        assert abs(fd - g[i]) <= 2e-2 * max(1e-3, abs(g[i])) + 1e-6, (i, fd, g[i])
