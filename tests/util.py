"""Helpers shared by the tests: seeded inputs and error norms."""
import numpy as np


def seeded_src(n, seed, constrained=None):
    """src ~ U[-1,1] from numpy's PCG64(seed); zero at constrained DoFs."""
    x = np.random.default_rng(seed).uniform(-1.0, 1.0, n)
    if constrained is not None:
        x[constrained.astype(bool)] = 0.0
    return x


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def dg_nodes(p):
    """Lattice of the P_p nodes in the library's cell order (barycentric / p)."""
    edges = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    lat = []
    for i in range(4):
        a = [0] * 4
        a[i] = p
        lat.append(a)
    for (i, j) in edges:
        for m in range(1, p):
            a = [0] * 4
            a[i], a[j] = p - m, m
            lat.append(a)
    if p == 3:
        for f in range(4):
            lat.append([0 if v == f else 1 for v in range(4)])
    return np.array(lat, np.float64) / p


def dg_interpolate(mesh, p, fn, n_components=1):
    """Nodal DG interpolant [cell][comp][k] of fn(points)->(n,) per component."""
    L = dg_nodes(p)
    xv, cells = mesh.vertices(), mesh.cells()
    pts = np.einsum("kv,cvd->ckd", L, xv[cells])  # [cell][k][3]
    vals = fn(pts.reshape(-1, 3)).reshape(len(cells), len(L))
    return np.repeat(vals[:, None, :], n_components, axis=1).reshape(-1)
