#!/usr/bin/env python3
"""Write tests/golden/element_matrices.json: exact element matrices.

The reference ships no golden vectors (no test directory; its only checks are
printed self-consistency norms, CG/cells_batched/application.cc:1937-1940).
These fixtures pin the oracle's basis, geometry and quadrature instead: the
P1-P3 Lagrange stiffness and mass matrices of two tetrahedra with rational
vertices, computed here in exact rational arithmetic by an independent route
(monomial Vandermonde inverse, exact monomial integrals on the reference tet,
affine pull-back K_ij = |det J| sum_ab (J^-1 J^-T)_ab int d_a phi_i d_b phi_j).

Node convention (the library's DoF format): vertices; edges (0,1),(0,2),(0,3),
(1,2),(1,3),(2,3) walked from the lower local vertex, p-1 nodes each; for P3
one node per face f = 0..3 (face f opposite vertex f).
"""
from fractions import Fraction as F
import json
import math
import os

TETS = {
    "reference": [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)],
    "skewed": [(F(0), F(0), F(0)), (F(1, 2), F(1, 8), F(0)), (F(1, 5), F(2, 3), F(1, 7)),
               (F(1, 9), F(1, 4), F(3, 4))],
}


def lattice(p):
    edges = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    out = []
    for i in range(4):
        a = [0] * 4
        a[i] = p
        out.append(a)
    for (i, j) in edges:
        for m in range(1, p):
            a = [0] * 4
            a[i], a[j] = p - m, m
            out.append(a)
    if p == 3:
        for f in range(4):
            out.append([0 if v == f else 1 for v in range(4)])
    return out


def monos(p):
    return [(a, b, c) for a in range(p + 1) for b in range(p + 1 - a) for c in range(p + 1 - a - b)]


def inverse(M):
    n = len(M)
    A = [[F(x) for x in row] + [F(int(i == j)) for j in range(n)] for i, row in enumerate(M)]
    for c in range(n):
        r = next(r for r in range(c, n) if A[r][c] != 0)
        A[c], A[r] = A[r], A[c]
        pv = A[c][c]
        A[c] = [x / pv for x in A[c]]
        for r in range(n):
            if r != c and A[r][c] != 0:
                f = A[r][c]
                A[r] = [x - f * y for x, y in zip(A[r], A[c])]
    return [row[n:] for row in A]


def basis(p):
    """phi_k as dict monomial -> coefficient."""
    L = lattice(p)
    ms = monos(p)
    V = [[F(l[1], p) ** m[0] * F(l[2], p) ** m[1] * F(l[3], p) ** m[2] for m in ms] for l in L]
    Vi = inverse(V)
    return [{ms[m]: Vi[m][k] for m in range(len(ms)) if Vi[m][k] != 0} for k in range(len(L))]


def deriv(poly, a):
    out = {}
    for m, c in poly.items():
        if m[a]:
            mm = list(m)
            mm[a] -= 1
            out[tuple(mm)] = out.get(tuple(mm), 0) + c * m[a]
    return out


def integral(p1, p2):
    s = F(0)
    for m1, c1 in p1.items():
        for m2, c2 in p2.items():
            i, j, k = (m1[0] + m2[0], m1[1] + m2[1], m1[2] + m2[2])
            s += c1 * c2 * F(math.factorial(i) * math.factorial(j) * math.factorial(k),
                             math.factorial(i + j + k + 3))
    return s


def element(p, verts):
    v = [[F(x) for x in vv] for vv in verts]
    J = [[v[j + 1][i] - v[0][i] for j in range(3)] for i in range(3)]
    det = (J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0])
           + J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]))
    Ji = inverse(J)
    Gm = [[sum(Ji[a][c] * Ji[b][c] for c in range(3)) for b in range(3)] for a in range(3)]
    B = basis(p)
    dB = [[deriv(phi, a) for a in range(3)] for phi in B]
    K = len(B)
    stiff = [[abs(det) * sum(Gm[a][b] * integral(dB[i][a], dB[j][b]) for a in range(3) for b in range(3))
              for j in range(K)] for i in range(K)]
    mass = [[abs(det) * integral(B[i], B[j]) for j in range(K)] for i in range(K)]
    return stiff, mass


def main():
    out = {"tets": {k: [[float(x) for x in v] for v in vs] for k, vs in TETS.items()}, "matrices": {}}
    for name, verts in TETS.items():
        for p in (1, 2, 3):
            s, m = element(p, verts)
            out["matrices"][f"{name}/P{p}"] = {"stiffness": [[float(x) for x in r] for r in s],
                                               "mass": [[float(x) for x in r] for r in m]}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "element_matrices.json")
    with open(path, "w") as fh:
        json.dump(out, fh)
    print("wrote", path)


if __name__ == "__main__":
    main()
