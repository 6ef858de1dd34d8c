#!/usr/bin/env python3
"""Generate fast_rules.h: symmetric positive quadrature rules for the CPU port.

TEST INFRASTRUCTURE ONLY (the CPU baseline).  The reference evaluates its
cell and face integrals with deal.II's QGaussSimplex(p+1) (exact to degree
2p+1).  On affine cells with constant coefficients every integrand of the
operators is a polynomial of degree 2p-2 (Laplace cell term) or 2p (mass and
face terms), so any rule of that exactness gives the same operator.  The CPU
port takes the smallest positive fully symmetric rules of those degrees, so
it does no more quadrature work than the reference's algorithm would:

  tetrahedron  degree 1: 1 point, 2: 4 points, 5: 14 points
  triangle     degree 2: 3 points, 4: 6 points, 6: 12 points

Each rule's orbit parameters are found here by solving its moment equations
(Newton/least squares from rough starting values), then every monomial up to
the rule's degree is checked against its exact integral.  Points are written
in barycentric coordinates, weights normalised to sum 1 (multiply by the
element's measure).
"""
import itertools
import math
import os

import numpy as np
from scipy.optimize import least_squares

HERE = os.path.dirname(os.path.abspath(__file__))


def tet_orbit(kind, a):
    if kind == "S4":
        return [(0.25, 0.25, 0.25, 0.25)]
    if kind == "S31":
        b = 1 - 3 * a
        return sorted(set(itertools.permutations((a, a, a, b))))
    if kind == "S22":
        b = 0.5 - a
        return sorted(set(itertools.permutations((a, a, b, b))))
    raise ValueError(kind)


def tri_orbit(kind, a, c=None):
    if kind == "S3":
        return [(1 / 3, 1 / 3, 1 / 3)]
    if kind == "S21":
        return sorted(set(itertools.permutations((a, a, 1 - 2 * a))))
    if kind == "S111":
        return sorted(set(itertools.permutations((a, c, 1 - a - c))))
    raise ValueError(kind)


def exact_tet(e):
    # integral over the unit tet of x^a y^b z^c divided by its volume 1/6
    a, b, c = e
    return 6.0 * math.factorial(a) * math.factorial(b) * math.factorial(c) / math.factorial(a + b + c + 3)


def exact_tri(e):
    a, b = e
    return 2.0 * math.factorial(a) * math.factorial(b) / math.factorial(a + b + 2)


def monomials(dim, deg):
    return [e for e in itertools.product(range(deg + 1), repeat=dim) if sum(e) <= deg]


def build(orbits, params, weights, tet):
    pts, ws = [], []
    k = 0
    for (kind, npar), w in zip(orbits, weights):
        par = params[k:k + npar]
        k += npar
        orb = (tet_orbit if tet else tri_orbit)(kind, *par) if npar else (tet_orbit if tet else tri_orbit)(kind, 0)
        pts += orb
        ws += [w] * len(orb)
    return np.array(pts), np.array(ws)


def residual(x, orbits, deg, tet):
    npar = sum(n for _, n in orbits)
    pts, ws = build(orbits, x[:npar], x[npar:], tet)
    dim = 3 if tet else 2
    cart = pts[:, 1:]  # barycentric (l0, l1, l2[, l3]) -> cartesian (l1, l2[, l3])
    r = []
    for e in monomials(dim, deg):
        v = np.prod(cart ** np.array(e), axis=1)
        r.append(ws @ v - (exact_tet(e) if tet else exact_tri(e)))
    return np.array(r)


def solve(orbits, deg, tet, guess):
    sol = least_squares(residual, np.array(guess, float), args=(orbits, deg, tet), xtol=1e-15, ftol=1e-15,
                        gtol=1e-15, max_nfev=20000)
    npar = sum(n for _, n in orbits)
    pts, ws = build(orbits, sol.x[:npar], sol.x[npar:], tet)
    res = np.abs(residual(sol.x, orbits, deg, tet)).max()
    assert res < 1e-14, (orbits, res)
    assert np.all(ws > 0) and np.all(pts >= -1e-15), (orbits, ws, pts)
    assert abs(ws.sum() - 1) < 1e-14
    return pts, ws


RULES = {
    # name: (tet?, degree, orbits [(kind, n_params)], starting values [params..., weights...])
    "tet1": (True, 1, [("S4", 0)], [1.0]),
    "tet4": (True, 2, [("S31", 1)], [0.14, 0.25]),
    "tet14": (True, 5, [("S31", 1), ("S31", 1), ("S22", 1)], [0.09, 0.31, 0.045, 0.07, 0.11, 0.04]),
    "tri3": (False, 2, [("S21", 1)], [1 / 6, 1 / 3]),
    "tri6": (False, 4, [("S21", 1), ("S21", 1)], [0.09, 0.44, 0.11, 0.22]),
    "tri12": (False, 6, [("S21", 1), ("S21", 1), ("S111", 2)], [0.063, 0.249, 0.053, 0.31, 0.05, 0.12, 0.08]),
}


def main():
    out = ["// Generated by gen_rules.py: symmetric positive quadrature rules for the CPU",
           "// port (barycentric points, weights summing to 1).  Do not edit.",
           "#pragma once", ""]
    for name, (tet, deg, orbits, guess) in RULES.items():
        pts, ws = solve(orbits, deg, tet, guess)
        n, d = pts.shape
        out.append(f"// {'tetrahedron' if tet else 'triangle'}, exact to degree {deg}")
        out.append(f"static const int kRule_{name}_n = {n};")
        out.append(f"static const double kRule_{name}_pts[{n}][{d}] = {{")
        out += ["  {" + ", ".join(f"{v:.17g}" for v in p) + "}," for p in pts]
        out.append("};")
        out.append(f"static const double kRule_{name}_w[{n}] = {{")
        out.append("  " + ", ".join(f"{w:.17g}" for w in ws))
        out.append("};")
        out.append("")
    with open(os.path.join(HERE, "fast_rules.h"), "w") as f:
        f.write("\n".join(out))


if __name__ == "__main__":
    main()
