#!/usr/bin/env python3
"""Generate the reference-element tables of the tetrahedral Lagrange spaces P1-P3.

Everything is computed in exact rational arithmetic (``fractions.Fraction``)
and only rounded to double when written out.  Two files are produced next to
this script:

* ``ref_tables.h``   constexpr host/device tables (node lattice, nodal-gradient
  matrices, reference masses, face node lists, face masses, p-embeddings);
* ``ref_kernels.cuh`` straight-line device functions that apply those matrices
  with every structural zero removed and every +-1 folded, so that the cell and
  face kernels run on compile-time constants only.

Conventions (the DoF format every other part of the library relies on)
-----------------------------------------------------------------------
Reference tetrahedron V0=(0,0,0), V1=(1,0,0), V2=(0,1,0), V3=(0,0,1); the
barycentric coordinates are l0 = 1-x-y-z, l1 = x, l2 = y, l3 = z.  A node of
P_q is a multi-index (a0,a1,a2,a3) with sum q and position (a1,a2,a3)/q.
Node order inside a cell: the 4 vertices; then the edges (0,1),(0,2),(0,3),
(1,2),(1,3),(2,3), each walked from its lower to its higher local vertex; then
the faces f=0..3 (face f is opposite vertex f), interior face nodes in
canonical face order; then interior nodes (none for q<=3).  This is the same
vertex/edge/face/interior grouping as deal.II's FE_SimplexP
(FE_SimplexP::FE_SimplexP in deal.II, used at CG/cells_batched/application.cc:1610),
with an edge order of our own.

Canonical face order: the three local vertices of face f in ascending order
(u0<u1<u2); a face node has face-barycentric index b=(a_u0,a_u1,a_u2) and
nodes are sorted by descending b0, then descending b1.  Cells store their
vertices sorted by global vertex id, so both cells that share a face list its
nodes in the same physical order.

P0 (the gradient space of P1) has a single node, the constant function.

Face matrices are normalised so that the integral over a physical face F of a
product of traces equals 2|F| * (the reference-triangle integral), i.e. the
tables already contain the factor 2 and kernels multiply by |F|.
"""
from fractions import Fraction as Fr
from itertools import product
import math
import os
import sys

EDGES = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]


def face_vertices(f):
    return [v for v in range(4) if v != f]


def nodes(q):
    """Multi-indices (a0,a1,a2,a3) of the P_q Lagrange nodes in cell order."""
    if q == 0:
        return [None]
    out = []
    for i in range(4):
        a = [0, 0, 0, 0]
        a[i] = q
        out.append(tuple(a))
    for (i, j) in EDGES:
        for m in range(1, q):
            a = [0, 0, 0, 0]
            a[i] = q - m
            a[j] = m
            out.append(tuple(a))
    for f in range(4):
        fv = face_vertices(f)
        interior = []
        for a in all_multi(q):
            if a[f] == 0 and all(a[v] >= 1 for v in fv):
                interior.append(a)
        interior.sort(key=lambda a: (-a[fv[0]], -a[fv[1]]))
        out.extend(interior)
    for a in all_multi(q):
        if all(x >= 1 for x in a):
            out.append(a)
    assert len(out) == len(set(out)) == n_nodes(q), (q, len(out))
    return out


def all_multi(q):
    res = []
    for a1 in range(q + 1):
        for a2 in range(q + 1 - a1):
            for a3 in range(q + 1 - a1 - a2):
                res.append((q - a1 - a2 - a3, a1, a2, a3))
    return res


def n_nodes(q):
    return (q + 1) * (q + 2) * (q + 3) // 6


def node_pos(a, q):
    if q == 0:
        return (Fr(1, 4), Fr(1, 4), Fr(1, 4))
    return (Fr(a[1], q), Fr(a[2], q), Fr(a[3], q))


def monomials3(q):
    return [(i, j, k) for i in range(q + 1) for j in range(q + 1 - i)
            for k in range(q + 1 - i - j)]


def monomials2(q):
    return [(i, j) for i in range(q + 1) for j in range(q + 1 - i)]


def solve_inverse(V):
    """Exact inverse of a square Fraction matrix by Gauss-Jordan."""
    n = len(V)
    A = [list(row) + [Fr(int(i == j)) for j in range(n)] for i, row in enumerate(V)]
    for c in range(n):
        p = next(r for r in range(c, n) if A[r][c] != 0)
        A[c], A[p] = A[p], A[c]
        piv = A[c][c]
        A[c] = [x / piv for x in A[c]]
        for r in range(n):
            if r != c and A[r][c] != 0:
                fac = A[r][c]
                A[r] = [x - fac * y for x, y in zip(A[r], A[c])]
    return [row[n:] for row in A]


class Basis3:
    """Lagrange basis of P_q on the reference tet as monomial coefficients."""

    def __init__(self, q):
        self.q = q
        self.nodes = nodes(q)
        self.mono = monomials3(q)
        V = [[mono_eval3(m, node_pos(a, q)) for m in self.mono] for a in self.nodes]
        Vi = solve_inverse(V)
        # phi_n = sum_m Vi[m][n] * mono_m
        self.coef = [[Vi[m][n] for m in range(len(self.mono))] for n in range(len(self.nodes))]

    def value(self, n, x):
        return sum(c * mono_eval3(m, x) for c, m in zip(self.coef[n], self.mono))

    def grad(self, n, a, x):
        s = Fr(0)
        for c, m in zip(self.coef[n], self.mono):
            if m[a] == 0 or c == 0:
                continue
            mm = list(m)
            e = mm[a]
            mm[a] -= 1
            s += c * e * mono_eval3(tuple(mm), x)
        return s

    def poly(self, n):
        return {m: c for c, m in zip(self.coef[n], self.mono) if c != 0}


def mono_eval3(m, x):
    return x[0] ** m[0] * x[1] ** m[1] * x[2] ** m[2]


def tet_int(m):
    """Exact integral of x^i y^j z^k over the reference tet."""
    i, j, k = m
    return Fr(math.factorial(i) * math.factorial(j) * math.factorial(k),
              math.factorial(i + j + k + 3))


def tri_int(m):
    i, j = m
    return Fr(math.factorial(i) * math.factorial(j), math.factorial(i + j + 2))


def poly_mul(p1, p2):
    out = {}
    for m1, c1 in p1.items():
        for m2, c2 in p2.items():
            m = tuple(a + b for a, b in zip(m1, m2))
            out[m] = out.get(m, Fr(0)) + c1 * c2
    return out


def mass3(B1, B2):
    M = []
    for i in range(len(B1.nodes)):
        row = []
        for j in range(len(B2.nodes)):
            pp = poly_mul(B1.poly(i), B2.poly(j))
            row.append(sum(c * tet_int(m) for m, c in pp.items()))
        M.append(row)
    return M


def face_nodes(q, f):
    """Indices (into the cell node list of P_q) of the nodes on face f, canonical order."""
    if q == 0:
        return [0]
    fv = face_vertices(f)
    nl = nodes(q)
    idx = [n for n, a in enumerate(nl) if a[f] == 0]
    idx.sort(key=lambda n: (-nl[n][fv[0]], -nl[n][fv[1]]))
    return idx


class Basis2:
    """Lagrange basis of P_q on the reference triangle in canonical face order."""

    def __init__(self, q):
        self.q = q
        if q == 0:
            self.pts = [(Fr(1, 3), Fr(1, 3))]
            self.coef = [[Fr(1)]]
            self.mono = [(0, 0)]
            return
        bs = []
        for b0 in range(q, -1, -1):
            for b1 in range(q - b0, -1, -1):
                bs.append((b0, b1, q - b0 - b1))
        self.pts = [(Fr(b[1], q), Fr(b[2], q)) for b in bs]
        self.mono = monomials2(q)
        V = [[p[0] ** m[0] * p[1] ** m[1] for m in self.mono] for p in self.pts]
        Vi = solve_inverse(V)
        self.coef = [[Vi[m][n] for m in range(len(self.mono))] for n in range(len(self.pts))]

    def poly(self, n):
        return {m: c for c, m in zip(self.coef[n], self.mono) if c != 0}


def mass2(B1, B2):
    M = []
    for i in range(len(B1.coef)):
        row = []
        for j in range(len(B2.coef)):
            pp = poly_mul(B1.poly(i), B2.poly(j))
            row.append(2 * sum(c * tri_int(m) for m, c in pp.items()))
        M.append(row)
    return M


def check_face_trace(q, f):
    """The trace of the 3D basis on face f equals the 2D basis (canonical order)."""
    if q == 0:
        return
    B3 = Basis3(q)
    B2 = Basis2(q)
    fv = face_vertices(f)
    verts = [(Fr(0), Fr(0), Fr(0)), (Fr(1), Fr(0), Fr(0)), (Fr(0), Fr(1), Fr(0)), (Fr(0), Fr(0), Fr(1))]
    fn = face_nodes(q, f)
    # sample points on the face
    for (s, t) in [(Fr(1, 7), Fr(2, 9)), (Fr(3, 11), Fr(1, 5)), (Fr(0), Fr(1, 3))]:
        x = tuple(verts[fv[0]][d] * (1 - s - t) + verts[fv[1]][d] * s + verts[fv[2]][d] * t
                  for d in range(3))
        for i, n in enumerate(fn):
            v3 = B3.value(n, x)
            v2 = sum(c * s ** m[0] * t ** m[1] for c, m in zip(B2.coef[i], B2.mono))
            assert v3 == v2, (q, f, i)
        on = set(fn)
        for n in range(len(B3.nodes)):
            if n not in on:
                assert B3.value(n, x) == 0


def fmt(x):
    v = float(x)
    if v == 0:
        return "0.0"
    return repr(v)


def build(pmax=3):
    data = {}
    for p in range(1, pmax + 1):
        Bp = Basis3(p)
        Bq = Basis3(p - 1) if p > 1 else None
        qnodes = nodes(p - 1) if p > 1 else [None]
        qpos = [node_pos(a, p - 1) if p > 1 else node_pos(None, 0) for a in qnodes]
        K, KQ = n_nodes(p), (n_nodes(p - 1) if p > 1 else 1)
        D = [[[Bp.grad(i, a, qpos[m]) for i in range(K)] for m in range(KQ)] for a in range(3)]
        if p > 1:
            MQ = mass3(Bq, Bq)
        else:
            MQ = [[Fr(1, 6)]]
        MP = mass3(Bp, Bp)
        NF, NFQ = (p + 1) * (p + 2) // 2, (p * (p + 1) // 2 if p > 1 else 1)
        FN = [face_nodes(p, f) for f in range(4)]
        FNQ = [face_nodes(p - 1, f) if p > 1 else [0] for f in range(4)]
        for f in range(4):
            check_face_trace(p, f)
            if p > 1:
                check_face_trace(p - 1, f)
        B2p, B2q = Basis2(p), Basis2(p - 1)
        MFPP = mass2(B2p, B2p)
        MFPQ = mass2(B2p, B2q)
        EMB = None
        if p > 1:
            EMB = [[Bq.value(j, node_pos(Bp.nodes[i], p)) for j in range(KQ)] for i in range(K)]
        # consistency: D applied to the nodal interpolant of x_a gives 1 for d/dx_a
        for a in range(3):
            lin = [node_pos(nd, p)[a] for nd in Bp.nodes]
            for b in range(3):
                for m in range(KQ):
                    v = sum(D[b][m][i] * lin[i] for i in range(K))
                    assert v == (1 if a == b else 0)
        data[p] = dict(K=K, KQ=KQ, NF=NF, NFQ=NFQ, D=D, MQ=MQ, MP=MP, FN=FN, FNQ=FNQ,
                       MFPP=MFPP, MFPQ=MFPQ, EMB=EMB,
                       NODES=[node_pos(a, p) for a in Bp.nodes],
                       LATTICE=Bp.nodes, MONO=Bp.mono, COEF=Bp.coef)
    return data


def arr(name, ctype, values, shape):
    def rec(v, depth):
        if depth == len(shape):
            return fmt(v) if ctype == "double" else str(v)
        return "{" + ", ".join(rec(x, depth + 1) for x in v) + "}"
    dims = "".join(f"[{s}]" for s in shape)
    return f"  static constexpr {ctype} {name}{dims} = {rec(values, 0)};\n"


def write_tables(data, path):
    out = []
    out.append("// Generated by gen_tables.py from exact rational arithmetic. Do not edit.\n")
    out.append("// Reference-element tables of the tetrahedral Lagrange spaces P1-P3; the\n")
    out.append("// node, edge and face conventions are documented in gen_tables.py.\n")
    out.append("#pragma once\n\nnamespace sfem {\nnamespace ref {\n\n")
    out.append("template <int P> struct Tables;\n\n")
    for p, d in data.items():
        out.append(f"template <> struct Tables<{p}> {{\n")
        out.append(f"  static constexpr int K = {d['K']};    // P{p} nodes per cell\n")
        out.append(f"  static constexpr int KQ = {d['KQ']};   // P{p-1} nodes (gradient space)\n")
        out.append(f"  static constexpr int NF = {d['NF']};   // P{p} nodes per face\n")
        out.append(f"  static constexpr int NFQ = {d['NFQ']};  // P{p-1} nodes per face\n")
        out.append(arr("NODES", "double", d["NODES"], [d["K"], 3]))
        out.append(arr("LATTICE", "int", [list(a) for a in d["LATTICE"]], [d["K"], 4]))
        out.append(arr("D", "double", d["D"], [3, d["KQ"], d["K"]]))
        out.append(arr("MQ", "double", d["MQ"], [d["KQ"], d["KQ"]]))
        out.append(arr("MP", "double", d["MP"], [d["K"], d["K"]]))
        out.append(arr("FN", "int", d["FN"], [4, d["NF"]]))
        out.append(arr("FNQ", "int", d["FNQ"], [4, d["NFQ"]]))
        out.append(arr("MFPP", "double", d["MFPP"], [d["NF"], d["NF"]]))
        out.append(arr("MFPQ", "double", d["MFPQ"], [d["NF"], d["NFQ"]]))
        if d["EMB"] is not None:
            kq = len(d["EMB"][0])
            out.append(arr("EMB", "double", d["EMB"], [d["K"], kq]))
        # basis polynomials: phi_n(x,y,z) = sum_m COEF[n][m] x^MONO[m][0] y^MONO[m][1] z^MONO[m][2]
        out.append(arr("MONO", "int", [list(m) for m in d["MONO"]], [len(d["MONO"]), 3]))
        out.append(arr("COEF", "double", d["COEF"], [d["K"], len(d["MONO"])]))
        out.append("};\n\n")
    out.append("}  // namespace ref\n}  // namespace sfem\n")
    with open(path, "w") as fh:
        fh.write("".join(out))


def emit_matvec(lines, A, rows, cols, out_expr, in_expr, accumulate, transpose=False):
    """Emit out[r] (+)= sum_c A[r][c] in[c] with zeros removed."""
    nnz = 0
    for r in range(rows):
        terms = []
        for c in range(cols):
            a = A[c][r] if transpose else A[r][c]
            if a == 0:
                continue
            nnz += 1
            x = in_expr(c)
            if a == 1:
                terms.append(("+", x))
            elif a == -1:
                terms.append(("-", x))
            else:
                terms.append(("+", f"T({fmt(a)}) * {x}"))
        o = out_expr(r)
        if not terms:
            if not accumulate:
                lines.append(f"  {o} = T(0);")
            continue
        if accumulate:
            for s, t in terms:
                lines.append(f"  {o} {s}= {t};")
        else:
            s0, t0 = terms[0]
            expr = (t0 if s0 == "+" else f"-({t0})")
            for s, t in terms[1:]:
                expr += f" {s} {t}"
            lines.append(f"  {o} = {expr};")
    return nnz


def write_kernels(data, path):
    L = []
    L.append("// Generated by gen_tables.py from exact rational arithmetic. Do not edit.")
    L.append("// Straight-line applications of the reference matrices of ref_tables.h:")
    L.append("// structural zeros are removed and +-1 entries folded, so cell and face")
    L.append("// kernels issue only FMAs on compile-time constants.")
    L.append("#pragma once\n")
    L.append("namespace sfem {\nnamespace gen {\n")
    stats = []
    for p, d in data.items():
        K, KQ, NF, NFQ = d["K"], d["KQ"], d["NF"], d["NFQ"]
        # nodal gradient: g[a][m] = sum_i D[a][m][i] u[i]
        L.append(f"// P{p}: reference gradient in the P{p-1} nodal basis, g[a*{KQ}+m] = (D_a u)_m")
        L.append(f"template <typename T> __host__ __device__ __forceinline__ void grad_P{p}(const T (&u)[{K}], T (&g)[{3*KQ}]) {{")
        nz = 0
        for a in range(3):
            nz += emit_matvec(L, d["D"][a], KQ, K, lambda r, a=a: f"g[{a*KQ + r}]", lambda c: f"u[{c}]", False)
        L.append("}")
        stats.append((p, "grad", nz, 3 * KQ * K))
        L.append(f"// P{p}: y += sum_a D_a^T h_a")
        L.append(f"template <typename T> __host__ __device__ __forceinline__ void gradT_P{p}(const T (&h)[{3*KQ}], T (&y)[{K}]) {{")
        # y[i] += sum_{a,m} D[a][m][i] h[a*KQ+m]
        DT = [[d["D"][a][m][i] for a in range(3) for m in range(KQ)] for i in range(K)]
        nz = emit_matvec(L, DT, K, 3 * KQ, lambda r: f"y[{r}]", lambda c: f"h[{c}]", True)
        L.append("}")
        stats.append((p, "gradT", nz, 3 * KQ * K))
        L.append(f"// P{p}: o = MQ w (reference-tet mass of P{p-1}), one gradient component")
        L.append(f"template <typename T> __host__ __device__ __forceinline__ void massQ_P{p}(const T* w, T* o) {{")
        emit_matvec(L, d["MQ"], KQ, KQ, lambda r: f"o[{r}]", lambda c: f"w[{c}]", False)
        L.append("}")
        L.append(f"// P{p}: y += MP u (reference-tet mass of P{p})")
        L.append(f"template <typename T> __host__ __device__ __forceinline__ void massP_P{p}(const T* u, T s, T* y) {{")
        # y += s * MP u  -> compute t = MP u then scale
        L.append(f"  T t[{K}];")
        emit_matvec(L, d["MP"], K, K, lambda r: f"t[{r}]", lambda c: f"u[{c}]", False)
        L.append(f"  for (int i = 0; i < {K}; ++i) y[i] += s * t[i];")
        L.append("}")
        L.append(f"// P{p}: o = MFPP j (face mass P{p} x P{p}, factor 2 included)")
        L.append(f"template <typename T> __host__ __device__ __forceinline__ void facePP_P{p}(const T* j, T* o) {{")
        emit_matvec(L, d["MFPP"], NF, NF, lambda r: f"o[{r}]", lambda c: f"j[{c}]", False)
        L.append("}")
        L.append(f"// P{p}: o += MFPQ a (face mass P{p} x P{p-1})")
        L.append(f"template <typename T> __host__ __device__ __forceinline__ void facePQ_P{p}(const T* a, T* o) {{")
        emit_matvec(L, d["MFPQ"], NF, NFQ, lambda r: f"o[{r}]", lambda c: f"a[{c}]", True)
        L.append("}")
        L.append(f"// P{p}: o = MFPQ^T j (face mass P{p-1} x P{p})")
        L.append(f"template <typename T> __host__ __device__ __forceinline__ void faceQP_P{p}(const T* j, T* o) {{")
        emit_matvec(L, d["MFPQ"], NFQ, NF, lambda r: f"o[{r}]", lambda c: f"j[{c}]", False, transpose=True)
        L.append("}")
        L.append("")
    # single-row functions for warp-split kernels: a switch on the row index
    # that folds away once the caller's loops are unrolled
    for p, d in data.items():
        K, KQ, NF, NFQ = d["K"], d["KQ"], d["NF"], d["NFQ"]

        def row_switch(name, sig, rows, body_of_row):
            L.append(f"template <typename T> __host__ __device__ __forceinline__ T {name}({sig}) {{")
            L.append("  switch (r) {")
            for r in range(rows):
                L.append(f"    case {r}: return {body_of_row(r)};")
            L.append("  }")
            L.append("  return T(0);")
            L.append("}")

        def lin(coefs, term):
            parts = []
            for c, a in coefs:
                if a == 0:
                    continue
                t = term(c)
                if a == 1:
                    parts.append(f"+ {t}")
                elif a == -1:
                    parts.append(f"- {t}")
                else:
                    parts.append(f"+ T({fmt(a)}) * {t}")
            if not parts:
                return "T(0)"
            s = " ".join(parts)
            return s[2:] if s.startswith("+ ") else "-" + s[2:] if False else ("T(0) " + s if s.startswith("-") else s[2:])

        # grad row r = a*KQ + m from u[i*us]
        row_switch(f"grad_row_P{p}", "int r, const T* u, int us", 3 * KQ,
                   lambda r: lin([(i, d["D"][r // KQ][r % KQ][i]) for i in range(K)], lambda i: f"u[{i} * us]"))
        # gradT row i from h[(a*KQ+m)*hs]
        row_switch(f"gradT_row_P{p}", "int r, const T* h, int hs", K,
                   lambda i: lin([(a * KQ + m, d["D"][a][m][i]) for a in range(3) for m in range(KQ)],
                                 lambda c: f"h[{c} * hs]"))
        # MQ row m from w[n]
        row_switch(f"massQ_row_P{p}", "int r, const T* w", KQ,
                   lambda m: lin([(n, d["MQ"][m][n]) for n in range(KQ)], lambda n: f"w[{n}]"))
        # MP row i from u[j*us]
        row_switch(f"massP_row_P{p}", "int r, const T* u, int us", K,
                   lambda i: lin([(j, d["MP"][i][j]) for j in range(K)], lambda j: f"u[{j} * us]"))
        # position of cell node i on face f (P_p) / of P_{p-1} node m on face f, -1 if absent
        cases = " ".join(f"case {f*K+i}: return {d['FN'][f].index(i) if i in d['FN'][f] else -1};"
                         for f in range(4) for i in range(K))
        L.append(f"__host__ __device__ __forceinline__ constexpr int face_pos_P{p}(int f, int i) "
                 f"{{ switch (f * {K} + i) {{ {cases} }} return -1; }}")
        cases = " ".join(f"case {f*KQ+m}: return {d['FNQ'][f].index(m) if m in d['FNQ'][f] else -1};"
                         for f in range(4) for m in range(KQ))
        L.append(f"__host__ __device__ __forceinline__ constexpr int faceq_pos_P{p}(int f, int m) "
                 f"{{ switch (f * {KQ} + m) {{ {cases} }} return -1; }}")
        L.append("")
    # dispatch struct and runtime face-node tables
    for p, d in data.items():
        K, KQ, NF, NFQ = d["K"], d["KQ"], d["NF"], d["NFQ"]
        L.append(f"// P{p} face node lists for runtime (neighbour) face indices")
        fn = ", ".join("{" + ", ".join(str(x) for x in row) + "}" for row in d["FN"])
        L.append(f"static __constant__ int8_t cFN_P{p}[4][{NF}] = {{{fn}}};")
    L.append("")
    L.append("template <int P> struct Ops;")
    for p, d in data.items():
        K, KQ, NF, NFQ = d["K"], d["KQ"], d["NF"], d["NFQ"]
        L.append(f"template <> struct Ops<{p}> {{")
        L.append(f"  static constexpr int K = {K}, KQ = {KQ}, NF = {NF}, NFQ = {NFQ};")
        L.append(f"  template <class T> static __device__ __forceinline__ void grad(const T (&u)[{K}], T (&g)[{3*KQ}]) {{ grad_P{p}(u, g); }}")
        L.append(f"  template <class T> static __device__ __forceinline__ void gradT(const T (&h)[{3*KQ}], T (&y)[{K}]) {{ gradT_P{p}(h, y); }}")
        L.append(f"  template <class T> static __device__ __forceinline__ void massQ(const T* w, T* o) {{ massQ_P{p}(w, o); }}")
        L.append(f"  template <class T> static __device__ __forceinline__ void massP(const T* u, T s, T* y) {{ massP_P{p}(u, s, y); }}")
        L.append(f"  template <class T> static __device__ __forceinline__ void facePP(const T* j, T* o) {{ facePP_P{p}(j, o); }}")
        L.append(f"  template <class T> static __device__ __forceinline__ void facePQ(const T* a, T* o) {{ facePQ_P{p}(a, o); }}")
        L.append(f"  template <class T> static __device__ __forceinline__ void faceQP(const T* j, T* o) {{ faceQP_P{p}(j, o); }}")
        L.append(f"  static __device__ __forceinline__ int fn_runtime(int f, int i) {{ return cFN_P{p}[f][i]; }}")
        L.append(f"  template <class T> static __device__ __forceinline__ T grad_row(int r, const T* u, int us) {{ return grad_row_P{p}(r, u, us); }}")
        L.append(f"  template <class T> static __device__ __forceinline__ T gradT_row(int r, const T* h, int hs) {{ return gradT_row_P{p}(r, h, hs); }}")
        L.append(f"  template <class T> static __device__ __forceinline__ T massQ_row(int r, const T* w) {{ return massQ_row_P{p}(r, w); }}")
        L.append(f"  template <class T> static __device__ __forceinline__ T massP_row(int r, const T* u, int us) {{ return massP_row_P{p}(r, u, us); }}")
        L.append(f"  static __host__ __device__ __forceinline__ constexpr int face_pos(int f, int i) {{ return face_pos_P{p}(f, i); }}")
        L.append(f"  static __host__ __device__ __forceinline__ constexpr int faceq_pos(int f, int m) {{ return faceq_pos_P{p}(f, m); }}")
        cases = " ".join(f"case {f*NF+i}: return {d['FN'][f][i]};" for f in range(4) for i in range(NF))
        L.append(f"  static __host__ __device__ __forceinline__ constexpr int fn(int f, int i) {{ switch (f * {NF} + i) {{ {cases} }} return 0; }}")
        cases = " ".join(f"case {f*NFQ+i}: return {d['FNQ'][f][i]};" for f in range(4) for i in range(NFQ))
        L.append(f"  static __host__ __device__ __forceinline__ constexpr int fnq(int f, int m) {{ switch (f * {NFQ} + m) {{ {cases} }} return 0; }}")
        L.append("};")
    L.append("")
    L.append("}  // namespace gen\n}  // namespace sfem")
    with open(path, "w") as fh:
        fh.write("\n".join(L) + "\n")
    return stats


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    data = build()
    write_tables(data, os.path.join(here, "ref_tables.h"))
    stats = write_kernels(data, os.path.join(here, "ref_kernels.cuh"))
    for s in stats:
        print("P%d %-6s nonzeros %4d of %4d" % s)


if __name__ == "__main__":
    sys.exit(main())
