"""Matrix-free hybrid multigrid-preconditioned CG on the host cores.

TEST INFRASTRUCTURE ONLY: bench.py times it as the CPU baseline of the
multigrid solve, tests check its iteration counts against the assembled
restatement (mg_oracle.MGOracle).  The product never imports it.

It restates the reference's MultigridPreconditioner + SolverCG
(CG/cells_batched/application_ph.cc:1754-2023) the way the reference runs it
on a CPU: every level operator matrix-free (fast.FastOperator, the optimized
SIMD/OpenMP cell loop), point-Jacobi Chebyshev smoothing with a Lanczos
eigenvalue estimate (:1909-1932), nodal-interpolation transfers
(MGTwoLevelTransfer, :1900-1907) and a direct coarse solve (the limit of the
reference's AMG on its 125-DoF coarse grid, :1934-1946), FP64 outer CG to
||r|| <= rtol ||b|| (:1949-1980).  Level sequence "ph": P1 on the coarsest
Kuhn mesh .. P1 on the fine mesh, then P2 .. Pp on the fine mesh.  Vectors are
float64 torch CPU tensors (multithreaded element-wise work); transfers are
sparse matrices assembled once.
"""
import warnings

import numpy as np
import torch

import fast
import oracle as orc


def lattice(p):
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


class Level:
    def __init__(self, mesh, p):
        self.mesh, self.p = mesh, p
        self.op = fast.FastOperator(mesh, p, orc.CG)
        self.cd, cm = mesh.cg_dofs(p)
        self.constrained = torch.from_numpy(cm.astype(bool))
        self.n = self.op.n
        d = self.op.diagonal()
        self.invd = torch.from_numpy(np.where(np.abs(d) > 1e-10, 1.0 / d, 1.0))
        self._out = np.empty(self.n)

    def vmult(self, x):
        y = torch.empty(self.n, dtype=torch.float64)
        self.op.vmult(x.numpy(), y.numpy())
        return y


def _csr(rows, cols, vals, shape):
    warnings.filterwarnings("ignore", message="Sparse (CSR tensor support|invariant checks)")
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    crow = np.zeros(shape[0] + 1, np.int64)
    np.add.at(crow, rows + 1, 1)
    return torch.sparse_csr_tensor(torch.from_numpy(np.cumsum(crow)), torch.from_numpy(cols.astype(np.int64)),
                                   torch.from_numpy(vals), size=shape, dtype=torch.float64)


def p_transfer(fine, coarse):
    """P_{q-1} -> P_q on one mesh: the coarse function at the fine nodes, each
    fine DoF from the first cell that holds it; constrained DoFs left out."""
    K = fine.cd.shape[1]
    E = np.empty((K, coarse.cd.shape[1]))
    for i, xi in enumerate(lattice(fine.p)[:, 1:]):
        E[i], _ = orc.basis(coarse.p, xi)
    flat = fine.cd.ravel()
    _, first = np.unique(flat, return_index=True)
    cells, nodes = first // K, first % K
    rows = np.repeat(flat[first], coarse.cd.shape[1])
    cols = coarse.cd[cells].ravel()
    vals = E[nodes].ravel()
    keep = (~fine.constrained.numpy()[rows]) & (~coarse.constrained.numpy()[cols]) & (np.abs(vals) > 1e-14)
    return _csr(rows[keep], cols[keep], vals[keep], (fine.n, coarse.n))


def h_transfer(fine, coarse):
    """P1 on the n-hex Kuhn mesh -> P1 on its 2n refinement: a fine vertex is a
    coarse vertex or the midpoint of a coarse Kuhn edge (i,j,k)-(i+a,j+b,k+c)."""
    nf = fine.mesh.n[0]
    nc = nf // 2

    def vdof(level, nn):
        vd = np.empty((nn + 1) ** 3, np.int64)
        vd[level.mesh.cells().ravel()] = level.cd.ravel()
        return vd

    vf, vc = vdof(fine, nf), vdof(coarse, nc)
    I = np.arange(nf + 1)
    K3, J3, I3 = np.meshgrid(I, I, I, indexing="ij")
    lo = [I3 // 2, J3 // 2, K3 // 2]
    hi = [(I3 + 1) // 2, (J3 + 1) // 2, (K3 + 1) // 2]
    cid = lambda q: (q[0] + (nc + 1) * (q[1] + (nc + 1) * q[2])).ravel()
    fid = (I3 + (nf + 1) * (J3 + (nf + 1) * K3)).ravel()
    a, b = cid(lo), cid(hi)
    same = a == b
    rows = np.concatenate([vf[fid], vf[fid[~same]]])
    cols = np.concatenate([vc[a], vc[b[~same]]])
    vals = np.concatenate([np.where(same, 1.0, 0.5), np.full((~same).sum(), 0.5)])
    keep = (~fine.constrained.numpy()[rows]) & (~coarse.constrained.numpy()[cols])
    return _csr(rows[keep], cols[keep], vals[keep], (fine.n, coarse.n))


class FastMG:
    """V-cycle over the "ph" ladder; degree = Chebyshev degree."""

    def __init__(self, n, p, coarse_n=4, degree=3, smoothing_range=20.0, eig_iterations=10, eig_safety=1.2,
                 seed=0, jitter=0.0):
        H = int(round(np.log2(n // coarse_n)))
        meshes = [orc.KuhnMesh(n >> k, jitter=jitter if k == 0 else 0.0, seed=0) for k in range(H + 1)]
        seq = [(meshes[k], 1) for k in range(H, -1, -1)] + [(meshes[0], q) for q in range(2, p + 1)]
        self.levels = [Level(m, q) for (m, q) in seq]
        self.P = [None]
        for l in range(1, len(self.levels)):
            f, c = self.levels[l], self.levels[l - 1]
            self.P.append(p_transfer(f, c) if f.mesh is c.mesh else h_transfer(f, c))
        self.PT = [None] + [P.to_dense().T.to_sparse_csr() if P.shape[0] < 4096 else
                            P.to_sparse_coo().t().coalesce().to_sparse_csr() for P in self.P[1:]]
        self.degree = degree
        rng = np.random.default_rng(seed)
        for L in self.levels[1:]:
            L.lmax = eig_safety * self._lanczos_max(L, eig_iterations, rng)
            L.lmin = L.lmax / smoothing_range
        C = self.levels[0]
        A = np.stack([C.vmult(torch.from_numpy(e)).numpy() for e in np.eye(C.n)], axis=1)
        self.coarse_inv = torch.from_numpy(np.linalg.inv(A))

    @staticmethod
    def _lanczos_max(L, its, rng):
        b = torch.from_numpy(rng.uniform(-1, 1, L.n))
        b[L.constrained] = 0
        r = b.clone()
        z = L.invd * r
        p = z.clone()
        rz = float(r @ z)
        al, be = [], []
        for _ in range(its):
            q = L.vmult(p)
            a = rz / float(p @ q)
            al.append(a)
            r -= a * q
            z = L.invd * r
            rzn = float(r @ z)
            be.append(rzn / rz)
            p = z + be[-1] * p
            rz = rzn
        k = len(al)
        T = np.zeros((k, k))
        for i in range(k):
            T[i, i] = 1 / al[i] + (be[i - 1] / al[i - 1] if i > 0 else 0)
            if i + 1 < k:
                T[i, i + 1] = T[i + 1, i] = np.sqrt(be[i]) / al[i]
        return np.linalg.eigvalsh(T).max()

    def _smooth(self, L, x, b, zero):
        theta, delta = 0.5 * (L.lmax + L.lmin), 0.5 * (L.lmax - L.lmin)
        if zero:
            d = L.invd * b / theta
            x = d.clone()
        else:
            d = L.invd * (b - L.vmult(x)) / theta
            x = x + d
        rho = delta / theta
        for _ in range(1, self.degree):
            rn = 1.0 / (2 * theta / delta - rho)
            d = rn * rho * d + 2 * rn / delta * (L.invd * (b - L.vmult(x)))
            x = x + d
            rho = rn
        return x

    def vcycle(self, b, l=None):
        l = len(self.levels) - 1 if l is None else l
        if l == 0:
            return self.coarse_inv @ b
        L = self.levels[l]
        x = self._smooth(L, None, b, True)
        r = b - L.vmult(x)
        xc = self.vcycle(self.PT[l] @ r, l - 1)
        x = x + self.P[l] @ xc
        return self._smooth(L, x, b, False)

    def solve(self, b, rtol=1e-8, max_iterations=100):
        """MG-preconditioned CG from x = 0; returns (x, iterations)."""
        A = self.levels[-1]
        x = torch.zeros_like(b)
        r = b.clone()
        bn = float(torch.linalg.norm(b))
        z = self.vcycle(r)
        p = z.clone()
        rz = float(r @ z)
        for it in range(1, max_iterations + 1):
            q = A.vmult(p)
            a = rz / float(p @ q)
            x += a * p
            r -= a * q
            if float(torch.linalg.norm(r)) <= rtol * bn:
                return x, it
            z = self.vcycle(r)
            rzn = float(r @ z)
            p = z + (rzn / rz) * p
            rz = rzn
        return x, max_iterations

