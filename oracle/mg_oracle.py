"""CPU restatement of the reference's hybrid multigrid-preconditioned CG.

TEST INFRASTRUCTURE ONLY.  Follows the reference's MultigridPreconditioner
(CG/cells_batched/application_ph.cc:1754-2023, h-then-p order
application_hp.cc:1735-2008) and SolverCG (:1949-1980):
  - levels P1 on the coarsest mesh .. P1 on the fine mesh, then P2 .. Pp (ph),
    or P1 .. Pp on the coarsest mesh, then Pp on finer meshes (hp);
  - level matrices assembled from the oracle's element matrices, constrained
    rows/columns replaced by the identity (ones_on_diagonal);
  - transfers = nodal interpolation of the coarse space at the fine nodes
    (MGTwoLevelTransfer), restriction = transpose, constrained DoFs excluded;
  - PreconditionChebyshev with a point-Jacobi inner preconditioner, degree d,
    lambda_max from a Lanczos estimate of eig_iterations CG steps times 1.2,
    lambda_min = lambda_max / smoothing_range;
  - a direct coarse solve (the reference's AMG on a 125-DoF coarse grid
    reduces to an exact solve for the purpose of counting iterations);
  - PCG stopping at ||r|| <= rtol ||b||;
  - DG hierarchies (DGMGOracle): DG P_p .. P_pc by cell-local embeddings, a
    c-transfer from CG P_pc, then the CG ladder
    (DG/cells_batched/application_phc.cc:3396-3652).
Meshes must be unjittered (nested Kuhn refinement).  Parity status: unpinned
against the reference (deal.II and Trilinos are absent); checked against the
GPU solver's iteration counts.
"""
import numpy as np
import scipy.sparse as sp

import oracle as orc

PERMS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


def lattice_nodes(p):
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
    def __init__(self, mesh, p, weak=False):
        """weak: boundary imposed by Nitsche terms, no constrained DoFs (the CG
        levels of DG/cells_batched/application_phc.cc:1799-1832)."""
        self.mesh, self.p = mesh, p
        self.cd, self.cm = mesh.cg_dofs(p)
        if weak:
            self.cm = np.zeros_like(self.cm)
        self.n = len(self.cm)
        o = orc.Oracle(mesh.vertices(), mesh.cells(), p, orc.CG, cell_dofs=self.cd, constrained=self.cm,
                       weak_bc=weak)
        K = self.cd.shape[1]
        rows, cols, vals = [], [], []
        free = ~self.cm.astype(bool)
        for c in range(mesh.n_cells):
            Ae = o.cell_matrix(c)
            g = self.cd[c]
            ok = free[g]
            gi, gj = np.meshgrid(g, g, indexing="ij")
            mask = np.outer(ok, ok)
            rows.append(gi[mask])
            cols.append(gj[mask])
            vals.append(Ae[mask])
        A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                          shape=(self.n, self.n)).tocsr()
        A = A + sp.diags(self.cm.astype(np.float64))
        self.A = A.tocsr()
        d = self.A.diagonal()
        self.invd = np.where(np.abs(d) > 1e-10, 1.0 / d, 1.0)
        # support points
        L = lattice_nodes(p)
        xv, cells = mesh.vertices(), mesh.cells()
        self.pts = np.zeros((self.n, 3))
        for c in range(mesh.n_cells):
            self.pts[self.cd[c]] = L @ xv[cells[c]]


def transfer(fine, coarse):
    """Prolongation matrix coarse -> fine (interpolation at fine nodes)."""
    mc = coarse.mesh
    n = np.array(mc.n)
    lo, hi = np.array(mc.lo), np.array(mc.hi)
    cells = mc.cells()
    xv = mc.vertices()
    # coarse cell by (hex, type)
    lat_v = np.round((xv - lo) / (hi - lo) * n).astype(int)
    table = {}
    for c in range(mc.n_cells):
        cen = lat_v[cells[c]].mean(0)
        h = np.floor(cen).astype(int)
        f = cen - h
        t = next(i for i, pm in enumerate(PERMS) if f[pm[0]] >= f[pm[1]] >= f[pm[2]])
        table[(h[0], h[1], h[2], t)] = c
    rows, cols, vals = [], [], []
    ffree = ~fine.cm.astype(bool)
    cfree = ~coarse.cm.astype(bool)
    for i in np.nonzero(ffree)[0]:
        X = (fine.pts[i] - lo) / (hi - lo) * n
        h = np.minimum(np.floor(X).astype(int), n - 1)
        f = X - h
        t = next(k for k, pm in enumerate(PERMS) if f[pm[0]] >= f[pm[1]] - 1e-12 and f[pm[1]] >= f[pm[2]] - 1e-12)
        c = table[(h[0], h[1], h[2], t)]
        v = xv[cells[c]]
        J = (v[1:] - v[0]).T
        xi = np.linalg.solve(J, fine.pts[i] - v[0])
        phi, _ = orc.basis(coarse.p, xi)
        for j, w in zip(coarse.cd[c], phi):
            if cfree[j] and abs(w) > 1e-14:
                rows.append(i)
                cols.append(j)
                vals.append(w)
    return sp.coo_matrix((vals, (rows, cols)), shape=(fine.n, coarse.n)).tocsr()


class MGOracle:
    def __init__(self, make_mesh, n, p, order="ph", coarse_n=4, degree=3, smoothing_range=20.0,
                 eig_iterations=10, eig_safety=1.2, seed=0, weak=False):
        H = int(round(np.log2(n // coarse_n)))
        meshes = [make_mesh(n >> k) for k in range(H + 1)]  # fine .. coarse
        seq = []
        if order == "ph":
            seq += [(meshes[k], 1) for k in range(H, -1, -1)]
            seq += [(meshes[0], q) for q in range(2, p + 1)]
        else:
            seq += [(meshes[H], q) for q in range(1, p + 1)]
            seq += [(meshes[k], p) for k in range(H - 1, -1, -1)]
        self.levels = [Level(m, q, weak) for (m, q) in seq]
        self.P = [None] + [transfer(self.levels[l], self.levels[l - 1]) for l in range(1, len(self.levels))]
        self.degree = degree
        rng = np.random.default_rng(seed)
        for L in self.levels[1:]:
            L.lmax = eig_safety * self._lanczos_max(L, eig_iterations, rng)
            L.lmin = L.lmax / smoothing_range
        self.coarse_inv = np.linalg.inv(self.levels[0].A.toarray())

    @staticmethod
    def _lanczos_max(L, its, rng):
        b = rng.uniform(-1, 1, L.n)
        b[L.cm.astype(bool)] = 0
        r = b.copy()
        z = L.invd * r
        p = z.copy()
        rz = r @ z
        al, be = [], []
        for _ in range(its):
            q = L.A @ p
            a = rz / (p @ q)
            al.append(a)
            r -= a * q
            z = L.invd * r
            rzn = r @ z
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
            x = d.copy()
        else:
            d = L.invd * (b - L.A @ x) / theta
            x = x + d
        rho = delta / theta
        for _ in range(1, self.degree):
            rn = 1.0 / (2 * theta / delta - rho)
            d = rn * rho * d + 2 * rn / delta * (L.invd * (b - L.A @ x))
            x = x + d
            rho = rn
        return x

    def vcycle(self, b, l=None):
        l = len(self.levels) - 1 if l is None else l
        if l == 0:
            return self.coarse_inv @ b
        L = self.levels[l]
        x = self._smooth(L, None, b, True)
        r = b - L.A @ x
        xc = self.vcycle(self.P[l].T @ r, l - 1)
        x = x + self.P[l] @ xc
        return self._smooth(L, x, b, False)


class DGLevel:
    """DG level (FE_SimplexDGP, SIPG) assembled by probing the oracle's vmult.
    A DG row of cell c couples only to cell c and its face neighbours, so the
    cells are given a distance-2 colouring and one probe per (colour, local
    DoF) recovers all columns of that colour; small meshes only."""

    def __init__(self, mesh, p):
        o = orc.for_mesh(mesh, p, orc.DG)
        self.mesh, self.p, self.n = mesh, p, o.n
        C = mesh.n_cells
        K = self.n // C
        nb, _ = mesh.neighbors()
        adj = [set(int(v) for v in nb[c] if v >= 0) for c in range(C)]
        color = np.full(C, -1)
        for c in range(C):
            near = set(adj[c])
            for a in adj[c]:
                near |= adj[a]
            used = {color[a] for a in near if color[a] >= 0}
            color[c] = next(k for k in range(len(used) + 1) if k not in used)
        rows, cols, vals = [], [], []
        for k in range(color.max() + 1):
            cells = np.nonzero(color == k)[0]
            for i in range(K):
                e = np.zeros(self.n)
                e[cells * K + i] = 1.0
                y = o.vmult(e)
                for c in cells:
                    for a in [c] + sorted(adj[c]):
                        blk = y[a * K:(a + 1) * K]
                        nz = np.nonzero(blk)[0]
                        rows.append(a * K + nz)
                        cols.append(np.full(nz.size, c * K + i))
                        vals.append(blk[nz])
        self.A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                               shape=(self.n, self.n)).tocsr()
        self.cm = np.zeros(self.n, np.uint8)
        d = self.A.diagonal()
        self.invd = np.where(np.abs(d) > 1e-10, 1.0 / d, 1.0)


def embedding(p):
    """Nodal interpolation of P_{p-1} at the P_p nodes, [K_p][K_{p-1}]."""
    L = lattice_nodes(p)
    return np.array([orc.basis(p - 1, lam[1:])[0] for lam in L])


class DGMGOracle(MGOracle):
    """DG multigrid of DG/cells_batched/application_phc.cc:3396-3652: DG levels
    P_p .. P_pc on the fine mesh (cell-local embeddings), a c-transfer from CG
    P_pc on the same mesh (continuous nodal values copied into every cell,
    constrained nodes as 0), then the CG ladder of MGOracle.  pc = 1
    (c_transfer 0, phc) or p (c_transfer 1, cph / chp).  The CG levels keep the
    strong homogeneous Dirichlet constraints of the CG operator, or with
    weak_cg take the reference's weak boundary terms and no constraints."""

    def __init__(self, make_mesh, n, p, c_transfer=0, order="ph", coarse_n=4, degree=3, smoothing_range=20.0,
                 eig_iterations=10, eig_safety=1.2, seed=0, weak_cg=False):
        pc = 1 if c_transfer == 0 else p
        super().__init__(make_mesh, n, pc, order=order, coarse_n=coarse_n, degree=degree,
                         smoothing_range=smoothing_range, eig_iterations=eig_iterations, eig_safety=eig_safety,
                         seed=seed, weak=weak_cg)
        mesh = make_mesh(n)
        cgtop = self.levels[-1]
        rng = np.random.default_rng(seed + 1)
        for q in range(pc, p + 1):
            L = DGLevel(mesh, q)
            C = mesh.n_cells
            if q == pc:
                K = cgtop.cd.shape[1]
                free = ~cgtop.cm.astype(bool)
                r = np.arange(C * K)
                g = cgtop.cd.reshape(-1)
                ok = free[g]
                P = sp.coo_matrix((np.ones(ok.sum()), (r[ok], g[ok])), shape=(L.n, cgtop.n)).tocsr()
            else:
                E = embedding(q)
                P = sp.kron(sp.identity(C, format="csr"), sp.csr_matrix(E)).tocsr()
            L.lmax = eig_safety * self._lanczos_max(L, eig_iterations, rng)
            L.lmin = L.lmax / smoothing_range
            self.levels.append(L)
            self.P.append(P)


def pcg(A, b, precond, rtol, maxit):
    x = np.zeros_like(b)
    r = b.copy()
    bn = np.linalg.norm(b)
    z = precond(r)
    p = z.copy()
    rz = r @ z
    for it in range(1, maxit + 1):
        q = A(p)
        a = rz / (p @ q)
        x += a * p
        r -= a * q
        if np.linalg.norm(r) <= rtol * bn:
            return x, it
        z = precond(r)
        rzn = r @ z
        p = z + (rzn / rz) * p
        rz = rzn
    return x, maxit
