"""ctypes binding of liboracle.so, the CPU restatement used as the checker.

TEST INFRASTRUCTURE ONLY (tests/, __graft_entry__.smoke(), bench.py's CPU
baseline leg).  See oracle.h for what it restates and its parity status.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
CG, DG, HELMHOLTZ = 0, 1, 2


class Params(C.Structure):
    _fields_ = [("degree", C.c_int32), ("kind", C.c_int32), ("n_components", C.c_int32),
                ("penalty", C.c_int32), ("mass", C.c_double), ("quad_points", C.c_int32),
                ("n_threads", C.c_int32), ("weak_bc", C.c_int32)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.oracle_create.restype = C.c_int
        L.oracle_create.argtypes = [C.POINTER(Params), C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_void_p)]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_vmult.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_vmult_cells.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64]
        L.oracle_diagonal.argtypes = [C.c_void_p, C.c_void_p]
        L.oracle_cell_matrix.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        L.oracle_check_cg_numbering.restype = C.c_int64
        L.oracle_check_cg_numbering.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_basis.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_n_dofs.restype = C.c_int64
        L.oracle_n_dofs.argtypes = [C.c_void_p]
        L.oracle_quadrature_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.oracle_set_p2_geometry.restype = C.c_int
        L.oracle_set_p2_geometry.argtypes = [C.c_void_p, C.c_void_p]
        L.oracle_kuhn_mesh.restype = C.c_int
        L.oracle_kuhn_mesh.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_uint64, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_cg_numbering.restype = C.c_int64
        L.oracle_cg_numbering.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                          C.c_void_p]
        _lib = L
    return _lib


class Oracle:
    """FP64 CPU operator on the same mesh arrays as the product."""

    def __init__(self, x, cells, degree, kind, cell_dofs=None, constrained=None, n_components=1,
                 penalty=0, mass=1e5, quad_points=0, n_threads=0, weak_bc=False):
        self.x = np.ascontiguousarray(x, np.float64)
        self.cells = np.ascontiguousarray(cells, np.int32)
        p = Params(degree, kind, n_components, penalty, mass, quad_points, n_threads, int(bool(weak_bc)))
        self.kind = kind
        if kind == CG:
            self.cell_dofs = np.ascontiguousarray(cell_dofs, np.int32)
            self.constrained = np.ascontiguousarray(constrained, np.uint8)
            nd = len(self.constrained)
            cdp, cmp = self.cell_dofs.ctypes.data, self.constrained.ctypes.data
        else:
            nd, cdp, cmp = 0, None, None
        h = C.c_void_p()
        rc = lib().oracle_create(C.byref(p), len(self.x), self.x.ctypes.data, len(self.cells),
                                 self.cells.ctypes.data, cdp, cmp, nd, C.byref(h))
        if rc != 0:
            raise RuntimeError(f"oracle_create failed: {rc}")
        self.h = h
        self.n = lib().oracle_n_dofs(h)
        self.K = (degree + 1) * (degree + 2) * (degree + 3) // 6
        self.nc = n_components

    def set_p2_geometry(self, edge_nodes):
        """CG on curved cells: quadratic geometry from the edge nodes [n_cells][6][3]."""
        self._edge = np.ascontiguousarray(edge_nodes, np.float64)
        if lib().oracle_set_p2_geometry(self.h, self._edge.ctypes.data) != 0:
            raise RuntimeError("oracle_set_p2_geometry failed")

    def vmult(self, src):
        src = np.ascontiguousarray(src, np.float64)
        dst = np.empty(self.n, np.float64)
        lib().oracle_vmult(self.h, src.ctypes.data, dst.ctypes.data)
        return dst

    def vmult_cells(self, src, dst, c0, c1):
        """Contributions of cells [c0, c1) into dst (a timing sample)."""
        lib().oracle_vmult_cells(self.h, src.ctypes.data, dst.ctypes.data, c0, c1)

    def diagonal(self):
        d = np.empty(self.n, np.float64)
        lib().oracle_diagonal(self.h, d.ctypes.data)
        return d

    def cell_matrix(self, c):
        n = self.K * self.nc
        m = np.empty((n, n), np.float64)
        lib().oracle_cell_matrix(self.h, c, m.ctypes.data)
        return m

    def check_cg_numbering(self, lo, hi):
        lo = np.ascontiguousarray(lo, np.float64)
        hi = np.ascontiguousarray(hi, np.float64)
        return lib().oracle_check_cg_numbering(self.h, lo.ctypes.data, hi.ctypes.data)

    def quadrature_sizes(self):
        a, b = C.c_int32(), C.c_int32()
        lib().oracle_quadrature_sizes(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.oracle_destroy(self.h)
            self.h = None


def basis(degree, xi):
    K = (degree + 1) * (degree + 2) * (degree + 3) // 6
    v = np.empty(K)
    g = np.empty((K, 3))
    xi = np.ascontiguousarray(xi, np.float64)
    lib().oracle_basis(degree, xi.ctypes.data, v.ctypes.data, g.ctypes.data)
    return v, g


class KuhnMesh:
    """The benchmark mesh made by the oracle's own generator (mesh.c), with
    the accessors of the product's Mesh (vertices, cells, neighbors, cg_dofs),
    so the CPU checker and baseline never need the product library."""

    def __init__(self, n, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), jitter=0.0, seed=0):
        if isinstance(n, int):
            n = (n, n, n)
        self.n = tuple(int(v) for v in n)
        self.lo, self.hi, self.jitter, self.seed = tuple(lo), tuple(hi), jitter, seed
        nv = (self.n[0] + 1) * (self.n[1] + 1) * (self.n[2] + 1)
        self.n_vertices = nv
        self.n_cells = 6 * self.n[0] * self.n[1] * self.n[2]
        self._x = np.empty((nv, 3), np.float64)
        self._cells = np.empty((self.n_cells, 4), np.int32)
        self._nb = np.empty((self.n_cells, 4), np.int32)
        self._nbf = np.empty((self.n_cells, 4), np.int8)
        nn = np.array(self.n, np.int32)
        lo_, hi_ = np.array(lo, np.float64), np.array(hi, np.float64)
        rc = lib().oracle_kuhn_mesh(nn.ctypes.data, lo_.ctypes.data, hi_.ctypes.data, float(jitter), int(seed),
                                    self._x.ctypes.data, self._cells.ctypes.data, self._nb.ctypes.data,
                                    self._nbf.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"oracle_kuhn_mesh failed: {rc}")
        self.n_boundary_faces = int((self._nb < 0).sum())
        self.n_interior_faces = (4 * self.n_cells - self.n_boundary_faces) // 2
        self._dofs = {}

    def vertices(self):
        return self._x

    def cells(self):
        return self._cells

    def neighbors(self):
        return self._nb, self._nbf

    def cg_dofs(self, degree):
        if degree not in self._dofs:
            n = lib().oracle_cg_numbering(self.n_vertices, self.n_cells, self._cells.ctypes.data,
                                          self._nb.ctypes.data, degree, None, None)
            if n < 0:
                raise RuntimeError(f"oracle_cg_numbering failed: {n}")
            k = (degree + 1) * (degree + 2) * (degree + 3) // 6
            cd = np.empty((self.n_cells, k), np.int32)
            cm = np.empty(n, np.uint8)
            lib().oracle_cg_numbering(self.n_vertices, self.n_cells, self._cells.ctypes.data,
                                      self._nb.ctypes.data, degree, cd.ctypes.data, cm.ctypes.data)
            self._dofs[degree] = (cd, cm)
        return self._dofs[degree]


def for_mesh(mesh, degree, kind, **kw):
    """Oracle on a simplexfem.Mesh or a KuhnMesh (CG uses the mesh's own CG numbering)."""
    if kind == CG:
        cd, cm = mesh.cg_dofs(degree)
        return Oracle(mesh.vertices(), mesh.cells(), degree, CG, cell_dofs=cd, constrained=cm, **kw)
    return Oracle(mesh.vertices(), mesh.cells(), degree, kind, **kw)
