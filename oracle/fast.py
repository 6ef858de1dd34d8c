"""ctypes binding of the optimized CPU restatement (fast.cpp).

TEST INFRASTRUCTURE ONLY: bench.py times it as the CPU baseline and the
reference arm; tests check it against the scalar oracle.  It loads the
AVX-512 build when the host has AVX-512 (x86-64-v4), else the AVX2 build.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
CG, DG, HELMHOLTZ = 0, 1, 2


class Params(C.Structure):
    _fields_ = [("degree", C.c_int32), ("kind", C.c_int32), ("n_components", C.c_int32),
                ("penalty", C.c_int32), ("mass", C.c_double), ("n_threads", C.c_int32)]


def host_isa():
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        return "avx2"
    need = ("avx512f", "avx512dq", "avx512bw", "avx512vl", "avx512cd")
    return "avx512" if all(f in flags for f in need) else "avx2"


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, f"liboracle_fast_{host_isa()}.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", _HERE], check=True)
        L = C.CDLL(path)
        L.fast_create.restype = C.c_int
        L.fast_create.argtypes = [C.POINTER(Params), C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_void_p)]
        L.fast_destroy.argtypes = [C.c_void_p]
        L.fast_n_dofs.restype = C.c_int64
        L.fast_n_dofs.argtypes = [C.c_void_p]
        L.fast_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int32)] * 4
        L.fast_vmult.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.fast_diagonal.restype = C.c_int
        L.fast_diagonal.argtypes = [C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


class FastOperator:
    """The reference's optimized vmult on the host cores (FP64)."""

    def __init__(self, mesh, degree, kind, n_components=1, penalty=0, mass=1e5, n_threads=0):
        self.x = np.ascontiguousarray(mesh.vertices(), np.float64)
        self.cells = np.ascontiguousarray(mesh.cells(), np.int32)
        nb, nbf = mesh.neighbors()
        self.nb = np.ascontiguousarray(nb, np.int32)
        self.nbf = np.ascontiguousarray(nbf, np.int8)
        if kind == CG:
            cd, cm = mesh.cg_dofs(degree)
            self.cd = np.ascontiguousarray(cd, np.int32)
            self.cm = np.ascontiguousarray(cm, np.uint8)
            cdp, cmp_, nd = self.cd.ctypes.data, self.cm.ctypes.data, len(self.cm)
        else:
            cdp, cmp_, nd = None, None, 0
        nc = n_components if kind == HELMHOLTZ else 1
        p = Params(degree, kind, nc, penalty, mass, n_threads)
        h = C.c_void_p()
        rc = lib().fast_create(C.byref(p), len(self.x), self.x.ctypes.data, len(self.cells), self.cells.ctypes.data,
                               self.nb.ctypes.data, self.nbf.ctypes.data, cdp, cmp_, nd, C.byref(h))
        if rc != 0:
            raise RuntimeError(f"fast_create failed: {rc}")
        self.h = h
        self.n = lib().fast_n_dofs(h)
        a, b, c, d = (C.c_int32() for _ in range(4))
        lib().fast_info(h, C.byref(a), C.byref(b), C.byref(c), C.byref(d))
        self.n_cell_points, self.n_face_points, self.lanes, self.threads = a.value, b.value, c.value, d.value
        self.isa = host_isa()

    def vmult(self, src, dst=None):
        src = np.ascontiguousarray(src, np.float64)
        if dst is None:
            dst = np.empty(self.n, np.float64)
        lib().fast_vmult(self.h, src.ctypes.data, dst.ctypes.data)
        return dst

    def diagonal(self):
        """CG only: the operator's diagonal (1 on constrained rows)."""
        d = np.empty(self.n, np.float64)
        if lib().fast_diagonal(self.h, d.ctypes.data) != 0:
            raise RuntimeError("fast_diagonal: CG operators only")
        return d

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fast_destroy(self.h)
            self.h = None
