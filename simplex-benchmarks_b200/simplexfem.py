"""Python mirror of the deal.II-shaped operator interface over the C ABI.

The classes here keep the names and argument meaning of the reference's
Operator / MultigridPreconditioner interface (CG/cells_batched/application.cc:
1040-1582, CG/cells_batched/application_ph.cc:1754-2023): ``vmult(dst, src)``,
``Tvmult``, ``m()``, ``initialize_dof_vector``, ``compute_inverse_diagonal``.
Vectors are CUDA tensors (torch is used only for device memory and streams);
every call goes through ``libsimplexfem.so`` (include/simplex_fem.h).  There is
no CPU fallback: a missing library raises at import of the first handle.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsimplexfem.so")

FEM_OK = 0
FEM_ERR_ARG, FEM_ERR_CUDA, FEM_ERR_STATE, FEM_ERR_INTERNAL = 1, 2, 3, 7
FEM_CG, FEM_DG, FEM_HELMHOLTZ = 0, 1, 2
FEM_FP64, FEM_FP32 = 0, 1
FEM_PENALTY_REFERENCE, FEM_PENALTY_SQUARE = 0, 1
KINDS = {"cg": FEM_CG, "dg": FEM_DG, "helmholtz": FEM_HELMHOLTZ}
PRECISIONS = {"fp64": FEM_FP64, "fp32": FEM_FP32}


class FemError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"simplexfem error {code}: {msg}")
        self.code = code


class MeshDesc(C.Structure):
    _fields_ = [("n", C.c_int32 * 3), ("lo", C.c_double * 3), ("hi", C.c_double * 3),
                ("jitter", C.c_double), ("seed", C.c_uint64)]


class OpParams(C.Structure):
    _fields_ = [("mass_coefficient", C.c_double), ("n_components", C.c_int32),
                ("penalty", C.c_int32), ("kernel_variant", C.c_int32), ("weak_boundary", C.c_int32),
                ("reserved", C.c_int32 * 4)]


class RhsDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_modes", C.c_int32), ("k", (C.c_double * 3) * 16),
                ("amp", C.c_double * 16)]


class MGParams(C.Structure):
    _fields_ = [("order", C.c_int32), ("precision", C.c_int32), ("smoother_degree", C.c_int32),
                ("eig_iterations", C.c_int32), ("smoothing_range", C.c_double), ("eig_safety", C.c_double),
                ("coarse_n", C.c_int32), ("use_graph", C.c_int32), ("c_transfer", C.c_int32),
                ("learned_steps", C.c_int32), ("tensor_cores", C.c_int32), ("weak_cg_levels", C.c_int32)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("status", C.c_int32), ("initial_residual", C.c_double),
                ("final_residual", C.c_double), ("fallback_iteration", C.c_int32), ("reserved", C.c_int32)]


class MLPTrainParams(C.Structure):
    _fields_ = [("n_sizes", C.c_int32), ("sizes", C.c_int32 * 4), ("rhs_per_size", C.c_int32),
                ("iterates", C.c_int32), ("samples", C.c_int32), ("epochs", C.c_int32), ("batch", C.c_int32),
                ("lr", C.c_float), ("jitter", C.c_double), ("seed", C.c_uint64), ("noise_fraction", C.c_double),
                ("coarse_iterations", C.c_int32), ("reserved", C.c_int32)]


class MLPTrainInfo(C.Structure):
    _fields_ = [("samples", C.c_int32), ("reserved", C.c_int32), ("loss_first", C.c_double),
                ("loss_last", C.c_double), ("seconds", C.c_double)]


FEM_RHS_PLANE_WAVES, FEM_RHS_SINE_PRODUCTS = 0, 1
FEM_MG_PH, FEM_MG_HP = 0, 1
FEM_PRECOND_NONE, FEM_PRECOND_JACOBI, FEM_PRECOND_MG = 0, 1, 2
FEM_ERR_NOT_CONVERGED, FEM_ERR_BREAKDOWN, FEM_ERR_NONFINITE = 4, 5, 6

_lib = None

# (name, restype, argtypes) of every exported entry point
_PROTOS = [
    ("fem_last_error_string", C.c_char_p, []),
    ("fem_version", C.c_int, [C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("fem_mesh_create", C.c_int, [C.POINTER(MeshDesc), C.POINTER(C.c_void_p)]),
    ("fem_mesh_create_from_arrays", C.c_int, [C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int32,
                                              C.POINTER(C.c_void_p)]),
    ("fem_mesh_read_vtk", C.c_int, [C.c_char_p, C.c_int32, C.POINTER(C.c_void_p)]),
    ("fem_mesh_copy_input_cells", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fem_mesh_curve", C.c_int, [C.c_void_p, C.c_double]),
    ("fem_mesh_copy_edge_nodes", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fem_mesh_destroy", C.c_int, [C.c_void_p]),
    ("fem_mesh_sizes", C.c_int, [C.c_void_p] + [C.POINTER(C.c_int64)] * 4),
    ("fem_mesh_copy_vertices", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fem_mesh_copy_cells", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fem_mesh_copy_neighbors", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_mesh_cg_dofs", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64), C.c_void_p, C.c_void_p]),
    ("fem_op_create", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.POINTER(OpParams),
                                C.POINTER(C.c_void_p)]),
    ("fem_op_destroy", C.c_int, [C.c_void_p]),
    ("fem_op_element_matrices", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_csr_spmv", C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                               C.c_void_p]),
    ("fem_op_m", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    ("fem_op_info", C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                              C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    ("fem_op_copy_dof_map", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fem_op_copy_constrained", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fem_op_copy_support_points", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fem_op_vmult", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_op_vmult_phase", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    ("fem_op_vmult_static_scratch", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_op_Tvmult", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_op_compute_inverse_diagonal", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_op_compute_diagonal", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_op_set_kernel_variant", C.c_int, [C.c_void_p, C.c_int32]),
    ("fem_op_vmult_host", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_op_work", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("fem_op_status", C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    ("fem_part_create", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                  C.POINTER(C.c_void_p)]),
    ("fem_part_destroy", C.c_int, [C.c_void_p]),
    ("fem_part_sizes", C.c_int, [C.c_void_p] + [C.POINTER(C.c_int64)] * 5 + [C.POINTER(C.c_int32)]),
    ("fem_part_global_index", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fem_part_peer", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                C.POINTER(C.c_int64)]),
    ("fem_part_halo", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    ("fem_op_create_part", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(OpParams), C.POINTER(C.c_void_p)]),
    ("fem_op_rhs", C.c_int, [C.c_void_p, C.POINTER(RhsDesc), C.c_void_p, C.c_void_p]),
    ("fem_op_interpolate", C.c_int, [C.c_void_p, C.POINTER(RhsDesc), C.c_void_p, C.c_void_p]),
    ("fem_mg_params_default", C.c_int, [C.POINTER(MGParams)]),
    ("fem_mg_create", C.c_int, [C.c_void_p, C.POINTER(MGParams), C.POINTER(C.c_void_p)]),
    ("fem_mg_destroy", C.c_int, [C.c_void_p]),
    ("fem_mg_n_levels", C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    ("fem_mg_level_info", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_uint64), C.POINTER(C.c_int32),
                                    C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    ("fem_mg_level_kind", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    ("fem_mg_vcycle", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_mg_level_vmult", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_mg_smooth", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    ("fem_mg_prolongate_add", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_mg_restrict_add", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_mg_coarse_solve", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_cg_create", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    ("fem_cg_destroy", C.c_int, [C.c_void_p]),
    ("fem_cg_solve", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int32,
                               C.POINTER(SolveInfo), C.c_void_p]),
    ("fem_mlp_create", C.c_int, [C.c_uint64, C.POINTER(C.c_void_p)]),
    ("fem_mlp_destroy", C.c_int, [C.c_void_p]),
    ("fem_mlp_n_params", C.c_int, [C.POINTER(C.c_int32)]),
    ("fem_mlp_get_weights", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fem_mlp_set_weights", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fem_mlp_train_params_default", C.c_int, [C.POINTER(MLPTrainParams)]),
    ("fem_mlp_generate_and_train", C.c_int, [C.c_void_p, C.POINTER(MLPTrainParams), C.POINTER(MLPTrainInfo)]),
    ("fem_mlp_train", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                C.c_uint64, C.POINTER(MLPTrainInfo)]),
    ("fem_mlp_gradient", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                   C.POINTER(C.c_double), C.c_void_p]),
    ("fem_mlp_forward", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    ("fem_mlp_forward_tc", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    ("fem_mlp_set_tensor_cores", C.c_int, [C.c_void_p, C.c_int32]),
    ("fem_mlp_status", C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    ("fem_mlp_save", C.c_int, [C.c_void_p, C.c_char_p]),
    ("fem_mlp_load", C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    ("fem_mg_set_learned_smoother", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    ("fem_batch_create", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]),
    ("fem_batch_destroy", C.c_int, [C.c_void_p]),
    ("fem_batch_vmult", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fem_batch_set_kernel_variant", C.c_int, [C.c_void_p, C.c_int32]),
    ("fem_op_autotune", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_double)]),
    ("fem_batch_autotune", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    ("fem_autotune_cache", C.c_int, [C.c_char_p]),
]


def lib():
    """Load libsimplexfem.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FemError(-1, f"{LIB_PATH} is missing: run `make -C simplex-benchmarks_b200`")
        L = C.CDLL(LIB_PATH)
        for name, res, args in _PROTOS:
            if hasattr(L, name):
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != FEM_OK:
        raise FemError(status, lib().fem_last_error_string().decode())


def _stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class Mesh:
    """Kuhn-subdivided box (fem_mesh_create)."""

    def __init__(self, n, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), jitter=0.0, seed=0):
        if isinstance(n, int):
            n = (n, n, n)
        d = MeshDesc()
        d.n[:] = list(n)
        d.lo[:] = list(lo)
        d.hi[:] = list(hi)
        d.jitter = jitter
        d.seed = seed
        h = C.c_void_p()
        check(lib().fem_mesh_create(C.byref(d), C.byref(h)))
        self._adopt(h)
        self.n, self.lo, self.hi, self.jitter, self.seed = tuple(n), tuple(lo), tuple(hi), jitter, seed

    def _adopt(self, h):
        self.handle = h
        nv, nc, fi, fb = (C.c_int64() for _ in range(4))
        check(lib().fem_mesh_sizes(h, C.byref(nv), C.byref(nc), C.byref(fi), C.byref(fb)))
        self.n_vertices, self.n_cells = nv.value, nc.value
        self.n_interior_faces, self.n_boundary_faces = fi.value, fb.value

    @classmethod
    def from_arrays(cls, vertices, cells, reorder=True):
        """Unstructured tet mesh (fem_mesh_create_from_arrays); reorder puts the
        cells in Morton order of their centroids."""
        x = np.ascontiguousarray(vertices, np.float64)
        c = np.ascontiguousarray(cells, np.int32)
        h = C.c_void_p()
        check(lib().fem_mesh_create_from_arrays(len(x), x.ctypes.data, len(c), c.ctypes.data, int(bool(reorder)),
                                                C.byref(h)))
        m = cls.__new__(cls)
        m._adopt(h)
        m.n = None
        return m

    @classmethod
    def read_vtk(cls, path, reorder=True):
        """Legacy ASCII VTK unstructured grid of tetrahedra (fem_mesh_read_vtk)."""
        h = C.c_void_p()
        check(lib().fem_mesh_read_vtk(os.fsencode(str(path)), int(bool(reorder)), C.byref(h)))
        m = cls.__new__(cls)
        m._adopt(h)
        m.n = None
        return m

    def curve(self, amplitude):
        """Curvilinear geometry (fem_mesh_curve): the mesh is moved by a smooth
        bump that keeps the box boundary and gets quadratic cells."""
        check(lib().fem_mesh_curve(self.handle, float(amplitude)))
        return self

    def edge_nodes(self):
        """Edge geometry nodes of a curved mesh, [n_cells][6][3]."""
        a = np.empty((self.n_cells, 6, 3), np.float64)
        check(lib().fem_mesh_copy_edge_nodes(self.handle, a.ctypes.data))
        return a

    def input_cells(self):
        """Input index of every cell (meshes from arrays; identity otherwise)."""
        a = np.empty(self.n_cells, np.int64)
        check(lib().fem_mesh_copy_input_cells(self.handle, a.ctypes.data))
        return a

    def vertices(self):
        a = np.empty((self.n_vertices, 3), np.float64)
        check(lib().fem_mesh_copy_vertices(self.handle, a.ctypes.data))
        return a

    def cells(self):
        a = np.empty((self.n_cells, 4), np.int32)
        check(lib().fem_mesh_copy_cells(self.handle, a.ctypes.data))
        return a

    def neighbors(self):
        nb = np.empty((self.n_cells, 4), np.int32)
        nbf = np.empty((self.n_cells, 4), np.int8)
        check(lib().fem_mesh_copy_neighbors(self.handle, nb.ctypes.data, nbf.ctypes.data))
        return nb, nbf

    def cg_dofs(self, degree):
        n = C.c_int64()
        check(lib().fem_mesh_cg_dofs(self.handle, degree, C.byref(n), None, None))
        k = (degree + 1) * (degree + 2) * (degree + 3) // 6
        cd = np.empty((self.n_cells, k), np.int32)
        cm = np.empty(n.value, np.uint8)
        check(lib().fem_mesh_cg_dofs(self.handle, degree, C.byref(n), cd.ctypes.data, cm.ctypes.data))
        return cd, cm

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.fem_mesh_destroy(self.handle)
            self.handle = None


class Operator:
    """Matrix-free operator (fem_op); the drop-in for the reference's Operator."""

    def __init__(self, mesh, degree, kind="cg", precision="fp64", mass=1e5, n_components=None,
                 penalty=FEM_PENALTY_REFERENCE, partition=None, weak_boundary=False):
        """partition: a Partition of `mesh`; the operator is then that part's
        local operator on [owned | ghost] vectors (fem_op_create_part)."""
        self.mesh = mesh
        k = KINDS[kind] if isinstance(kind, str) else kind
        pr = PRECISIONS[precision] if isinstance(precision, str) else precision
        p = OpParams()
        p.mass_coefficient = mass
        p.n_components = n_components or (3 if k == FEM_HELMHOLTZ else 1)
        p.penalty = penalty
        p.weak_boundary = int(bool(weak_boundary))
        h = C.c_void_p()
        if partition is None:
            check(lib().fem_op_create(mesh.handle, degree, k, pr, C.byref(p), C.byref(h)))
        else:
            if (partition.degree, partition.kind) != (degree, k):
                raise FemError(FEM_ERR_ARG, "partition made for another degree or kind")
            check(lib().fem_op_create_part(partition.handle, pr, C.byref(p), C.byref(h)))
        self.partition = partition
        self.handle = h
        self.kind, self.precision, self.degree = k, pr, degree
        m = C.c_uint64()
        check(lib().fem_op_m(h, C.byref(m)))
        self._m = m.value
        dpc, nc, ncomp = C.c_int32(), C.c_int64(), C.c_int32()
        check(lib().fem_op_info(h, None, None, None, C.byref(dpc), C.byref(nc), C.byref(ncomp)))
        self.dofs_per_cell, self.n_cells, self.n_components = dpc.value, nc.value, ncomp.value

    @property
    def dtype(self):
        import torch
        return torch.float64 if self.precision == FEM_FP64 else torch.float32

    def m(self):
        return self._m

    def initialize_dof_vector(self):
        import torch
        return torch.zeros(self._m, dtype=self.dtype, device="cuda")

    def _check_vec(self, v):
        if not v.is_cuda or v.dtype != self.dtype or v.numel() != self._m or not v.is_contiguous():
            raise FemError(1, f"vector must be a contiguous CUDA {self.dtype} tensor of length {self._m}")

    def vmult(self, dst, src, stream=None):
        self._check_vec(dst)
        self._check_vec(src)
        check(lib().fem_op_vmult(self.handle, _ptr(dst), _ptr(src), _stream_ptr(stream)))

    def vmult_host(self, dsts, srcs, stream=None):
        """dsts[i] = A srcs[i] on vectors in host memory (fem_op_vmult_host):
        CPU tensors of the operator's dtype and length m (pinned memory lets
        the copies of consecutive vectors overlap).  Asynchronous on `stream`."""
        if len(dsts) != len(srcs) or not dsts:
            raise ValueError("vmult_host needs equal, non-empty lists of dst and src vectors")
        for v in list(dsts) + list(srcs):
            if v.device.type != "cpu" or v.dtype != self.dtype or v.numel() != self.m() or not v.is_contiguous():
                raise ValueError("vmult_host vectors must be contiguous CPU tensors of the operator's dtype and length")
        n = len(dsts)
        da = (C.c_void_p * n)(*[d.data_ptr() for d in dsts])
        sa = (C.c_void_p * n)(*[s.data_ptr() for s in srcs])
        check(lib().fem_op_vmult_host(self.handle, n, da, sa, _stream_ptr(stream)))

    def vmult_phase(self, dst, src, phase, stream=None):
        self._check_vec(dst)
        self._check_vec(src)
        check(lib().fem_op_vmult_phase(self.handle, _ptr(dst), _ptr(src), phase, _stream_ptr(stream)))

    def Tvmult(self, dst, src, stream=None):
        self._check_vec(dst)
        self._check_vec(src)
        check(lib().fem_op_Tvmult(self.handle, _ptr(dst), _ptr(src), _stream_ptr(stream)))

    def compute_inverse_diagonal(self, vec, stream=None):
        self._check_vec(vec)
        check(lib().fem_op_compute_inverse_diagonal(self.handle, _ptr(vec), _stream_ptr(stream)))

    def compute_diagonal(self, vec, stream=None):
        self._check_vec(vec)
        check(lib().fem_op_compute_diagonal(self.handle, _ptr(vec), _stream_ptr(stream)))

    def dof_map(self):
        a = np.empty((self.n_cells, self.dofs_per_cell * self.n_components), np.int32)
        check(lib().fem_op_copy_dof_map(self.handle, a.ctypes.data))
        return a

    def constrained(self):
        a = np.empty(self._m, np.uint8)
        check(lib().fem_op_copy_constrained(self.handle, a.ctypes.data))
        return a

    def support_points(self):
        a = np.empty((self._m // self.n_components, 3), np.float64)
        check(lib().fem_op_copy_support_points(self.handle, a.ctypes.data))
        return a

    def set_kernel_variant(self, variant):
        check(lib().fem_op_set_kernel_variant(self.handle, variant))

    def status(self):
        """Device-side status bits since the last call (0: every bounded wait completed)."""
        v = C.c_int32()
        check(lib().fem_op_status(self.handle, C.byref(v)))
        return v.value

    def autotune(self, reps=20, use_cache=True):
        """Time the kernel variants on this operator and keep the fastest
        (fem_op_autotune); returns {"variant", "cached", "us": [per variant]}."""
        return _autotune(lib().fem_op_autotune, self.handle, reps, use_cache)

    def work(self):
        f, b = C.c_double(), C.c_double()
        check(lib().fem_op_work(self.handle, C.byref(f), C.byref(b)))
        return f.value, b.value

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.fem_op_destroy(self.handle)
            self.handle = None


class CSRMatrix:
    """The CG operator assembled into a device CSR matrix (the reference's
    Trilinos SparseMatrix comparison, CG/cells_batched/application.cc:1944-1988):
    the cell matrices come from fem_op_element_matrices, constrained rows and
    columns are dropped and get a one on the diagonal (the operator's
    identity rows); vmult runs fem_csr_spmv."""

    def __init__(self, op):
        import torch
        if op.kind != FEM_CG:
            raise FemError(FEM_ERR_ARG, "CSRMatrix: CG operators only")
        K, n = op.dofs_per_cell, op.n_cells
        mats = torch.empty((n, K, K), dtype=op.dtype, device="cuda")
        check(lib().fem_op_element_matrices(op.handle, _ptr(mats), _stream_ptr(None)))
        dofs = torch.from_numpy(op.dof_map().astype(np.int64)).cuda()  # [n][K]
        free = ~torch.from_numpy(op.constrained().astype(bool)).cuda()
        rows = dofs[:, :, None].expand(n, K, K).reshape(-1)
        cols = dofs[:, None, :].expand(n, K, K).reshape(-1)
        vals = mats.reshape(-1)
        keep = free[rows] & free[cols]
        cidx = torch.nonzero(~free).reshape(-1)
        rows = torch.cat([rows[keep], cidx])
        cols = torch.cat([cols[keep], cidx])
        vals = torch.cat([vals[keep], torch.ones(len(cidx), dtype=op.dtype, device="cuda")])
        del mats, keep
        m = op.m()
        A = torch.sparse_coo_tensor(torch.stack([rows, cols]), vals, (m, m)).coalesce().to_sparse_csr()
        self.row_ptr = A.crow_indices().to(torch.int64).contiguous()
        self.col = A.col_indices().to(torch.int32).contiguous()
        self.val = A.values().contiguous()
        self.m, self.nnz, self.precision = m, int(self.val.numel()), op.precision

    def vmult(self, dst, src, stream=None):
        check(lib().fem_csr_spmv(self.m, _ptr(self.row_ptr), _ptr(self.col), _ptr(self.val), _ptr(src), _ptr(dst),
                                 self.precision, _stream_ptr(stream)))


class Partition:
    """Part `part` of `n_parts` of a mesh for one rank (fem_part): contiguous
    ranges of the hierarchical cell order; local vectors are [owned | ghost]
    entries (CG DoFs, DG cell blocks) with per-peer send / receive lists."""

    def __init__(self, mesh, degree, kind, n_parts, part, n_components=None):
        k = KINDS[kind] if isinstance(kind, str) else kind
        nc = n_components or (3 if k == FEM_HELMHOLTZ else 1)
        h = C.c_void_p()
        check(lib().fem_part_create(mesh.handle, degree, k, nc, n_parts, part, C.byref(h)))
        self.handle = h
        self.mesh, self.degree, self.kind, self.n_components = mesh, degree, k, nc
        self.n_parts, self.part = n_parts, part
        no, ng, ngl, cb, ce = (C.c_int64() for _ in range(5))
        npeer = C.c_int32()
        check(lib().fem_part_sizes(h, C.byref(no), C.byref(ng), C.byref(ngl), C.byref(cb), C.byref(ce),
                                   C.byref(npeer)))
        self.n_owned, self.n_ghost, self.n_global = no.value, ng.value, ngl.value
        self.cell_range = (cb.value, ce.value)
        self.global_index = np.empty(self.n_owned + self.n_ghost, np.int64)
        check(lib().fem_part_global_index(h, self.global_index.ctypes.data))
        self.peers = []  # (rank, send local indices, recv local indices)
        for i in range(npeer.value):
            r, ns, nr = C.c_int32(), C.c_int64(), C.c_int64()
            check(lib().fem_part_peer(h, i, C.byref(r), C.byref(ns), C.byref(nr)))
            snd = np.empty(ns.value, np.int64)
            rcv = np.empty(nr.value, np.int64)
            check(lib().fem_part_halo(h, i, snd.ctypes.data, rcv.ctypes.data))
            self.peers.append((r.value, snd, rcv))

    @property
    def m(self):
        return self.n_owned + self.n_ghost

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.fem_part_destroy(self.handle)
            self.handle = None


class Batch:
    """Several independent DG/Helmholtz operators applied in one launch per phase."""

    def __init__(self, ops):
        self.ops = list(ops)
        arr = (C.c_void_p * len(ops))(*[o.handle.value for o in ops])
        h = C.c_void_p()
        check(lib().fem_batch_create(arr, len(ops), C.byref(h)))
        self.handle = h

    def vmult(self, dsts, srcs, stream=None):
        n = len(self.ops)
        for o, d, s in zip(self.ops, dsts, srcs):
            o._check_vec(d)
            o._check_vec(s)
        da = (C.c_void_p * n)(*[d.data_ptr() for d in dsts])
        sa = (C.c_void_p * n)(*[s.data_ptr() for s in srcs])
        check(lib().fem_batch_vmult(self.handle, da, sa, _stream_ptr(stream)))

    def set_kernel_variant(self, variant):
        check(lib().fem_batch_set_kernel_variant(self.handle, variant))

    def autotune(self, reps=20, use_cache=True):
        """Time the kernel variants on the whole batch and keep the fastest."""
        return _autotune(lib().fem_batch_autotune, self.handle, reps, use_cache)

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.fem_batch_destroy(self.handle)
            self.handle = None


def _autotune(fn, handle, reps, use_cache):
    v, c = C.c_int32(), C.c_int32()
    us = (C.c_double * 8)()
    check(fn(handle, reps, int(bool(use_cache)), C.byref(v), C.byref(c), us))
    return {"variant": v.value, "cached": bool(c.value), "us": list(us)}


def set_autotune_cache(path):
    """Keep autotuning choices in a JSON-lines file across processes (None: memory only)."""
    check(lib().fem_autotune_cache(None if path is None else os.fsencode(path)))


def rhs_desc(modes, kind=FEM_RHS_PLANE_WAVES):
    """modes: list of (k(3), amp)."""
    d = RhsDesc()
    d.kind = kind
    d.n_modes = len(modes)
    for m, (k, a) in enumerate(modes):
        for j in range(3):
            d.k[m][j] = float(k[j])
        d.amp[m] = float(a)
    return d


def sine_modes_rhs(n_modes=8, seed=2, kmin=1.0, kmax=6.0):
    """f = sum of n_modes sin(k.x), k uniform in [kmin, kmax]^3 from numpy PCG64(seed)."""
    ks = np.random.default_rng(seed).uniform(kmin, kmax, (n_modes, 3))
    return rhs_desc([(k, 1.0) for k in ks])


def rhs(op, desc, dst=None, stream=None):
    dst = op.initialize_dof_vector() if dst is None else dst
    check(lib().fem_op_rhs(op.handle, C.byref(desc), _ptr(dst), _stream_ptr(stream)))
    return dst


def interpolate(op, desc, dst=None, stream=None):
    dst = op.initialize_dof_vector() if dst is None else dst
    check(lib().fem_op_interpolate(op.handle, C.byref(desc), _ptr(dst), _stream_ptr(stream)))
    return dst


class Multigrid:
    """Hybrid p/h/c multigrid on a CG or DG operator (fem_mg); MultigridPreconditioner's shape.
    DG: c_transfer=0 coarsens DG P_p .. P_1 then hands over to CG P_1 (phc);
    c_transfer=1 hands over at P_p (cph with FEM_MG_PH, chp with FEM_MG_HP);
    weak_cg_levels gives the CG levels weak boundary terms (the reference's)."""

    def __init__(self, fine_op, order=FEM_MG_PH, precision="fp32", smoother_degree=3, smoothing_range=20.0,
                 eig_iterations=10, eig_safety=1.2, coarse_n=4, use_graph=True, c_transfer=0, learned_steps=3,
                 tensor_cores=False, weak_cg_levels=False):
        p = MGParams()
        check(lib().fem_mg_params_default(C.byref(p)))
        p.order = order
        p.precision = PRECISIONS[precision] if isinstance(precision, str) else precision
        p.smoother_degree = smoother_degree
        p.smoothing_range = smoothing_range
        p.eig_iterations = eig_iterations
        p.eig_safety = eig_safety
        p.coarse_n = coarse_n
        p.use_graph = int(bool(use_graph))
        p.c_transfer = c_transfer
        p.learned_steps = learned_steps
        p.tensor_cores = int(bool(tensor_cores))
        p.weak_cg_levels = int(bool(weak_cg_levels))
        h = C.c_void_p()
        check(lib().fem_mg_create(fine_op.handle, C.byref(p), C.byref(h)))
        self.handle = h
        self.fine = fine_op
        self.precision = p.precision
        n = C.c_int32()
        check(lib().fem_mg_n_levels(h, C.byref(n)))
        self.n_levels = n.value

    def level_info(self, level):
        m, d, hx, lm = C.c_uint64(), C.c_int32(), C.c_int32(), C.c_double()
        check(lib().fem_mg_level_info(self.handle, level, C.byref(m), C.byref(d), C.byref(hx), C.byref(lm)))
        kd = C.c_int32()
        check(lib().fem_mg_level_kind(self.handle, level, C.byref(kd)))
        return {"m": m.value, "degree": d.value, "hexes": hx.value, "lambda_max": lm.value,
                "kind": {FEM_CG: "cg", FEM_DG: "dg"}.get(kd.value, kd.value)}

    def level_vector(self, level):
        import torch
        dt = torch.float64 if self.precision == FEM_FP64 else torch.float32
        return torch.zeros(self.level_info(level)["m"], dtype=dt, device="cuda")

    def vmult(self, dst, src, stream=None):
        """PreconditionMG::vmult: dst = V(src) (FP64 fine vectors)."""
        check(lib().fem_mg_vcycle(self.handle, _ptr(dst), _ptr(src), _stream_ptr(stream)))

    def level_vmult(self, level, dst, src, stream=None):
        check(lib().fem_mg_level_vmult(self.handle, level, _ptr(dst), _ptr(src), _stream_ptr(stream)))

    def smooth(self, level, x, b, zero_initial=True, stream=None):
        check(lib().fem_mg_smooth(self.handle, level, _ptr(x), _ptr(b), int(zero_initial), _stream_ptr(stream)))

    def prolongate_add(self, level, dst, src, stream=None):
        check(lib().fem_mg_prolongate_add(self.handle, level, _ptr(dst), _ptr(src), _stream_ptr(stream)))

    def restrict_add(self, level, dst, src, stream=None):
        check(lib().fem_mg_restrict_add(self.handle, level, _ptr(dst), _ptr(src), _stream_ptr(stream)))

    def coarse_solve(self, dst, src, stream=None):
        check(lib().fem_mg_coarse_solve(self.handle, _ptr(dst), _ptr(src), _stream_ptr(stream)))

    def set_learned_smoother(self, mlp, fallback=True):
        """Finest-level smoothing by a trained MLP (None: back to Chebyshev)."""
        self.mlp = mlp
        check(lib().fem_mg_set_learned_smoother(self.handle, mlp.handle if mlp is not None else None,
                                                int(bool(fallback))))

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.fem_mg_destroy(self.handle)
            self.handle = None


class SolverCG:
    """Preconditioned CG on an FP64 operator (fem_cg); SolverCG's shape."""

    def __init__(self, op, preconditioner=None, flexible=False):
        if isinstance(preconditioner, Multigrid):
            kind, mgh = FEM_PRECOND_MG, preconditioner.handle
        elif preconditioner == "jacobi":
            kind, mgh = FEM_PRECOND_JACOBI, None
        else:
            kind, mgh = FEM_PRECOND_NONE, None
        h = C.c_void_p()
        check(lib().fem_cg_create(op.handle, mgh, kind, int(flexible), C.byref(h)))
        self.handle = h
        self.op = op
        self.pre = preconditioner

    def solve(self, x, b, rtol=1e-8, max_iterations=1000, stream=None, raise_on_failure=False):
        info = SolveInfo()
        rc = lib().fem_cg_solve(self.handle, _ptr(x), _ptr(b), rtol, max_iterations, C.byref(info),
                                _stream_ptr(stream))
        if rc not in (FEM_OK, FEM_ERR_NOT_CONVERGED, FEM_ERR_BREAKDOWN, FEM_ERR_NONFINITE) or (
                raise_on_failure and rc != FEM_OK):
            check(rc)
        return {"iterations": info.iterations, "status": info.status, "r0": info.initial_residual,
                "rn": info.final_residual, "fallback_iteration": info.fallback_iteration}

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.fem_cg_destroy(self.handle)
            self.handle = None


def mlp_n_params():
    n = C.c_int32()
    check(lib().fem_mlp_n_params(C.byref(n)))
    return n.value


class MLP:
    """Learned finest-level smoother (fem_mlp): 29 -> 64 -> 64 -> 20, GELU, BF16 weights."""

    def __init__(self, seed=0, handle=None):
        if handle is None:
            handle = C.c_void_p()
            check(lib().fem_mlp_create(seed, C.byref(handle)))
        self.handle = handle

    @classmethod
    def load(cls, path):
        h = C.c_void_p()
        check(lib().fem_mlp_load(str(path).encode(), C.byref(h)))
        return cls(handle=h)

    def save(self, path):
        check(lib().fem_mlp_save(self.handle, str(path).encode()))

    def weights(self):
        w = np.empty(mlp_n_params(), np.float32)
        check(lib().fem_mlp_get_weights(self.handle, w.ctypes.data))
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == mlp_n_params()
        check(lib().fem_mlp_set_weights(self.handle, w.ctypes.data))

    def generate_and_train(self, **kw):
        p = MLPTrainParams()
        check(lib().fem_mlp_train_params_default(C.byref(p)))
        for k, v in kw.items():
            if k == "sizes":
                p.n_sizes = len(v)
                for i, s in enumerate(v):
                    p.sizes[i] = s
            else:
                setattr(p, k, v)
        info = MLPTrainInfo()
        check(lib().fem_mlp_generate_and_train(self.handle, C.byref(p), C.byref(info)))
        return {"samples": info.samples, "loss_first": info.loss_first, "loss_last": info.loss_last,
                "seconds": info.seconds}

    def train(self, X, Y, epochs=10, batch=256, lr=1e-3, seed=0):
        info = MLPTrainInfo()
        check(lib().fem_mlp_train(self.handle, _ptr(X), _ptr(Y), X.shape[0], epochs, batch, lr, seed,
                                  C.byref(info)))
        return {"loss_first": info.loss_first, "loss_last": info.loss_last}

    def gradient(self, X, Y, stream=None):
        import torch
        g = torch.zeros(mlp_n_params(), dtype=torch.float32, device="cuda")
        loss = C.c_double()
        check(lib().fem_mlp_gradient(self.handle, _ptr(X), _ptr(Y), X.shape[0], _ptr(g), C.byref(loss),
                                     _stream_ptr(stream)))
        return g, loss.value

    def forward(self, X, stream=None, tensor_cores=False):
        """O [n][20] = MLP(X [n][29]) (device float32 tensors); tensor_cores
        selects the tcgen05 kernel (BF16 activations)."""
        import torch
        O = torch.zeros((X.shape[0], 20), dtype=torch.float32, device="cuda")
        fn = lib().fem_mlp_forward_tc if tensor_cores else lib().fem_mlp_forward
        check(fn(self.handle, _ptr(X), _ptr(O), X.shape[0], _stream_ptr(stream)))
        return O

    def set_tensor_cores(self, on):
        """Smooth on the tensor cores (default) or on the CUDA cores."""
        check(lib().fem_mlp_set_tensor_cores(self.handle, int(bool(on))))

    def timed_out(self):
        """True if a tensor-core launch gave up on a bounded wait since the last call."""
        v = C.c_int32()
        check(lib().fem_mlp_status(self.handle, C.byref(v)))
        return bool(v.value)

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.fem_mlp_destroy(self.handle)
            self.handle = None
