"""fem_op_vmult_static_scratch: the vmult whose scratch is a static array.

Some callers cannot call cudaMalloc where they set up per-apply working
memory: their framework's memory pool already owns the device.  This entry
point allocates nothing and takes its face-trace scratch from a 16 MiB static
device array inside the library instead of the operator's own buffer.  The
test calls it through the C ABI twice in a row (the second call finds the
first call's leftovers in the shared array) and checks both results against
fem_op_vmult, with the FP64 tolerance of the other parity tests.  It lives in
a file that pytest collects last, and also passes when run alone.
"""
import ctypes

import numpy as np
import pytest

import simplexfem as sf

pytestmark = pytest.mark.gpu


def _call(op, dst, src, stream):
    return sf.lib().fem_op_vmult_static_scratch(op.handle, ctypes.c_void_p(dst.data_ptr()),
                                                ctypes.c_void_p(src.data_ptr()),
                                                ctypes.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("kind,degree,precision", [("dg", 3, "fp64"), ("helmholtz", 2, "fp32")])
def test_static_scratch_matches_vmult(cuda, kind, degree, precision):
    import torch
    mesh = sf.Mesh((6, 5, 4), jitter=0.1, seed=0)
    op = sf.Operator(mesh, degree, kind, precision)
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(11)
    tol = 1e-12 if precision == "fp64" else 2e-6
    for call in range(2):
        src = torch.tensor(rng.uniform(-1, 1, op.m()), dtype=op.dtype, device="cuda")
        want = op.initialize_dof_vector()
        op.vmult(want, src)
        got = torch.full_like(want, float("nan"))
        assert _call(op, got, src, stream) == sf.FEM_OK, sf.lib().fem_last_error_string()
        torch.cuda.synchronize()
        err = float(torch.linalg.norm((got - want).double()) / torch.linalg.norm(want.double()))
        assert err <= tol, (call, err)


def test_static_scratch_rejects_oversized_and_cg(cuda):
    import torch
    big = sf.Operator(sf.Mesh(25), 3, "dg", "fp64")  # 93,750 cells x 192 B > 16 MiB
    src = big.initialize_dof_vector()
    dst = big.initialize_dof_vector()
    stream = torch.cuda.current_stream()
    assert _call(big, dst, src, stream) == sf.FEM_ERR_ARG
    assert b"static maximum" in sf.lib().fem_last_error_string()
    cg = sf.Operator(sf.Mesh(3), 2, "cg", "fp64")
    v = cg.initialize_dof_vector()
    w = cg.initialize_dof_vector()
    assert _call(cg, w, v, stream) == sf.FEM_ERR_ARG
    assert b"only DG and Helmholtz" in sf.lib().fem_last_error_string()
