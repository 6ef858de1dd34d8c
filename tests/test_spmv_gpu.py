"""Assembled-matrix comparison: the CG operator as a device CSR matrix.

The reference times a Trilinos sparse matrix-vector product beside its
matrix-free vmult (CG/cells_batched/application.cc:1944-1988).  Here the cell
matrices of the GPU operator (fem_op_element_matrices) are assembled into a
CSR matrix with the operator's identity rows, and fem_csr_spmv must give the
matrix-free vmult: relative l2 <= 1e-12 in FP64 (and against the oracle),
<= 2e-6 in FP32.
"""
import numpy as np
import pytest

import oracle as orc
import simplexfem as sf
from util import rel_l2, seeded_src

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_csr_spmv_equals_matrix_free(cuda, p, precision):
    import torch
    mesh = sf.Mesh((6, 5, 7), jitter=0.1, seed=8)
    op = sf.Operator(mesh, p, "cg", precision)
    A = sf.CSRMatrix(op)
    cm = op.constrained().astype(bool)
    assert A.m == op.m() and A.nnz > op.m()
    x = seeded_src(op.m(), 9)
    src = torch.tensor(x, dtype=op.dtype, device="cuda")
    y_mf, y_sp = op.initialize_dof_vector(), op.initialize_dof_vector()
    op.vmult(y_mf, src)
    A.vmult(y_sp, src)
    torch.cuda.synchronize()
    tol = 1e-12 if precision == "fp64" else 2e-6
    assert rel_l2(y_sp.double().cpu().numpy(), y_mf.double().cpu().numpy()) <= tol
    if precision == "fp64":
        ref = orc.for_mesh(mesh, p, orc.CG).vmult(x)
        assert rel_l2(y_sp.cpu().numpy(), ref) <= 1e-12
    # constrained rows are identity rows
    assert np.array_equal(y_sp.double().cpu().numpy()[cm], src.double().cpu().numpy()[cm])


def test_element_matrices_rejected_for_dg(cuda):
    op = sf.Operator(sf.Mesh(2), 2, "dg")
    with pytest.raises(sf.FemError):
        sf.CSRMatrix(op)
