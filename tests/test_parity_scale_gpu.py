"""GPU parity at the shapes the benchmarks run, against the CPU oracle.

The small-mesh parity tests (test_parity_gpu.py) give every CTA of the
persistent CG cube kernels at most one 4x4x4-hex cube, so the software
pipeline that prefetches the next cube (cp.async gather into the second
buffer, metric and DoF codes one cube ahead) never runs there.  These tests
use meshes with more cubes than the persistent grid can hold CTAs, the
32-problem Helmholtz batch at its own sizes (8^3 .. 40^3), and a sampled
check of the 128^3 CG P2 vmult.

Tolerances as in test_parity_gpu.py: relative l2 <= 1e-12 in FP64 (the
reference's "optimized vs generic should be 0" check,
CG/cells_batched/application.cc:1937-1940), <= 2e-6 for FP32 operators on the
rounded input, <= 3e-3 for the TF32 tensor-core cube kernel.
"""
import numpy as np
import pytest

import oracle as orc
import simplexfem as sf
from util import rel_l2, seeded_src

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 2e-6}


def run_product(op, x):
    import torch
    src = torch.tensor(x, dtype=op.dtype, device="cuda")
    dst = op.initialize_dof_vector()
    op.vmult(dst, src)
    torch.cuda.synchronize()
    return dst.double().cpu().numpy()


def rounded(op, x):
    return x.astype(np.float32).astype(np.float64) if op.precision == sf.FEM_FP32 else x


# 48^3 hexes = 1,728 cubes and 40 x 48 x 44 = 1,320 cubes.  The persistent
# grid is min(cubes, SMs x resident CTAs); a 384-thread CTA allows at most 5
# per SM (2,048 threads), i.e. at most 740 CTAs on 148 SMs, so every CTA runs
# at least one pipelined cube switch.
MULTI_CUBE_SHAPES = [(48, 48, 48), (40, 48, 44)]


@pytest.fixture(scope="module")
def multi_cube_meshes():
    return {s: sf.Mesh(s, jitter=0.1, seed=9) for s in MULTI_CUBE_SHAPES}


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("shape", MULTI_CUBE_SHAPES)
def test_cube_kernel_pipelined_path(cuda, multi_cube_meshes, shape, p, precision):
    """Cube kernel (variant 3 and its reduce schedules 5, 6, 7) with several
    cubes per persistent CTA, against the oracle."""
    mesh = multi_cube_meshes[shape]
    op = sf.Operator(mesh, p, "cg", precision)
    assert mesh.n_cells // 384 > 740
    x = seeded_src(op.m(), 4, op.constrained())
    ref = orc.for_mesh(mesh, p, orc.CG).vmult(rounded(op, x))
    for v in (3, 5, 6, 7):
        op.set_kernel_variant(v)
        err = rel_l2(run_product(op, x), ref)
        assert err <= TOL[precision], (v, err)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_cube_tc_kernel_pipelined_path(cuda, multi_cube_meshes, p):
    """TF32 tensor-core cube kernel (variant 8) with several cubes per CTA."""
    mesh = multi_cube_meshes[(48, 48, 48)]
    op = sf.Operator(mesh, p, "cg", "fp32")
    op.set_kernel_variant(8)
    x = seeded_src(op.m(), 4, op.constrained())
    ref = orc.for_mesh(mesh, p, orc.CG).vmult(rounded(op, x))
    err = rel_l2(run_product(op, x), ref)
    assert err <= 3e-3, err
    assert op.status() == 0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_config4_batch_at_its_own_sizes(cuda, precision):
    """The 32-problem Helmholtz batch (DG P2 x 3 components, n_i = 8 +
    floor(32 i / 31) hexes per direction, src_i ~ U[-1,1] from seed 100 + i),
    applied in one batched launch per pass: every problem equals its own
    vmult bit for bit, and the smallest (8^3) and largest (40^3) problems
    match the oracle."""
    import torch
    sizes = [8 + (32 * i) // 31 for i in range(32)]
    meshes = [sf.Mesh(n) for n in sizes]
    ops = [sf.Operator(m, 2, "helmholtz", precision) for m in meshes]
    xs = [seeded_src(o.m(), 100 + i) for i, o in enumerate(ops)]
    srcs = [torch.tensor(x, dtype=o.dtype, device="cuda") for x, o in zip(xs, ops)]
    outs = [o.initialize_dof_vector() for o in ops]
    b = sf.Batch(ops)
    for variant in (0, 1, 4):
        if variant:
            b.set_kernel_variant(variant)
        b.vmult(outs, srcs)
        torch.cuda.synchronize()
        for i in (0, 31):
            o = orc.for_mesh(meshes[i], 2, orc.HELMHOLTZ, n_components=3)
            err = rel_l2(outs[i].double().cpu().numpy(), o.vmult(rounded(ops[i], xs[i])))
            assert err <= TOL[precision], (variant, sizes[i], err)
        for i in range(0, 32, 5):
            ref = ops[i].initialize_dof_vector()
            ops[i].set_kernel_variant(variant)
            ops[i].vmult(ref, srcs[i])
            torch.cuda.synchronize()
            assert torch.equal(ref, outs[i]), (variant, sizes[i])


def test_config1L_sampled_rows(cuda):
    """CG P2 on 128^3 x 6 tets (16,974,593 DoFs, jitter 0.1h seed 0, src
    U[-1,1] seed 1 zeroed at constrained DoFs), FP64, the benchmark's default
    kernel.  The oracle applies three slices of 150,000 cells each; every
    unconstrained DoF whose cells all lie inside a slice gets its full row
    there, and those rows are compared with the GPU result."""
    mesh = sf.Mesh(128, jitter=0.1, seed=0)
    op = sf.Operator(mesh, 2, "cg", "fp64")
    assert op.m() == 16974593
    cm = op.constrained()
    x = seeded_src(op.m(), 1, cm)
    y = run_product(op, x)
    cd, cm2 = mesh.cg_dofs(2)
    assert np.array_equal(cm, cm2)
    o = orc.Oracle(mesh.vertices(), mesh.cells(), 2, orc.CG, cell_dofs=cd, constrained=cm)
    touches = np.bincount(cd.ravel(), minlength=op.m())
    free = cm == 0
    checked = 0
    for c0 in (0, mesh.n_cells // 2 - 75_000, mesh.n_cells - 150_000):
        c1 = c0 + 150_000
        dst = np.zeros(op.m())
        o.vmult_cells(x, dst, c0, c1)
        inside = np.bincount(cd[c0:c1].ravel(), minlength=op.m())
        rows = (inside == touches) & (inside > 0) & free
        assert rows.sum() > 100_000
        checked += int(rows.sum())
        assert rel_l2(y[rows], dst[rows]) <= 1e-12
    assert checked > 300_000
