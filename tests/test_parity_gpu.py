"""GPU vmult parity against the CPU oracle, through the C ABI.

Tolerances: relative l2 <= 1e-12 for FP64 (the bar of the reference's own
"optimized vs generic" check, CG/cells_batched/application.cc:1937-1940, which
prints a difference that "should be 0"), <= 2e-6 for FP32 operators compared
with the FP64 oracle on the same (rounded) input.
"""
import numpy as np
import pytest

import oracle as orc
import simplexfem as sf
from util import dg_interpolate, rel_l2, seeded_src

pytestmark = pytest.mark.gpu

KIND = {"cg": orc.CG, "dg": orc.DG, "helmholtz": orc.HELMHOLTZ}
TOL = {"fp64": 1e-12, "fp32": 2e-6}


def run_product(op, x):
    import torch
    src = torch.tensor(x, dtype=op.dtype, device="cuda")
    dst = op.initialize_dof_vector()
    op.vmult(dst, src)
    torch.cuda.synchronize()
    return dst.double().cpu().numpy()


def oracle_input(op, x):
    """The FP64 value of the input the product actually sees."""
    return x.astype(np.float32).astype(np.float64) if op.precision == sf.FEM_FP32 else x


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("kind", ["cg", "dg", "helmholtz"])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_vmult_parity_small(cuda, p, kind, precision):
    mesh = sf.Mesh((5, 4, 3), jitter=0.1, seed=0)
    op = sf.Operator(mesh, p, kind, precision)
    o = orc.for_mesh(mesh, p, KIND[kind], n_components=op.n_components)
    assert o.n == op.m()
    x = seeded_src(op.m(), 1)
    y = run_product(op, x)
    ref = o.vmult(oracle_input(op, x))
    assert rel_l2(y, ref) <= TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("variant", [1, 2])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_cg_kernel_variants(cuda, p, variant, precision):
    """Thread-per-cell (1) and thread-per-hex (2, one atomic per distinct DoF of
    the hex's 6 tets) CG kernels against the oracle."""
    mesh = sf.Mesh((6, 5, 7), jitter=0.1, seed=3)
    op = sf.Operator(mesh, p, "cg", precision)
    op.set_kernel_variant(variant)
    x = seeded_src(op.m(), 1)
    y = run_product(op, x)
    ref = orc.for_mesh(mesh, p, orc.CG).vmult(oracle_input(op, x))
    assert rel_l2(y, ref) <= TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("shape", [(8, 8, 8), (8, 4, 12)])
def test_cg_cube_kernel(cuda, p, precision, shape):
    """Cube-block CG kernel (variant 3: 4x4x4 hexes per CTA, interior DoFs
    stored, cube-surface DoFs added atomically) against the oracle, with each
    of its DoF-reduction schedules (variants 5, 6, 7)."""
    mesh = sf.Mesh(shape, jitter=0.1, seed=5)
    op = sf.Operator(mesh, p, "cg", precision)
    ref = orc.for_mesh(mesh, p, orc.CG).vmult(oracle_input(op, seeded_src(op.m(), 2)))
    for v in (3, 5, 6, 7):
        op.set_kernel_variant(v)
        y = run_product(op, seeded_src(op.m(), 2))
        assert rel_l2(y, ref) <= TOL[precision], v


def test_cg_autotuner_times_the_cube_schedules(cuda):
    """CG autotuning times cell, hex and the three cube schedules; the winner
    still matches the oracle."""
    sf.set_autotune_cache(None)
    mesh = sf.Mesh((8, 8, 8), jitter=0.1, seed=5)
    op = sf.Operator(mesh, 2, "cg", "fp64")
    r = op.autotune(reps=3, use_cache=False)
    assert r["variant"] in (1, 2, 5, 6, 7)
    assert all(r["us"][v - 1] > 0 for v in (1, 2, 5, 6, 7)) and r["us"][2] == 0 and r["us"][3] == 0
    x = seeded_src(op.m(), 2)
    ref = orc.for_mesh(mesh, 2, orc.CG).vmult(oracle_input(op, x))
    assert rel_l2(run_product(op, x), ref) <= TOL["fp64"]


def test_config1_cg_p2_full_size(cuda):
    """16^3 x 6 tets, CG P2, jitter 0.1 (seed 0), src U[-1,1] (seed 1), FP64."""
    mesh = sf.Mesh(16, jitter=0.1, seed=0)
    op = sf.Operator(mesh, 2, "cg", "fp64")
    assert op.m() == 35937
    x = seeded_src(op.m(), 1)
    y = run_product(op, x)
    ref = orc.for_mesh(mesh, 2, orc.CG).vmult(x)
    assert rel_l2(y, ref) <= 1e-12


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_config2_dg_p3_full_size(cuda, precision):
    """32^3 x 6 tets, DG P3 SIPG, 3,932,160 DoFs, FP64 and FP32 vs the FP64 oracle."""
    mesh = sf.Mesh(32, jitter=0.1, seed=0)
    op = sf.Operator(mesh, 3, "dg", precision)
    assert op.m() == 3932160
    x = seeded_src(op.m(), 1)
    y = run_product(op, x)
    ref = orc.for_mesh(mesh, 3, orc.DG).vmult(oracle_input(op, x))
    assert rel_l2(y, ref) <= TOL[precision]


@pytest.mark.parametrize("kind", ["cg", "dg", "helmholtz"])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_diagonal_parity(cuda, p, kind):
    import torch
    mesh = sf.Mesh(3, jitter=0.1, seed=2)
    op = sf.Operator(mesh, p, kind, "fp64")
    d = op.initialize_dof_vector()
    op.compute_diagonal(d)
    ref = orc.for_mesh(mesh, p, KIND[kind], n_components=op.n_components).diagonal()
    assert rel_l2(d.cpu().numpy(), ref) <= 1e-12
    inv = op.initialize_dof_vector()
    op.compute_inverse_diagonal(inv)
    r = np.where(np.abs(ref) > 1e-10, 1.0 / ref, 1.0)
    assert rel_l2(inv.cpu().numpy(), r) <= 1e-12
    torch.cuda.synchronize()


def test_cg_constrained_rows_are_identity(cuda):
    mesh = sf.Mesh(4, jitter=0.1, seed=0)
    op = sf.Operator(mesh, 2, "cg")
    x = seeded_src(op.m(), 7)
    y = run_product(op, x)
    c = op.constrained().astype(bool)
    assert c.sum() > 0 and np.array_equal(y[c], x[c])


def test_dg_deterministic(cuda):
    mesh = sf.Mesh(6, jitter=0.1, seed=0)
    op = sf.Operator(mesh, 3, "dg")
    x = seeded_src(op.m(), 3)
    assert np.array_equal(run_product(op, x), run_product(op, x))


def test_repeated_vmults_stable(cuda):
    """100 back-to-back vmults (the reference's timing loop) give the same result."""
    import torch
    mesh = sf.Mesh(8, jitter=0.1, seed=0)
    op = sf.Operator(mesh, 3, "dg")
    src = torch.tensor(seeded_src(op.m(), 1), device="cuda")
    dst = op.initialize_dof_vector()
    op.vmult(dst, src)
    first = dst.clone()
    for _ in range(100):
        op.vmult(dst, src)
    torch.cuda.synchronize()
    assert torch.equal(first, dst)


def test_dg_linear_consistency_full_size(cuda):
    """Size-independent property at 32^3: interior cells annihilate linears."""
    import torch
    mesh = sf.Mesh(32, jitter=0.1, seed=0)
    op = sf.Operator(mesh, 3, "dg")
    u = dg_interpolate(mesh, 3, lambda X: 1.0 + 2 * X[:, 0] - 3 * X[:, 1] + 0.5 * X[:, 2])
    y = run_product(op, u).reshape(mesh.n_cells, -1)
    nb, _ = mesh.neighbors()
    inner = np.all(nb >= 0, axis=1)
    assert np.abs(y[inner]).max() < 1e-11 * np.abs(y).max()
    torch.cuda.synchronize()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_matches_single(cuda, precision):
    """Uneven Helmholtz problems in one launch equal their individual vmults."""
    import torch
    ops, srcs = [], []
    for i, n in enumerate([2, 3, 5, 4]):
        mesh = sf.Mesh(n, jitter=0.1, seed=i)
        op = sf.Operator(mesh, 2, "helmholtz", precision)
        ops.append(op)
        srcs.append(torch.tensor(seeded_src(op.m(), 100 + i), dtype=op.dtype, device="cuda"))
    b = sf.Batch(ops)
    outs = [o.initialize_dof_vector() for o in ops]
    b.vmult(outs, srcs)
    for o, s, d in zip(ops, srcs, outs):
        ref = o.initialize_dof_vector()
        o.vmult(ref, s)
        torch.cuda.synchronize()
        assert torch.equal(ref, d)
    # and one of them against the oracle
    o0 = orc.for_mesh(ops[2].mesh, 2, orc.HELMHOLTZ, n_components=3)
    x = srcs[2].double().cpu().numpy()
    assert rel_l2(outs[2].double().cpu().numpy(), o0.vmult(x)) <= TOL[precision]


def test_autotuner_picks_a_variant_and_caches_it(cuda, tmp_path):
    """The autotuner times the DG kernel variants, keeps the fastest, records it
    in the cache file, and a second operator of the same shape reuses it; the
    tuned operator still matches the oracle."""
    sf.set_autotune_cache(str(tmp_path / "tune.jsonl"))
    try:
        mesh = sf.Mesh((6, 5, 4), jitter=0.1, seed=0)
        op = sf.Operator(mesh, 3, "dg", "fp64")
        r = op.autotune(reps=5)
        assert r["variant"] in (1, 2, 3) and not r["cached"]
        assert all(t > 0 for t in r["us"][:5]) and r["us"][r["variant"] - 1] == min(r["us"][:5])
        op2 = sf.Operator(mesh, 3, "dg", "fp64")
        r2 = op2.autotune(reps=5)
        assert r2["cached"] and r2["variant"] == r["variant"]
        assert (tmp_path / "tune.jsonl").read_text().count("variant") == 1
        x = seeded_src(op.m(), 1)
        ref = orc.for_mesh(mesh, 3, orc.DG).vmult(x)
        assert rel_l2(run_product(op2, x), ref) <= 1e-12
        # batch of uneven Helmholtz problems
        import torch
        meshes = [sf.Mesh(n) for n in (3, 4, 5)]
        ops = [sf.Operator(m, 2, "helmholtz", "fp64") for m in meshes]
        b = sf.Batch(ops)
        rb = b.autotune(reps=3)
        assert rb["variant"] in (1, 2, 3)
        xs = [torch.tensor(seeded_src(o.m(), 7 + i), device="cuda") for i, o in enumerate(ops)]
        ys = [o.initialize_dof_vector() for o in ops]
        b.vmult(ys, xs)
        for o, x_, y_ in zip(ops, xs, ys):
            z = o.initialize_dof_vector()
            o.vmult(z, x_)
            torch.cuda.synchronize()
            assert rel_l2(y_.cpu().numpy(), z.cpu().numpy()) <= 1e-13
    finally:
        sf.set_autotune_cache(None)


@pytest.mark.parametrize("variant,shape", [(4, (6, 5, 7)), (8, (8, 8, 8)), (8, (8, 4, 12)), (8, (6, 5, 7))])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_cg_tf32_tensor_core_variant(cuda, p, variant, shape):
    """FP32 CG operator on the TF32 tensor cores: per cell (variant 4, one
    [128 cells x K] x [K x 6K] tcgen05 product per tile) and per cube (variant
    8, three tiles of 128 tets per 4x4x4-hex cube with the cube kernel's gather
    and reduction; on a mesh without whole cubes it runs as variant 4).  TF32
    keeps 10 mantissa bits: rel l2 <= 3e-3 against the FP64 oracle."""
    mesh = sf.Mesh(shape, jitter=0.1, seed=3)
    op = sf.Operator(mesh, p, "cg", "fp32")
    op.set_kernel_variant(variant)
    x = seeded_src(op.m(), 1)
    y = run_product(op, x)
    assert op.status() == 0
    ref = orc.for_mesh(mesh, p, orc.CG).vmult(oracle_input(op, x))
    assert rel_l2(y, ref) <= 3e-3
    with pytest.raises(sf.FemError):
        sf.Operator(mesh, p, "cg", "fp64").set_kernel_variant(variant)


@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5, 7, 9, 11])
@pytest.mark.parametrize("kind", ["dg", "helmholtz"])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_dg_kernel_variants(cuda, p, kind, variant):
    """Every DG / Helmholtz kernel shape (the autotuner's candidates) against
    the oracle, FP64.  On 360 cells most faces of the phase-split forms (7, 9)
    and of the prefetching form (11) cross a block boundary, so both
    neighbour paths (shared memory and the published cross-block traces) run."""
    mesh = sf.Mesh((5, 4, 3), jitter=0.1, seed=2)
    op = sf.Operator(mesh, p, kind, "fp64")
    op.set_kernel_variant(variant)
    x = seeded_src(op.m(), 4)
    y = run_product(op, x)
    ref = orc.for_mesh(mesh, p, KIND[kind], n_components=op.n_components).vmult(x)
    assert rel_l2(y, ref) <= 1e-12


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_dg_kernel_variants_config2_full_size(cuda, precision):
    """Every scalar DG kernel shape on the headline workload (DG P3, 32^3 x 6
    tets, src U[-1,1] seed 1) against the oracle."""
    mesh = sf.Mesh(32, jitter=0.1, seed=0)
    op = sf.Operator(mesh, 3, "dg", precision)
    x = seeded_src(op.m(), 1)
    ref = orc.for_mesh(mesh, 3, orc.DG).vmult(oracle_input(op, x))
    for v in (1, 2, 3, 4, 5, 7, 9, 11):
        op.set_kernel_variant(v)
        err = rel_l2(run_product(op, x), ref)
        assert err <= TOL[precision], (v, err)
    # the bulk-copy trace pass of the scalar forms reports no bounded-wait timeout
    assert op.status() == 0


@pytest.mark.parametrize("kind", ["dg", "helmholtz"])
def test_batch_many_right_hand_sides_one_operator(cuda, kind):
    """One operator listed several times in a batch applies it to several
    vectors in one launch (each repeat gets its own trace scratch); every
    result equals a separate vmult."""
    import torch
    mesh = sf.Mesh((5, 4, 3), jitter=0.1, seed=1)
    op = sf.Operator(mesh, 2, kind, "fp64")
    b = sf.Batch([op, op, op])
    xs = [torch.tensor(seeded_src(op.m(), 20 + i), device="cuda") for i in range(3)]
    ys = [op.initialize_dof_vector() for _ in range(3)]
    b.vmult(ys, xs)
    for x_, y_ in zip(xs, ys):
        z = op.initialize_dof_vector()
        op.vmult(z, x_)
        torch.cuda.synchronize()
        assert rel_l2(y_.cpu().numpy(), z.cpu().numpy()) <= 1e-13


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("kind,p", [("cg", 2), ("dg", 3)])
def test_vmult_on_host_vectors(cuda, kind, p, precision):
    """fem_op_vmult_host: five host vectors through the double-buffered
    copy-in / apply / copy-out pipeline (pinned and pageable memory, and a
    second call on another stream) give the device vmult of each (bit for bit
    for DG; CG adds with atomics, so only up to the order of the sums), and
    the FP64 result matches the oracle."""
    import torch
    mesh = sf.Mesh((6, 5, 4), jitter=0.1, seed=2)
    op = sf.Operator(mesh, p, kind, precision)
    xs = [seeded_src(op.m(), 30 + i) for i in range(5)]
    want = [run_product(op, x) for x in xs]
    for pinned, stream in ((True, None), (False, None), (True, torch.cuda.Stream())):
        hs = [torch.tensor(x, dtype=op.dtype) for x in xs]
        hd = [torch.full((op.m(),), float("nan"), dtype=op.dtype) for _ in xs]
        if pinned:
            hs = [h.pin_memory() for h in hs]
            hd = [h.pin_memory() for h in hd]
        op.vmult_host(hd, hs, stream)
        torch.cuda.synchronize()
        for h, w in zip(hd, want):
            if kind == "dg":
                assert np.array_equal(h.double().numpy(), w)
            else:
                assert rel_l2(h.double().numpy(), w) <= (1e-14 if precision == "fp64" else 1e-6)
    if precision == "fp64":
        ref = orc.for_mesh(mesh, p, KIND[kind]).vmult(xs[0])
        assert rel_l2(want[0], ref) <= TOL["fp64"]
    with pytest.raises(ValueError):
        op.vmult_host([torch.empty(op.m(), dtype=op.dtype)], [torch.empty(op.m() + 1, dtype=op.dtype)])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("kind,p", [("dg", 3), ("helmholtz", 2)])
def test_dg_vmult_on_unaligned_views(cuda, kind, p, precision):
    """DG / Helmholtz vmult on vectors that start one element into a larger
    buffer (not 16-byte aligned): the row staging falls back from 16-byte to
    value-by-value copies, and the result equals the vmult on aligned vectors
    bit for bit."""
    import torch
    mesh = sf.Mesh((5, 4, 3), jitter=0.1, seed=2)
    op = sf.Operator(mesh, p, kind, precision)
    x = torch.tensor(seeded_src(op.m(), 5), dtype=op.dtype, device="cuda")
    y = op.initialize_dof_vector()
    op.vmult(y, x)
    bx = torch.zeros(op.m() + 1, dtype=op.dtype, device="cuda")
    bx[1:] = x
    by = torch.zeros(op.m() + 1, dtype=op.dtype, device="cuda")
    op.vmult(by[1:], bx[1:])
    torch.cuda.synchronize()
    assert torch.equal(by[1:], y)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_dg_trace_pass_forms(cuda, p, precision):
    """The scalar DG trace pass takes bulk copies when every copy starts
    16-byte aligned and moves whole 16-byte units, else the form without bulk
    copies.  4x4x4 hexes: 384 cells, whole 128-cell blocks.  3x3x3 hexes:
    162 cells, a last block of 34 cells; in FP32 the metric rows start at
    648-byte offsets, so that pass runs without bulk copies.  Every case
    against the oracle, and no bounded-wait timeout reported."""
    for shape in ((4, 4, 4), (3, 3, 3)):
        mesh = sf.Mesh(shape, jitter=0.1, seed=3)
        op = sf.Operator(mesh, p, "dg", precision)
        x = seeded_src(op.m(), 7)
        ref = orc.for_mesh(mesh, p, orc.DG).vmult(oracle_input(op, x))
        err = rel_l2(run_product(op, x), ref)
        assert err <= TOL[precision], (shape, err)
        assert op.status() == 0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_cg_three_component_operator(cuda, p, precision):
    """CG vector Laplacian with 3 interleaved components (the reference's
    components-batched CG operator, CG/components_batched/application.cc:
    1025-1216): every component equals the scalar oracle on that component's
    values; constrained rows are identity rows; the diagonal repeats the
    scalar one."""
    import torch
    mesh = sf.Mesh((5, 4, 6), jitter=0.1, seed=12)
    op = sf.Operator(mesh, p, "cg", precision, n_components=3)
    o = orc.for_mesh(mesh, p, orc.CG)
    assert op.m() == 3 * o.n and op.n_components == 3
    x = seeded_src(op.m(), 13)
    y = run_product(op, x)
    xr = oracle_input(op, x)
    for comp in range(3):
        assert rel_l2(y[comp::3], o.vmult(xr[comp::3])) <= TOL[precision], comp
    cm = op.constrained().astype(bool)
    assert cm.sum() == 3 * o.constrained.sum()
    d = op.initialize_dof_vector()
    op.compute_diagonal(d)
    torch.cuda.synchronize()
    dd = d.double().cpu().numpy()
    for comp in range(3):
        assert rel_l2(dd[comp::3], o.diagonal()) <= TOL[precision]
    with pytest.raises(sf.FemError):
        sf.Multigrid(op)
