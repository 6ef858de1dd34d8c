"""Partitioned GPU operators (fem_op_create_part) against the whole operator.

Every part's local operator runs on the one GPU, one after the other (none
waits on another); the ghost update and the CG compress between them follow
the partition's send / receive lists exactly as distributed.HaloExchange
moves them between ranks.  The owned rows of all parts together must equal
the single-operator vmult and the oracle (relative l2 <= 1e-12 in FP64, the
tolerance of the other parity tests), for 2, 3 and 4 parts.
"""
import numpy as np
import pytest
import torch

import oracle as orc
import simplexfem as sf
from util import rel_l2, seeded_src

pytestmark = pytest.mark.gpu

CASES = [("cg", 1, 1), ("cg", 2, 1), ("cg", 3, 1), ("dg", 3, 1), ("dg", 2, 1), ("helmholtz", 2, 3)]
OKIND = {"cg": orc.CG, "dg": orc.DG, "helmholtz": orc.HELMHOLTZ}


def partitioned_vmult(mesh, p, kind, nc, n_parts, x, precision="fp64", variant=0):
    parts = [sf.Partition(mesh, p, kind, n_parts, r, n_components=nc) for r in range(n_parts)]
    ops = [sf.Operator(mesh, p, kind, precision, partition=P) for P in parts]
    if variant:
        for o in ops:
            o.set_kernel_variant(variant)
    dt = ops[0].dtype
    xs = []
    for P in parts:
        v = torch.full((P.m,), float("nan"), dtype=dt, device="cuda")
        v[:P.n_owned] = torch.tensor(x[P.global_index[:P.n_owned]], dtype=dt, device="cuda")
        xs.append(v)
    # ghost update along the lists: part r's send to q fills q's receive from r
    for r, P in enumerate(parts):
        for q, snd, _ in P.peers:
            rcv = {a: c for a, _, c in parts[q].peers}[r]
            xs[q][torch.as_tensor(rcv, device="cuda")] = xs[r][torch.as_tensor(snd, device="cuda")]
    ys = [o.initialize_dof_vector() for o in ops]
    for o, a, y in zip(ops, xs, ys):
        assert o.m() == a.numel()
        o.vmult(y, a)
    torch.cuda.synchronize()
    if kind == "cg":
        # compress: the ghost contributions go back to their owners
        for r, P in enumerate(parts):
            for q, snd, _ in P.peers:
                rcv = {a: c for a, _, c in parts[q].peers}[r]
                ys[r].index_add_(0, torch.as_tensor(snd, device="cuda"), ys[q][torch.as_tensor(rcv, device="cuda")])
    out = np.zeros(parts[0].n_global)
    for P, y in zip(parts, ys):
        out[P.global_index[:P.n_owned]] = y[:P.n_owned].double().cpu().numpy()
    return out


@pytest.mark.parametrize("n_parts", [2, 3, 4])
@pytest.mark.parametrize("kind,p,nc", CASES)
def test_partitioned_vmult_equals_whole(cuda, kind, p, nc, n_parts):
    mesh = sf.Mesh((8, 8, 12), jitter=0.1, seed=1)
    whole = sf.Operator(mesh, p, kind, "fp64", n_components=nc)
    x = seeded_src(whole.m(), 3, whole.constrained() if kind == "cg" else None)
    y = partitioned_vmult(mesh, p, kind, nc, n_parts, x)
    src = torch.tensor(x, device="cuda")
    dst = whole.initialize_dof_vector()
    whole.vmult(dst, src)
    torch.cuda.synchronize()
    assert rel_l2(y, dst.cpu().numpy()) <= 1e-12
    ref = orc.for_mesh(mesh, p, OKIND[kind], n_components=nc).vmult(x)
    assert rel_l2(y, ref) <= 1e-12


@pytest.mark.parametrize("variant", [1, 2, 7, 9])
def test_partitioned_dg_kernel_variants(cuda, variant):
    """The DG kernel shapes on partitions (ghost cells at the end of the local
    cell order, faces to cells outside the local mesh)."""
    mesh = sf.Mesh((8, 8, 8), jitter=0.1, seed=2)
    x = seeded_src(mesh.n_cells * 20, 5)
    y = partitioned_vmult(mesh, 3, "dg", 1, 3, x, variant=variant)
    ref = orc.for_mesh(mesh, 3, orc.DG).vmult(x)
    assert rel_l2(y, ref) <= 1e-12


def test_partitioned_config2_fp32(cuda):
    """The headline mesh (DG P3 32^3) in 4 parts, FP32 operator."""
    mesh = sf.Mesh(32, jitter=0.1, seed=0)
    x = seeded_src(mesh.n_cells * 20, 1)
    y = partitioned_vmult(mesh, 3, "dg", 1, 4, x, precision="fp32")
    ref = orc.for_mesh(mesh, 3, orc.DG).vmult(x.astype(np.float32).astype(np.float64))
    assert rel_l2(y, ref) <= 2e-6
