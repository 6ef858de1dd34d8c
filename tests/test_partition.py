"""Domain decomposition on the host: partition lists and the halo exchange.

The reference partitions its triangulation over MPI ranks (z-order,
CG/cells_batched/application.cc:1773-1801) and exchanges ghosts inside
MatrixFree::loop (update_ghost_values / compress(add),
DG/cells_batched/application.cc:1303-1316).  These tests need no GPU:
  * the partition lists (simplexfem.Partition, host-only C++) cover every
    global entry exactly once as owned, and every send list matches the
    peer's receive list entry by entry;
  * 2 and 3 gloo ranks exchange ghosts with distributed.HaloExchange; each
    rank then applies the oracle to its own cells only (the stand-in for its
    local GPU operator), compresses, and its owned rows must equal the
    oracle's global vmult.  Tolerance 1e-12 (FP64).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as orc
import simplexfem as sf

KINDS = [("cg", 2, 1), ("cg", 3, 1), ("dg", 3, 1), ("helmholtz", 2, 3)]
OKIND = {"cg": orc.CG, "dg": orc.DG, "helmholtz": orc.HELMHOLTZ}


def _mesh(shape=(8, 8, 8)):
    return sf.Mesh(shape, jitter=0.1, seed=4)


@pytest.mark.parametrize("n_parts", [1, 2, 3, 5])
@pytest.mark.parametrize("kind,p,nc", KINDS)
def test_partition_lists(kind, p, nc, n_parts):
    mesh = _mesh((8, 6, 8))
    parts = [sf.Partition(mesh, p, kind, n_parts, r, n_components=nc) for r in range(n_parts)]
    n_global = parts[0].n_global
    owned = np.concatenate([P.global_index[:P.n_owned] for P in parts])
    assert len(owned) == n_global and np.array_equal(np.sort(owned), np.arange(n_global))
    # contiguous cell ranges
    assert parts[0].cell_range[0] == 0 and parts[-1].cell_range[1] == mesh.n_cells
    for a, b in zip(parts, parts[1:]):
        assert a.cell_range[1] == b.cell_range[0]
    owner = np.empty(n_global, np.int64)
    for r, P in enumerate(parts):
        owner[P.global_index[:P.n_owned]] = r
    for r, P in enumerate(parts):
        g = P.global_index
        assert np.all(owner[g[P.n_owned:]] != r)
        peers = {q: (s, rc) for q, s, rc in P.peers}
        for q, (s, rc) in peers.items():
            Q = parts[q]
            qs, qr = {x: (a, b) for x, a, b in Q.peers}[r]
            assert np.array_equal(g[s], Q.global_index[qr])       # r -> q ghost update
            assert np.array_equal(g[rc], Q.global_index[qs])      # q -> r ghost update
            assert np.all(np.diff(g[s]) > 0) and np.all(owner[g[rc]] == q)
        # every ghost is received from its owner
        got = np.concatenate([rc for _, _, rc in P.peers]) if P.peers else np.array([], np.int64)
        assert np.array_equal(np.sort(got), np.arange(P.n_owned, P.m))


def test_partition_cuts_at_cubes():
    """Parts of a mesh of 4x4x4-hex cubes are whole cubes (384 tets)."""
    mesh = _mesh((16, 8, 8))
    for n_parts in (2, 3, 4, 7):
        for r in range(n_parts):
            b, e = sf.Partition(mesh, 2, "cg", n_parts, r).cell_range
            assert b % 384 == 0 and (e % 384 == 0 or e == mesh.n_cells)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, kind, p, nc, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import distributed as fd
        mesh = _mesh()
        P = sf.Partition(mesh, p, kind, world, rank, n_components=nc)
        o = orc.for_mesh(mesh, p, OKIND[kind], n_components=nc)
        x = np.random.default_rng(11).uniform(-1, 1, P.n_global)
        if kind == "cg":
            cm = mesh.cg_dofs(p)[1].astype(bool)
            x[cm] = 0.0
        g = P.global_index
        local = torch.full((P.m,), float("nan"), dtype=torch.float64)
        local[:P.n_owned] = torch.from_numpy(x[g[:P.n_owned]])
        halo = fd.HaloExchange(P, "cpu")
        halo.update_ghosts(local)
        ghosts_ok = bool(torch.equal(local, torch.from_numpy(x[g])))
        # this rank's cells only, on its own local values
        xs = np.zeros(P.n_global)
        xs[g] = local.numpy()
        ys = np.zeros(P.n_global)
        o.vmult_cells(xs, ys, *P.cell_range)
        y = torch.from_numpy(ys[g].copy())
        if kind == "cg":
            y[P.n_owned:][torch.from_numpy(cm[g[P.n_owned:]])] = 0.0  # identity rows belong to the owner
            halo.compress_add(y)
        ref = o.vmult(x)[g[:P.n_owned]]
        err = float(np.linalg.norm(y[:P.n_owned].numpy() - ref) / max(np.linalg.norm(ref), 1e-300))
        out.put((rank, ghosts_ok, err))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("kind,p,nc", KINDS)
def test_gloo_halo_exchange_and_partitioned_vmult(kind, p, nc, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, kind, p, nc, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for rank, ghosts_ok, err in res:
        assert ghosts_ok, rank
        assert err <= 1e-12, (rank, err)
