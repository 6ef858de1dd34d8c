"""Domain-decomposed operators over torch.distributed (one rank per GPU).

The reference runs one MPI rank per core on a z-order partitioned
triangulation; MatrixFree::cell_loop / loop update the ghost values of src
before the cell and face integrals and add the ghost contributions of dst back
to their owners afterwards (compress(VectorOperation::add); DG/cells_batched/
application.cc:1303-1316, CG/cells_batched/application.cc:1154-1176), and
SolverCG reduces its dot products over all ranks.  Here:

  * ``Partition`` (simplexfem) cuts the hierarchical cell order into
    contiguous parts and gives every rank its [owned | ghost] local layout and
    per-peer send / receive lists;
  * ``HaloExchange`` moves the ghost entries with grouped point-to-point
    transfers (``batch_isend_irecv``: NCCL over NVLink / NVSwitch between GPUs,
    gloo between CPU ranks), one exchange per vmult;
  * ``DistributedOperator`` is the vmult of one rank: ghost update, the local
    GPU operator (fem_op_create_part), and for CG the compress;
  * ``solve_cg`` is the Jacobi-preconditioned CG of the reference's SolverCG
    on these vectors, with its dot products all-reduced (two reductions of
    1 and 2 scalars per step).

Every rank takes the same collective steps in the same order.
"""
import torch
import torch.distributed as dist

import simplexfem as sf


class HaloExchange:
    """Ghost update (owner -> ghost copy) and compress (ghost -> owner add) of
    a partition's local vectors.  Works on CUDA tensors with NCCL and on CPU
    tensors with gloo; the index lists live on `device`."""

    def __init__(self, partition, device, group=None):
        self.part = partition
        self.group = group
        self.peers = []
        for rank, send, recv in partition.peers:
            s = torch.as_tensor(send, dtype=torch.int64).to(device)
            r = torch.as_tensor(recv, dtype=torch.int64).to(device)
            self.peers.append((rank, s, r))

    def _exchange(self, v, out_idx, in_idx):
        """Send v[out_idx] to each peer, return what each peer sent (in_idx-sized)."""
        ops, bufs = [], []
        for rank, s, r in self.peers:
            src_idx, dst_idx = out_idx(s, r), in_idx(s, r)
            buf = torch.empty(len(dst_idx), dtype=v.dtype, device=v.device)
            if len(src_idx):
                ops.append(dist.P2POp(dist.isend, v.index_select(0, src_idx), rank, self.group))
            if len(dst_idx):
                ops.append(dist.P2POp(dist.irecv, buf, rank, self.group))
            bufs.append(buf)
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        return bufs

    def update_ghosts(self, v):
        """v[ghosts] = the owners' values (the reference's update_ghost_values)."""
        bufs = self._exchange(v, lambda s, r: s, lambda s, r: r)
        for (rank, s, r), buf in zip(self.peers, bufs):
            if len(r):
                v.index_copy_(0, r, buf)

    def compress_add(self, v, zero_ghosts=True):
        """v[owned] += the ghost copies held by other ranks (compress(add))."""
        bufs = self._exchange(v, lambda s, r: r, lambda s, r: s)
        for (rank, s, r), buf in zip(self.peers, bufs):
            if len(s):
                v.index_add_(0, s, buf)
        if zero_ghosts:
            v[self.part.n_owned:] = 0


class DistributedOperator:
    """One rank's share of the operator on a mesh partitioned over the ranks
    of `group` (default: the world).  Vectors are this rank's local vectors,
    [owned | ghost] of length ``m()``; the owned entries are the rank's rows."""

    def __init__(self, mesh, degree, kind="cg", precision="fp64", group=None, **op_kw):
        self.group = group
        rank = dist.get_rank(group)
        world = dist.get_world_size(group)
        nc = op_kw.get("n_components")
        self.partition = sf.Partition(mesh, degree, kind, world, rank, n_components=nc)
        self.op = sf.Operator(mesh, degree, kind, precision, partition=self.partition, **op_kw)
        self.halo = HaloExchange(self.partition, "cuda", group)
        self.kind = self.op.kind
        self.n_owned = self.partition.n_owned

    def m(self):
        return self.partition.m

    def initialize_dof_vector(self):
        return self.op.initialize_dof_vector()

    def vmult(self, dst, src, stream=None):
        """dst = A src on the owned rows; src's ghosts are refreshed first."""
        self.halo.update_ghosts(src)
        self.op.vmult(dst, src, stream)
        if self.kind == sf.FEM_CG:
            self.halo.compress_add(dst)

    def dots(self, *pairs):
        """Global dot products of pairs of local vectors (owned entries only),
        reduced over the ranks in one all-reduce."""
        n = self.n_owned
        d = torch.stack([torch.dot(a[:n].double(), b[:n].double()) for a, b in pairs])
        dist.all_reduce(d, group=self.group)
        return [float(v) for v in d.cpu()]

    def inverse_diagonal(self):
        """1 / diag(A) on the owned entries (CG: the local diagonals of the
        ranks sharing a DoF are added into its owner first)."""
        d = self.initialize_dof_vector()
        self.op.compute_diagonal(d)
        if self.kind == sf.FEM_CG:
            self.halo.compress_add(d)
        d[self.n_owned:] = 1.0
        return torch.where(d.abs() < 1e-10, torch.ones_like(d), 1.0 / d)

    def scatter(self, x_global):
        """This rank's local vector (owned and ghost entries) of a global vector."""
        idx = torch.as_tensor(self.partition.global_index, device=x_global.device)
        return x_global.index_select(0, idx).to(self.op.dtype)


def solve_cg(dop, x, b, rtol=1e-8, max_iterations=1000, jacobi=True):
    """Preconditioned CG (the reference's SolverCG with a point-Jacobi
    preconditioner) on the local vectors of a DistributedOperator; stops when
    ||r|| <= rtol ||b||.  Returns iterations and the final relative residual."""
    inv = dop.inverse_diagonal() if jacobi else None
    r = b.clone()
    ax = dop.initialize_dof_vector()
    dop.vmult(ax, x)
    r -= ax
    r[dop.n_owned:] = 0
    z = r * inv if jacobi else r.clone()
    p = z.clone()
    bb, rz, rr = dop.dots((b, b), (r, z), (r, r))
    bnorm, res = bb ** 0.5, rr ** 0.5
    it = 0
    while res > rtol * bnorm and it < max_iterations:
        dop.vmult(ax, p)
        (pap,) = dop.dots((p, ax))
        alpha = rz / pap
        x += alpha * p
        r -= alpha * ax
        r[dop.n_owned:] = 0
        z = r * inv if jacobi else r.clone()
        rz_new, rr = dop.dots((r, z), (r, r))
        p = z + (rz_new / rz) * p
        rz, res = rz_new, rr ** 0.5
        it += 1
    return {"iterations": it, "relative_residual": res / bnorm}
