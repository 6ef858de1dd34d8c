"""GPU operators on unstructured meshes and hand-computed penalty values.

* Operators on a mesh from arrays (vertices relabelled, cells shuffled,
  each cell's vertices permuted, then Morton-reordered) against the oracle on
  the same arrays: FP64 relative l2 <= 1e-12.
* Known-answer tests of the interior-face penalty on a hand-built pair of
  tetrahedra, computed here from the geometry alone (independent of the
  library and of the oracle).  With u = 1 on cell A and 0 on cell B (DG P1),
  every gradient vanishes and the basis sums to one on each cell, so
      sum over B's DoFs of (A u) = -sigma_F |F|,
      sum over A's DoFs of (A u) =  sigma_F |F| + sum_boundary 2 sigma_b |F_b| (+ m |A|),
  where F is the shared face.  The SIPG operator uses
  sigma = (p+1)(p+3)/3 max(tau_A, tau_B), tau = (sum_f w_f |F_f|) / |K| with
  w = 1 on boundary faces and 1/2 on interior ones
  (DG/cells_batched/application.cc:1191-1245); the Helmholtz operator uses
  sigma = (p+1)(p+3)/3 * 1/2 (1/h_A + 1/h_B), h = 3 |K| / |F| the height
  over the face, i.e. the reading of |(n J^-1)[dim-1]| as the inverse length
  normal to the face (application_helmholtz.cc:694-701, 1329-1333).
"""
import numpy as np
import pytest

import oracle as orc
import simplexfem as sf
from test_mesh_input import scrambled
from util import rel_l2, seeded_src

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,p,nc", [("cg", 1, 1), ("cg", 2, 1), ("cg", 3, 1), ("dg", 1, 1), ("dg", 2, 1),
                                       ("dg", 3, 1), ("helmholtz", 2, 3)])
def test_operator_on_unstructured_mesh(cuda, kind, p, nc):
    import torch
    m0 = sf.Mesh((6, 5, 7), jitter=0.15, seed=21)
    x2, c2, _ = scrambled(m0, seed=9)
    mesh = sf.Mesh.from_arrays(x2, c2, reorder=True)
    okind = {"cg": orc.CG, "dg": orc.DG, "helmholtz": orc.HELMHOLTZ}[kind]
    op = sf.Operator(mesh, p, kind, "fp64", n_components=nc)
    x = seeded_src(op.m(), 6, op.constrained() if kind == "cg" else None)
    dst = op.initialize_dof_vector()
    op.vmult(dst, torch.tensor(x, device="cuda"))
    torch.cuda.synchronize()
    ref = orc.for_mesh(mesh, p, okind, n_components=nc).vmult(x)
    assert rel_l2(dst.cpu().numpy(), ref) <= 1e-12


def _tet_pair():
    # A = (0,1,2,3) above the shared face (0,1,2), B = (0,1,2,4) below it
    x = np.array([[0.0, 0.0, 0.0], [1.1, 0.1, 0.0], [0.2, 0.9, 0.05], [0.3, 0.25, 0.8], [0.4, 0.3, -0.5]])
    cells = np.array([[0, 1, 2, 3], [0, 1, 2, 4]], np.int32)
    return x, cells


def _vol(x, c):
    return abs(np.linalg.det(x[c[1:]] - x[c[0]])) / 6.0


def _area(x, f):
    return 0.5 * np.linalg.norm(np.cross(x[f[1]] - x[f[0]], x[f[2]] - x[f[0]]))


def _faces(c):
    return [[c[j] for j in range(4) if j != i] for i in range(4)]


@pytest.mark.parametrize("kind", ["dg", "helmholtz"])
def test_penalty_known_answer_on_a_tet_pair(cuda, kind):
    import torch
    x, cells = _tet_pair()
    mesh = sf.Mesh.from_arrays(x, cells, reorder=False)
    assert mesh.n_interior_faces == 1 and mesh.n_boundary_faces == 6
    mass = 7.0
    op = sf.Operator(mesh, 1, kind, "fp64", mass=mass, n_components=1)
    p, factor = 1, (1 + 1) * (1 + 3) / 3.0
    shared = [0, 1, 2]
    F = _area(x, shared)
    vol = [_vol(x, c) for c in cells]
    bnd = [[f for f in _faces(c) if sorted(f) != shared] for c in cells]
    if kind == "dg":
        tau = [(0.5 * F + sum(_area(x, f) for f in bnd[k])) / vol[k] for k in range(2)]
        sigma_F = factor * max(tau)
        sigma_b = [[factor * tau[0]] * 3, [factor * tau[1]] * 3]
    else:
        h = [3.0 * vol[k] / F for k in range(2)]
        sigma_F = factor * 0.5 * (1.0 / h[0] + 1.0 / h[1])
        sigma_b = [[factor * _area(x, f) / (3.0 * vol[k]) for f in bnd[k]] for k in range(2)]
    u = np.zeros(op.m())
    u[:4] = 1.0  # cell A is first (input order kept)
    y = op.initialize_dof_vector()
    op.vmult(y, torch.tensor(u, device="cuda"))
    torch.cuda.synchronize()
    y = y.cpu().numpy()
    want_B = -sigma_F * F
    want_A = sigma_F * F + sum(2.0 * s * _area(x, f) for s, f in zip(sigma_b[0], bnd[0]))
    if kind == "helmholtz":
        want_A += mass * vol[0]
    assert abs(y[4:].sum() - want_B) <= 1e-12 * abs(want_B)
    assert abs(y[:4].sum() - want_A) <= 1e-12 * abs(want_A)
