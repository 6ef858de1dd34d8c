"""Hybrid multigrid and preconditioned CG on the GPU, against the CPU oracle.

The north-star bar for the solver is the same CG iteration count +-1 at the
same tolerance; the oracle is oracle/mg_oracle.py (assembled level matrices,
interpolation transfers, Chebyshev-Jacobi, direct coarse solve).
"""
import numpy as np
import pytest

import mg_oracle as mgo
import oracle as orc
import simplexfem as sf
from util import rel_l2

pytestmark = pytest.mark.gpu


def torch_vec(x, dtype="fp64"):
    import torch
    return torch.tensor(x, dtype=torch.float64 if dtype == "fp64" else torch.float32, device="cuda")


@pytest.mark.parametrize("order", [sf.FEM_MG_PH, sf.FEM_MG_HP])
def test_transfer_is_transpose(cuda, order):
    mesh = sf.Mesh(8)
    op = sf.Operator(mesh, 3, "cg")
    mg = sf.Multigrid(op, order=order, precision="fp64")
    rng = np.random.default_rng(0)
    for l in range(1, mg.n_levels):
        nf, nc = mg.level_info(l)["m"], mg.level_info(l - 1)["m"]
        xc, yf = torch_vec(rng.uniform(-1, 1, nc)), torch_vec(rng.uniform(-1, 1, nf))
        Pxc, Ryf = mg.level_vector(l), mg.level_vector(l - 1)
        mg.prolongate_add(l, Pxc, xc)
        mg.restrict_add(l, Ryf, yf)
        a, b = float(Pxc @ yf), float(xc @ Ryf)
        assert abs(a - b) <= 1e-12 * max(abs(a), 1.0), (l, a, b)


@pytest.mark.parametrize("p,order,prec", [(2, "ph", "fp64"), (3, "ph", "fp64"), (3, "ph", "fp32"),
                                          (3, "hp", "fp64"), (2, "ph", "fp32")])
def test_mg_cg_iterations_match_oracle(cuda, p, order, prec):
    n = 8
    mesh = sf.Mesh(n)
    op = sf.Operator(mesh, p, "cg")
    mg = sf.Multigrid(op, order=sf.FEM_MG_PH if order == "ph" else sf.FEM_MG_HP, precision=prec)
    b = sf.rhs(op, sf.sine_modes_rhs())
    x = op.initialize_dof_vector()
    res = sf.SolverCG(op, mg).solve(x, b, rtol=1e-8)
    assert res["status"] == sf.FEM_OK
    M = mgo.MGOracle(lambda k: sf.Mesh(k), n, p, order=order)
    top = M.levels[-1]
    _, its = mgo.pcg(lambda v: top.A @ v, b.cpu().numpy(), M.vcycle, 1e-8, 100)
    assert abs(res["iterations"] - its) <= 1, (res["iterations"], its)
    # the GPU solution satisfies the oracle's system
    xs = x.cpu().numpy()
    bb = b.cpu().numpy()
    assert np.linalg.norm(bb - top.A @ xs) <= 1.01e-8 * np.linalg.norm(bb)


def test_jacobi_cg_matches_oracle(cuda):
    mesh = sf.Mesh(6, jitter=0.1, seed=0)
    op = sf.Operator(mesh, 2, "cg")
    b = sf.rhs(op, sf.sine_modes_rhs())
    x = op.initialize_dof_vector()
    res = sf.SolverCG(op, "jacobi").solve(x, b, rtol=1e-8, max_iterations=500)
    assert res["status"] == sf.FEM_OK
    o = orc.for_mesh(mesh, 2, orc.CG)
    invd = 1.0 / o.diagonal()
    _, its = mgo.pcg(o.vmult, b.cpu().numpy(), lambda r: invd * r, 1e-8, 500)
    assert abs(res["iterations"] - its) <= 1, (res["iterations"], its)


@pytest.mark.parametrize("p", [2, 3])
def test_mms_convergence(cuda, p):
    """-Laplace u = 3 pi^2 prod sin(pi x_d) on the unit cube, u = prod sin(pi x_d)."""
    f = sf.rhs_desc([((np.pi,) * 3, 3 * np.pi ** 2)], kind=sf.FEM_RHS_SINE_PRODUCTS)
    u = sf.rhs_desc([((np.pi,) * 3, 1.0)], kind=sf.FEM_RHS_SINE_PRODUCTS)
    errs = []
    for n in (8, 16):
        op = sf.Operator(sf.Mesh(n), p, "cg")
        b = sf.rhs(op, f)
        x = op.initialize_dof_vector()
        res = sf.SolverCG(op, sf.Multigrid(op, precision="fp64")).solve(x, b, rtol=1e-12)
        assert res["status"] == sf.FEM_OK
        errs.append(float((x - sf.interpolate(op, u)).abs().max()))
    assert errs[0] / errs[1] > 2 ** (p + 1) * 0.75, errs


def test_vcycle_graph_matches_eager(cuda):
    import torch
    mesh = sf.Mesh(8)
    op = sf.Operator(mesh, 3, "cg")
    src = sf.rhs(op, sf.sine_modes_rhs())
    outs = []
    for graph in (True, False):
        mg = sf.Multigrid(op, precision="fp64", use_graph=graph)
        dst = op.initialize_dof_vector()
        mg.vmult(dst, src)
        mg.vmult(dst, src)
        torch.cuda.synchronize()
        outs.append(dst.cpu().numpy())
    assert rel_l2(outs[0], outs[1]) <= 1e-12


def test_solver_reports_failures(cuda):
    import torch
    mesh = sf.Mesh(4)
    op = sf.Operator(mesh, 2, "cg")
    b = sf.rhs(op, sf.sine_modes_rhs())
    x = op.initialize_dof_vector()
    cg = sf.SolverCG(op, "jacobi")
    r = cg.solve(x, b, rtol=1e-12, max_iterations=2)
    assert r["status"] == sf.FEM_ERR_NOT_CONVERGED and r["iterations"] == 2
    bad = b.clone()
    bad[int(torch.nonzero(bad)[0])] = float("nan")  # fault injected on the host side
    x.zero_()
    r = cg.solve(x, bad, rtol=1e-8)
    assert r["status"] == sf.FEM_ERR_NONFINITE


def test_rhs_matches_quadrature(cuda):
    """b_i = (f, phi_i) against a numpy quadrature with the oracle basis."""
    mesh = sf.Mesh(3, jitter=0.1, seed=4)
    op = sf.Operator(mesh, 2, "cg")
    # smooth modes: the library's p+3 point rule and the 9-point check rule
    # then agree to rounding, so any difference is a bug, not quadrature error
    desc = sf.sine_modes_rhs(n_modes=3, seed=9, kmin=0.2, kmax=1.0)
    b = sf.rhs(op, desc).cpu().numpy()
    cd, cm = mesh.cg_dofs(2)
    xv, cells = mesh.vertices(), mesh.cells()
    g, w = np.polynomial.legendre.leggauss(9)
    g, w = 0.5 * (g + 1), 0.5 * w
    ks = [np.array(desc.k[m][:]) for m in range(desc.n_modes)]
    ref = np.zeros(len(cm))
    for c in range(mesh.n_cells):
        v = xv[cells[c]]
        J = (v[1:] - v[0]).T
        det = abs(np.linalg.det(J))
        loc = np.zeros(10)
        for a, wa in zip(g, w):
            for bq, wb in zip(g, w):
                for cq, wc in zip(g, w):
                    xi = np.array([a, bq * (1 - a), cq * (1 - a) * (1 - bq)])
                    wt = wa * wb * wc * (1 - a) ** 2 * (1 - bq) * det
                    X = v[0] + J @ xi
                    fx = sum(np.sin(k @ X) for k in ks)
                    phi, _ = orc.basis(2, xi)
                    loc += wt * fx * phi
        for i in range(10):
            if not cm[cd[c, i]]:
                ref[cd[c, i]] += loc[i]
    assert rel_l2(b, ref) <= 1e-9


def test_config3_full_size(cuda):
    """64^3 x 6 tets, CG P3 (7,189,057 DoFs), 8 sine modes (seed 2), rel. residual 1e-8:
    mixed (FP32 levels) and all-FP64 MG reach it in the same iterations +-1, and the
    residual recomputed through vmult confirms it."""
    import torch
    mesh = sf.Mesh(64)
    op = sf.Operator(mesh, 3, "cg")
    assert op.m() == 7189057
    b = sf.rhs(op, sf.sine_modes_rhs())
    its = {}
    for prec in ("fp32", "fp64"):
        mg = sf.Multigrid(op, precision=prec, smoother_degree=3)
        x = op.initialize_dof_vector()
        res = sf.SolverCG(op, mg).solve(x, b, rtol=1e-8)
        assert res["status"] == sf.FEM_OK
        its[prec] = res["iterations"]
        r = op.initialize_dof_vector()
        op.vmult(r, x)
        torch.cuda.synchronize()
        assert float(torch.linalg.norm(b - r) / torch.linalg.norm(b)) <= 1.01e-8
        del mg
    assert abs(its["fp32"] - its["fp64"]) <= 1 and its["fp32"] <= 12, its


@pytest.mark.parametrize("p,c_transfer,order", [(2, 0, sf.FEM_MG_PH), (3, 0, sf.FEM_MG_PH),
                                                (3, 1, sf.FEM_MG_PH), (3, 1, sf.FEM_MG_HP)])
@pytest.mark.parametrize("weak", [False, True])
def test_dg_multigrid_iterations_match_oracle(cuda, p, c_transfer, order, weak):
    """DG (SIPG) P_p solved by CG with the p/c/h multigrid (phc: DG P_p .. P_1,
    CG P_1, h-levels; cph/chp: CG P_p right below DG P_p): iteration count to
    1e-8 within +-1 of the CPU oracle's multigrid on the same problem.  weak:
    the CG levels carry the reference's weak boundary terms and no constrained
    DoFs (DG/cells_batched/application_phc.cc:1737-1744,1799-1832)."""
    import torch
    n = 4
    mesh = sf.Mesh(n)
    op = sf.Operator(mesh, p, "dg")
    mg = sf.Multigrid(op, order=order, precision="fp64", coarse_n=2, c_transfer=c_transfer, weak_cg_levels=weak)
    kinds = [mg.level_info(l)["kind"] for l in range(mg.n_levels)]
    assert kinds[-1] == "dg" and kinds[0] == "cg"
    assert kinds.count("dg") == (p if c_transfer == 0 else 1)
    rng = np.random.default_rng(5)
    bh = rng.uniform(-1, 1, op.m())
    b = torch.tensor(bh, device="cuda")
    x = op.initialize_dof_vector()
    res = sf.SolverCG(op, mg).solve(x, b, rtol=1e-8, max_iterations=100)
    assert res["status"] == sf.FEM_OK, res
    M = mgo.DGMGOracle(lambda k: sf.Mesh(k), n, p, c_transfer=c_transfer,
                       order="ph" if order == sf.FEM_MG_PH else "hp", coarse_n=2, weak_cg=weak)
    top = M.levels[-1]
    _, its = mgo.pcg(lambda v: top.A @ v, bh, M.vcycle, 1e-8, 100)
    assert abs(res["iterations"] - its) <= 1, (res["iterations"], its)
    xs = x.cpu().numpy()
    assert np.linalg.norm(top.A @ xs - bh) <= 1.1e-8 * np.linalg.norm(bh)


def test_mg_with_tf32_tensor_core_levels(cuda):
    """Mixed multigrid whose FP32 CG levels run on the TF32 tensor cores reaches
    1e-8 (the outer CG stays FP64) within 2 iterations of the CUDA-core levels."""
    import torch
    mesh = sf.Mesh(16)
    op = sf.Operator(mesh, 3, "cg")
    b = sf.rhs(op, sf.sine_modes_rhs())
    its = {}
    for tc in (False, True):
        mg = sf.Multigrid(op, precision="fp32", tensor_cores=tc)
        x = op.initialize_dof_vector()
        r = sf.SolverCG(op, mg).solve(x, b, rtol=1e-8, max_iterations=100)
        assert r["status"] == sf.FEM_OK, r
        its[tc] = r["iterations"]
    assert its[True] <= its[False] + 2, its


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 5, 6, 7])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_cg_weak_boundary_operator(cuda, p, variant):
    """CG operator with weak (Nitsche) boundary terms and no constrained DoFs
    (fem_op_params.weak_boundary), every cell-kernel form plus the boundary
    kernel, and its diagonal, against the oracle's weak mode (FP64, 1e-12)."""
    import torch
    mesh = sf.Mesh((8, 8, 4), jitter=0.1, seed=6)
    op = sf.Operator(mesh, p, "cg", "fp64", weak_boundary=True)
    assert op.constrained().sum() == 0
    op.set_kernel_variant(variant)
    cd, cm = mesh.cg_dofs(p)
    o = orc.Oracle(mesh.vertices(), mesh.cells(), p, orc.CG, cell_dofs=cd, constrained=cm, weak_bc=True)
    x = np.random.default_rng(3).uniform(-1, 1, op.m())
    y = op.initialize_dof_vector()
    op.vmult(y, torch.tensor(x, device="cuda"))
    d = op.initialize_dof_vector()
    op.compute_diagonal(d)
    torch.cuda.synchronize()
    assert rel_l2(y.cpu().numpy(), o.vmult(x)) <= 1e-12
    assert rel_l2(d.cpu().numpy(), o.diagonal()) <= 1e-12
