"""Jacobi preconditioners (point: the reference's diagonal one; block: the
inverse of each cell's diagonal block) built on the device, checked against
the oracle, and their effect inside GMRES."""
import ctypes as C

import numpy as np
import pytest

import oracle
from conftest import rel_err

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("d,L,T,kind", [(2, 4, 2, "random"), (3, 3, 3, "advdiff"),
                                        (4, 3, 4, "advdiff")])
def test_block_and_point_apply_match_oracle(cuda, d, L, T, kind):
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(d, L, T, kind=kind, seed=5)
    dt = 0.05 if kind == "random" else 1e-3
    pntr, iA = op.row_ptr.astype(np.int32), op.iA()
    blocks = oracle.diagonal_blocks(d, 3, pntr, op.col, T, iA, op.vA)
    ts = 3 ** d
    inv = np.linalg.inv(np.eye(ts)[None] - dt * blocks)
    pc = oracle.point_jacobi_diag(d, 3, pntr, op.col, T, iA, op.vA)
    v = np.random.default_rng(7).uniform(-1, 1, op.N)
    expect_block = np.einsum("cij,cj->ci", inv, v.reshape(-1, ts)).ravel()
    expect_point = v / (1.0 - dt * pc)
    for mat in (op.kronmult_matrix(), op.kronmult_matrix(expanded=True)):
        z = torch.zeros(op.N, dtype=torch.float64, device="cuda")
        pb = ab.JacobiPreconditioner(mat, dt, kind="block")
        pb.apply(_dev(v), z)
        torch.cuda.synchronize()
        assert rel_err(z.cpu().numpy(), expect_block) < 1e-12
        pp = ab.JacobiPreconditioner(mat, dt, kind="point")
        pp.apply(_dev(v), z)
        torch.cuda.synchronize()
        assert rel_err(z.cpu().numpy(), expect_point) < 1e-14


def test_block_jacobi_gmres_fewer_iterations(cuda):
    """Block Jacobi inside (flexible) GMRES reaches the same FP64 residual
    as plain GMRES in fewer iterations, in FP64 and with the FP32 operator
    (iterative refinement); the point version converges too."""
    import asgard_b200 as ab
    import torch
    d, L, T, dt = 3, 6, 3, 4e-3
    op = ab.SparseGridOperator(d, L, T, kind="advdiff")
    mat = op.kronmult_matrix()
    b = _dev(np.random.default_rng(1).uniform(-1, 1, op.N))
    x0 = torch.zeros_like(b)
    plain = ab.simple_gmres_euler(dt, mat, x0, b, restart=50, max_iter=200,
                                  tol=1e-10, tol_mode="rel")
    assert plain.true_relres <= 1e-10
    res = {}
    for kind in ("block", "point"):
        pc = ab.JacobiPreconditioner(mat, dt, kind=kind)
        for prec in ("fp64", "fp32"):
            x = torch.zeros_like(b)
            info = ab.simple_gmres_euler(dt, mat, x, b, restart=50, max_iter=200,
                                         tol=1e-10, tol_mode="rel",
                                         precision=prec, precond=pc)
            assert info.status == 0
            assert info.true_relres <= 1e-10, (kind, prec, info)
            assert info.precond_calls > 0
            res[(kind, prec)] = info.iterations
    # the block preconditioner's gain (CPU study: 439 -> 192 iterations here)
    assert res[("block", "fp64")] < 0.7 * plain.iterations, (res, plain.iterations)
    assert ab.lib.asgk_device_status(1) == 0


def test_jacobi_errors(cuda):
    import asgard_b200 as ab
    # a singular diagonal block: one cell, identity factors, dt = 1 -> I - K = 0
    d, n, T = 1, 3, 1
    vA = np.eye(3).ravel(order="F")
    mat = ab.kronmult_matrix.from_csr(d, n, 1, 1, T, [0, 1], [0], [0], vA)
    with pytest.raises(ab.AsgkError):
        ab.JacobiPreconditioner(mat, 1.0, kind="block")
    with pytest.raises(ab.AsgkError):
        ab.JacobiPreconditioner(mat, 1.0, kind="point")
    # block inverses are limited to n^d <= 81
    op = ab.SparseGridOperator(5, 2, 2, kind="random")
    with pytest.raises(ab.AsgkError):
        ab.JacobiPreconditioner(op.kronmult_matrix(), 1e-3, kind="block")
    ab.JacobiPreconditioner(op.kronmult_matrix(), 1e-3, kind="point")
    with pytest.raises(ValueError):
        ab.JacobiPreconditioner(mat, 1e-3, kind="ilu")
    # non-square plans have no backward-Euler operator
    rect = ab.kronmult_matrix.from_csr(1, 3, 1, 2, 1, [0, 1], [1], [0], vA)
    with pytest.raises(ab.AsgkError):
        ab.JacobiPreconditioner(rect, 1e-3, kind="point")


def test_preconditioner_of_another_plan_is_refused(cuda):
    """A Jacobi preconditioner built on a smaller plan would index past the
    solve's vectors: the solve, the implicit loop and the IMEX loop refuse it
    before any kernel launches; the IMEX loop also refuses stage
    preconditioners built for other step sizes."""
    import torch
    import asgard_b200 as ab
    small = ab.SparseGridOperator(3, 3, 3, kind="advdiff")
    big = ab.SparseGridOperator(3, 4, 3, kind="advdiff")
    ms, mb = small.kronmult_matrix(), big.kronmult_matrix()
    dt = 1e-3
    pcs = {k: ab.JacobiPreconditioner(ms, dt, kind=k) for k in ("point", "block")}
    b = torch.ones(big.N, dtype=torch.float64, device="cuda")
    x = torch.zeros_like(b)
    torch.cuda.synchronize()
    for kind, pc in pcs.items():
        before = ab.launch_count()
        with pytest.raises(ab.AsgkError):
            ab.simple_gmres_euler(dt, mb, x, b, 10, 2, 1e-10, precond=pc)
        with pytest.raises(ab.AsgkError):
            ab.implicit_advance(dt, mb, x, 1, restart=10, max_iter=2, tol=1e-10,
                                precond=pc)
        with pytest.raises(ab.AsgkError):
            ab.imex_advance(dt, mb, mb, x, 1, restart=10, max_iter=2, tol=1e-10,
                            precond=(pc, None))
        assert ab.launch_count() == before, kind
    # right shape, wrong step: stage 1 inverts I - dt K, stage 2 I - dt/2 K
    p1 = ab.JacobiPreconditioner(mb, dt, kind="point")
    p2 = ab.JacobiPreconditioner(mb, dt / 2, kind="point")
    with pytest.raises(ab.AsgkError):
        ab.imex_advance(dt, mb, mb, x, 1, restart=10, max_iter=2, tol=1e-10,
                        precond=(p2, p1))
    ab.imex_advance(dt, mb, mb, x, 1, restart=10, max_iter=2, tol=1e-10,
                    precond=(p1, p2))
    # the learned preconditioner's base must fit the network's cells
    net = ab.LearnedPreconditioner(big)
    with pytest.raises(ab.AsgkError):
        net.set_base(pcs["point"])


@pytest.mark.parametrize("d,L,T", [(2, 6, 2), (3, 5, 3), (4, 4, 4), (4, 7, 4)])
def test_kron_block_jacobi_equals_dense_block(cuda, d, L, T):
    """The Kronecker-sum form of the cell-block inverse (eigendecompositions
    of the 3x3 factors) applies the same map as the dense inverse, and
    GMRES takes the same iterations with either."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(d, L, T, kind="advdiff")
    g = op.kronmult_matrix(mode="global")
    dt = 1e-3
    blk = ab.JacobiPreconditioner(g, dt, kind="block")
    kr = ab.JacobiPreconditioner(g, dt, kind="kron")
    v = torch.from_numpy(np.random.default_rng(d).uniform(-1, 1, op.N)).cuda()
    za, zb = torch.zeros_like(v), torch.zeros_like(v)
    blk.apply(v, za)
    kr.apply(v, zb)
    torch.cuda.synchronize()
    assert (torch.linalg.norm(za - zb) / torch.linalg.norm(za)).item() < 1e-12
    b = torch.from_numpy(np.random.default_rng(5).uniform(-1, 1, op.N)).cuda()
    its = []
    for pc in (blk, kr):
        for prec in ("fp64", "fp32"):
            x = torch.zeros_like(b)
            info = ab.simple_gmres_euler(dt, g, x, b, 50, 300, 1e-10, tol_mode="rel",
                                         precision=prec, precond=pc)
            assert info.status == 0 and info.true_relres <= 1e-10
            its.append(info.iterations)
    assert abs(its[0] - its[2]) <= 1 and abs(its[1] - its[3]) <= 2, its


def _cell_block(op, c):
    """K_cc = sum_t (x)_k A_{t,k} over cell c's own pair (dimension 0
    slowest, column-major factors)."""
    d, T, n = op.d, op.terms, 3
    iA = op.iA()
    p = [q for q in range(op.row_ptr[c], op.row_ptr[c + 1]) if op.col[q] == c][0]
    K = 0.0
    for t in range(T):
        m = np.ones((1, 1))
        for k in range(d):
            off = iA[(p * T + t) * d + k]
            m = np.kron(m, op.vA[off:off + n * n].reshape(n, n, order="F"))
        K = K + m
    return K


@pytest.mark.parametrize("d,L,T", [(5, 3, 5), (6, 2, 6)])
def test_kron_block_jacobi_beyond_dense_blocks(cuda, d, L, T):
    """d = 5, 6: the dense inverse is not built (n^d > 81), the Kronecker-sum
    form is; it is exact on each cell's block (checked against the oracle's
    blocks) and lowers the iteration count; pair plans and terms acting in
    several dimensions are refused."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(d, L, T, kind="advdiff")
    g = op.kronmult_matrix(mode="global")
    dt = 5e-4
    with pytest.raises(ab.AsgkError):
        ab.JacobiPreconditioner(g, dt, kind="block")
    kr = ab.JacobiPreconditioner(g, dt, kind="kron")
    # cell c's block times z_c must give back v_c
    v = np.random.default_rng(2).uniform(-1, 1, op.N)
    z = torch.zeros(op.N, dtype=torch.float64, device="cuda")
    kr.apply(torch.from_numpy(v).cuda(), z)
    torch.cuda.synchronize()
    zn, ts = z.cpu().numpy(), 3 ** d
    for c in (0, op.rows // 2, op.rows - 1):
        Dc = np.eye(ts) - dt * _cell_block(op, c)
        r = Dc @ zn[c * ts:(c + 1) * ts] - v[c * ts:(c + 1) * ts]
        assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(v[c * ts:(c + 1) * ts])
    b = torch.from_numpy(np.random.default_rng(6).uniform(-1, 1, op.N)).cuda()
    its = []
    for pc in (None, kr):
        x = torch.zeros_like(b)
        info = ab.simple_gmres_euler(dt, g, x, b, 50, 300, 1e-10, tol_mode="rel",
                                     precision="fp32", precond=pc)
        assert info.status == 0 and info.true_relres <= 1e-10
        its.append(info.iterations)
    assert its[1] < its[0], its
    with pytest.raises(ab.AsgkError):
        ab.JacobiPreconditioner(op.kronmult_matrix(), dt, kind="kron")
    r = ab.SparseGridOperator(2, 3, 2, kind="random")
    with pytest.raises(ab.AsgkError):
        ab.JacobiPreconditioner(r.kronmult_matrix(mode="global"), dt, kind="kron")


@pytest.mark.parametrize("d,L,T", [(1, 5, 2), (2, 5, 2), (3, 4, 3), (4, 3, 4),
                                   (5, 2, 4), (6, 2, 6)])
def test_line_jacobi_matches_oracle(cuda, d, L, T):
    """The line preconditioner (exact pencil solves along the dimensions with
    symmetric operators, chained) applies the oracle's dense-algebra
    definition (oracle.line_jacobi_apply) to FP64 accuracy; in GMRES its
    FP32 and FP64 forms reach the 1e-10 FP64 residual in fewer iterations
    than the cell-block inverse."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(d, L, T, kind="advdiff")
    g = op.kronmult_matrix(mode="global")
    dt = 1e-3
    line_dims = oracle.line_dimensions(d, L, T, op.vA)
    if not line_dims:
        with pytest.raises(ab.AsgkError):
            ab.JacobiPreconditioner(g, dt, kind="line")
        return
    ln = ab.JacobiPreconditioner(g, dt, kind="line")
    v = np.random.default_rng(d + 7).uniform(-1, 1, op.N)
    expect = oracle.line_jacobi_apply(d, L, op.table, T, op.vA, dt, v)
    vd = torch.from_numpy(v).cuda()
    z = torch.zeros_like(vd)
    ln.apply(vd, z)
    torch.cuda.synchronize()
    assert rel_err(z.cpu().numpy(), expect) < 1e-12
    assert np.array_equal(vd.cpu().numpy(), v)     # v only read
    b = torch.from_numpy(np.random.default_rng(5).uniform(-1, 1, op.N)).cuda()
    kr = ab.JacobiPreconditioner(g, dt, kind="kron")
    its = {}
    for name, pc in (("line", ln), ("kron", kr)):
        for prec in ("fp64", "fp32"):
            x = torch.zeros_like(b)
            info = ab.simple_gmres_euler(dt, g, x, b, 50, 300, 1e-10, tol_mode="rel",
                                         precision=prec, precond=pc)
            assert info.status == 0 and info.true_relres <= 1e-10, (name, prec, info)
            its[(name, prec)] = info.iterations
    assert its[("line", "fp64")] <= its[("kron", "fp64")], its
    assert its[("line", "fp32")] <= its[("kron", "fp32")] + 2, its
