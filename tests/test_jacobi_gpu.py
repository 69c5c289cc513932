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
