"""The implicit time loop (GMRES branch of the reference's implicit_advance,
src/time_advance.cpp:308-470) with the state resident on the device,
checked step by step against the oracle's GMRES run in the same loop."""
import numpy as np
import pytest

import oracle
from conftest import rel_err

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _oracle_loop(op, dt, x, forcing, steps, restart, max_outer, tol):
    """x_{k+1} solves (I - dt K) x_{k+1} = x_k + dt f_k from the initial
    guess x_k + dt f_k (the reference's fx(x) copy)."""
    pntr = op.row_ptr.astype(np.int32)
    iA = op.iA()
    its = []
    for k in range(steps):
        f = None if forcing is None else (forcing if forcing.ndim == 1 else forcing[k])
        b = x + dt * f if f is not None else x.copy()
        x = b.copy()
        _, it = oracle.gmres_euler(op.d, 3, pntr, op.col, op.terms, iA, op.vA, dt,
                                   x, b, restart, max_outer, tol)
        its.append(it)
    return x, its


@pytest.mark.parametrize("per_step", [False, True])
def test_implicit_advance_matches_oracle_loop(cuda, per_step):
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(3, 4, 3, kind="advdiff")
    mat = op.kronmult_matrix()
    dt, steps = 1e-2, 5
    rng = np.random.default_rng(11)
    x0 = rng.uniform(-1, 1, op.N)
    forcing = rng.uniform(-1, 1, (steps, op.N) if per_step else op.N)
    expect, its = _oracle_loop(op, dt, x0.copy(), forcing, steps, 20, 50, 1e-12)
    x = _dev(x0)
    infos = ab.implicit_advance(dt, mat, x, steps, forcing=_dev(forcing),
                                restart=20, max_iter=50, tol=1e-12)
    torch.cuda.synchronize()
    assert len(infos) == steps
    for info, it in zip(infos, its):
        assert info.status == 0 and info.error <= 1e-12
        assert abs(info.iterations - it) <= 1
    assert rel_err(x.cpu().numpy(), expect) < 1e-10


def test_implicit_advance_preconditioned_mixed_precision(cuda):
    """Block Jacobi + FP32 operator in FP64 refinement (relative 1e-10 per
    step) reaches the FP64 plain loop's state; a global-form plan too."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(3, 5, 3, kind="advdiff")
    dt, steps = 4e-3, 4
    rng = np.random.default_rng(3)
    x0 = rng.uniform(-1, 1, op.N)
    f = _dev(rng.uniform(-1, 1, op.N))
    pm = op.kronmult_matrix()
    xr = _dev(x0)
    ab.implicit_advance(dt, pm, xr, steps, forcing=f, restart=50, max_iter=200,
                        tol=1e-12, tol_mode="rel")
    for mat in (pm, op.kronmult_matrix(mode="global")):
        pc = ab.JacobiPreconditioner(mat, dt, kind="block")
        x = _dev(x0)
        infos = ab.implicit_advance(dt, mat, x, steps, forcing=f, restart=50,
                                    max_iter=200, tol=1e-10, tol_mode="rel",
                                    precision="fp32", precond=pc)
        torch.cuda.synchronize()
        assert all(i.status == 0 and i.true_relres <= 1e-10 for i in infos)
        assert (torch.linalg.norm(x - xr) / torch.linalg.norm(xr)).item() < 1e-8


def test_implicit_advance_no_forcing_and_errors(cuda):
    """Without forcing the loop is x_{k+1} = (I - dt K)^-1 x_k; a solve that
    stops short of the tolerance is reported in its step's status and the
    loop goes on (as the reference's); bad arguments raise."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(2, 4, 2, kind="advdiff")
    mat = op.kronmult_matrix()
    dt = 1e-2
    x0 = np.random.default_rng(5).uniform(-1, 1, op.N)
    expect, _ = _oracle_loop(op, dt, x0.copy(), None, 3, 20, 50, 1e-12)
    x = _dev(x0)
    ab.implicit_advance(dt, mat, x, 3, restart=20, max_iter=50, tol=1e-12)
    torch.cuda.synchronize()
    assert rel_err(x.cpu().numpy(), expect) < 1e-10
    short = ab.implicit_advance(dt, mat, _dev(x0), 3, restart=2, max_iter=1,
                                tol=1e-14)
    assert len(short) == 3
    assert all(i.status == 6 and i.iterations == 3 for i in short)
    with pytest.raises(ValueError):
        ab.implicit_advance(dt, mat, _dev(x0), 3,
                            forcing=_dev(np.zeros((2, op.N))))
    assert ab.implicit_advance(dt, mat, _dev(x0), 0) == []
