"""The oracle's IMEX step (the reference's imex_advance,
src/time_advance.cpp:477-990, over the oracle kronmult and GMRES) against a
dense restatement: explicit SSP-RK2 stages and exact backward-Euler solves."""
import numpy as np
import pytest

import oracle
from conftest import rel_err


def _op(d, level, terms, kind, nu, seed):
    from asgard_b200.operators import SparseGridOperator
    op = SparseGridOperator(d, level, terms, kind=kind, nu=nu, seed=seed)
    return op, (op.row_ptr.astype(np.int32), op.col, op.terms, op.iA(), op.vA.copy())


def _dense(op, t):
    pntr, indx, terms, iA, vA = t
    N = op.N
    A = np.zeros((N, N))
    for j in range(N):
        e = np.zeros(N)
        e[j] = 1.0
        y = np.zeros(N)
        oracle.kronmult(op.d, 3, pntr, indx, terms, iA, vA, 1.0, e, 0.0, y)
        A[:, j] = y
    return A


@pytest.mark.parametrize("with_implicit", [False, True])
def test_oracle_imex_matches_dense_restatement(with_implicit):
    ope, E = _op(2, 3, 2, "advdiff", 0.1, 0)
    opi, I_ = _op(2, 3, 2, "advdiff", 0.5, 1)
    dt, steps = 2e-3, 3
    rng = np.random.default_rng(5)
    x0 = rng.uniform(-1, 1, ope.N)
    Ed = _dense(ope, E)
    Id = _dense(opi, I_)
    eye = np.eye(ope.N)
    xd = x0.copy()
    for _ in range(steps):
        f1 = xd + dt * Ed @ xd
        if with_implicit:
            f1 = np.linalg.solve(eye - dt * Id, f1)
        f2s = 0.5 * (xd + f1 + dt * Ed @ f1)
        xd = np.linalg.solve(eye - 0.5 * dt * Id, f2s) if with_implicit else f2s
    x = x0.copy()
    its = oracle.imex_advance(2, 3, E, I_ if with_implicit else None, dt, x, steps,
                              30, 50, 1e-13)
    assert len(its) == steps
    assert all((a > 0 and b > 0) if with_implicit else (a == 0 and b == 0) for a, b in its)
    assert rel_err(x, xd) < 1e-11
