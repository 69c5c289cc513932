"""The reference's global-Kronecker implicit path, compiled from its own
sources in KRON_MODE_GLOBAL (``make -C oracle ref_gsolve``), as a checker:

* on the benchmark's synthetic advection/diffusion operators its element
  table, operator and diagonal preconditioner equal the oracle's restatements
  (the preconditioner bit for bit: this pins ``oracle.point_jacobi_diag``,
  the restatement of build_preconditioner, src/asgard_kronmult_matrix.cpp:
  1015-1067, to the reference's own code);
* on the reference's built-in PDEs its preconditioner equals the restatement
  applied to the same PDE's local-kron operator (the reference's own
  make_kronmult_sparse output), and its global operator equals that local
  operator;
* its simple_gmres_euler (src/solver.cpp:93-117) with the tolerance the
  benchmark's reference arm uses reaches a true relative residual of 1e-10.
"""
import numpy as np
import pytest

import oracle
from conftest import rel_err

pytestmark = pytest.mark.skipif(
    not oracle.ref_gsolve_available(),
    reason="reference global-kron solver not built (make -C oracle ref_gsolve)")


def _synthetic(d, L, T):
    import asgard_b200.operators as O
    return O.SparseGridOperator(d, L, T, kind="advdiff", nu=0.1)


@pytest.mark.parametrize("d,L,T", [(1, 6, 2), (2, 5, 3), (3, 4, 3), (4, 3, 4),
                                   (6, 2, 6)])
def test_synthetic_operator_matches_oracle(d, L, T):
    op = _synthetic(d, L, T)
    R = oracle.RefGlobalSolver.synthetic(d, L, T, 0.1)
    assert R.N == op.N and R.cells == op.rows
    assert np.array_equal(R.table(), oracle.sparse_grid(d, L))
    x = np.random.default_rng(d).uniform(-1, 1, op.N)
    y, _ = R.apply(1.0, x)
    pntr = op.row_ptr.astype(np.int32)
    expect = oracle.kronmult(d, 3, pntr, op.col, T, op.iA(), op.vA, 1.0, x,
                             0.0, np.zeros(op.N))
    assert rel_err(y, expect) <= 1e-13
    # the reference's build_preconditioner and the restatement: bit for bit
    pc = R.precond()
    pco = oracle.point_jacobi_diag(d, 3, pntr, op.col, T, op.iA(), op.vA)
    assert np.array_equal(pc, pco)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("name,d,L", [("continuity_2", 2, 4), ("continuity_3", 3, 3),
                                      ("diffusion_2", 2, 3), ("continuity_6", 6, 2)])
def test_builtin_pde_preconditioner_and_operator(name, d, L):
    """Global-kron mode (its preconditioner, its global product) against the
    local-kron mode of the same PDE (the reference's pair list, iA, vA)."""
    G = oracle.RefGlobalSolver.builtin(name, d, L, 3)
    P = oracle.RefPDE(name, L, 3, d)
    assert np.array_equal(G.table(), P.table)
    pc = G.precond()
    pco = oracle.point_jacobi_diag(d, 3, P.pntr, P.indx, P.terms, P.iA, P.vA)
    assert rel_err(pc, pco) <= 1e-14
    x = np.random.default_rng(3).uniform(-1, 1, G.N)
    y, _ = G.apply(1.0, x)
    y_local = P.apply(1.0, x, 0.0, np.zeros(G.N))
    assert rel_err(y, y_local) <= 1e-12


def test_reference_solve_reaches_the_target_residual():
    """The reference arm's tolerance: TOL * ||b|| / max |1 - dt pc| on the
    reference's left-preconditioned estimate gives a true relative residual
    <= TOL; consecutive one-cycle calls give the same solution as one call."""
    d, L, T, dt = 2, 5, 3, 1e-3
    R = oracle.RefGlobalSolver.synthetic(d, L, T, 0.1)
    b = np.random.default_rng(5).uniform(-1, 1, R.N)
    m = np.abs(1 - dt * R.precond()).max()
    tol = 1e-10 * np.linalg.norm(b) / m
    x1 = np.zeros(R.N)
    err, its, _ = R.gmres_euler(dt, x1, b, 20, 100, tol)
    assert err <= tol
    Kx, _ = R.apply(1.0, x1)
    assert np.linalg.norm(b - (x1 - dt * Kx)) <= 1e-10 * np.linalg.norm(b)
    # one restart cycle per call, from the current x
    x2 = np.zeros(R.N)
    total = 0
    for _ in range(100):
        e2, i2, _ = R.gmres_euler(dt, x2, b, 20, 1, tol)
        total += i2
        if e2 <= tol:
            break
    assert total == its
    assert rel_err(x2, x1) <= 1e-14
