"""The tensor-core (BF16 operands, FP32 accumulation in TMEM) form of the
global operator, precision "bf16": exact on BF16-representable inputs to the
FP32 accumulation error, within BF16 rounding on general inputs, every pencil
class (one to 128 cells: one and two MMA halves, one to six K chunks), the
apply's alpha/beta/Euler forms, value updates, and FP64 refinement around it
reaching the 1e-10 residual."""
import numpy as np
import pytest

import oracle
from conftest import rel_err

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _apply(mat, alpha, x, beta, y, precision="fp64"):
    import torch
    yd = _dev(y)
    mat.apply(alpha, _dev(x), beta, yd, precision=precision)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def _bf16(a):
    import torch
    return torch.from_numpy(np.asarray(a, np.float64)).to(torch.bfloat16).double().numpy()


def _exact_operator(d, L, T):
    """advdiff structure with factor values rounded to BF16 (one term per
    dimension, so each dimension's pre-summed block is one factor: exact)."""
    import asgard_b200 as ab
    op = ab.SparseGridOperator(d, L, T, kind="advdiff")
    op.vA = _bf16(op.vA)
    return op


# (d, level, terms): level 7 in d=2 has pencils of 128 cells (384 x 384
# class matrix: two N halves, six K chunks); d=4/5/6 cover every dimension
# stride; d=1 is the single-dimension epilogue
CASES = [(1, 7, 1), (2, 7, 2), (3, 5, 3), (4, 4, 4), (5, 3, 5), (6, 3, 6)]


@pytest.mark.parametrize("d,L,T", CASES)
def test_bf16_exact_on_representable_inputs(cuda, d, L, T):
    """BF16 products of BF16 numbers are exact; what remains is the FP32
    accumulation: within 1e-6 of the oracle's FP64 kronmult."""
    op = _exact_operator(d, L, T)
    g = op.kronmult_matrix(mode="global")
    rng = np.random.default_rng(10 + d)
    x = _bf16(rng.uniform(-1, 1, op.N))
    y0 = rng.uniform(-1, 1, op.N)
    expect = oracle.kronmult(d, 3, op.row_ptr.astype(np.int32), op.col, T,
                             op.iA(), op.vA, 0.7, x, -1.3, y0.copy())
    got = _apply(g, 0.7, x, -1.3, y0, "bf16")
    assert rel_err(got, expect) < 1e-6
    # beta = 0 never reads y (NaN there stays out)
    ynan = np.full(op.N, np.nan)
    got0 = _apply(g, 1.0, x, 0.0, ynan, "bf16")
    assert np.isfinite(got0).all()
    assert rel_err(got0, _apply(g, 1.0, x, 0.0, ynan, "fp64")) < 1e-6


@pytest.mark.parametrize("d,L,T", [(2, 7, 2), (4, 5, 4), (6, 4, 6)])
def test_bf16_general_inputs_within_rounding(cuda, d, L, T):
    """General operands: the BF16 rounding of x and of the class matrices
    (2^-9 relative each) bounds the error against FP64; the same bits on
    every call."""
    import asgard_b200 as ab
    op = ab.SparseGridOperator(d, L, T, kind="advdiff")
    g = op.kronmult_matrix(mode="global")
    rng = np.random.default_rng(20 + d)
    x = rng.uniform(-1, 1, op.N)
    y0 = rng.uniform(-1, 1, op.N)
    ref = _apply(g, 1.0, x, 0.5, y0, "fp64")
    held = g.device_bytes()
    a = _apply(g, 1.0, x, 0.5, y0, "bf16")
    b = _apply(g, 1.0, x, 0.5, y0, "bf16")
    assert rel_err(a, ref) < 1e-2
    assert np.array_equal(a, b)
    # the tensor-core tables built by the first BF16 call are reported:
    # at least the BF16 copy of x and the FP32 sum vector
    assert g.device_bytes() >= held + 6 * op.N


def test_bf16_euler_form_and_value_update(cuda):
    """apply_euler (x - dt K x) in BF16, an identity term, and new values
    through update_stored_coefficients (the class matrices are rewritten)."""
    import asgard_b200 as ab
    import torch
    d, L, T = 3, 5, 4
    op = _exact_operator(d, L, 3)
    pntr, indx = ab.connect_1d(L)
    rows = np.repeat(np.arange(len(pntr) - 1), np.diff(pntr))
    # a fourth term that is the identity in every dimension
    vA = op.vA.reshape(len(indx), 3, d, 9)
    eye = np.where((rows == indx)[:, None], np.eye(3).ravel(order="F")[None, :], 0.0)
    v4 = np.concatenate([vA, np.repeat(eye[:, None, None, :], d, axis=2)], axis=1)
    op4 = ab.SparseGridOperator(d, L, T, kind="advdiff")
    op4.vA = np.ascontiguousarray(v4).reshape(-1)
    g = op4.kronmult_matrix(mode="global")
    rng = np.random.default_rng(3)
    x = _bf16(rng.uniform(-1, 1, op4.N))
    y0 = rng.uniform(-1, 1, op4.N)
    dt = 1e-3
    ya, yb = _dev(y0), _dev(y0)
    g.apply_euler(dt, 0.8, _dev(x), 0.3, ya, precision="fp64")
    g.apply_euler(dt, 0.8, _dev(x), 0.3, yb, precision="bf16")
    torch.cuda.synchronize()
    assert rel_err(yb.cpu().numpy(), ya.cpu().numpy()) < 1e-6
    # new values: the acting factors scaled by 2 (still exact in BF16; the
    # identity factors stay, so every term acts in the same dimensions)
    v2 = v4.copy()
    for t in range(3):
        v2[:, t, t % d] *= 2.0
    g.update_stored_coefficients(np.ascontiguousarray(v2).reshape(-1))
    got = _apply(g, 1.0, x, 0.0, y0, "bf16")
    ref = _apply(g, 1.0, x, 0.0, y0, "fp64")
    assert rel_err(got, ref) < 1e-6


@pytest.mark.parametrize("d,L,T,dt", [(3, 6, 3, 1e-3), (4, 5, 4, 1e-3)])
def test_bf16_refinement_reaches_fp64_residual(cuda, d, L, T, dt):
    """FP64 iterative refinement around inner solves with the tensor-core
    operator reaches the 1e-10 FP64 relative residual, with and without the
    line preconditioner; the solution agrees with the FP64 solve."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(d, L, T, kind="advdiff", nu=0.1)
    g = op.kronmult_matrix(mode="global")
    rng = np.random.default_rng(7)
    b = _dev(rng.uniform(-1, 1, op.N))
    x64 = torch.zeros_like(b)
    i64 = ab.simple_gmres_euler(dt, g, x64, b, 50, 200, 1e-10, tol_mode="rel")
    assert i64.status == 0
    for pc in (None, ab.JacobiPreconditioner(g, dt, kind="line")):
        xb = torch.zeros_like(b)
        ib = ab.simple_gmres_euler(dt, g, xb, b, 50, 200, 1e-10, tol_mode="rel",
                                   precision="bf16", precond=pc)
        assert ib.status == 0 and ib.true_relres <= 1e-10, ib
        assert ib.matvecs_low > 0 and ib.outer_steps >= 2
        assert rel_err(xb.cpu().numpy(), x64.cpu().numpy()) < 1e-8


def test_bf16_refused_where_the_pencil_form_does_not_apply(cuda):
    """The tensor-core form needs a global plan whose terms act in one
    dimension each: a connected-pair plan, and a global plan with a term
    acting in several dimensions (upper/lower chains), refuse precision
    "bf16" with ASGK_ERR_UNSUPPORTED in the apply and in the solve, and the
    solve leaves x untouched."""
    import asgard_b200 as ab
    import torch
    from asgard_b200._lib import AsgkError
    op = ab.SparseGridOperator(3, 4, 3, kind="advdiff")
    pairs = op.kronmult_matrix()
    opr = ab.SparseGridOperator(3, 4, 2, kind="random", seed=3)  # all-direction terms
    chains = opr.kronmult_matrix(mode="global")
    x = torch.rand(op.N, dtype=torch.float64, device="cuda")
    for m in (pairs, chains):
        y = torch.zeros_like(x)
        with pytest.raises(AsgkError) as e:
            m.apply(1.0, x, 0.0, y, precision="bf16")
        assert e.value.status == 2   # ASGK_ERR_UNSUPPORTED
        x0 = torch.zeros_like(x)
        with pytest.raises(AsgkError) as e:
            ab.simple_gmres_euler(1e-3, m, x0, x, 20, 5, 1e-10, tol_mode="rel",
                                  precision="bf16")
        assert e.value.status == 2
        assert not x0.any()
