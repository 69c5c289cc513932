"""Global Kronecker form: the same operator as the connected-pair
kronmult -- terms acting in one dimension in one pass, terms acting in
several as chains of masked 1D passes -- checked against the oracle, the
pair plan and the reference's own global product, inside GMRES, and its
error cases."""
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


@pytest.mark.parametrize("d,L,T", [(1, 6, 2), (2, 6, 3), (3, 5, 3), (4, 4, 4),
                                   (5, 3, 5), (6, 3, 6), (4, 7, 4)])
def test_global_matches_oracle_and_pairs(cuda, d, L, T):
    import asgard_b200 as ab
    op = ab.SparseGridOperator(d, L, T, kind="advdiff")
    g = op.kronmult_matrix(mode="global")
    rng = np.random.default_rng(d)
    x = rng.uniform(-1, 1, op.N)
    y0 = rng.uniform(-1, 1, op.N)
    if op.nnz < 3_000_000:
        expect = oracle.kronmult(d, 3, op.row_ptr.astype(np.int32), op.col, T,
                                 op.iA(), op.vA, 0.7, x, -1.3, y0.copy())
    else:   # d=4 level 7: the pair plan is the reference
        expect = _apply(op.kronmult_matrix(), 0.7, x, -1.3, y0)
    assert rel_err(_apply(g, 0.7, x, -1.3, y0), expect) < 1e-13
    assert rel_err(_apply(g, 0.7, x, 0.0, y0), _apply(op.kronmult_matrix(), 0.7, x, 0.0, y0)) < 1e-13
    assert rel_err(_apply(g, 0.7, x, -1.3, y0, "fp32"), expect) < 1e-5
    # num_pairs: the single-direction pairs; flops: one contraction each
    assert g.num_pairs() < op.nnz or d == 1
    assert g.flops() == 2 * 3 ** (d + 1) * g.num_pairs()
    assert g.num_batch() == op.rows * op.rows


def test_global_euler_identity_term_and_update(cuda):
    """The fused Euler form, a term that is the identity in every dimension
    (it adds x), and update_stored_coefficients."""
    import asgard_b200 as ab
    import torch
    d, L, T = 3, 5, 4
    op = ab.SparseGridOperator(d, L, T, kind="advdiff")
    pntr, indx = ab.connect_1d(L)
    rows = np.repeat(np.arange(len(pntr) - 1), np.diff(pntr))
    vA = op.vA.reshape(len(indx), T, d, 9).copy()
    eye = np.where((rows == indx)[:, None], np.eye(3).ravel(order="F")[None, :], 0.0)
    vA[:, 3, 3 % d] = eye          # term 3 is now the identity everywhere
    vA = vA.ravel()
    g = ab.kronmult_matrix.from_global(d, 3, L, op.table, T, vA)
    rng = np.random.default_rng(3)
    x, y0 = rng.uniform(-1, 1, op.N), rng.uniform(-1, 1, op.N)
    kx = oracle.kronmult(d, 3, op.row_ptr.astype(np.int32), op.col, T, op.iA(),
                         vA, 1.0, x, 0.0, np.zeros(op.N))
    dt, alpha, beta = 1e-3, -1.0, 0.5
    yd = _dev(y0)
    g.apply_euler(dt, alpha, _dev(x), beta, yd)
    torch.cuda.synchronize()
    assert rel_err(yd.cpu().numpy(), beta * y0 + alpha * (x - dt * kx)) < 1e-13
    # new values: 2x the factors of the acting dimensions
    vA2 = vA.reshape(len(indx), T, d, 9).copy()
    for t in range(3):
        vA2[:, t, t % d] *= 2.0
    vA2 = vA2.ravel()
    g.update_stored_coefficients(vA2)
    kx2 = oracle.kronmult(d, 3, op.row_ptr.astype(np.int32), op.col, T, op.iA(),
                          vA2, 1.0, x, 0.0, np.zeros(op.N))
    assert rel_err(_apply(g, 1.0, x, 0.0, y0), kx2) < 1e-13


def test_global_gmres_matches_pair_gmres(cuda):
    """Solves with the global plan take the pair plan's iterations (+-1) and
    reach the same solution, plain and with block Jacobi (built from the
    global plan's diagonal pairs)."""
    import asgard_b200 as ab
    import torch
    d, L, T, dt = 3, 6, 3, 4e-3
    op = ab.SparseGridOperator(d, L, T, kind="advdiff")
    pm, gm = op.kronmult_matrix(), op.kronmult_matrix(mode="global")
    b = _dev(np.random.default_rng(1).uniform(-1, 1, op.N))
    for kind in (None, "block"):
        infos, xs = [], []
        for mat in (pm, gm):
            pc = ab.JacobiPreconditioner(mat, dt, kind=kind) if kind else None
            x = torch.zeros_like(b)
            info = ab.simple_gmres_euler(dt, mat, x, b, 50, 200, 1e-10,
                                         tol_mode="rel", precond=pc)
            assert info.status == 0 and info.true_relres <= 1e-10
            infos.append(info)
            xs.append(x)
        assert abs(infos[0].iterations - infos[1].iterations) <= 1, (kind, infos)
        assert (torch.linalg.norm(xs[0] - xs[1]) / torch.linalg.norm(xs[0])).item() < 1e-9


@pytest.mark.parametrize("d,L,T", [(1, 5, 2), (2, 5, 2), (3, 4, 3), (4, 3, 2), (5, 2, 2)])
def test_global_multi_direction_terms(cuda, d, L, T):
    """Terms acting in every dimension (random factors): the chains of
    masked 1D passes (the reference's upper/lower permutations) give the
    connected-pair operator, FP64 and FP32, and the Euler form."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(d, L, T, kind="random")
    g = op.kronmult_matrix(mode="global")
    rng = np.random.default_rng(d + 10)
    x, y0 = rng.uniform(-1, 1, op.N), rng.uniform(-1, 1, op.N)
    expect = oracle.kronmult(d, 3, op.row_ptr.astype(np.int32), op.col, T,
                             op.iA(), op.vA, 0.7, x, -1.3, y0.copy())
    assert rel_err(_apply(g, 0.7, x, -1.3, y0), expect) < 1e-13
    assert rel_err(_apply(g, 0.7, x, -1.3, y0, "fp32"), expect) < 1e-5
    pm = op.kronmult_matrix()
    ya, yb = _dev(y0), _dev(y0)
    g.apply_euler(1e-3, -1.0, _dev(x), 0.5, ya)
    pm.apply_euler(1e-3, -1.0, _dev(x), 0.5, yb)
    torch.cuda.synchronize()
    assert rel_err(ya.cpu().numpy(), yb.cpu().numpy()) < 1e-13
    assert g.num_pairs() > 0 and g.flops() == 2 * 3 ** (d + 1) * g.num_pairs()


def test_global_mixed_terms_gmres_and_updates(cuda):
    """Single-direction (advection/diffusion), all-direction (random) and
    identity terms in one operator; GMRES with block-Jacobi matches the pair
    plan; new values with the same active dimensions are taken, a term that
    changes its active dimensions is refused; unknown modes raise."""
    import asgard_b200 as ab
    import torch
    d, L, dt = 3, 5, 4e-3
    a = ab.SparseGridOperator(d, L, 3, kind="advdiff")
    r = ab.SparseGridOperator(d, L, 2, kind="random")
    nconn = len(ab.connect_1d(L)[1])
    va = a.vA.reshape(nconn, 3, d, 9)
    vr = 0.05 * r.vA.reshape(nconn, 2, d, 9)
    vA = np.concatenate([va, vr], axis=1).ravel()
    T = 5
    g = ab.kronmult_matrix.from_global(d, 3, L, a.table, T, vA)
    pm = ab.kronmult_matrix.from_conn(d, 3, a.rows, a.rows, T, a.row_ptr, a.col, a.conn, vA)
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, a.N)
    assert rel_err(_apply(g, 1.0, x, 0.0, np.zeros(a.N)),
                   _apply(pm, 1.0, x, 0.0, np.zeros(a.N))) < 1e-13
    b = _dev(rng.uniform(-1, 1, a.N))
    infos, xs = [], []
    for mat in (pm, g):
        pc = ab.JacobiPreconditioner(mat, dt, kind="block")
        xx = torch.zeros_like(b)
        info = ab.simple_gmres_euler(dt, mat, xx, b, 50, 200, 1e-10, tol_mode="rel",
                                     precision="fp32", precond=pc)
        assert info.status == 0 and info.true_relres <= 1e-10
        infos.append(info)
        xs.append(xx)
    assert abs(infos[0].iterations - infos[1].iterations) <= 1
    assert (torch.linalg.norm(xs[0] - xs[1]) / torch.linalg.norm(xs[0])).item() < 1e-9
    v2 = vA.reshape(nconn, T, d, 9).copy()
    v2[:, 3:] *= 1.5                       # same active dimensions
    v2 = v2.ravel()
    g.update_stored_coefficients(v2)
    pm.update_stored_coefficients(v2)
    assert rel_err(_apply(g, 1.0, x, 0.0, np.zeros(a.N)),
                   _apply(pm, 1.0, x, 0.0, np.zeros(a.N))) < 1e-13
    v3 = v2.reshape(nconn, T, d, 9).copy()
    v3[:, 0, (0 + 1) % d] = v3[:, 1, 1 % d]  # term 0 now acts in two dimensions
    with pytest.raises(ab.AsgkError):
        g.update_stored_coefficients(v3.ravel())
    with pytest.raises(ValueError):
        a.kronmult_matrix(mode="blocked")


@pytest.mark.skipif(not oracle.ref_global_available(),
                    reason="reference global-kron library not built")
@pytest.mark.parametrize("d,L,T,kind", [(2, 6, 3, "advdiff"), (3, 5, 3, "advdiff"),
                                        (4, 5, 4, "advdiff"), (2, 5, 2, "random"),
                                        (3, 4, 2, "random"), (4, 3, 2, "random")])
def test_global_matches_reference_global_kron(cuda, d, L, T, kind):
    """The GPU global form against the reference's own global Kronecker
    product (global_cpu compiled from its sources), single-direction terms
    and terms acting in every dimension (its upper/lower permutations)."""
    import asgard_b200 as ab
    op = ab.SparseGridOperator(d, L, T, kind=kind)
    x = np.random.default_rng(7).uniform(-1, 1, op.N)
    y_ref, _ = oracle.ref_global_apply(d, 3, L, op.table, T, op.vA, x)
    g = op.kronmult_matrix(mode="global")
    assert rel_err(_apply(g, 1.0, x, 0.0, np.zeros(op.N)), y_ref) < 1e-13


def test_value_update_changing_identity_terms_drops_recorded_cycles(cuda):
    """A term that is the identity in every dimension enters the global
    form's launches as a scalar that recorded GMRES cycles hold; an update
    that makes it a real term must not replay those recordings: the solve
    after the update equals a solve on a plan built from the new values."""
    import asgard_b200 as ab
    import torch
    from asgard_b200.operators import connect_1d, factor_values, sparse_grid
    d, L, T = 3, 5, 3
    pntr, indx = connect_1d(L)
    rows = np.repeat(np.arange(len(pntr) - 1), np.diff(pntr))
    eye = np.where((rows == indx)[:, None], np.eye(3).ravel(order="F")[None, :], 0.0)
    vA = factor_values(d, L, T).reshape(len(indx), T, d, 9)
    vA[:, 2] = eye[:, None, :]                 # term 2: identity everywhere
    v0 = np.ascontiguousarray(vA.reshape(-1))
    v1 = vA.copy()
    v1[:, 2, 0] *= 1.5                         # term 2 now scales dimension 0
    v1 = np.ascontiguousarray(v1.reshape(-1))
    table = sparse_grid(d, L)
    b = torch.from_numpy(np.random.default_rng(2).uniform(-1, 1, table.shape[0] * 27)).cuda()
    dt = 2e-3

    def solve(mat):
        x = torch.zeros_like(b)
        info = ab.simple_gmres_euler(dt, mat, x, b, 30, 100, 1e-11, tol_mode="rel")
        assert info.status == 0
        return x.cpu().numpy(), info.iterations

    mat = ab.kronmult_matrix.from_global(d, 3, L, table, T, v0)
    solve(mat)                                 # records the cycles
    mat.update_stored_coefficients(v1)
    x_upd, it_upd = solve(mat)
    x_new, it_new = solve(ab.kronmult_matrix.from_global(d, 3, L, table, T, v1))
    assert it_upd == it_new
    assert np.array_equal(x_upd, x_new)


def test_global_cell_kernel_misaligned_and_aliasing_free_input(cuda):
    """d >= 5 applies read x through an FP32 copy in FP32: an input that is
    only 8-byte aligned (a column of an odd-length system) gives the same
    result as an aligned copy of it."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(5, 3, 4, kind="advdiff")
    g = op.kronmult_matrix(mode="global")
    x = np.random.default_rng(9).uniform(-1, 1, op.N)
    buf = torch.zeros(op.N + 1, dtype=torch.float64, device="cuda")
    buf[1:] = _dev(x)
    xs = buf[1:]                      # 8 bytes past a 256-byte boundary
    assert xs.data_ptr() % 16 == 8
    for prec in ("fp32", "fp64"):
        ya, yb = torch.zeros_like(xs), torch.zeros_like(xs)
        g.apply(1.0, xs, 0.0, ya, precision=prec)
        g.apply(1.0, _dev(x), 0.0, yb, precision=prec)
        torch.cuda.synchronize()
        assert torch.equal(ya, yb), prec
