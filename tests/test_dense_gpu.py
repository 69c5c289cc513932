"""Dense kron mode on the GPU (the reference's dense kronmult_matrix and
gpu_dense): the reference's dense-test shapes against fixtures the reference
made, offsets, host vectors, coefficient updates, the empty matrix, bad
element tables, and the dense form of a sparse-grid operator against its
pair form, in apply and in GMRES."""
import numpy as np
import pytest

import oracle
from conftest import golden, rel_err, rmse_close
from test_dense_oracle import OFFSET, dense_keys

pytestmark = pytest.mark.gpu

DENSE = np.load(golden("dense_data.npz"))


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("tag,d,n,terms,rg", dense_keys())
def test_dense_plan_reference_test_data(cuda, tag, d, n, terms, rg):
    """y <- y + K x over every cell pair (test_kronmult_dense,
    src/asgard_kronmult_matrix_tests.cpp:118-176): FP64 within 1e-13 of the
    reference's cpu_dense, FP32 vectors and arithmetic within the
    reference test's 100-ulp rmse of its explicit Kronecker answer."""
    import asgard_b200 as ab
    import torch
    dt = np.float64 if tag == "f64" else np.float32
    a = oracle.make_kronmult_welem(d, n, terms, rg, dt)
    key = f"{tag}_{d}_{n}_{terms}_{rg}"
    rows = a["rows"]
    mat = ab.kronmult_matrix.from_dense(d, n, rows, rows, terms,
                                        [t.astype(np.float64) for t in a["terms"]],
                                        a["elem"], 0, 0, rg)
    assert mat.is_dense() and mat.kind() == "dense"
    assert mat.num_batch() == rows * rows == mat.num_pairs()
    assert mat.flops() == 2 * n ** (d + 1) * d * terms * rows * rows
    y = _dev(a["y"])
    mat.apply(1.0, _dev(a["x"]), 1.0, y)
    torch.cuda.synchronize()
    got = y.cpu().numpy()
    eps = np.finfo(dt).eps
    if tag == "f64":
        assert rel_err(got, DENSE[key + "_cpu_dense_y"]) < 1e-13
    assert rmse_close(got, DENSE[key + "_ref_y"], 100 * eps)


def test_dense_plan_offsets_non_square_and_host(cuda):
    """Rows and columns from different parts of the element table, general
    alpha/beta, on device and on host vectors."""
    import asgard_b200 as ab
    import torch
    c = OFFSET
    a = oracle.make_kronmult_welem(c["d"], c["n"], c["terms"], c["index_range"])
    ts = c["n"] ** c["d"]
    x = a["x"][c["col_offset"] * ts:(c["col_offset"] + c["cols"]) * ts].copy()
    y0 = a["y"][c["row_offset"] * ts:(c["row_offset"] + c["rows"]) * ts].copy()
    mat = ab.kronmult_matrix.from_dense(c["d"], c["n"], c["rows"], c["cols"],
                                        c["terms"], a["terms"], a["elem"],
                                        c["row_offset"], c["col_offset"],
                                        c["index_range"])
    assert mat.input_size() == c["cols"] * ts and mat.output_size() == c["rows"] * ts
    yd = _dev(y0)
    mat.apply(c["alpha"], _dev(x), c["beta"], yd)
    torch.cuda.synchronize()
    assert rel_err(yd.cpu().numpy(), DENSE["offset_y"]) < 1e-13
    yh = y0.copy()
    mat.apply(c["alpha"], x, c["beta"], yh, resource="host")
    assert rel_err(yh, DENSE["offset_y"]) < 1e-13
    # the Euler form needs a square operator
    with pytest.raises(ab.AsgkError):
        mat.apply_euler(1e-3, 1.0, _dev(x), 0.0, _dev(y0))


def test_dense_plan_update_and_alpha_beta_cases(cuda):
    """update_stored_coefficients with per-term arrays, and the alpha/beta
    cases the reference dispatches separately (src/device/asgard_kronmult_cpu.cpp:517-580)."""
    import asgard_b200 as ab
    import torch
    d, n, terms, rg = 3, 3, 3, 3
    a = oracle.make_kronmult_welem(d, n, terms, rg)
    rows = a["rows"]
    mat = ab.kronmult_matrix.from_dense(d, n, rows, rows, terms, a["terms"],
                                        a["elem"], 0, 0, rg)
    for alpha, beta in [(1.0, 0.0), (-1.0, 0.0), (0.3, 0.0), (1.0, 1.0),
                        (-1.0, -1.0), (0.3, 2.0)]:
        expect = oracle.kronmult_dense(d, n, rows, rows, a["terms"], a["elem"],
                                       0, 0, rg, alpha, a["x"], beta, a["y"].copy())
        y = _dev(a["y"])
        mat.apply(alpha, _dev(a["x"]), beta, y)
        torch.cuda.synchronize()
        assert rel_err(y.cpu().numpy(), expect) < 1e-13, (alpha, beta)
    new = [t * (1.5 + i) for i, t in enumerate(a["terms"])]
    mat.update_stored_coefficients(new)
    expect = oracle.kronmult_dense(d, n, rows, rows, new, a["elem"], 0, 0, rg,
                                   1.0, a["x"], 0.0, np.zeros_like(a["y"]))
    y = _dev(np.zeros_like(a["y"]))
    mat.apply(1.0, _dev(a["x"]), 0.0, y)
    torch.cuda.synchronize()
    assert rel_err(y.cpu().numpy(), expect) < 1e-13
    with pytest.raises(ab.AsgkError):      # wrong number of terms
        mat.update_stored_coefficients(new[:2])


def test_dense_plan_empty_and_bad_tables(cuda):
    """num_terms == 0 is the reference's empty matrix (apply scales y,
    src/asgard_kronmult_matrix.hpp:344-349); element tables with 1D indices
    outside num_1d_blocks -- as the reference's own (4, n, 2, 3) and
    (6, n, 2, 2) dense tests make them -- and short tables are refused."""
    import asgard_b200 as ab
    import torch
    e = ab.kronmult_matrix.from_dense(2, 3, 4, 4, 0, [], np.zeros((4, 2), np.int32), 0, 0, 2)
    y0 = np.random.default_rng(0).uniform(-1, 1, 4 * 9)
    y = _dev(y0)
    e.apply(1.0, _dev(np.ones(36)), 2.0, y)
    torch.cuda.synchronize()
    assert np.array_equal(y.cpu().numpy(), 2.0 * y0)
    for (d, rg) in [(4, 3), (6, 2)]:
        a = oracle.make_kronmult_welem(d, 2, 1, rg)
        with pytest.raises(ab.AsgkError):
            ab.kronmult_matrix.from_dense(d, 2, a["rows"], a["rows"], 1,
                                          a["terms"], a["elem"], 0, 0, rg)
    a = oracle.make_kronmult_welem(2, 2, 1, 5)
    with pytest.raises(ab.AsgkError):      # rows past the end of elem
        ab.kronmult_matrix.from_dense(2, 2, 20, 20, 1, a["terms"], a["elem"],
                                      10, 0, 5)


@pytest.mark.parametrize("d,L,T", [(2, 6, 3), (3, 5, 3), (4, 4, 4), (5, 3, 4),
                                   (6, 2, 6)])
def test_dense_form_matches_pair_form(cuda, d, L, T):
    """The dense form of a sparse-grid operator (full 1D operators, every
    cell pair) against its connected-pair plan: FP64, FP32 and Euler."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(d, L, T, kind="advdiff")
    dm, pm = op.kronmult_matrix(mode="dense"), op.kronmult_matrix()
    assert dm.num_pairs() == op.rows * op.rows
    rng = np.random.default_rng(d)
    x, y0 = _dev(rng.uniform(-1, 1, op.N)), rng.uniform(-1, 1, op.N)
    for prec, tol in (("fp64", 1e-13), ("fp32", 1e-5)):
        ya, yb = _dev(y0), _dev(y0)
        dm.apply(0.7, x, -1.3, ya, precision=prec)
        pm.apply(0.7, x, -1.3, yb, precision=prec)
        torch.cuda.synchronize()
        assert rel_err(ya.cpu().numpy(), yb.cpu().numpy()) < tol, prec
    ya, yb = _dev(y0), _dev(y0)
    dm.apply_euler(1e-3, -1.0, x, 0.5, ya)
    pm.apply_euler(1e-3, -1.0, x, 0.5, yb)
    torch.cuda.synchronize()
    assert rel_err(ya.cpu().numpy(), yb.cpu().numpy()) < 1e-13


def test_dense_form_in_gmres(cuda):
    """simple_gmres_euler over the dense form takes the pair form's
    iterations (+-1) to the same solution, plain and block-Jacobi."""
    import asgard_b200 as ab
    import torch
    d, L, T, dt = 3, 5, 3, 4e-3
    op = ab.SparseGridOperator(d, L, T, kind="advdiff")
    pm, dm = op.kronmult_matrix(), op.kronmult_matrix(mode="dense")
    b = _dev(np.random.default_rng(2).uniform(-1, 1, op.N))
    for kind in (None, "block"):
        infos, xs = [], []
        for mat in (pm, dm):
            pc = ab.JacobiPreconditioner(mat, dt, kind=kind) if kind else None
            x = torch.zeros_like(b)
            info = ab.simple_gmres_euler(dt, mat, x, b, 50, 200, 1e-10,
                                         tol_mode="rel", precond=pc)
            assert info.status == 0 and info.true_relres <= 1e-10
            infos.append(info)
            xs.append(x)
        assert abs(infos[0].iterations - infos[1].iterations) <= 1, (kind, infos)
        assert (torch.linalg.norm(xs[0] - xs[1]) / torch.linalg.norm(xs[0])).item() < 1e-9
