"""Dense kron mode on the CPU: the restatement of kronmult::cpu_dense and of
the reference's dense-test data generator (make_kronmult_welem) pinned
against fixtures made by the reference (tests/golden/dense_data.npz) and
against the reference compiled from its sources."""
import hashlib

import numpy as np
import pytest

import oracle
from conftest import golden, rmse_close

DENSE = np.load(golden("dense_data.npz"))
# the non-square offset case of the fixture (tests/golden/make_golden.py)
OFFSET = dict(d=2, n=3, terms=2, index_range=5, rows=10, cols=12,
              row_offset=5, col_offset=9, alpha=0.7, beta=-1.3)


def dense_keys():
    out = []
    for k in DENSE.files:
        if k.endswith("_ref_y"):
            tag, d, n, terms, rg = k[:-len("_ref_y")].split("_")
            out.append((tag, int(d), int(n), int(terms), int(rg)))
    return sorted(out)


def test_dense_fixture_covers_the_reference_shapes():
    keys = dense_keys()
    assert len(keys) == 2 * 26
    assert {k[1] for k in keys} == {1, 2, 3, 5, 6}


@pytest.mark.parametrize("tag,d,n,terms,rg", dense_keys())
def test_oracle_dense_reference_test_data(tag, d, n, terms, rg):
    """make_kronmult_welem regenerated bit-exactly; the oracle's cpu_dense
    equals the reference's cpu_dense (bit-exact, n = 1 within one ulp: the
    reference has a separate n = 1 path) and the explicit Kronecker answer
    (src/asgard_kronmult_matrix_tests.cpp:118-176, 100 ulp rmse)."""
    dt = np.float64 if tag == "f64" else np.float32
    a = oracle.make_kronmult_welem(d, n, terms, rg, dt)
    key = f"{tag}_{d}_{n}_{terms}_{rg}"
    h = hashlib.sha256()
    for arr in (a["elem"], *a["terms"], a["x"], a["y"]):
        h.update(np.ascontiguousarray(arr).tobytes())
    assert h.hexdigest() == bytes(DENSE[key + "_inputs_sha256"]).decode()
    y = a["y"].copy()
    oracle.kronmult_dense(d, n, a["rows"], a["rows"], a["terms"], a["elem"],
                          0, 0, rg, dt(1.0), a["x"], dt(1.0), y)
    eps = np.finfo(dt).eps
    if n == 1:
        assert np.abs(y - DENSE[key + "_cpu_dense_y"]).max() <= 4 * eps * np.abs(y).max()
    else:
        assert np.array_equal(y, DENSE[key + "_cpu_dense_y"])
    assert rmse_close(y, DENSE[key + "_ref_y"], 100 * eps)


def test_oracle_dense_offsets_non_square():
    """Rows and columns from different parts of the element table
    (row_offset / col_offset, rows != cols), alpha and beta general."""
    c = OFFSET
    a = oracle.make_kronmult_welem(c["d"], c["n"], c["terms"], c["index_range"])
    ts = c["n"] ** c["d"]
    x = a["x"][c["col_offset"] * ts:(c["col_offset"] + c["cols"]) * ts].copy()
    y = a["y"][c["row_offset"] * ts:(c["row_offset"] + c["rows"]) * ts].copy()
    oracle.kronmult_dense(c["d"], c["n"], c["rows"], c["cols"], a["terms"],
                          a["elem"], c["row_offset"], c["col_offset"],
                          c["index_range"], c["alpha"], x, c["beta"], y)
    assert np.array_equal(y, DENSE["offset_y"])


@pytest.mark.parametrize("d,L,T", [(1, 5, 2), (2, 4, 3), (3, 3, 3)])
def test_dense_form_of_a_sparse_grid_equals_its_pair_form(d, L, T):
    """The dense form (full 1D operators, zero between unconnected cells)
    of a sparse-grid operator is the connected-pair operator: the extra
    pairs add exact zeros."""
    import asgard_b200.operators as O
    op = O.SparseGridOperator(d, L, T, kind="advdiff")
    terms, nb = op.dense_terms()
    rng = np.random.default_rng(d)
    x, y0 = rng.uniform(-1, 1, op.N), rng.uniform(-1, 1, op.N)
    ys = oracle.kronmult(d, 3, op.row_ptr.astype(np.int32), op.col, T, op.iA(),
                         op.vA, 0.7, x, -1.3, y0.copy())
    yd = oracle.kronmult_dense(d, 3, op.rows, op.rows, terms, op.elem(), 0, 0,
                               nb, 0.7, x, -1.3, y0.copy())
    assert np.array_equal(ys, yd)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference not built here")
def test_oracle_dense_matches_compiled_reference():
    """The restatement against the reference's kronmult_matrix (dense
    constructor, cpu_dense) on generated data, every alpha/beta case."""
    R = oracle.ref()
    for (d, n, terms, rg) in [(2, 3, 2, 5), (3, 2, 3, 3), (5, 3, 2, 1)]:
        a = oracle.make_kronmult_welem(d, n, terms, rg)
        b = oracle.ref_make_kronmult_welem(d, n, terms, rg, want_ref=False)
        assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["elem"], b["elem"])
        for alpha, beta in [(1.0, 0.0), (-1.0, 1.0), (0.7, -1.0), (2.5, 0.3)]:
            y1, y2 = a["y"].copy(), a["y"].copy()
            rows = a["rows"]
            oracle.kronmult_dense(d, n, rows, rows, a["terms"], a["elem"], 0, 0,
                                  rg, alpha, a["x"], beta, y1)
            oracle.kronmult_dense(d, n, rows, rows, a["terms"], a["elem"], 0, 0,
                                  rg, alpha, a["x"], beta, y2, lib=R)
            assert np.allclose(y1, y2, rtol=0, atol=1e-14 * np.abs(y2).max())


def test_reference_dense_tables_out_of_range():
    """make_kronmult_welem writes base-d digits, so the reference's own
    (4, n, 2, 3) and (6, n, 2, 2) dense tests index past index_range (their
    answer reads outside the coefficient arrays); these tables are what the
    GPU constructor must reject."""
    for (d, rg) in [(4, 3), (6, 2)]:
        a = oracle.make_kronmult_welem(d, 2, 1, rg)
        assert a["elem"].max() >= rg
    for (d, rg) in [(1, 7), (2, 5), (3, 3), (5, 1)]:
        a = oracle.make_kronmult_welem(d, 2, 1, rg)
        assert a["elem"].max() < rg
