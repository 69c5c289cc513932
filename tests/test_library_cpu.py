"""CPU-side checks of the product library: it loads, exports every symbol the
C header declares, and its host-side sparse-grid builder reproduces the
reference builder (golden fixtures) and the oracle."""
import os
import re

import numpy as np
import pytest

import oracle
from conftest import ROOT, golden


def header_symbols():
    text = open(os.path.join(ROOT, "include", "asgard_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(asgk_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import asgard_b200
    syms = header_symbols()
    assert len(syms) >= 15
    missing = [s for s in syms if not hasattr(asgard_b200.lib, s)]
    assert not missing, missing


def test_cpp_dropin_compiles_and_links(tmp_path):
    """The C++ drop-in program (the reference-side usage of the header-only
    mirror over the C ABI) compiles and links against the in-tree library
    with g++ alone; the GPU test runs it."""
    from test_cpp_dropin_gpu import compile_dropin
    r = compile_dropin(tmp_path / "dropin")
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "dropin").exists()


def test_imex_rejects_invalid_arguments_without_device_work():
    """asgk_imex_advance checks its arguments before any CUDA call: no
    explicit plan, no state vector, or no info array for a positive step
    count are ASGK_ERR_INVALID; zero steps need no info."""
    import ctypes as C
    import asgard_b200 as ab
    inv = 1  # ASGK_ERR_INVALID
    call = lambda plan, x, steps, info: ab.lib.asgk_imex_advance(
        plan, None, 1e-3, x, steps, 10, 10, 1e-10, 0, 0, None, None, None, None,
        None, info, None)
    dummy = C.c_double(0.0)
    assert call(None, C.addressof(dummy), 1, None) == inv
    assert call(C.addressof(dummy), None, 1, None) == inv
    assert call(C.addressof(dummy), C.addressof(dummy), 1, None) == inv
    assert call(C.addressof(dummy), C.addressof(dummy), -1, None) == inv


def test_gmres_settings_set_and_restore():
    """The process-wide GMRES settings (no device work): defaults, a change
    reported back, and the restore from the returned dict."""
    import asgard_b200 as ab
    old = ab.gmres_settings()
    assert old == {"graphs": True, "node_steps": 16, "fp32_basis": True,
                   "bf16_inner_tol": 1e-3}
    try:
        assert ab.gmres_settings(graphs=False, node_steps=3, fp32_basis=False,
                                 bf16_inner_tol=1e-2) == old
        assert ab.gmres_settings() == {"graphs": False, "node_steps": 3,
                                       "fp32_basis": False, "bf16_inner_tol": 1e-2}
        ab.gmres_settings(node_steps=0)  # below 1: only read
        assert ab.gmres_settings()["node_steps"] == 3
        ab.gmres_settings(bf16_inner_tol=2.0)  # outside (0, 1): only read
        assert ab.gmres_settings()["bf16_inner_tol"] == 1e-2
    finally:
        ab.gmres_settings(**old)
    assert ab.gmres_settings() == old


@pytest.mark.parametrize("name", ["continuity_2_L4", "continuity_3_L3",
                                  "continuity_6_L2", "diffusion_2_L3"])
def test_builder_matches_reference_builder(name):
    import asgard_b200 as ab
    z = np.load(golden(f"pde_{name}.npz"))
    d, n, L, terms = int(z["d"]), int(z["n"]), int(z["level"]), int(z["terms"])
    table = ab.sparse_grid(d, L)
    assert np.array_equal(table, z["table"])
    row_ptr, col, conn = ab.build_pairs(d, L, table)
    assert np.array_equal(row_ptr, z["pntr"].astype(np.int64))
    assert np.array_equal(col, z["indx"])
    assert np.array_equal(ab.expand_iA(conn, d, n, terms), z["iA"])


@pytest.mark.parametrize("d,L", [(1, 7), (2, 6), (3, 5), (4, 5), (5, 4), (6, 3)])
def test_builder_matches_oracle(d, L):
    import asgard_b200 as ab
    t1 = ab.sparse_grid(d, L)
    t2 = oracle.sparse_grid(d, L)
    assert np.array_equal(t1, t2)
    r1, c1, k1 = ab.build_pairs(d, L, t1)
    r2, c2, k2 = oracle.build_pairs(d, L, t2)
    assert np.array_equal(r1, r2.astype(np.int64))
    assert np.array_equal(c1, c2)
    assert np.array_equal(k1, k2)


def test_connect_1d_matches_oracle():
    import asgard_b200 as ab
    for L in range(0, 10):
        p1, i1 = ab.connect_1d(L)
        if L == 0:
            assert len(p1) == 2
            continue
        p2, i2 = oracle.connect_1d(L)
        assert np.array_equal(p1, p2) and np.array_equal(i1, i2)


def test_sparse_grid_sizes():
    """Cell and pair counts of the benchmark grids (n = 3)."""
    import asgard_b200 as ab
    assert ab.sparse_grid(2, 6).shape[0] == 256
    assert ab.sparse_grid(4, 7).shape[0] == 4048
    assert ab.sparse_grid(5, 7).shape[0] == 8472
    assert ab.sparse_grid(6, 7).shape[0] == 16172
    r, c, k = ab.build_pairs(2, 6, ab.sparse_grid(2, 6))
    assert len(c) == 38512


def test_advdiff_factors_use_reference_blocks():
    """Level-7 advection/diffusion factors equal the stored reference blocks."""
    import asgard_b200 as ab
    vA = ab.factor_values(2, 7, 2, "advdiff", nu=0.1).reshape(-1, 2, 2, 9)
    ops = ab.operators.ops1d()
    assert np.array_equal(vA[:, 0, 0], ops["adv"])
    assert np.allclose(vA[:, 1, 1], 0.1 * ops["dif"], rtol=0, atol=0)
    pntr, indx = ab.connect_1d(7)
    rows = np.repeat(np.arange(len(pntr) - 1), np.diff(pntr))
    diag = rows == indx
    assert np.array_equal(vA[diag, 0, 1], np.tile(np.eye(3).ravel(), (diag.sum(), 1)))
    assert not vA[~diag, 0, 1].any()


def test_invalid_plans_are_rejected():
    import asgard_b200 as ab
    from asgard_b200._lib import AsgkError
    # column out of range, factor offset out of range, bad dimension
    with pytest.raises(AsgkError):
        ab.kronmult_matrix.from_csr(2, 2, 1, 1, 1, [0, 1], [1], [0, 0], np.zeros(4))
    with pytest.raises(AsgkError):
        ab.kronmult_matrix.from_csr(2, 2, 1, 1, 1, [0, 1], [0], [0, 1], np.zeros(4))
    with pytest.raises(AsgkError):
        ab.kronmult_matrix.from_csr(7, 2, 1, 1, 1, [0, 1], [0], [0] * 7, np.zeros(4))
    with pytest.raises(AsgkError):
        ab.kronmult_matrix.from_pairs(2, 2, 1, 1, 1, [1], [0], [0, 0], np.zeros(4))


def test_default_gmres_restarts():
    """default_gmres_restarts (src/solver.cpp:142-152)."""
    import asgard_b200 as ab
    assert ab.default_gmres_restarts(5) == 5
    assert ab.default_gmres_restarts(1000) == 200
    n = 11789388
    assert ab.default_gmres_restarts(n) == max(10, min(200, int(512 / (n * 8 / 1048576))))


def test_cpp_dropin_header_compiles(tmp_path):
    """The C++ drop-in header and its driver compile and link against the
    library (running them needs a GPU: tests/test_cpp_dropin_gpu.py)."""
    from test_cpp_dropin_gpu import compile_dropin
    r = compile_dropin(tmp_path / "dropin")
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("d,L", [(2, 5), (3, 4), (4, 3)])
def test_direction_pairs_are_the_single_dimension_pairs(d, L):
    """asgk_direction_pairs lists, per cell, exactly the connected pairs whose
    cells differ in at most one dimension (the diagonal pair once per
    dimension), with that dimension's 1D connection."""
    import ctypes as C
    from asgard_b200 import lib, operators as O
    table = np.ascontiguousarray(O.sparse_grid(d, L), dtype=np.int32)
    cells = table.shape[0]
    rp, col, conn = O.build_pairs(d, L, table)
    conn = conn.reshape(-1, d)
    nnz = C.c_int64()
    assert lib.asgk_direction_pairs(d, L, cells, table.ctypes.data, C.byref(nnz),
                                    None, None, None, None) == 0
    n = nnz.value
    ptr = np.zeros(cells + 1, np.int64)
    gcol, gdim, gconn = (np.zeros(n, np.int32) for _ in range(3))
    assert lib.asgk_direction_pairs(d, L, cells, table.ctypes.data, C.byref(nnz),
                                    ptr.ctypes.data, gcol.ctypes.data,
                                    gdim.ctypes.data, gconn.ctypes.data) == 0
    lv, ps = table[:, :d], table[:, d:]
    for r in range(cells):
        got = {(int(c), int(k), int(j)) for c, k, j in
               zip(gcol[ptr[r]:ptr[r + 1]], gdim[ptr[r]:ptr[r + 1]], gconn[ptr[r]:ptr[r + 1]])}
        want = set()
        for p in range(rp[r], rp[r + 1]):
            c = int(col[p])
            diff = [k for k in range(d) if lv[r, k] != lv[c, k] or ps[r, k] != ps[c, k]]
            if len(diff) == 1:
                want.add((c, diff[0], int(conn[p, diff[0]])))
            elif not diff:
                want |= {(c, k, int(conn[p, k])) for k in range(d)}
        assert got == want, r


@pytest.mark.parametrize("d,L,T", [(2, 5, 2), (3, 4, 3), (4, 3, 2)])
def test_bench_pencil_gemm_flops(d, L, T):
    """The bench's count of the tensor-core form's useful flops: along each
    dimension with terms, a cell of a standard sparse grid lies in a pencil
    of 2^(L - s) cells (s: its levels summed over the other dimensions), so
    sum over pencils of 2 (3p)^2 3^(d-1) = sum over cells of 2 * 9 p * 3^(d-1)."""
    import bench
    import asgard_b200 as ab
    op = ab.SparseGridOperator(d, L, T, kind="advdiff")
    lev = op.table[:, :d].astype(np.int64)
    expect = 0
    for k in sorted({t % d for t in range(T)}):
        s = lev.sum(axis=1) - lev[:, k]
        p = 2 ** (L - s)
        expect += int((2 * 9 * p * 3 ** (d - 1)).sum())
    assert bench.pencil_gemm_flops(op) == expect
