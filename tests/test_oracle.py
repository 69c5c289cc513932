"""Pins the C restatement (oracle/) against the reference: golden fixtures made
by the reference itself, and the reference library when it was built here."""
import hashlib
import json

import numpy as np
import pytest

import oracle
from conftest import golden, rmse_close

KRON = np.load(golden("kronmult_data.npz"))


def kron_keys():
    out = []
    for k in KRON.files:
        if k.endswith("_ref_y"):
            tag, d, n, rows, terms, mats = k[:-len("_ref_y")].split("_")
            out.append((tag, int(d), int(n), int(rows), int(terms), int(mats)))
    return sorted(out)


@pytest.mark.parametrize("tag,d,n,rows,terms,mats", kron_keys())
def test_oracle_kronmult_reference_test_data(tag, d, n, rows, terms, mats):
    """make_kronmult_data (minstd_rand(42)) regenerated bit-exactly, and the
    oracle's pair kronmult against the reference's explicit Kronecker answer
    (src/asgard_kronmult_matrix_tests.cpp:14-118, 100 ulp rmse)."""
    dt = np.float64 if tag == "f64" else np.float32
    data = oracle.make_kronmult_data(d, n, rows, terms, mats, dt)
    key = f"{tag}_{d}_{n}_{rows}_{terms}_{mats}"
    h = hashlib.sha256()
    for a in (data["iA"], data["vA"], data["x"], data["y"]):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == bytes(KRON[key + "_inputs_sha256"]).decode()
    y = data["y"].copy()
    oracle.kronmult(d, n, data["pntr"], data["indx"], terms, data["iA"],
                    data["vA"], 1.0, data["x"], 1.0, y)
    eps = np.finfo(dt).eps
    assert rmse_close(y, KRON[key + "_ref_y"], 100 * eps)


PDES = ["continuity_2_L4", "continuity_3_L3", "continuity_6_L2", "diffusion_2_L3"]


@pytest.mark.parametrize("name", PDES)
def test_oracle_builder_matches_reference_builder(name):
    """Element table, pair list, iA of the reference's make_kronmult_sparse."""
    z = np.load(golden(f"pde_{name}.npz"))
    d, n, L, terms = int(z["d"]), int(z["n"]), int(z["level"]), int(z["terms"])
    table = oracle.sparse_grid(d, L)
    assert np.array_equal(table, z["table"])
    pntr, indx, conn = oracle.build_pairs(d, L, table)
    assert np.array_equal(pntr, z["pntr"])
    assert np.array_equal(indx, z["indx"])
    assert np.array_equal(oracle.expand_iA(d, n, terms, conn), z["iA"])


@pytest.mark.parametrize("name", PDES)
def test_oracle_apply_matches_reference_apply(name):
    z = np.load(golden(f"pde_{name}.npz"))
    d, n, terms = int(z["d"]), int(z["n"]), int(z["terms"])
    N = (len(z["pntr"]) - 1) * n ** d
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, N)
    y0 = rng.uniform(-1, 1, N)
    y = oracle.kronmult(d, n, z["pntr"], z["indx"], terms, z["iA"], z["vA"],
                        1.0, x, 0.0, np.zeros(N))
    assert np.array_equal(y, z["y"])  # same summation order: bit-exact
    y2 = oracle.kronmult(d, n, z["pntr"], z["indx"], terms, z["iA"], z["vA"],
                         -0.5, x, 2.0, y0.copy())
    assert np.array_equal(y2, z["y_ab"])


@pytest.mark.parametrize("name", ["continuity_2_L4", "continuity_3_L3", "diffusion_2_L3"])
def test_oracle_gmres_euler_matches_reference(name):
    """simple_gmres_euler: same iteration count, solution to 1e-12."""
    z = np.load(golden(f"pde_{name}.npz"))
    d, n, terms = int(z["d"]), int(z["n"]), int(z["terms"])
    N = (len(z["pntr"]) - 1) * n ** d
    rng = np.random.default_rng(7)
    rng.uniform(-1, 1, N)
    rng.uniform(-1, 1, N)
    b = rng.uniform(-1, 1, N)
    x = np.zeros(N)
    err, its = oracle.gmres_euler(d, n, z["pntr"], z["indx"], terms, z["iA"],
                                  z["vA"], float(z["dt"]), x, b, 20, 50, 1e-12)
    assert its == int(z["gmres_iters"])
    assert err <= 1e-12
    assert np.linalg.norm(x - z["gmres_x"]) <= 1e-12 * max(1, np.linalg.norm(z["gmres_x"]))


def test_oracle_gmres_known_answers():
    """The 3x3 systems of src/solver_tests.cpp:141-213."""
    case = json.load(open(golden("gmres_3x3.json")))
    A = np.array(case["A"])
    for k in ("1", "2"):
        x = np.zeros(3)
        err, its = oracle.gmres_dense(A, x, np.array(case["b" + k]), 3, 3,
                                      np.finfo(np.float64).eps)
        assert err < np.finfo(np.float64).eps
        assert its == case["ref_iters" + k]
        assert rmse_close(x, case["x" + k], 10 * np.finfo(np.float64).eps)
        assert rmse_close(x, case["ref_x" + k], 10 * np.finfo(np.float64).eps)


def test_oracle_kronecker_known_answers():
    """Known-answer Kronecker products (src/asgard_kronmult_matrix_tests.cpp:178-193)."""
    import ctypes as C
    A = np.array([1, 2, 3, 4], dtype=np.float64)
    B = np.array([10, 20, 30, 40], dtype=np.float64)
    gold = [10, 20, 20, 40, 30, 40, 60, 80, 30, 60, 40, 80, 90, 120, 120, 160]
    # K = A (x) B applied to unit vectors gives its columns
    lib = oracle.oracle()
    lib.orc_reference_kronmult_one.restype = None
    K = np.zeros(16)
    for c in range(4):
        e = np.zeros(4)
        e[c] = 1
        y = np.zeros(4)
        pa = (C.c_void_p * 2)(A.ctypes.data, B.ctypes.data)
        lib.orc_reference_kronmult_one(2, 2, pa, e.ctypes.data_as(C.c_void_p),
                                       y.ctypes.data_as(C.c_void_p))
        K[c * 4:(c + 1) * 4] = y
    assert np.array_equal(K, gold)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference not built here")
def test_oracle_matches_compiled_reference():
    """connect_1d for levels 1..9 and cpu_sparse on random data, bit-exact."""
    R = oracle.ref()
    for L in range(1, 10):
        p1, i1 = oracle.connect_1d(L)
        p2, i2 = oracle.connect_1d(L, lib=R)
        assert np.array_equal(p1, p2) and np.array_equal(i1, i2)
    for (d, n, rows, terms, mats) in [(2, 3, 12, 3, 7), (4, 3, 6, 2, 7), (6, 2, 5, 2, 7)]:
        data = oracle.make_kronmult_data(d, n, rows, terms, mats)
        y1 = data["y"].copy()
        y2 = data["y"].copy()
        oracle.kronmult(d, n, data["pntr"], data["indx"], terms, data["iA"],
                        data["vA"], 0.7, data["x"], -1.0, y1)
        oracle.kronmult(d, n, data["pntr"], data["indx"], terms, data["iA"],
                        data["vA"], 0.7, data["x"], -1.0, y2, lib=R)
        assert np.array_equal(y1, y2)


def test_oracle_planted_mistake_is_caught():
    """A wrong factor in the oracle's input must change the answer well above
    the parity tolerance (guards against a vacuous comparison)."""
    data = oracle.make_kronmult_data(3, 3, 6, 2, 7)
    y1 = oracle.kronmult(3, 3, data["pntr"], data["indx"], 2, data["iA"],
                         data["vA"], 1.0, data["x"], 0.0, np.zeros_like(data["y"]))
    vA = data["vA"].copy()
    vA[4] += 1e-6
    y2 = oracle.kronmult(3, 3, data["pntr"], data["indx"], 2, data["iA"], vA,
                         1.0, data["x"], 0.0, np.zeros_like(data["y"]))
    assert np.linalg.norm(y1 - y2) / np.linalg.norm(y1) > 1e-9


def test_mlp_oracle_gradient_matches_finite_differences():
    """The float64 network oracle's backward pass against central finite
    differences (it is the checker of the GPU gradients)."""
    from oracle import mlp_oracle
    rng = np.random.default_rng(0)
    ts, d, H = 5, 3, 6
    nparams = sum(int(np.prod(s)) for _, s in mlp_oracle.layout(ts, d, H))
    p = rng.normal(0, 0.5, nparams)
    X = rng.normal(0, 1, (4, ts + d))
    T = rng.normal(0, 1, (4, ts))
    _, _, g = mlp_oracle.forward_backward(p, ts, d, H, X, T)
    h = 1e-6
    for i in rng.choice(nparams, 40, replace=False):
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp_oracle.forward_backward(pp, ts, d, H, X, T)[1] -
              mlp_oracle.forward_backward(pm, ts, d, H, X, T)[1]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd))


def test_mlp_oracle_is_linear_in_the_residual():
    from oracle import mlp_oracle
    rng = np.random.default_rng(1)
    ts, d, H = 9, 2, 8
    nparams = sum(int(np.prod(s)) for _, s in mlp_oracle.layout(ts, d, H))
    p = rng.normal(0, 0.5, nparams)
    lam = rng.uniform(0, 1, (3, d))
    u1, u2 = rng.normal(0, 1, (3, ts)), rng.normal(0, 1, (3, ts))
    Z = np.zeros((3, ts))
    f = lambda u: mlp_oracle.forward_backward(p, ts, d, H, np.hstack([u, lam]), Z)[0]
    assert np.allclose(f(2 * u1 - 3 * u2), 2 * f(u1) - 3 * f(u2), atol=1e-12)


def test_jacobi_restatements_against_dense_assembly():
    """The point-Jacobi diagonal and the cell-diagonal blocks of the oracle
    equal the diagonal entries / blocks of K assembled column by column from
    the oracle's kronmult (d = 2, level 3, random factors)."""
    import asgard_b200.operators as O
    d, L, T = 2, 3, 2
    op = O.SparseGridOperator(d, L, T, kind="random", seed=4)
    pntr, iA = op.row_ptr.astype(np.int32), op.iA()
    ts, N = 3 ** d, op.N
    K = np.zeros((N, N))
    for j in range(N):
        e = np.zeros(N)
        e[j] = 1.0
        K[:, j] = oracle.kronmult(d, 3, pntr, op.col, T, iA, op.vA, 1.0, e, 0.0, np.zeros(N))
    blocks = oracle.diagonal_blocks(d, 3, pntr, op.col, T, iA, op.vA)
    for c in range(op.rows):
        assert np.allclose(blocks[c], K[c * ts:(c + 1) * ts, c * ts:(c + 1) * ts], rtol=0, atol=1e-14)
    pc = oracle.point_jacobi_diag(d, 3, pntr, op.col, T, iA, op.vA)
    assert np.allclose(pc, np.diag(K), rtol=0, atol=1e-14)


@pytest.mark.skipif(not oracle.ref_global_available(),
                    reason="reference global-kron library not built (make -C oracle ref_global)")
@pytest.mark.parametrize("d,L,T,kind", [(1, 5, 2, "advdiff"), (2, 5, 3, "advdiff"),
                                        (3, 4, 3, "advdiff"), (4, 3, 4, "advdiff"),
                                        (2, 4, 2, "random"), (3, 4, 2, "random"),
                                        (4, 3, 2, "random")])
def test_reference_global_kron_equals_pair_kronmult(d, L, T, kind):
    """The reference's global Kronecker product (compiled from its sources in
    KRON_MODE_GLOBAL) and the connected-pair kronmult give the same operator,
    for terms acting in one dimension each (advection/diffusion factors) and
    for terms acting in every dimension (random factors, its upper/lower
    permutations) -- the identity the global form of this library rests on."""
    import asgard_b200.operators as O
    op = O.SparseGridOperator(d, L, T, kind=kind)
    x = np.random.default_rng(d).uniform(-1, 1, op.N)
    y_ref, _ = oracle.ref_global_apply(d, 3, L, op.table, T, op.vA, x)
    y_pair = oracle.kronmult(d, 3, op.row_ptr.astype(np.int32), op.col, T,
                             op.iA(), op.vA, 1.0, x, 0.0, np.zeros(op.N))
    assert np.linalg.norm(y_ref - y_pair) <= 1e-13 * np.linalg.norm(y_pair)
