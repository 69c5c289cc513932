"""Parity of the CUDA kronmult (through the C ABI) with the oracle and with the
reference's own answers.

Tolerances: FP64 results within 1e-13 relative (L2) of the oracle; the
reference tests' rmse criterion at 100 ulp against their explicit-Kronecker
answers; FP32 arithmetic within 1e-5 relative."""
import numpy as np
import pytest

import oracle
from conftest import golden, rel_err, rmse_close

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-13
FP32_TOL = 1e-5

# the reference's GPU sparse test shapes (src/asgard_kronmult_matrix_tests.cpp:307-378)
REF_GPU_SHAPES = (
    [(1, n, 11, 2, 7) for n in range(1, 11)]
    + [(2, n, 13, 2, 7) for n in list(range(1, 21)) + list(range(22, 33))]
    + [(3, n, 17, 3, 7) for n in range(1, 11)]
    + [(4, n, 10, 3, 7) for n in range(1, 6)]
    + [(5, n, 10, 2, 7) for n in range(1, 5)]
    + [(6, n, 8, 2, 7) for n in range(1, 5)]
)


def to_dev(a, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def gpu_apply(mat, alpha, x, beta, y, precision="fp64"):
    import torch
    xd, yd = to_dev(x), to_dev(y)
    mat.apply(alpha, xd, beta, yd, precision=precision)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def pair_format(data, rows, ts):
    iy = np.repeat(np.arange(rows), rows).astype(np.int32) * ts
    ix = np.tile(np.arange(rows), rows).astype(np.int32) * ts
    return iy, ix


@pytest.mark.parametrize("d,n,rows,terms,mats", REF_GPU_SHAPES)
def test_reference_gpu_test_shapes_fp64(cuda, d, n, rows, terms, mats):
    import asgard_b200 as ab
    data = oracle.make_kronmult_data(d, n, rows, terms, mats, np.float64)
    ts = n ** d
    expect = oracle.kronmult(d, n, data["pntr"], data["indx"], terms,
                             data["iA"], data["vA"], 1.0, data["x"], 1.0,
                             data["y"].copy())
    # the reference GPU test builds the pair format (row_indx, col_indx)
    iy, ix = pair_format(data, rows, ts)
    mat = ab.kronmult_matrix.from_pairs(d, n, rows, rows, terms, iy, ix,
                                        data["iA"], data["vA"])
    got = gpu_apply(mat, 1.0, data["x"], 1.0, data["y"])
    assert rel_err(got, expect) < FP64_TOL
    assert rmse_close(got, expect, 100 * np.finfo(np.float64).eps)
    # and the CPU (CSR) format
    mat2 = ab.kronmult_matrix.from_csr(d, n, rows, rows, terms, data["pntr"],
                                       data["indx"], data["iA"], data["vA"])
    got2 = gpu_apply(mat2, 1.0, data["x"], 1.0, data["y"])
    assert rel_err(got2, expect) < FP64_TOL


KRON = np.load(golden("kronmult_data.npz"))


@pytest.mark.parametrize("key", sorted(k[:-6] for k in KRON.files if k.endswith("_ref_y")))
def test_reference_explicit_kronecker_answers(cuda, key):
    """Against the reference's own explicit-Kronecker answers, at the reference
    tests' 100-ulp rmse (src/asgard_kronmult_matrix_tests.cpp:115)."""
    import asgard_b200 as ab
    import torch
    tag, d, n, rows, terms, mats = key.split("_")
    d, n, rows, terms, mats = map(int, (d, n, rows, terms, mats))
    dt = np.float64 if tag == "f64" else np.float32
    data = oracle.make_kronmult_data(d, n, rows, terms, mats, dt)
    mat = ab.kronmult_matrix.from_csr(d, n, rows, rows, terms, data["pntr"],
                                      data["indx"], data["iA"],
                                      data["vA"].astype(np.float64))
    xd, yd = to_dev(data["x"]), to_dev(data["y"])
    mat.apply(1.0, xd, 1.0, yd)
    torch.cuda.synchronize()
    got = yd.cpu().numpy()
    assert rmse_close(got, KRON[key + "_ref_y"], 100 * np.finfo(dt).eps)


@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (1.0, 1.0), (-1.0, 1.0),
                                        (0.3, -1.0), (-2.5, 2.0), (1.0, -1.0)])
def test_alpha_beta_cases(cuda, alpha, beta):
    import asgard_b200 as ab
    d, n, rows, terms, mats = 4, 3, 7, 3, 7
    data = oracle.make_kronmult_data(d, n, rows, terms, mats)
    y0 = data["y"].copy()
    if beta == 0.0:
        y0[::7] = np.nan  # beta = 0 overwrites y, NaNs included
    expect = oracle.kronmult(d, n, data["pntr"], data["indx"], terms,
                             data["iA"], data["vA"], alpha, data["x"], beta,
                             y0.copy())
    mat = ab.kronmult_matrix.from_csr(d, n, rows, rows, terms, data["pntr"],
                                      data["indx"], data["iA"], data["vA"])
    got = gpu_apply(mat, alpha, data["x"], beta, y0)
    assert np.isfinite(got).all()
    assert rel_err(got, expect) < FP64_TOL


PDES = ["continuity_2_L4", "continuity_3_L3", "continuity_6_L2", "diffusion_2_L3"]


@pytest.mark.parametrize("name", PDES)
def test_reference_pde_operators(cuda, name):
    """Operators built by the reference's make_kronmult_sparse: y = K x and
    y = 2 y0 - 0.5 K x against the reference's own apply."""
    import asgard_b200 as ab
    z = np.load(golden(f"pde_{name}.npz"))
    d, n, terms = int(z["d"]), int(z["n"]), int(z["terms"])
    rows = len(z["pntr"]) - 1
    N = rows * n ** d
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, N)
    y0 = rng.uniform(-1, 1, N)
    mat = ab.kronmult_matrix.from_csr(d, n, rows, rows, terms, z["pntr"],
                                      z["indx"], z["iA"], z["vA"])
    assert rel_err(gpu_apply(mat, 1.0, x, 0.0, np.zeros(N)), z["y"]) < FP64_TOL
    assert rel_err(gpu_apply(mat, -0.5, x, 2.0, y0), z["y_ab"]) < FP64_TOL
    # same operator through the library's own builder (conn format)
    L = int(z["level"])
    table = ab.sparse_grid(d, L)
    rp, col, conn = ab.build_pairs(d, L, table)
    mat2 = ab.kronmult_matrix.from_conn(d, n, rows, rows, terms, rp, col, conn,
                                        z["vA"])
    assert rel_err(gpu_apply(mat2, 1.0, x, 0.0, np.zeros(N)), z["y"]) < FP64_TOL


def test_config1_against_dense_assembly(cuda):
    """d=2, n=3, level 6, 3 terms, random factors: y = K x against the dense
    FP64 assembly of the whole operator."""
    import asgard_b200 as ab
    op = ab.SparseGridOperator(2, 6, 3, kind="random", seed=0)
    assert (op.rows, op.nnz) == (256, 38512)
    iA = op.iA()
    K = np.zeros(op.N * op.N)
    oracle.oracle().orc_assemble_dense(2, 3, op.rows, op.row_ptr.astype(np.int32),
                                       op.col, 3, iA, op.vA, K)
    K = K.reshape(op.N, op.N, order="F")
    x = np.random.default_rng(1).uniform(-1, 1, op.N)
    expect = K @ x
    got = gpu_apply(op.kronmult_matrix(), 1.0, x, 0.0, np.zeros(op.N))
    assert rel_err(got, expect) < FP64_TOL
    got2 = gpu_apply(op.kronmult_matrix(expanded=True), 1.0, x, 0.0, np.zeros(op.N))
    assert rel_err(got2, expect) < FP64_TOL


@pytest.mark.parametrize("d,L,terms,kind", [(2, 7, 2, "advdiff"), (3, 5, 3, "advdiff"),
                                            (4, 4, 4, "advdiff"), (5, 3, 4, "random"),
                                            (6, 2, 6, "advdiff"), (6, 3, 2, "random")])
def test_sparse_grid_operators_fp64_fp32(cuda, d, L, terms, kind):
    import asgard_b200 as ab
    op = ab.SparseGridOperator(d, L, terms, kind=kind, seed=3)
    iA = op.iA()
    pntr = op.row_ptr.astype(np.int32)
    x = np.random.default_rng(2).uniform(-1, 1, op.N)
    y0 = np.random.default_rng(3).uniform(-1, 1, op.N)
    expect = oracle.kronmult(d, 3, pntr, op.col, terms, iA, op.vA, 0.7, x,
                             -1.3, y0.copy())
    mat = op.kronmult_matrix()
    assert rel_err(gpu_apply(mat, 0.7, x, -1.3, y0), expect) < FP64_TOL
    mat_e = op.kronmult_matrix(expanded=True)
    assert rel_err(gpu_apply(mat_e, 0.7, x, -1.3, y0), expect) < FP64_TOL
    # FP32 arithmetic on FP64 vectors, and FP32 vectors
    assert rel_err(gpu_apply(mat, 0.7, x, -1.3, y0, precision="fp32"), expect) < FP32_TOL
    import torch
    xf, yf = to_dev(x.astype(np.float32)), to_dev(y0.astype(np.float32))
    mat.apply(0.7, xf, -1.3, yf)
    torch.cuda.synchronize()
    assert rel_err(yf.cpu().numpy(), expect) < FP32_TOL


def test_euler_operator(cuda):
    """y = beta*y + alpha*(x - dt*K*x), the matvec of simple_gmres_euler."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(3, 5, 3, kind="advdiff")
    mat = op.kronmult_matrix()
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, op.N)
    y0 = rng.uniform(-1, 1, op.N)
    dt, alpha, beta = 1e-3, -1.0, 1.0
    kx = oracle.kronmult(3, 3, op.row_ptr.astype(np.int32), op.col, 3, op.iA(),
                         op.vA, 1.0, x, 0.0, np.zeros(op.N))
    expect = beta * y0 + alpha * (x - dt * kx)
    xd, yd = to_dev(x), to_dev(y0)
    mat.apply_euler(dt, alpha, xd, beta, yd)
    torch.cuda.synchronize()
    assert rel_err(yd.cpu().numpy(), expect) < FP64_TOL


def test_host_resource_apply(cuda):
    """apply<resource::host>: host vectors copied in and out inside the call."""
    import asgard_b200 as ab
    op = ab.SparseGridOperator(4, 4, 4, kind="advdiff")
    mat = op.kronmult_matrix()
    x = np.random.default_rng(9).uniform(-1, 1, op.N)
    y = np.random.default_rng(10).uniform(-1, 1, op.N)
    expect = oracle.kronmult(4, 3, op.row_ptr.astype(np.int32), op.col, 4,
                             op.iA(), op.vA, 1.0, x, 1.0, y.copy())
    mat.apply(1.0, x, 1.0, y, resource="host")
    assert rel_err(y, expect) < FP64_TOL


def test_host_apply_in_caller_workspace(cuda):
    """set_workspace (src/asgard_kronmult_matrix.hpp:301-307): host applies
    stage x and y in the caller's device buffers, which two plans share;
    buffers shorter than input_size / output_size are refused."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(3, 4, 3, kind="advdiff")
    m1, m2 = op.kronmult_matrix(), op.kronmult_matrix(mode="dense")
    wx = torch.zeros(op.N, dtype=torch.float64, device="cuda")
    wy = torch.zeros(op.N, dtype=torch.float64, device="cuda")
    m1.set_workspace(wx, wy)
    m2.set_workspace(wx, wy)
    rng = np.random.default_rng(4)
    x, y0 = rng.uniform(-1, 1, op.N), rng.uniform(-1, 1, op.N)
    expect = oracle.kronmult(3, 3, op.row_ptr.astype(np.int32), op.col, 3,
                             op.iA(), op.vA, 0.5, x, -2.0, y0.copy())
    for m in (m1, m2):
        y = y0.copy()
        m.apply(0.5, x, -2.0, y, resource="host")
        assert rel_err(y, expect) < FP64_TOL
        assert np.array_equal(wx.cpu().numpy(), x)
    with pytest.raises(ab.AsgkError):
        m1.set_workspace(wx[:-1], wy)


def test_empty_rows_and_no_terms(cuda):
    import asgard_b200 as ab
    # 3 output cells, the middle one without pairs
    d, n, terms = 2, 3, 2
    rng = np.random.default_rng(0)
    pntr = np.array([0, 2, 2, 3])
    indx = np.array([0, 2, 1], np.int32)
    vA = rng.uniform(-1, 1, 9 * 5)
    iA = (rng.integers(0, 5, size=3 * terms * d) * 9).astype(np.int32)
    x = rng.uniform(-1, 1, 27)
    y0 = rng.uniform(-1, 1, 27)
    expect = oracle.kronmult(d, n, pntr.astype(np.int32), indx, terms, iA, vA,
                             1.0, x, 2.0, y0.copy())
    mat = ab.kronmult_matrix.from_csr(d, n, 3, 3, terms, pntr, indx, iA, vA)
    got = gpu_apply(mat, 1.0, x, 2.0, y0)
    assert rel_err(got, expect) < FP64_TOL
    assert np.allclose(got[9:18], 2.0 * y0[9:18], rtol=0, atol=0)
    # no terms: only beta scales y (src/asgard_kronmult_matrix.hpp:344-349)
    mat0 = ab.kronmult_matrix.from_csr(d, n, 3, 3, 0, pntr, indx, [], vA)
    assert np.array_equal(gpu_apply(mat0, 1.0, x, -3.0, y0), -3.0 * y0)


def test_full_size_properties(cuda):
    """d=4, level 7 (12.3 M pairs, the benchmark operator): linearity
    K(a x1 + b x2) = a K x1 + b K x2, Euler identity and run-to-run
    bit-reproducibility (no atomics)."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(4, 7, 4, kind="advdiff")
    mat = op.kronmult_matrix()
    g = torch.Generator(device="cuda").manual_seed(0)
    x1 = torch.rand(op.N, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    x2 = torch.rand(op.N, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    a, b = 0.75, -1.25
    y1 = torch.zeros_like(x1)
    y2 = torch.zeros_like(x1)
    y3 = torch.zeros_like(x1)
    mat.apply(1.0, x1, 0.0, y1)
    mat.apply(1.0, x2, 0.0, y2)
    mat.apply(1.0, a * x1 + b * x2, 0.0, y3)
    lhs, rhs = y3, a * y1 + b * y2
    assert (torch.linalg.norm(lhs - rhs) / torch.linalg.norm(rhs)).item() < 1e-13
    y1b = torch.zeros_like(x1)
    mat.apply(1.0, x1, 0.0, y1b)
    assert torch.equal(y1, y1b)
    ye = torch.zeros_like(x1)
    mat.apply_euler(1e-3, 1.0, x1, 0.0, ye)
    assert (torch.linalg.norm(ye - (x1 - 1e-3 * y1)) / torch.linalg.norm(ye)).item() < 1e-14


@pytest.mark.parametrize("d,L", [(3, 4), (4, 3), (4, 4)])
def test_staged_kernel_alignment_and_status(cuda, d, L):
    """The n = 3, d = 3/4 kernel copies x tensors to shared memory in 16-byte
    aligned pieces: x views offset by one double and odd or even cell counts
    (63 / 104 / 192 cells here) take the same result, in FP64 and FP32, and
    no bounded wait in the kernel expires."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(d, L, d, kind="advdiff", seed=1)
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, op.N)
    y0 = rng.uniform(-1, 1, op.N)
    expect = oracle.kronmult(d, 3, op.row_ptr.astype(np.int32), op.col, d,
                             op.iA(), op.vA, -0.4, x, 0.5, y0.copy())
    for mat in (op.kronmult_matrix(), op.kronmult_matrix(expanded=True)):
        for off in (0, 1):
            buf = torch.zeros(op.N + 2, dtype=torch.float64, device="cuda")
            xd = buf[off:off + op.N]
            xd.copy_(torch.from_numpy(x))
            for prec, tol in (("fp64", FP64_TOL), ("fp32", FP32_TOL)):
                yd = to_dev(y0)
                mat.apply(-0.4, xd, 0.5, yd, precision=prec)
                torch.cuda.synchronize()
                assert rel_err(yd.cpu().numpy(), expect) < tol, (off, prec)
            # the input is left untouched
            assert torch.equal(xd.cpu(), torch.from_numpy(x))
    assert ab.lib.asgk_device_status(1) == 0


@pytest.mark.parametrize("d,L,T", [(1, 6, 2), (2, 5, 2), (3, 5, 3), (4, 4, 4),
                                   (5, 3, 3), (6, 3, 2), (4, 7, 4)])
def test_device_built_pairs_match_host_built(cuda, d, L, T):
    """asgk_plan_create_grid (connected pairs found on the GPU) makes the
    plan the host builder makes: the same pairs in the same order, so the
    applies agree bit for bit, FP64, FP32 and Euler."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(d, L, T, kind="advdiff")
    mh = op.kronmult_matrix()
    md = ab.kronmult_matrix.from_grid(d, 3, L, T, op.vA)
    assert md.num_pairs() == mh.num_pairs() == op.nnz
    assert md.num_rows == op.rows and md.output_size() == op.N
    rng = np.random.default_rng(d)
    x, y0 = to_dev(rng.uniform(-1, 1, op.N)), rng.uniform(-1, 1, op.N)
    for prec in ("fp64", "fp32"):
        ya, yb = to_dev(y0), to_dev(y0)
        mh.apply(0.7, x, -1.3, ya, precision=prec)
        md.apply(0.7, x, -1.3, yb, precision=prec)
        torch.cuda.synchronize()
        assert np.array_equal(ya.cpu().numpy(), yb.cpu().numpy()), prec
    ya, yb = to_dev(y0), to_dev(y0)
    mh.apply_euler(1e-3, -1.0, x, 0.5, ya)
    md.apply_euler(1e-3, -1.0, x, 0.5, yb)
    torch.cuda.synchronize()
    assert np.array_equal(ya.cpu().numpy(), yb.cpu().numpy())
