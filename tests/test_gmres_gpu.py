"""Device-resident GMRES through the C ABI against the oracle and the
reference's known answers."""
import json

import numpy as np
import pytest

import oracle
from conftest import golden, rel_err, rmse_close

pytestmark = pytest.mark.gpu


def to_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def test_gmres_known_answers(cuda):
    """The 3x3 systems of src/solver_tests.cpp:141-213 (no preconditioner):
    error below machine epsilon, x equal to the gold answer."""
    import asgard_b200 as ab
    case = json.load(open(golden("gmres_3x3.json")))
    A = np.array(case["A"])
    eps = np.finfo(np.float64).eps
    for k in ("1", "2"):
        x = np.zeros(3)
        info = ab.simple_gmres(A, x, np.array(case["b" + k]), None, 3, 3, eps)
        assert info.error < eps
        assert info.iterations == case["ref_iters" + k]
        assert rmse_close(x, case["x" + k], 10 * eps)


def test_gmres_known_answers_preconditioned(cuda):
    """The point-Jacobi preconditioned 3x3 cases of src/solver_tests.cpp:
    175-213 through the reference's dense preconditioner (LU of M applied on
    the left): error below machine epsilon and x equal to the gold answer, as
    the reference's test requires.  Iterations: the reference's count
    (reference-made fixture) or one more restart cycle -- after 3 Arnoldi
    steps on a 3x3 system the estimated residual is rounding noise around
    the machine-epsilon tolerance, so one cycle more or less depends on the
    last bits of the device's dot products."""
    import asgard_b200 as ab
    case = json.load(open(golden("gmres_3x3.json")))
    A, M = np.array(case["A"]), np.array(case["M"])
    eps = np.finfo(np.float64).eps
    for k in ("1", "2"):
        x = np.zeros(3)
        info = ab.simple_gmres(A, x, np.array(case["b" + k]), M, 3, 3, eps)
        assert info.status == 0
        assert info.error < eps
        assert info.iterations in (case["ref_pre_iters" + k], case["ref_pre_iters" + k] + 4)
        assert rmse_close(x, case["x" + k], 10 * eps)
        assert rmse_close(x, case["ref_pre_x" + k], 10 * eps)
    # a singular M is refused before any device work
    with pytest.raises(ab.AsgkError):
        ab.simple_gmres(A, np.zeros(3), np.array(case["b1"]), np.zeros((3, 3)), 3, 3, eps)


@pytest.mark.parametrize("name", ["continuity_2_L4", "continuity_3_L3", "diffusion_2_L3"])
def test_gmres_euler_reference_pdes(cuda, name):
    """simple_gmres_euler on reference-built operators: the reference's answer
    (restart 20, 50 restarts, absolute tolerance 1e-12), same iteration count
    as the reference up to one step."""
    import asgard_b200 as ab
    import torch
    z = np.load(golden(f"pde_{name}.npz"))
    d, n, terms = int(z["d"]), int(z["n"]), int(z["terms"])
    rows = len(z["pntr"]) - 1
    N = rows * n ** d
    rng = np.random.default_rng(7)
    rng.uniform(-1, 1, N)
    rng.uniform(-1, 1, N)
    b = rng.uniform(-1, 1, N)
    mat = ab.kronmult_matrix.from_csr(d, n, rows, rows, terms, z["pntr"],
                                      z["indx"], z["iA"], z["vA"])
    x = torch.zeros(N, dtype=torch.float64, device="cuda")
    info = ab.simple_gmres_euler(float(z["dt"]), mat, x, to_dev(b), 20, 50, 1e-12)
    assert info.status == 0
    assert info.error <= 1e-12
    assert abs(info.iterations - int(z["gmres_iters"])) <= 1
    xs = x.cpu().numpy()
    assert rel_err(xs, z["gmres_x"]) < 1e-10
    assert info.true_relres < 1e-11


def test_gmres_euler_matches_oracle_iterations(cuda):
    """Synthetic advection/diffusion operator, reference (absolute) criterion:
    the oracle's restarted GMRES and the device GMRES agree."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(2, 6, 2, kind="advdiff", nu=0.1)
    b = np.random.default_rng(11).uniform(-1, 1, op.N)
    xo = np.zeros(op.N)
    err_o, its_o = oracle.gmres_euler(2, 3, op.row_ptr.astype(np.int32), op.col,
                                      2, op.iA(), op.vA, 1e-3, xo, b, 30, 40, 1e-9)
    x = torch.zeros(op.N, dtype=torch.float64, device="cuda")
    info = ab.simple_gmres_euler(1e-3, op.kronmult_matrix(), x, to_dev(b), 30, 40, 1e-9)
    assert info.status == 0
    assert abs(info.iterations - its_o) <= 2
    assert rel_err(x.cpu().numpy(), xo) < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gmres_relative_tolerance_true_residual(cuda, precision):
    """1e-10 relative residual, checked in FP64; the FP32 operator runs inside
    FP64 iterative refinement."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(3, 5, 3, kind="advdiff", nu=0.1)
    b = to_dev(np.random.default_rng(4).uniform(-1, 1, op.N))
    x = torch.zeros(op.N, dtype=torch.float64, device="cuda")
    info = ab.simple_gmres_euler(1e-3, op.kronmult_matrix(), x, b, 50, 100,
                                 1e-10, tol_mode="rel", precision=precision)
    assert info.status == 0
    assert info.true_relres <= 1e-10
    if precision == "fp32":
        assert info.matvecs_low > 0 and info.outer_steps >= 2


def test_gmres_restart_larger_than_system(cuda):
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(1, 2, 1, kind="random")
    x = torch.zeros(op.N, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        ab.simple_gmres_euler(1e-3, op.kronmult_matrix(), x, x.clone(), op.N + 1, 1, 1e-10)


def test_gmres_nonfinite_input_reports_status(cuda):
    """A NaN planted in b (host-side fault injection) ends the solve with a
    non-finite status instead of iterating on garbage."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(2, 4, 2, kind="advdiff")
    b = np.random.default_rng(0).uniform(-1, 1, op.N)
    b[5] = np.nan
    x = torch.zeros(op.N, dtype=torch.float64, device="cuda")
    info = ab.simple_gmres_euler(1e-3, op.kronmult_matrix(), x, to_dev(b), 10, 5, 1e-10)
    assert info.status == 7  # ASGK_ERR_NONFINITE


@pytest.mark.parametrize("n,k", [(1000, 1), (327888, 7), (50001, 51)])
def test_cgs_step_against_fp64_reference(cuda, n, k):
    """One Gram-Schmidt step (src/solver.cpp:233-245) against numpy in FP64."""
    import asgard_b200 as ab
    import torch
    rng = np.random.default_rng(n + k)
    V = rng.uniform(-1, 1, (k, n))
    w = rng.uniform(-1, 1, n)
    h_ref = V @ w
    w_ref = w - V.T @ h_ref
    Vd = torch.from_numpy(V).cuda()
    wd = torch.from_numpy(w).cuda()
    h, nrm = ab.cgs_step(Vd, k, wd)
    assert rel_err(h.cpu().numpy(), h_ref) < 1e-13
    assert rel_err(wd.cpu().numpy(), w_ref) < 1e-13
    assert abs(nrm - np.linalg.norm(w_ref)) <= 1e-13 * np.linalg.norm(w_ref)


@pytest.mark.parametrize("mode,precond,precision", [
    ("pairs", None, "fp64"), ("pairs", "point", "fp64"),
    ("global", "block", "fp32"), ("global", None, "fp32"), ("global", "kron", "fp32"),
    ("global", "line", "fp32"), ("global", "line", "fp64"), ("dense", "block", "fp64")])
def test_recorded_cycles_match_host_driven_cycles(cuda, mode, precond, precision):
    """Restart cycles run as recorded CUDA graphs (device-side Givens steps,
    one launch per cycle) give the host-driven loop's iterates bit for bit:
    same iteration counts, same solution, same reported residuals; and the
    launch counter sees every kernel the recorded cycles run."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(3, 5, 3, kind="advdiff")
    mat = op.kronmult_matrix(mode=mode)
    dt = 4e-3
    pc = ab.JacobiPreconditioner(mat, dt, kind=precond) if precond else None
    b = torch.from_numpy(np.random.default_rng(8).uniform(-1, 1, op.N)).cuda()
    out = {}
    try:
        for graphs in (0, 1):
            ab.lib.asgk_set_gmres_graphs(graphs)
            for rep in range(2):          # the second solve reuses the recording
                x = torch.zeros_like(b)
                l0 = ab.launch_count()
                info = ab.simple_gmres_euler(dt, mat, x, b, 30, 200, 1e-10,
                                             tol_mode="rel", precision=precision,
                                             precond=pc)
                torch.cuda.synchronize()
                out[(graphs, rep)] = (x.cpu().numpy(), info, ab.launch_count() - l0)
    finally:
        ab.lib.asgk_set_gmres_graphs(1)
    xh, ih, lh = out[(0, 1)]
    for rep in (0, 1):
        xg, ig, lg = out[(1, rep)]
        assert ig.status == 0 and ig.true_relres <= 1e-10
        assert ig.iterations == ih.iterations and ig.outer_steps == ih.outer_steps
        assert np.array_equal(xg, xh)
        assert ig.error == ih.error and ig.true_relres == ih.true_relres
        # every executed step's kernels are counted (operator, two
        # Gram-Schmidt passes, preconditioner or scaling: at least three)
        assert lg >= 3 * ig.iterations and lh >= 3 * ih.iterations


@pytest.mark.parametrize("precond", [None, "kron"])
def test_fp32_basis_gram_schmidt(cuda, precond):
    """FP32 inner solves orthogonalise against an FP32 copy of the basis
    (the default) or the FP64 basis: both reach the 1e-10 FP64 relative
    residual with nearly the same iteration counts, and the solutions agree
    to the accuracy the residual allows."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(3, 5, 3, kind="advdiff", nu=0.1)
    mat = op.kronmult_matrix(mode="global")
    dt = 1e-3
    pc = ab.JacobiPreconditioner(mat, dt, kind=precond) if precond else None
    b = to_dev(np.random.default_rng(12).uniform(-1, 1, op.N))
    res = {}
    try:
        for basis in (0, 1):
            ab.lib.asgk_set_gmres_basis(basis)
            x = torch.zeros_like(b)
            info = ab.simple_gmres_euler(dt, mat, x, b, 50, 200, 1e-10, tol_mode="rel",
                                         precision="fp32", precond=pc)
            assert info.status == 0 and info.true_relres <= 1e-10
            res[basis] = (x.cpu().numpy(), info)
    finally:
        ab.lib.asgk_set_gmres_basis(1)
    (x64, i64), (x32, i32) = res[0], res[1]
    assert abs(i32.iterations - i64.iterations) <= 2 + i64.iterations // 10, \
        (i32.iterations, i64.iterations)
    assert rel_err(x32, x64) < 1e-7


@pytest.mark.parametrize("precond,precision", [(None, "fp32"), ("kron", "fp32"),
                                               ("block", "fp64"), ("line", "fp32")])
def test_node_steps_give_the_same_iterates(cuda, precond, precision):
    """Recorded cycles with several Arnoldi steps per graph node (the kernels
    of steps after the cycle stopped skip themselves) give the iterates of
    one step per node bit for bit, whatever the node size and wherever the
    cycles stop inside a node."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(3, 5, 3, kind="advdiff")
    mat = op.kronmult_matrix(mode="global")
    dt = 4e-3
    pc = ab.JacobiPreconditioner(mat, dt, kind=precond) if precond else None
    b = torch.from_numpy(np.random.default_rng(21).uniform(-1, 1, op.N)).cuda()
    out = {}
    old = ab.lib.asgk_set_gmres_node_steps(0)
    try:
        for steps in (1, 3, 8, 30):
            ab.lib.asgk_set_gmres_node_steps(steps)
            x = torch.zeros_like(b)
            l0 = ab.launch_count()
            info = ab.simple_gmres_euler(dt, mat, x, b, 30, 200, 1e-10,
                                         tol_mode="rel", precision=precision,
                                         precond=pc)
            torch.cuda.synchronize()
            assert info.status == 0 and info.true_relres <= 1e-10
            out[steps] = (x.cpu().numpy(), info, ab.launch_count() - l0)
    finally:
        ab.lib.asgk_set_gmres_node_steps(old)
    x1, i1, l1 = out[1]
    for steps in (3, 8, 30):
        xs, i_s, ls = out[steps]
        assert i_s.iterations == i1.iterations and i_s.outer_steps == i1.outer_steps
        assert np.array_equal(xs, x1)
        assert i_s.error == i1.error and i_s.true_relres == i1.true_relres
        assert ls == l1  # skipped launches are not counted as work


@pytest.mark.parametrize("graphs", [0, 1])
def test_line_preconditioner_fused_fp32_copy(cuda, graphs):
    """At d >= 5 the line preconditioner's last pass also writes the FP32
    copy of its output that the FP32 global operator reads (no separate
    conversion pass): the iterates equal those with the separate pass bit
    for bit, host-driven and recorded."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(5, 4, 5, kind="advdiff", nu=0.1)
    mat = op.kronmult_matrix(mode="global")
    dt = 1e-3
    pc = ab.JacobiPreconditioner(mat, dt, kind="line")
    b = to_dev(np.random.default_rng(21).uniform(-1, 1, op.N))
    res = {}
    old_graphs = ab.lib.asgk_set_gmres_graphs(graphs)
    try:
        for fused in (0, 1):
            ab.lib.asgk_set_gmres_fused_copy(fused)
            x = torch.zeros_like(b)
            l0 = ab.launch_count()
            info = ab.simple_gmres_euler(dt, mat, x, b, 30, 200, 1e-10, tol_mode="rel",
                                         precision="fp32", precond=pc)
            torch.cuda.synchronize()
            assert info.status == 0 and info.true_relres <= 1e-10
            res[fused] = (x.cpu().numpy(), info, ab.launch_count() - l0)
    finally:
        ab.lib.asgk_set_gmres_fused_copy(1)
        ab.lib.asgk_set_gmres_graphs(old_graphs)
    (xs, i_s, ls), (xf, i_f, lf) = res[0], res[1]
    assert i_f.iterations == i_s.iterations and np.array_equal(xf, xs)
    assert i_f.true_relres == i_s.true_relres
    # one conversion launch fewer per preconditioned operator apply
    assert lf < ls
