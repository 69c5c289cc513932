"""Learned preconditioner: the GPU forward/backward kernels against the float64
oracle (oracle/mlp_oracle.py), training, and what the trained network gains
inside flexible GMRES over the same solve without it."""
import numpy as np
import pytest

from oracle import mlp_oracle

pytestmark = pytest.mark.gpu

# BF16 operands with FP32 accumulation: relative (L2) tolerances
FWD_TOL = 3e-2
GRAD_TOL = 6e-2


def _rel(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("d,hidden,rows", [(2, 32, 64), (4, 256, 300)])
def test_forward_backward_against_fp64_oracle(cuda, d, hidden, rows):
    import asgard_b200 as ab
    op = ab.SparseGridOperator(d, 3, d, kind="advdiff")
    pc = ab.LearnedPreconditioner(op, hidden=hidden, seed=5)
    rng = np.random.default_rng(d)
    X = rng.uniform(-1, 1, (rows, pc.dims[0])).astype(np.float32)
    T = rng.uniform(-1, 1, (rows, pc.dims[-1])).astype(np.float32)
    params = pc.get_params()
    # the oracle sees the same BF16-rounded inputs and weights the GEMMs use
    import torch
    bf = lambda a: torch.from_numpy(a).to(torch.bfloat16).float().numpy()
    Yg, lossg, gg = pc.forward_backward(X, T)
    Yo, losso, go = mlp_oracle.forward_backward(params, pc.dims, bf(X), T)
    assert _rel(Yg, Yo) < FWD_TOL
    assert abs(lossg - losso) / losso < FWD_TOL
    assert _rel(gg, go) < GRAD_TOL
    # per layer, weights and biases separately
    o = 0
    for l in range(4):
        nw = pc.dims[l] * pc.dims[l + 1]
        assert _rel(gg[o:o + nw], go[o:o + nw]) < GRAD_TOL, ("W", l)
        o += nw
        nb = pc.dims[l + 1]
        assert _rel(gg[o:o + nb], go[o:o + nb]) < GRAD_TOL, ("b", l)
        o += nb


def test_save_load_round_trip(cuda, tmp_path):
    import asgard_b200 as ab
    op = ab.SparseGridOperator(2, 3, 2, kind="advdiff")
    a = ab.LearnedPreconditioner(op, hidden=32, seed=1)
    b = ab.LearnedPreconditioner(op, hidden=32, seed=2)
    a.save(tmp_path / "pc.bin")
    b.load(tmp_path / "pc.bin")
    assert np.array_equal(a.get_params(), b.get_params())


def test_trained_preconditioner_reduces_iterations(cuda):
    """d=3, level 6: train on plain-GMRES solutions of random right-hand
    sides, then solve a new right-hand side to 1e-10 (FP64 relative residual)
    with and without the network."""
    import asgard_b200 as ab
    import torch
    op = ab.SparseGridOperator(3, 6, 3, kind="advdiff", nu=0.1)
    mat = op.kronmult_matrix()
    dt = 1e-3
    pc = ab.LearnedPreconditioner(op, seed=0)
    stats = pc.train(mat, dt, num_solves=12, epochs=40, batch=512, lr=1e-3)
    assert np.isfinite(stats["loss"])
    b = torch.rand(op.N, dtype=torch.float64, device="cuda",
                   generator=torch.Generator(device="cuda").manual_seed(99)) * 2 - 1
    x0 = torch.zeros_like(b)
    plain = ab.simple_gmres_euler(dt, mat, x0, b, 50, 200, 1e-10, tol_mode="rel")
    x1 = torch.zeros_like(b)
    learned = ab.simple_gmres_euler(dt, mat, x1, b, 50, 200, 1e-10,
                                    tol_mode="rel", precond=pc)
    assert plain.status == 0 and learned.status == 0
    assert learned.true_relres <= 1e-10
    assert learned.iterations < 0.7 * plain.iterations, (learned, plain)
    assert (torch.linalg.norm(x1 - x0) / torch.linalg.norm(x0)).item() < 1e-8
