"""The IMEX time loop (the reference's imex_advance,
src/time_advance.cpp:477-990) with the state resident on the device, against
the oracle's restatement of the same stages: explicit SSP-RK2 stages, two
backward-Euler GMRES solves per step, and the caller's hook where the
reference regenerates moments and coefficients."""
import numpy as np
import pytest

import oracle
from conftest import rel_err

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ops(d=3, level=4, terms=3):
    import asgard_b200 as ab
    ope = ab.SparseGridOperator(d, level, terms, kind="advdiff", nu=0.1, seed=0)
    opi = ab.SparseGridOperator(d, level, terms, kind="advdiff", nu=0.5, seed=1)
    tup = lambda op: (op.row_ptr.astype(np.int32), op.col, op.terms, op.iA(), op.vA.copy())
    return ope, opi, tup(ope), tup(opi)


@pytest.mark.parametrize("with_implicit", [True, False])
def test_imex_matches_oracle(cuda, with_implicit):
    import asgard_b200 as ab
    import torch
    ope, opi, E, I_ = _ops()
    dt, steps = 2e-3, 3
    x0 = np.random.default_rng(7).uniform(-1, 1, ope.N)
    xo = x0.copy()
    its = oracle.imex_advance(3, 3, E, I_ if with_implicit else None, dt, xo, steps,
                              30, 50, 1e-12)
    x = _dev(x0)
    infos = ab.imex_advance(dt, ope.kronmult_matrix(),
                            opi.kronmult_matrix() if with_implicit else None, x, steps,
                            restart=30, max_iter=50, tol=1e-12)
    torch.cuda.synchronize()
    assert len(infos) == steps
    for (i1, i2), (o1, o2) in zip(infos, its):
        if with_implicit:
            assert i1.status == 0 and i2.status == 0
            assert abs(i1.iterations - o1) <= 1 and abs(i2.iterations - o2) <= 1
        else:
            assert i1.iterations == 0 and i2.iterations == 0
    assert rel_err(x.cpu().numpy(), xo) < 1e-10


def test_imex_hook_events_and_coefficient_updates(cuda):
    """The hook sees the reference's vectors at its two events per stage, and
    coefficients it regenerates from a moment of f (here: the implicit
    factors scaled by 1 + tanh(mean f)/10) take effect in the next solve, as
    in the oracle given the same hook."""
    import asgard_b200 as ab
    import torch
    ope, opi, E, I_ = _ops()
    dt, steps = 2e-3, 2
    x0 = np.random.default_rng(9).uniform(-1, 1, ope.N)
    base = opi.vA.copy()
    mat_e, mat_i = ope.kronmult_matrix(), opi.kronmult_matrix()

    seen = []

    def hook_dev(step, stage, event, f):
        seen.append((step, stage, event, f.cpu().numpy().copy()))
        if event == ab.IMEX_BEFORE_IMPLICIT:
            m = float(f.mean())
            mat_i.update_stored_coefficients(base * (1.0 + np.tanh(m) / 10))

    oseen = []

    def hook_orc(step, stage, event, f):
        oseen.append((step, stage, event, f.copy()))
        if event == 1:
            I_[4][:] = base * (1.0 + np.tanh(f.mean()) / 10)

    xo = x0.copy()
    oracle.imex_advance(3, 3, E, I_, dt, xo, steps, 30, 50, 1e-12, hook=hook_orc)
    x = _dev(x0)
    infos = ab.imex_advance(dt, mat_e, mat_i, x, steps, restart=30, max_iter=50,
                            tol=1e-12, hook=hook_dev)
    torch.cuda.synchronize()
    assert all(a.status == 0 and b.status == 0 for a, b in infos)
    order = [(s, g, e) for s in range(steps) for g in (0, 1) for e in (0, 1)]
    assert [t[:3] for t in seen] == order and [t[:3] for t in oseen] == order
    assert np.array_equal(seen[0][3], x0)       # stage 1 reads f_0
    for a, b in zip(seen, oseen):
        assert rel_err(a[3], b[3]) < 1e-10
    assert rel_err(x.cpu().numpy(), xo) < 1e-10


def test_imex_preconditioned_mixed_precision(cuda):
    """Kronecker-sum Jacobi preconditioners for dt and dt/2 with the FP32
    operator in FP64 refinement (relative 1e-10 per solve) on global plans
    reach the FP64 unpreconditioned result."""
    import asgard_b200 as ab
    import torch
    ope, opi, _, _ = _ops(3, 5, 3)
    dt, steps = 2e-3, 2
    x0 = _dev(np.random.default_rng(4).uniform(-1, 1, ope.N))
    xr = x0.clone()
    ab.imex_advance(dt, ope.kronmult_matrix(), opi.kronmult_matrix(), xr, steps,
                    restart=50, max_iter=200, tol=1e-12, tol_mode="rel")
    gi = opi.kronmult_matrix(mode="global")
    pcs = (ab.JacobiPreconditioner(gi, dt, kind="kron"),
           ab.JacobiPreconditioner(gi, 0.5 * dt, kind="kron"))
    x = x0.clone()
    infos = ab.imex_advance(dt, ope.kronmult_matrix(mode="global"), gi, x, steps,
                            restart=50, max_iter=200, tol=1e-10, tol_mode="rel",
                            precision="fp32", precond=pcs)
    torch.cuda.synchronize()
    assert all(a.status == 0 and a.true_relres <= 1e-10 and
               b.status == 0 and b.true_relres <= 1e-10 for a, b in infos)
    assert (torch.linalg.norm(x - xr) / torch.linalg.norm(xr)).item() < 1e-8


def test_imex_hook_exception_stops_the_loop(cuda):
    import asgard_b200 as ab
    ope, opi, _, _ = _ops(2, 3, 2)
    x = _dev(np.ones(ope.N))
    calls = []

    def hook(step, stage, event, f):
        calls.append((step, stage, event))
        if (step, stage, event) == (0, 1, 0):
            raise KeyError("stop")

    with pytest.raises(KeyError):
        ab.imex_advance(1e-3, ope.kronmult_matrix(), opi.kronmult_matrix(), x, 3,
                        restart=20, max_iter=20, tol=1e-10, hook=hook)
    assert calls == [(0, 0, 0), (0, 0, 1), (0, 1, 0)]
