"""Times implicit-step GMRES solves on a synthetic sparse-grid operator.

    python -m asgard_b200.profile_solve --d 4 --level 7 --terms 4 --dt 1e-3 \
        --mode global --precond block --precision fp32 --solves 3 [--warmup 1]
        [--advance K | --imex K] [--trace] [--no-graphs]

Builds the operator (connected pairs or the global Kronecker form), the
preconditioner (none, point or block Jacobi), runs --warmup untimed and
--solves timed solves of (I - dt K) x = b to a 1e-10 FP64 relative residual
(GMRES restart 50, a new seeded b per solve) and prints one JSON line with
the seconds per solve (CUDA events), iterations and residuals.  --advance K
times K steps of the implicit time loop instead (x_{k+1} from x_k plus a
fixed forcing, each solve started from its right-hand side).  Used for
per-kernel captures of a solve (`ncu ... python -m asgard_b200.profile_solve`).
"""
from __future__ import annotations

import argparse
import json
import time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--d", type=int, default=4)
    ap.add_argument("--level", type=int, default=7)
    ap.add_argument("--terms", type=int, default=4)
    ap.add_argument("--dt", type=float, default=1e-3)
    ap.add_argument("--device-build", action="store_true",
                    help="connected pairs found on the GPU (from_grid) instead of "
                         "by the host builder; mode pairs only")
    ap.add_argument("--mode", default="global", choices=["pairs", "global"])
    ap.add_argument("--precond", default="block", choices=["none", "point", "block", "kron", "line"])
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32", "bf16"])
    ap.add_argument("--bf16-inner-tol", type=float, default=0.0,
                    help="inner relative tolerance of the bf16 solves (0: the default)")
    ap.add_argument("--restart", type=int, default=50)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--solves", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--no-graphs", action="store_true",
                    help="drive every GMRES cycle from the host (no recorded "
                         "cycles; the same kernels, for per-kernel captures)")
    ap.add_argument("--basis", default="fp32", choices=["fp32", "fp64"],
                    help="Krylov basis read by the Gram-Schmidt passes of FP32 "
                         "inner solves")
    ap.add_argument("--node-steps", type=int, default=0,
                    help="Arnoldi steps per node of a recorded cycle (0: the "
                         "library default)")
    ap.add_argument("--trace", action="store_true",
                    help="also run one solve under torch.profiler (CUPTI) and "
                         "print its kernels: launches, device time, share, and "
                         "device-busy against wall time (sees the kernels of "
                         "recorded cycles, which ncu's launch list does not)")
    ap.add_argument("--imex", type=int, default=0,
                    help="time that many steps of the IMEX loop (imex_advance: "
                         "the operator implicit, the operator scaled by 1e-3 "
                         "explicit, two solves per step) instead of "
                         "independent solves")
    ap.add_argument("--advance", type=int, default=0,
                    help="time that many steps of the implicit time loop "
                         "(implicit_advance, state resident) instead of "
                         "independent solves")
    args = ap.parse_args()

    import torch
    import asgard_b200 as ab

    ab.gmres_settings(graphs=not args.no_graphs, fp32_basis=args.basis == "fp32",
                      node_steps=args.node_steps if args.node_steps > 0 else None,
                      bf16_inner_tol=args.bf16_inner_tol if args.bf16_inner_tol > 0 else None)
    t0 = time.perf_counter()
    if args.device_build:
        from asgard_b200.operators import factor_values
        from types import SimpleNamespace
        vA = factor_values(args.d, args.level, args.terms)
        mat = ab.kronmult_matrix.from_grid(args.d, 3, args.level, args.terms, vA)
        op = SimpleNamespace(N=mat.output_size())
    else:
        op = ab.SparseGridOperator(args.d, args.level, args.terms)
        mat = op.kronmult_matrix(mode=args.mode)
    pc = None if args.precond == "none" else ab.JacobiPreconditioner(mat, args.dt, kind=args.precond)
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    g = torch.Generator(device="cuda").manual_seed(0)
    bs = [torch.rand(op.N, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
          for _ in range(args.warmup + args.solves)]

    def solve(b):
        x = torch.zeros_like(b)
        return ab.simple_gmres_euler(args.dt, mat, x, b, args.restart, 400, args.tol,
                                     tol_mode="rel", precision=args.precision,
                                     precond=pc)

    if args.advance > 0:
        x = bs[0].clone()
        f = bs[1] if len(bs) > 1 else None

        def advance(k):
            return ab.implicit_advance(args.dt, mat, x, k, forcing=f,
                                       restart=args.restart, max_iter=400,
                                       tol=args.tol, tol_mode="rel",
                                       precision=args.precision, precond=pc)
        advance(args.warmup)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        infos = advance(args.advance)
        e1.record()
        torch.cuda.synchronize()
        s = e0.elapsed_time(e1) / 1e3 / args.advance
        print(json.dumps({"d": args.d, "level": args.level, "terms": args.terms,
                          "mode": args.mode, "precond": args.precond, "basis": args.basis,
                      "node_steps": ab.gmres_settings()["node_steps"],
                          "precision": args.precision, "dofs": op.N,
                          "steps": args.advance, "s_per_step": s,
                          "steps_per_s": 1.0 / s,
                          "iterations": [i.iterations for i in infos],
                          "true_relres": max(i.true_relres for i in infos),
                          "setup_s": setup}))
        return

    if args.imex > 0:
        # the reference's two-stage IMEX step: the operator as the implicit
        # part, the same operator scaled by 1e-3 as the (non-stiff) explicit
        # part; preconditioners for dt and dt/2
        mat_e = op.kronmult_matrix(mode=args.mode)
        ve = op.vA.reshape(-1, op.terms, op.d, op.n * op.n).copy()
        for t in range(op.terms):      # term t acts in dimension t mod d
            ve[:, t, t % op.d] *= 1e-3
        mat_e.update_stored_coefficients(ve.reshape(-1))
        pcs = (None, None) if pc is None else (
            pc, ab.JacobiPreconditioner(mat, 0.5 * args.dt, kind=args.precond))
        x = bs[0].clone()

        def imex(k):
            return ab.imex_advance(args.dt, mat_e, mat, x, k, restart=args.restart,
                                   max_iter=400, tol=args.tol, tol_mode="rel",
                                   precision=args.precision, precond=pcs)
        imex(args.warmup)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        infos = imex(args.imex)
        e1.record()
        torch.cuda.synchronize()
        s = e0.elapsed_time(e1) / 1e3 / args.imex
        print(json.dumps({"d": args.d, "level": args.level, "terms": args.terms,
                          "mode": args.mode, "precond": args.precond, "basis": args.basis,
                          "precision": args.precision, "dofs": op.N,
                          "imex_steps": args.imex, "s_per_step": s,
                          "steps_per_s": 1.0 / s,
                          "iterations": [[a.iterations, b.iterations] for a, b in infos],
                          "true_relres": max(max(a.true_relres, b.true_relres)
                                             for a, b in infos),
                          "setup_s": setup}))
        return

    if args.trace:
        trace(solve, bs[0])

    for i in range(args.warmup):
        solve(bs[i])
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    infos = [solve(bs[args.warmup + i]) for i in range(args.solves)]
    e1.record()
    torch.cuda.synchronize()
    s = e0.elapsed_time(e1) / 1e3 / args.solves
    print(json.dumps({"d": args.d, "level": args.level, "terms": args.terms,
                      "mode": args.mode, "precond": args.precond, "basis": args.basis,
                      "node_steps": ab.gmres_settings()["node_steps"],
                      "precision": args.precision, "dofs": op.N,
                      "s_per_solve": s, "solves_per_s": 1.0 / s,
                      "iterations": [i.iterations for i in infos],
                      "outer_steps": [i.outer_steps for i in infos],
                      "true_relres": max(i.true_relres for i in infos),
                      "ms_per_iteration": s * 1e3 / (sum(i.iterations for i in infos) / len(infos)),
                      "setup_s": setup}))


def trace(solve, b):
    """One solve under torch.profiler: per-kernel launches and device time,
    device-busy time against the solve's wall time, and the idle time between
    consecutive device activities grouped by (previous, next) kernel."""
    import re
    import torch
    from torch.profiler import ProfilerActivity, profile
    solve(b)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    solve(b)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        info = solve(b)
        torch.cuda.synchronize()
    evs = [e for e in prof.events() if e.device_type.name == "CUDA"]
    spans = sorted((e.time_range.start, e.time_range.end) for e in evs)
    busy = sum(e - s for s, e in spans)

    def short(e):
        name = e.name.replace("(anonymous namespace)::", "").replace("asgk::", "")
        return re.sub(r"\(.*", "", name)

    per = {}
    for e in evs:
        c = per.setdefault(short(e), [0, 0.0])
        c[0] += 1
        c[1] += e.time_range.end - e.time_range.start
    # idle time between consecutive device activities, by transition
    order = sorted(evs, key=lambda e: e.time_range.start)
    gaps = {}
    for a, b in zip(order, order[1:]):
        g = max(0.0, b.time_range.start - a.time_range.end)
        key = short(a).split("<")[0].replace("void ", "") + " -> " + \
            short(b).split("<")[0].replace("void ", "")
        c = gaps.setdefault(key, [0, 0.0])
        c[0] += 1
        c[1] += g
    print(json.dumps({"trace": {
        "iterations": info.iterations, "wall_ms": wall * 1e3,
        "device_busy_ms": busy / 1e3,
        "first_to_last_ms": (spans[-1][1] - spans[0][0]) / 1e3,
        "kernels": [{"name": k, "launches": c, "ms": t / 1e3,
                     "us_per_launch": t / c, "share": t / busy}
                    for k, (c, t) in sorted(per.items(), key=lambda kv: -kv[1][1])],
        "gaps": [{"between": k, "count": c, "ms": t / 1e3, "us_each": t / c}
                 for k, (c, t) in sorted(gaps.items(), key=lambda kv: -kv[1][1])[:12]]}}))


if __name__ == "__main__":
    main()
