"""Times the kronmult apply kernel on a synthetic sparse-grid operator.

    python -m asgard_b200.profile_apply --d 4 --level 7 --terms 4 \
        --precision fp64 --reps 3 [--warmup 1] [--mode global|dense]
        [--jacobi point|block|kron|line]

Builds the operator (advection/diffusion factors unless --kind random), runs
--warmup untimed applies of the fused backward-Euler operator
y = x - dt*K*x, then --reps timed applies (CUDA events on the launching
stream) and prints one JSON line: ms per launch, algorithmic TFLOP/s
(2*d*T*n^(d+1) flops per pair -- every cell pair in the dense form;
2*n^(d+1) per single-direction pair in the global form) and the fraction of the measured FMA peak.
The kernel summaries of this repository were taken with this command under ncu.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--d", type=int, default=4)
    ap.add_argument("--level", type=int, default=7)
    ap.add_argument("--terms", type=int, default=4)
    ap.add_argument("--kind", default="advdiff")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32", "bf16"])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--peak", action="store_true", help="also measure the FMA peak")
    ap.add_argument("--device-build", action="store_true",
                    help="connected pairs found on the GPU (from_grid) instead of "
                         "by the host builder; mode pairs only")
    ap.add_argument("--jacobi", default=None, choices=["point", "block", "kron", "line"],
                    help="time the Jacobi preconditioner of that kind (built on the "
                         "--mode plan, dt 5e-4 at d >= 6 else 1e-3) instead of the operator")
    ap.add_argument("--mode", default="pairs", choices=["pairs", "global", "dense"],
                    help="connected-pair kronmult, the global Kronecker form, "
                         "or the dense form (every cell pair)")
    args = ap.parse_args()

    import torch
    import asgard_b200 as ab

    t0 = time.perf_counter()
    if args.device_build:
        from asgard_b200.operators import factor_values
        from types import SimpleNamespace
        vA = factor_values(args.d, args.level, args.terms, args.kind)
        mat = ab.kronmult_matrix.from_grid(args.d, 3, args.level, args.terms, vA)
        op = SimpleNamespace(rows=mat.num_rows, nnz=mat.num_pairs(),
                             N=mat.output_size())
    else:
        op = ab.SparseGridOperator(args.d, args.level, args.terms, kind=args.kind)
        mat = op.kronmult_matrix(mode=args.mode)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.rand(op.N, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    y = torch.zeros_like(x)
    if args.jacobi:
        t0 = time.perf_counter()
        pc = ab.JacobiPreconditioner(mat, 5e-4 if args.d >= 6 else 1e-3, kind=args.jacobi)
        torch.cuda.synchronize()
        t_pc = time.perf_counter() - t0
        for _ in range(args.warmup):
            pc.apply(x, y, precision=args.precision)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.reps):
            pc.apply(x, y, precision=args.precision)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.reps
        print(json.dumps({"d": args.d, "level": args.level, "terms": args.terms,
                          "jacobi": args.jacobi, "precision": args.precision,
                          "dofs": op.N, "ms_per_apply": ms, "setup_s": t_pc,
                          "algorithmic_GBps": 16 * op.N / ms / 1e6,
                          "device_bytes": pc.device_bytes()}))
        return
    for _ in range(args.warmup):
        mat.apply_euler(1e-3, 1.0, x, 0.0, y, precision=args.precision)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.reps):
        mat.apply_euler(1e-3, 1.0, x, 0.0, y, precision=args.precision)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.reps
    flops = mat.flops()
    out = {"d": args.d, "level": args.level, "terms": args.terms, "mode": args.mode,
           "num_pairs": mat.num_pairs(),
           "precision": args.precision, "cells": op.rows, "pairs": op.nnz,
           "dofs": op.N, "ms_per_launch": ms, "tflops": flops / ms / 1e9,
           "flops_per_launch": flops, "setup_s": t_setup,
           "device_bytes": mat.device_bytes()}
    if args.precision != "fp64":
        # the low-precision product K x against the FP64 one on the same x
        y64, ylo = torch.zeros_like(x), torch.zeros_like(x)
        mat.apply(1.0, x, 0.0, y64, precision="fp64")
        mat.apply(1.0, x, 0.0, ylo, precision=args.precision)
        torch.cuda.synchronize()
        out["rel_err_vs_fp64"] = float(torch.linalg.norm(ylo - y64) / torch.linalg.norm(y64))
    if args.peak:
        pk = C.c_double()
        ab.lib.asgk_measure_fma_peak(0 if args.precision == "fp64" else 1, C.byref(pk))
        out["fma_peak_tflops"] = pk.value
        out["frac"] = out["tflops"] / pk.value
    print(json.dumps(out))


if __name__ == "__main__":
    main()
