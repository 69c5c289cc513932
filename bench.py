"""Benchmark: implicit backward-Euler solves per second on one B200.

Workload (default ``d4``): d=4, n=3 (81 dofs per cell), level-7 sparse grid
(4048 cells, 327,888 dofs, 12,258,592 connected cell pairs), 4 terms of
advection/diffusion factors, solve (I - dt*K) x = b with dt = 1e-3,
b uniform in [-1, 1] (seeded, a new b every step), GMRES restart 50, until the
FP64 relative residual ||b - (I - dt K) x|| / ||b|| <= 1e-10.

A step is one solve by the framework's method: the operator in its global
Kronecker form (the reference's global_kron_matrix; the same operator as
the connected-pair kronmult, its terms acting in one dimension each),
block-Jacobi right preconditioning (each cell's diagonal block inverted
through the eigendecompositions of its 3x3 1D factors; the learned correction
on top of it is trained and kept only if its validation solve gains), FP32
operator inside
FP64 iterative refinement.  Timed beside it: the plain baseline -- FP64
GMRES with the connected-pair FP64 kronmult -- and the same
method on the connected-pair operator.  Inputs are resident in HBM when the
timed region starts; the plain baseline's operator (pair list + factor
indices, ~245 MB) is larger than L2; no extra L2 flush is done between
steps (the method's working set is L2-sized by design).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

For N > 1 (torchrun, one rank per GPU) every rank solves its own right-hand
sides on its own copy of the operator (replicas: the solve is not
sharded); value = solves of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "implicit-step solves/s at 1e-10 residual, learned+mixed vs plain FP64 (1 B200)"
WORKLOADS = {
    "d4": dict(d=4, level=7, terms=4, dt=1e-3, nu=0.1, kind="advdiff"),
    "d5": dict(d=5, level=7, terms=4, dt=1e-3, nu=0.1, kind="advdiff"),
    "d6": dict(d=6, level=7, terms=6, dt=5e-4, nu=0.1, kind="advdiff"),
    "d3": dict(d=3, level=7, terms=3, dt=1e-3, nu=0.1, kind="advdiff"),
}
RESTART = 50
TOL = 1e-10


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--workload", default="d4", choices=sorted(WORKLOADS))
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--method", default="learned-block-fp32",
                    choices=["learned-block-fp32", "learned-block-fp64",
                             "block-fp32", "block-fp64", "learned-fp32",
                             "learned-fp64", "fp32", "fp64"])
    ap.add_argument("--operator", default="global", choices=["global", "pairs"],
                    help="the method's operator form (plain FP64 always uses pairs)")
    ap.add_argument("--train-solves", type=int, default=1)
    ap.add_argument("--train-epochs", type=int, default=60)
    return ap.parse_args()


class ClockSampler:
    """SM clock and throttle reasons during the timed region: NVML read every
    10 ms from a thread (the default 20 steps last ~0.16 s; reading every 2 ms
    slowed the host-driven parts of the solves by ~5 %); `nvidia-smi -lms
    200` when NVML is unavailable.  Read-only."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
            "hw_thermal_slowdown": 0x40}

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.nvml = None
        self.samples = []

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.index)
        uuid = getattr(props, "uuid", None)
        if uuid is not None:
            try:
                return pynvml, pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(uuid))
            except Exception:
                pass
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        try:
            self.nvml, self.h = self._nvml_handle()
            get_reasons = getattr(self.nvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                self.nvml.nvmlDeviceGetCurrentClocksThrottleReasons
            self.max_mhz = float(self.nvml.nvmlDeviceGetMaxClockInfo(self.h, self.nvml.NVML_CLOCK_SM))
            self.stop_evt = threading.Event()

            def poll():
                while not self.stop_evt.is_set():
                    try:
                        sm = self.nvml.nvmlDeviceGetClockInfo(self.h, self.nvml.NVML_CLOCK_SM)
                        self.samples.append((float(sm), int(get_reasons(self.h))))
                    except Exception:
                        pass
                    time.sleep(0.01)
            self.t = threading.Thread(target=poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_evt.set()
            self.t.join(timeout=2)
            sm = sorted(s for s, _ in self.samples)
            reasons = sorted({nm for _, r in self.samples
                              for nm, bit in self.BITS.items() if r & bit})
            return {"sm_mhz": sm[len(sm) // 2] if sm else None,
                    "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(sm), "source": "NVML every 10 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi every 200 ms"}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


# ---------------------------------------------------------------- reference arm

def reference_arm(args):
    """The reference's own CPU paths (compiled from source into oracle/_ref),
    all host threads: kronmult_matrix<double>::apply on the CPU sparse format
    (local-kron mode) and, where its terms allow and the operator is small
    enough to set up, the global Kronecker product (global-kron mode,
    kronmult::global_cpu).  Each step times one full-operator product of
    each and converts it to solves/s with the iteration count of the
    reference GMRES algorithm on this workload; the line's value is the
    faster of the two (the reference's strongest CPU path)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import numpy as np
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference library oracle/_ref/libasgard_ref.so was not built"}))
        return
    R = oracle.ref()
    cfg = WORKLOADS[args.workload]
    from asgard_b200 import operators as ops
    d, L, T = cfg["d"], cfg["level"], cfg["terms"]
    table = ops.sparse_grid(d, L)
    row_ptr, col, conn = ops.build_pairs(d, L, table)
    vA = ops.factor_values(d, L, T, cfg["kind"], cfg["nu"])
    iA = ops.expand_iA(conn, d, 3, T)
    pntr = row_ptr.astype(np.int32)
    rows = len(pntr) - 1
    N = rows * 3 ** d
    x = np.random.default_rng(0).uniform(-1, 1, N)
    y = np.zeros(N)
    iters = _plain_iterations(args.workload)
    times = []
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.kronmult(d, 3, pntr, col, T, iA, vA, -cfg["dt"], x, 0.0, y, lib=R)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
    t_sparse = sorted(times)[len(times) // 2]
    cores = R.ref_num_threads()
    paths = {"cpu_sparse": {"apply_s": t_sparse, "value": 1.0 / (t_sparse * iters)}}
    g = _ref_global(d, L, T, table, vA, N)
    if g is not None:
        gtimes = [g.apply(x)[1] for _ in range(args.warmup + args.steps)][args.warmup:]
        t_global = sorted(gtimes)[len(gtimes) // 2]
        paths["global_cpu"] = {"apply_s": t_global, "value": 1.0 / (t_global * iters)}
    best = max(paths, key=lambda k: paths[k]["value"])
    value, t_apply = paths[best]["value"], paths[best]["apply_s"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_apply * iters * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": _config(args.workload),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores,
                         "kind": "reference",
                         "sample": f"{args.steps} full-operator products of the reference's "
                                   f"{best} (OpenMP {cores} threads); solves/s = "
                                   f"1/(median product time x {iters} GMRES iterations)"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "apply_s": t_apply, "gmres_iterations": iters, "paths": paths,
    }
    print(json.dumps(line))


def _ref_global(d, L, T, table, vA, N):
    """The reference's global product when built and affordable to set up
    (its pattern build is single-threaded host code: up to ~4 M unknowns)."""
    import oracle
    if not oracle.ref_global_available() or N > 4_000_000:
        return None
    try:
        return oracle.RefGlobal(d, 3, L, table, T, vA)
    except (OSError, ValueError):
        return None


# Iterations of the reference GMRES algorithm (restart 50, FP64, relative
# tolerance 1e-10, b uniform) on each workload, as this framework's plain
# FP64 GMRES measured them (same algorithm; bench line "plain_fp64"); the
# reference arm turns its CPU apply time into solves/s with them.
PLAIN_ITERATIONS = {"d4": 230}

# DRAM bytes per launch of the dominant kernel from one ncu capture
# (profiles/kron3_staged_d4_L7_fp64.md); None where none was taken.
KERNEL_TRAFFIC = {"d4": 254_243_328 + 4_232_704}
# the same for the global form's kernel (profiles/kron_global_rows_d4_L7.md)
GLOBAL_TRAFFIC = {"d4": 3_930_368 + 0}


def _measured_hbm_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


def _plain_iterations(workload):
    # other workloads reuse the d4 count (not measured on them)
    return PLAIN_ITERATIONS.get(workload, PLAIN_ITERATIONS["d4"])


def _config(workload):
    cfg = WORKLOADS[workload]
    return {"workload": f"d={cfg['d']} n=3 level {cfg['level']} sparse grid, "
                        f"{cfg['terms']} advection/diffusion terms (nu={cfg['nu']}), "
                        f"dt={cfg['dt']}, GMRES restart {RESTART}, rel tol {TOL}",
            "d": cfg["d"], "n": 3, "level": cfg["level"], "terms": cfg["terms"],
            "dt": cfg["dt"], "restart": RESTART, "tol": TOL,
            "l2": "operator data (pair list + indices) larger than L2; no flush"}


# ---------------------------------------------------------------- our arm

def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    import numpy as np
    import torch
    import asgard_b200 as ab

    from asgard_b200 import replicas
    world, rank, local = replicas.init("nccl")
    cfg = WORKLOADS[args.workload]
    d, L, T, dt = cfg["d"], cfg["level"], cfg["terms"], cfg["dt"]
    op = ab.SparseGridOperator(d, L, T, kind=cfg["kind"], nu=cfg["nu"])
    mat = op.kronmult_matrix()          # connected pairs: the plain baseline
    N = op.N
    # the method's operator: the global Kronecker form of the same operator
    # (terms acting in one dimension each) unless --operator pairs
    gmat = None
    if args.operator == "global":
        try:
            gmat = op.kronmult_matrix(mode="global")
        except ab.AsgkError:
            gmat = None
    mmat = gmat if gmat is not None else mat
    gen = torch.Generator(device="cuda").manual_seed(replicas.rhs_seed(rank))
    nb = args.warmup + args.steps
    B = [torch.rand(N, dtype=torch.float64, device="cuda", generator=gen) * 2 - 1
         for _ in range(max(nb, args.plain_steps + 1))]
    precision = "fp64" if args.method.endswith("fp64") else "fp32"
    # setup, not timed (like building the operator): the block-Jacobi
    # inverse -- through the eigendecompositions of each cell's 1D factors
    # on the global form (any d), else the dense per-cell inverses (n^d <= 81)
    # -- and the learned network's training
    base, base_form = None, None
    if "block" in args.method:
        if gmat is not None:
            try:
                base = ab.JacobiPreconditioner(gmat, dt, kind="kron")
                base_form = "Kronecker-sum form"
            except ab.AsgkError:
                base = None
        if base is None and 3 ** d <= 81:
            base = ab.JacobiPreconditioner(mmat, dt, kind="block")
            base_form = "dense cell inverses"
    pc, train_info = base, None
    if args.method.startswith("learned"):
        # plain FP64 GMRES solves of random right-hand sides give (v, e)
        # pairs, one row per cell, and the network trains on them on this
        # GPU; with a base it learns the correction e - base(v)
        t0 = time.perf_counter()
        net = ab.LearnedPreconditioner(op, seed=rank)
        if base is not None:
            net.set_base(base)
        if gmat is not None:
            from asgard_b200.operators import transpose_factor_values
            mat_T = ab.kronmult_matrix.from_global(
                d, 3, L, op.table, T, transpose_factor_values(op.vA, d, L, T))
        else:
            mat_T = op.kronmult_matrix_transposed()
        train_info = net.train(mmat, dt, num_solves=args.train_solves,
                               epochs=args.train_epochs, batch=1024, lr=1e-3,
                               seed=rank, mat_T=mat_T, residual_epochs=20)
        torch.cuda.synchronize()
        train_info["setup_s"] = time.perf_counter() - t0
        # the validation solve decides: without a gain the method continues
        # without the network (the base preconditioner, or none)
        if net.useful:
            pc = net
    learned = args.method.startswith("learned")
    dropped = " (learned correction dropped: no gain in its validation solve)"
    parts = []
    if learned and pc is not None and pc is not base:
        parts.append("learned preconditioner" + (" on block-Jacobi" if base is not None else ""))
    elif base is not None:
        parts.append(f"block-Jacobi preconditioner ({base_form})"
                     + (dropped if learned else ""))
    elif learned:
        parts.append("no preconditioner" + dropped)
    parts.append("FP32 operator, FP64 refinement" if precision == "fp32" else "FP64")
    parts.insert(0, "global Kronecker operator" if gmat is not None
                 else "connected-pair operator")
    method = dict(precision=precision, precond=pc, name=", ".join(parts))

    def solve(b, precision, precond=None, m=None):
        x = torch.zeros(N, dtype=torch.float64, device="cuda")
        info = ab.simple_gmres_euler(dt, m if m is not None else mmat, x, b,
                                     RESTART, 200, TOL,
                                     tol_mode="rel", precision=precision,
                                     precond=precond)
        return x, info

    # warm-up (method and plain)
    infos = []
    for i in range(args.warmup):
        _, info = solve(B[i], method["precision"], method["precond"])
        infos.append(info)
    _, pinfo = solve(B[0], "fp64", None, mat)

    # ---- timed: the method
    launches0 = ab.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    replicas.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    minfos = []
    for i in range(args.steps):
        _, info = solve(B[args.warmup + i], method["precision"], method["precond"])
        minfos.append(info)
    e1.record()
    replicas.barrier()
    clk = clocks.stop()
    launches = ab.launch_count() - launches0
    t_local = e0.elapsed_time(e1) / 1e3
    t_method = replicas.max_over_ranks(t_local)
    value = replicas.throughput(args.steps, t_local)

    # ---- timed: plain FP64 GMRES with the FP64 kronmult
    replicas.barrier()
    e0.record()
    pinfos = []
    for i in range(args.plain_steps):
        _, info = solve(B[i], "fp64", None, mat)
        pinfos.append(info)
    e1.record()
    replicas.barrier()
    t_local = e0.elapsed_time(e1) / 1e3
    t_plain = replicas.max_over_ranks(t_local)
    plain_value = replicas.throughput(args.plain_steps, t_local)

    # ---- timed: the same method on the connected-pair operator
    pair_method = None
    if gmat is not None:
        replicas.barrier()
        e0.record()
        qinfos = []
        for i in range(args.plain_steps):
            _, info = solve(B[i], method["precision"], method["precond"], mat)
            qinfos.append(info)
        e1.record()
        replicas.barrier()
        t_local = e0.elapsed_time(e1) / 1e3
        pair_method = {"value": replicas.throughput(args.plain_steps, t_local),
                       "unit": "solves/s",
                       "iterations": [i.iterations for i in qinfos],
                       "true_relres": max(i.true_relres for i in qinfos)}

    # ---- rooflines by CUDA events (average launch duration): the
    # connected-pair kronmult (FP64, the plain baseline's kernel, and FP32)
    # and the method's operator kernel
    xs = B[0]
    ys = torch.zeros_like(xs)
    flops = op.flops()
    reps = 5

    def time_apply(m, precision):
        m.apply_euler(dt, 1.0, xs, 0.0, ys, precision=precision)
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record()
        for _ in range(reps):
            m.apply_euler(dt, 1.0, xs, 0.0, ys, precision=precision)
        a1.record()
        torch.cuda.synchronize()
        return a0.elapsed_time(a1) / 1e3 / reps

    t64 = time_apply(mat, "fp64")
    t32 = time_apply(mat, "fp32")
    fp64_peak = ab._lib.C.c_double()
    ab.lib.asgk_measure_fma_peak(0, ab._lib.C.byref(fp64_peak))
    fp32_peak = ab._lib.C.c_double()
    ab.lib.asgk_measure_fma_peak(1, ab._lib.C.byref(fp32_peak))
    pair_kernel = (f"kron3_staged<d={d}, fp64> (+ x repack)" if d in (3, 4)
                   else f"kron3_rows<d={d}, fp64>")
    pair_roof = {"bound": "fp64", "kernel": pair_kernel,
                 "achieved": flops / t64 / 1e12, "peak": fp64_peak.value,
                 "peak_source": "measured live (FMA chain kernel)",
                 "unit": "TFLOP/s", "frac": flops / t64 / 1e12 / fp64_peak.value,
                 "traffic": KERNEL_TRAFFIC.get(args.workload),
                 "traffic_source": "ncu dram__bytes_read+write, one launch",
                 "ms_per_launch": t64 * 1e3, "flops_per_launch": flops,
                 "fp32_kernel": {"ms_per_launch": t32 * 1e3,
                                 "achieved": flops / t32 / 1e12,
                                 "peak": fp32_peak.value,
                                 "frac": flops / t32 / 1e12 / fp32_peak.value}}
    if gmat is not None:
        # the method's operator kernel: algorithmic bytes per launch are x
        # read once, y written, the neighbour lists and the pre-summed blocks
        tg = time_apply(gmat, method["precision"])
        nbytes = (16 * N + 8 * gmat.num_pairs() + 8 * (op.rows + 1)
                  + 48 * len(op.vA) // (9 * T))
        hbm = _measured_hbm_gbs()
        roofline = {"bound": "hbm",
                    "kernel": f"kron_global_rows<d={d}, {method['precision']}>",
                    "achieved": nbytes / tg / 1e9, "peak": hbm,
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs" if hbm != 6650.0
                                   else "fallback 6.65 TB/s",
                    "unit": "GB/s", "frac": nbytes / tg / 1e9 / hbm,
                    "traffic": GLOBAL_TRAFFIC.get(args.workload),
                    "traffic_source": "ncu dram__bytes_read+write, one launch",
                    "bytes_per_launch": nbytes, "ms_per_launch": tg * 1e3,
                    "note": "working set L2-resident; launch/latency bound",
                    "pair_kernel": pair_roof}
    else:
        roofline = pair_roof

    # ---- e2e through the public API with host buffers
    e2e_value = None
    hb = torch.empty(N, dtype=torch.float64, pin_memory=True)
    hx = torch.empty(N, dtype=torch.float64, pin_memory=True)
    hb.copy_(B[0].cpu())
    replicas.barrier()
    e0.record()
    for i in range(args.e2e_steps):
        bd = hb.to("cuda", non_blocking=True)
        x, _ = solve(bd, method["precision"], method["precond"])
        hx.copy_(x, non_blocking=True)
    e1.record()
    replicas.barrier()
    t_local = e0.elapsed_time(e1) / 1e3
    e2e_value = replicas.throughput(args.e2e_steps, t_local)

    # ---- CPU baseline (rank 0, N = 1): the reference compiled from source
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(op, cfg, pinfo.iterations)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_method / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": dict(_config(args.workload), method=args.method,
                           parallelism=f"replicas x{world}"),
            "plain_fp64": {"value": plain_value, "unit": "solves/s",
                           "iterations": pinfo.iterations,
                           "true_relres": max(i.true_relres for i in pinfos),
                           "ms_per_solve": t_plain / args.plain_steps * 1e3},
            "method": {"name": method["name"],
                       "iterations": [i.iterations for i in minfos],
                       "true_relres": max(i.true_relres for i in minfos),
                       "outer_steps": minfos[0].outer_steps,
                       "matvecs_low": minfos[0].matvecs_low,
                       "matvecs_fp64": minfos[0].matvecs_fp64,
                       "precond_calls": minfos[0].precond_calls,
                       "fallback": max(i.fallback for i in minfos),
                       "training": train_info,
                       "speedup_vs_plain": value / plain_value},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "solves/s",
                    "h2d_bytes_per_step": N * 8, "d2h_bytes_per_step": N * 8},
            "gpu_launches": launches,
            "pair_operator_method": pair_method,
            "roofline": roofline,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    replicas.shutdown()


def cpu_baseline(op, cfg, iters):
    """The reference's CPU paths on the host cores (bounded sample: one
    full-operator product each, converted with the plain iteration count):
    cpu_sparse (local-kron kronmult_matrix::apply) and, where available, the
    global Kronecker product; value = the faster."""
    import numpy as np
    import oracle
    if not oracle.ref_available():
        return {"value": None, "unit": "solves/s", "cores": 0, "kind": "reference",
                "sample": "reference library not built"}
    R = oracle.ref()
    iA = op.iA()
    pntr = op.row_ptr.astype(np.int32)
    x = np.random.default_rng(0).uniform(-1, 1, op.N)
    y = np.zeros(op.N)
    t0 = time.perf_counter()
    oracle.kronmult(op.d, 3, pntr, op.col, op.terms, iA, op.vA, -cfg["dt"], x,
                    0.0, y, lib=R)
    t_sparse = time.perf_counter() - t0
    cores = R.ref_num_threads()
    out = {"value": 1.0 / (t_sparse * iters), "unit": "solves/s",
           "cores": cores, "kind": "reference",
           "sample": f"1 full-operator product of the reference cpu_sparse kronmult "
                     f"({t_sparse:.3f} s, {cores} OpenMP threads) x {iters} GMRES iterations",
           "apply_s": t_sparse, "cpu_sparse_value": 1.0 / (t_sparse * iters)}
    g = _ref_global(op.d, op.level, op.terms, op.table, op.vA, op.N)
    if g is not None:
        _, t_global = g.apply(x, reps=3)
        out.update(value=1.0 / (t_global * iters), apply_s=t_global,
                   global_cpu_value=1.0 / (t_global * iters),
                   sample=f"best of 3 full-operator products of the reference's global "
                          f"Kronecker product ({t_global * 1e3:.1f} ms, {cores} OpenMP "
                          f"threads; cpu_sparse {t_sparse:.2f} s) x {iters} GMRES iterations")
    return out


if __name__ == "__main__":
    main()
