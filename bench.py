"""Benchmark: implicit backward-Euler solves per second on one B200.

Workload (default ``d6``): d=6, n=3 (729 dofs per cell), level-7 sparse grid
(16,172 cells, 11,789,388 dofs, 226,043,944 connected cell pairs), 6 terms
of advection/diffusion factors (term t acts in dimension t, even terms DG
advection, odd terms 0.1 x LDG diffusion), solve (I - dt*K) x = b with
dt = 5e-4, b uniform in [-1, 1] (seeded, a new b every step), GMRES restart
50, until the FP64 relative residual ||b - (I - dt K) x|| / ||b|| <= 1e-10.
``--workload d4`` is the d=4 level-7 configuration (4 terms, dt = 1e-3).

A step is one solve by the framework's method: the operator in its global
Kronecker form (the reference's global_kron_matrix; the same operator as
the connected-pair kronmult, its terms acting in one dimension each), right
preconditioning by exact solves along the pencils of the diffusion
dimensions, chained (the learned correction on top of it is trained and kept
only if its validation solve gains), FP32 operator inside FP64 iterative
refinement.  Timed beside it: the plain
baseline -- FP64 GMRES with the connected-pair FP64 kronmult (one solve by
default: about four minutes at d=6) -- and, at d <= 4, the same method on the
connected-pair operator.  Inputs are resident in HBM when the timed region
starts; at d=6 every vector (94 MB) and the plain baseline's pair list
(6.3 GB) are larger than L2, at d=4 the method's working set is L2-sized by
design; no extra L2 flush is done between steps.  ``e2e`` is the same
solves with b in pinned host memory and x read back into pinned host
memory every step, the copies on a second stream overlapping the
neighbouring steps' solves.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

For N > 1 (torchrun, one rank per GPU) every rank solves its own right-hand
sides on its own copy of the operator (replicas: the solve is not
sharded); value = solves of all ranks / max-over-ranks time.

``--impl reference`` runs the reference's own CPU path on the host cores:
its sparse grid, global Kronecker matrix, diagonal preconditioner and
solver::simple_gmres_euler, compiled from the reference sources into
oracle/_ref/libasgard_ref_gsolve.so; it imports nothing of this framework.
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
    "d6": dict(d=6, level=7, terms=6, dt=5e-4, nu=0.1, kind="advdiff"),
    "d5": dict(d=5, level=7, terms=4, dt=1e-3, nu=0.1, kind="advdiff"),
    "d4": dict(d=4, level=7, terms=4, dt=1e-3, nu=0.1, kind="advdiff"),
    "d3": dict(d=3, level=7, terms=3, dt=1e-3, nu=0.1, kind="advdiff"),
}
RESTART = 50
TOL = 1e-10

# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of
# each workload's operator kernels, from one ncu capture of that kernel on
# that workload; None where no capture was taken.
KERNEL_TRAFFIC = {
    ("pairs", "d4"): 254_243_328 + 4_232_704,
    ("global", "d4"): 3_930_368,
    ("global", "d6"): 71_265_792 + 54_134_016,
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--workload", default="d6", choices=sorted(WORKLOADS))
    ap.add_argument("--plain-steps", type=int, default=1,
                    help="timed plain FP64 solves (about 250 s each at d=6)")
    ap.add_argument("--pair-method-steps", type=int, default=None,
                    help="timed solves of the method on the connected-pair "
                         "operator (default 2 at d <= 4, 0 above)")
    ap.add_argument("--e2e-steps", type=int, default=None,
                    help="solves through host buffers (default: --steps)")
    ap.add_argument("--cpu-baseline", default="solve", choices=["solve", "none"],
                    help="solve: one full solve by the reference's CPU path "
                         "(rank 0, one GPU); none: skip")
    ap.add_argument("--method", default="learned-block-fp32",
                    choices=["learned-block-fp32", "learned-block-fp64",
                             "block-fp32", "block-fp64", "learned-fp32",
                             "learned-fp64", "fp32", "fp64"])
    ap.add_argument("--operator", default="global", choices=["global", "pairs"],
                    help="the method's operator form (plain FP64 always uses pairs)")
    ap.add_argument("--form-steps", type=int, default=3,
                    help="timed solves of the method with its inner operator in "
                         "FP32 and in BF16 on the tensor cores (0: skip)")
    ap.add_argument("--train-solves", type=int, default=1)
    ap.add_argument("--train-epochs", type=int, default=60)
    return ap.parse_args()


class ClockSampler:
    """SM clock and throttle reasons during the timed region: NVML read every
    10 ms from a thread (reading every 2 ms slowed the host-driven parts of
    the solves by ~5 %); `nvidia-smi -lms 200` when NVML is unavailable.
    Read-only."""

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


def _measured_hbm_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def _config(workload):
    cfg = WORKLOADS[workload]
    return {"workload": f"d={cfg['d']} n=3 level {cfg['level']} sparse grid, "
                        f"{cfg['terms']} advection/diffusion terms (diffusion "
                        f"scaled by nu={cfg['nu']}), dt={cfg['dt']}, GMRES "
                        f"restart {RESTART}, rel tol {TOL}",
            "d": cfg["d"], "n": 3, "level": cfg["level"], "terms": cfg["terms"],
            "dt": cfg["dt"], "nu": cfg["nu"], "restart": RESTART, "tol": TOL,
            "l2": ("vectors (94 MB) and the plain baseline's pair list larger "
                   "than L2; no flush" if cfg["d"] >= 6 else
                   "plain baseline's pair list larger than L2; the method's "
                   "working set L2-sized; no flush")}


# ---------------------------------------------------------------- reference arm

class ReferenceSolves:
    """The reference's implicit solve on the host cores, driven one GMRES
    restart cycle at a time: each call of its solver::simple_gmres_euler with
    max_iter = 1 runs one cycle (the residual b - (I - dt K) x, its diagonal
    preconditioner, up to 50 Arnoldi steps, the update of x) from the
    current x, which is what its own outer loop does between cycles; when a
    cycle meets the tolerance the solve is complete and the next starts from
    x = 0 with a new b.  The tolerance is the reference's (absolute, on its
    estimated left-preconditioned residual), set to TOL * ||b|| / max_i
    |1 - dt pc_i| so that the true relative residual ||b - (I - dt K) x|| /
    ||b|| is at most TOL (r = M r_prec with M = diag(1 - dt pc)); every
    completed solve's true residual is recomputed by the reference's apply."""

    def __init__(self, workload, seed=0):
        import numpy as np
        import oracle
        cfg = WORKLOADS[workload]
        self.np = np
        self.dt = cfg["dt"]
        t0 = time.perf_counter()
        self.R = oracle.RefGlobalSolver.synthetic(cfg["d"], cfg["level"],
                                                  cfg["terms"], cfg["nu"])
        self.setup_s = time.perf_counter() - t0
        pc = self.R.precond()
        self.mmax = float(np.abs(1.0 - self.dt * pc).max())
        self.rng = np.random.default_rng(seed)
        self.cores = oracle._gsolve_lib().ref_gsolve_num_threads()
        self.solves = []          # completed: iterations, seconds, true relres
        self._new_solve()

    def _new_solve(self):
        np = self.np
        self.b = self.rng.uniform(-1.0, 1.0, self.R.N)
        self.x = np.zeros(self.R.N)
        self.tol = TOL * float(np.linalg.norm(self.b)) / self.mmax
        self.its = 0
        self.sec = 0.0

    def cycle(self):
        """One restart cycle; returns (iterations, seconds)."""
        t0 = time.perf_counter()
        err, its, _ = self.R.gmres_euler(self.dt, self.x, self.b, RESTART, 1,
                                         self.tol)
        sec = time.perf_counter() - t0
        self.its += its
        self.sec += sec
        if err <= self.tol:
            np = self.np
            Kx, _ = self.R.apply(1.0, self.x)
            r = self.b - (self.x - self.dt * Kx)
            self.solves.append({"iterations": self.its, "seconds": self.sec,
                                "error": err, "true_relres":
                                float(np.linalg.norm(r) / np.linalg.norm(self.b))})
            self._new_solve()
        return its, sec

    def full_solve(self):
        """Cycles until the current solve completes; returns its record."""
        n = len(self.solves)
        while len(self.solves) == n:
            self.cycle()
        return self.solves[-1]


def reference_arm(args):
    """The reference's own CPU path (see ReferenceSolves), all host threads.
    A step is one GMRES restart cycle of the reference solver (a bounded
    sample: a full d=6 solve takes minutes on the host); the steps run
    consecutive real solves.  value = iterations per second over the timed
    steps / mean iterations of the solves completed in the run."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    if not oracle.ref_gsolve_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference library oracle/_ref/libasgard_ref_gsolve.so "
                          "was not built"}))
        return
    ref = ReferenceSolves(args.workload)
    for _ in range(args.warmup):
        ref.cycle()
    timed_its, timed_s, times = 0, 0.0, []
    for _ in range(args.steps):
        its, sec = ref.cycle()
        timed_its += its
        timed_s += sec
        times.append(sec)
    if not ref.solves:          # too few cycles in the run for one solve
        ref.full_solve()
    its_per_solve = sum(s["iterations"] for s in ref.solves) / len(ref.solves)
    value = (timed_its / timed_s) / its_per_solve
    line = {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": timed_s / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": _config(args.workload),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": ref.cores,
                         "kind": "reference",
                         "sample": f"{args.steps} GMRES restart cycles of the reference's "
                                   f"solver::simple_gmres_euler over its global_kron_matrix "
                                   f"(OpenMP {ref.cores} threads), consecutive real solves; "
                                   f"solves/s = timed iterations/s / {its_per_solve:.1f} "
                                   f"iterations per completed solve"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "step": "one GMRES restart cycle (up to 51 iterations in the reference's count)",
        "iterations_timed": timed_its, "seconds_timed": timed_s,
        "cycle_s": {"min": min(times), "max": max(times)},
        "solves": ref.solves, "setup_s": ref.setup_s,
        "solver": "reference solver::simple_gmres_euler(dt, matrix_entry::regular, "
                  "global_kron_matrix, ...), left diagonal preconditioner, "
                  f"absolute tol TOL*||b||/max|1-dt pc| (max |1-dt pc| = {ref.mmax:.4g})",
    }
    print(json.dumps(line))


# ---------------------------------------------------------------- our arm

def build_method(args, ab, op, mat, gmat, mmat, dt, rank):
    """Setup of the method, not timed (as the reference's matrix setup is
    not part of solves/s): the base preconditioner -- on the global form the
    line preconditioner (exact solves along the pencils of the diffusion
    dimensions, chained), else the cell-block inverse through the
    eigendecompositions of each cell's 1D factors, else the dense per-cell
    inverses (n^d <= 81) -- and the learned network's training.  Returns
    (method dict, training info)."""
    import torch
    d = op.d
    precision = "fp64" if args.method.endswith("fp64") else "fp32"
    base, base_form = None, None
    if "block" in args.method:
        if gmat is not None:
            for kind, form in (("line", "line solves along the diffusion dimensions"),
                               ("kron", "block-Jacobi, Kronecker-sum form")):
                try:
                    base = ab.JacobiPreconditioner(gmat, dt, kind=kind)
                    base_form = form
                    break
                except ab.AsgkError:
                    base = None
        if base is None and 3 ** d <= 81:
            base = ab.JacobiPreconditioner(mmat, dt, kind="block")
            base_form = "block-Jacobi, dense cell inverses"
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
                d, 3, op.level, op.table, op.terms,
                transpose_factor_values(op.vA, d, op.level, op.terms))
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
        parts.append("learned preconditioner" + (f" on {base_form}" if base is not None else ""))
    elif base is not None:
        parts.append(f"preconditioner: {base_form}" + (dropped if learned else ""))
    elif learned:
        parts.append("no preconditioner" + dropped)
    parts.append("FP32 operator, FP64 refinement" if precision == "fp32" else "FP64")
    parts.insert(0, "global Kronecker operator" if gmat is not None
                 else "connected-pair operator")
    return dict(precision=precision, precond=pc, name=", ".join(parts)), train_info


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    import torch
    import asgard_b200 as ab

    from asgard_b200 import replicas
    world, rank, local = replicas.init("nccl")
    cfg = WORKLOADS[args.workload]
    d, L, T, dt = cfg["d"], cfg["level"], cfg["terms"], cfg["dt"]
    pair_steps = (args.pair_method_steps if args.pair_method_steps is not None
                  else (2 if d <= 4 else 0))
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else args.steps
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
         for _ in range(max(nb, args.plain_steps, pair_steps))]
    method, train_info = build_method(args, ab, op, mat, gmat, mmat, dt, rank)

    def solve(b, precision, precond=None, m=None):
        x = torch.zeros(N, dtype=torch.float64, device="cuda")
        info = ab.simple_gmres_euler(dt, m if m is not None else mmat, x, b,
                                     RESTART, 200, TOL,
                                     tol_mode="rel", precision=precision,
                                     precond=precond)
        return x, info

    # warm-up: the method's solves; one FP64 apply of the plain operator
    for i in range(args.warmup):
        solve(B[i], method["precision"], method["precond"])
    ytmp = torch.empty_like(B[0])
    mat.apply_euler(dt, 1.0, B[0], 0.0, ytmp, precision="fp64")
    torch.cuda.synchronize()

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

    # ---- e2e through the public API with host buffers: every step copies
    # its own b from pinned host memory and reads its x back into pinned
    # host memory.  The copies run on a second stream, as a user streaming
    # many solves would issue them: step i+1's b travels while step i
    # solves, step i's x while step i+1 solves; the timed region ends after
    # the last read-back.
    hb = [torch.empty(N, dtype=torch.float64, pin_memory=True) for _ in range(e2e_steps)]
    for i, h in enumerate(hb):
        h.copy_(B[(args.warmup + i) % len(B)].cpu())
    hx = [torch.empty(N, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    main = torch.cuda.current_stream()
    copy = torch.cuda.Stream()
    bdev = [torch.empty(N, dtype=torch.float64, device="cuda") for _ in range(2)]
    b_in = [torch.cuda.Event() for _ in range(2)]    # b copied in
    b_free = [torch.cuda.Event() for _ in range(2)]  # its solve is done with it
    replicas.barrier()
    torch.cuda.synchronize()
    e0.record()
    copy.wait_stream(main)
    with torch.cuda.stream(copy):
        bdev[0].copy_(hb[0], non_blocking=True)
        b_in[0].record(copy)
    for i in range(e2e_steps):
        cur = i % 2
        if i + 1 < e2e_steps:
            nxt = (i + 1) % 2
            with torch.cuda.stream(copy):
                if i >= 1:
                    copy.wait_event(b_free[nxt])
                bdev[nxt].copy_(hb[i + 1], non_blocking=True)
                b_in[nxt].record(copy)
        main.wait_event(b_in[cur])
        x, _ = solve(bdev[cur], method["precision"], method["precond"])
        b_free[cur].record(main)
        done = torch.cuda.Event()
        done.record(main)
        with torch.cuda.stream(copy):
            copy.wait_event(done)
            hx[cur].copy_(x, non_blocking=True)
        x.record_stream(copy)
    main.wait_stream(copy)
    e1.record()
    replicas.barrier()
    t_local = e0.elapsed_time(e1) / 1e3
    e2e_value = replicas.throughput(e2e_steps, t_local)
    del hb

    # ---- timed: plain FP64 GMRES with the FP64 connected-pair kronmult
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
    plain_value = replicas.throughput(max(args.plain_steps, 0), t_local) \
        if args.plain_steps > 0 else None

    # ---- timed: the same method on the connected-pair operator
    pair_method = None
    if gmat is not None and pair_steps > 0:
        replicas.barrier()
        e0.record()
        qinfos = []
        for i in range(pair_steps):
            _, info = solve(B[i], method["precision"], method["precond"], mat)
            qinfos.append(info)
        e1.record()
        replicas.barrier()
        t_local = e0.elapsed_time(e1) / 1e3
        pair_method = {"value": replicas.throughput(pair_steps, t_local),
                       "unit": "solves/s",
                       "iterations": [i.iterations for i in qinfos],
                       "true_relres": max(i.true_relres for i in qinfos)}

    # ---- the inner operator in FP32 (CUDA cores) and in BF16 (tensor
    # cores): its error against the FP64 product and the method's solves
    forms = None
    if gmat is not None and args.form_steps > 0:
        forms = precision_forms(op, gmat, method, dt, B, args.form_steps, solve,
                                plain_value)

    roofline = rooflines(ab, op, mat, gmat, method, dt, args.workload, B[0])

    # ---- CPU baseline (rank 0, N = 1): the reference's own solve
    cpu = None
    if rank == 0 and world == 1 and args.cpu_baseline == "solve":
        cpu = cpu_baseline(args.workload)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_method / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": dict(_config(args.workload), method=args.method,
                           parallelism=f"replicas x{world}"),
            "plain_fp64": ({"value": plain_value, "unit": "solves/s",
                            "iterations": [i.iterations for i in pinfos],
                            "true_relres": max(i.true_relres for i in pinfos),
                            "ms_per_solve": t_plain / args.plain_steps * 1e3}
                           if pinfos else None),
            "method": {"name": method["name"],
                       "iterations": [i.iterations for i in minfos],
                       "true_relres": max(i.true_relres for i in minfos),
                       "outer_steps": minfos[0].outer_steps,
                       "matvecs_low": minfos[0].matvecs_low,
                       "matvecs_fp64": minfos[0].matvecs_fp64,
                       "precond_calls": minfos[0].precond_calls,
                       "fallback": max(i.fallback for i in minfos),
                       "training": train_info,
                       "speedup_vs_plain": (value / plain_value
                                            if plain_value else None)},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "solves/s",
                    "h2d_bytes_per_step": N * 8, "d2h_bytes_per_step": N * 8,
                    "steps": e2e_steps},
            "gpu_launches": launches,
            "pair_operator_method": pair_method,
            "precision_forms": forms,
            "roofline": roofline,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    replicas.shutdown()


def pencil_gemm_flops(op):
    """Useful flops of the tensor-core form per apply: along each dimension
    with terms, every pencil of p cells is a (3p x 3p) by (3p x 3^(d-1))
    product (2 flops per multiply-add; padding not counted)."""
    import numpy as np
    t = op.table.astype(np.int64)
    d, fib = op.d, 3 ** (op.d - 1)
    total = 0
    for k in sorted({tt % d for tt in range(op.terms)}):
        keep = [j for j in range(d) if j != k] + [d + j for j in range(d) if j != k]
        _, counts = np.unique(t[:, keep], axis=0, return_counts=True)
        total += int((2 * (3 * counts) ** 2 * fib).sum())
    return total


def _bf16_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "MEASURED_PEAKS.json bf16_tflops"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback 1.59 PFLOP/s"


def precision_forms(op, gmat, method, dt, B, steps, solve, plain_value):
    """The method (its preconditioner, FP64 refinement, recorded cycles) with
    the inner operator in FP32 on the CUDA cores and in BF16 on the tensor
    cores (FP32 accumulation): the inner product's relative error against
    the FP64 product on a seeded x, the apply time, and `steps` timed solves
    to the FP64 relative residual (each recomputed in FP64)."""
    import torch
    x = B[0]
    y64 = torch.zeros_like(x)
    gmat.apply(1.0, x, 0.0, y64, precision="fp64")
    ys = torch.zeros_like(x)
    out = {}
    for prec in ("fp32", "bf16"):
        gmat.apply(1.0, x, 0.0, ys, precision=prec)
        torch.cuda.synchronize()
        err = float(torch.linalg.norm(ys - y64) / torch.linalg.norm(y64))
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record()
        for _ in range(10):
            gmat.apply_euler(dt, 1.0, x, 0.0, ys, precision=prec)
        a1.record()
        torch.cuda.synchronize()
        apply_ms = a0.elapsed_time(a1) / 10
        solve(B[0], prec, method["precond"])        # warm-up: records the cycles
        torch.cuda.synchronize()
        a0.record()
        infos = [solve(B[(1 + i) % len(B)], prec, method["precond"])[1]
                 for i in range(steps)]
        a1.record()
        torch.cuda.synchronize()
        sec = a0.elapsed_time(a1) / 1e3
        out[prec] = {"operator_rel_err_vs_fp64": err, "apply_ms": apply_ms,
                     "value": steps / sec, "unit": "solves/s",
                     "iterations": [i.iterations for i in infos],
                     "outer_steps": [i.outer_steps for i in infos],
                     "true_relres": max(i.true_relres for i in infos),
                     "speedup_vs_plain": (steps / sec / plain_value
                                          if plain_value else None)}
    flops = pencil_gemm_flops(op)
    peak, src = _bf16_peak()
    ms = out["bf16"]["apply_ms"]
    out["bf16"]["tensor"] = {"kernel": f"k_tc_pencil<d={op.d}> (tcgen05.mma kind::f16, "
                                       f"+ BF16 conversion of x)",
                             "useful_flops_per_apply": flops,
                             "achieved": flops / ms / 1e9, "peak": peak,
                             "peak_source": src, "unit": "TFLOP/s",
                             "frac": flops / ms / 1e9 / peak}
    out["inner"] = ("FP64 iterative refinement; inner flexible GMRES to 1e-5 (fp32) / "
                    "1e-3 (bf16) relative with the method's preconditioner")
    return out


def rooflines(ab, op, mat, gmat, method, dt, workload, xs):
    """Average launch durations by CUDA events on the launching stream: the
    method's operator kernel (global form, algorithmic bytes against the
    measured HBM bandwidth) and the plain baseline's connected-pair kernel
    (algorithmic flops against the live-measured FP64 FMA peak)."""
    import torch
    d, N = op.d, op.N
    ys = torch.zeros_like(xs)
    flops = op.flops()

    def time_apply(m, precision, reps):
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

    preps = 5 if d <= 4 else 2
    t64 = time_apply(mat, "fp64", preps)
    t32 = time_apply(mat, "fp32", preps)
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
                 "traffic": KERNEL_TRAFFIC.get(("pairs", workload)),
                 "traffic_source": "ncu dram__bytes_read+write, one launch",
                 "ms_per_launch": t64 * 1e3, "flops_per_launch": flops,
                 "fp32_kernel": {"ms_per_launch": t32 * 1e3,
                                 "achieved": flops / t32 / 1e12,
                                 "peak": fp32_peak.value,
                                 "frac": flops / t32 / 1e12 / fp32_peak.value}}
    if gmat is None:
        return pair_roof
    # the method's operator kernel: algorithmic bytes per launch are x read
    # once, y written, the neighbour lists and the pre-summed blocks
    tg = time_apply(gmat, method["precision"], 10)
    nbytes = (16 * N + 8 * gmat.num_pairs() + 8 * (op.rows + 1)
              + 48 * len(op.vA) // (9 * op.terms))
    hbm, src = _measured_hbm_gbs()
    gk = ("kron_global_cell_dims" if method["precision"] == "fp32"
          else "kron_global_cell_ranges") if d >= 5 else "kron_global_rows"
    return {"bound": "hbm",
            "kernel": f"{gk}<d={d}, {method['precision']}>"
                      + (" (+ FP32 copy of x)" if d >= 5 and method["precision"] == "fp32"
                         else ""),
            "achieved": nbytes / tg / 1e9, "peak": hbm, "peak_source": src,
            "unit": "GB/s", "frac": nbytes / tg / 1e9 / hbm,
            "traffic": KERNEL_TRAFFIC.get(("global", workload)),
            "traffic_source": "ncu dram__bytes_read+write, one launch",
            "bytes_per_launch": nbytes, "ms_per_launch": tg * 1e3,
            "pair_kernel": pair_roof}


def cpu_baseline(workload):
    """One full solve by the reference's own CPU path (ReferenceSolves) on
    the host cores; value = 1 / its wall time.  Setup (the reference's
    global matrix and preconditioner) is not timed."""
    import oracle
    if not oracle.ref_gsolve_available():
        return {"value": None, "unit": "solves/s", "cores": 0, "kind": "reference",
                "sample": "reference library not built"}
    ref = ReferenceSolves(workload, seed=1)
    s = ref.full_solve()
    return {"value": 1.0 / s["seconds"], "unit": "solves/s", "cores": ref.cores,
            "kind": "reference",
            "sample": f"one full solve by the reference's solver::simple_gmres_euler "
                      f"over its global_kron_matrix ({s['iterations']} iterations, "
                      f"{s['seconds']:.1f} s, true relres {s['true_relres']:.2e}, "
                      f"OpenMP {ref.cores} threads)",
            "solve": s, "setup_s": ref.setup_s}


if __name__ == "__main__":
    main()
