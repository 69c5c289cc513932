"""Preconditioners of the backward-Euler operator, used on the right inside
(flexible) GMRES.

JacobiPreconditioner: the reference's diagonal preconditioner
(build_preconditioner, src/asgard_kronmult_matrix.cpp:1015-1067) or the
inverse of each cell's whole diagonal block, built on the device.

    pc = JacobiPreconditioner(mat, dt, kind="block")
    info = simple_gmres_euler(dt, mat, x, b, ..., precond=pc)

LearnedPreconditioner: a per-cell network trained on the GPU from plain
GMRES solves.  The network is
linear in the residual block and gated by the cell's levels (see
include/asgard_b200.h), so the preconditioner is a fixed linear operator.

    pc = LearnedPreconditioner(op)                  # op: SparseGridOperator
    stats = pc.train(mat, dt, num_solves=5)         # 5 x cells training rows
    info = simple_gmres_euler(dt, mat, x, b, ..., precond=pc)

Training data: (residual, GMRES-correction) pairs from plain FP64 GMRES solves
of random right-hand sides -- each restart cycle's residual r_k and the exact
correction x* - x_k -- one row per (pair, cell).  A solve with ~5 restart
cycles gives ~5 x cells rows (about 20k at d=4, level 7).
"""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np

from ._lib import check, lib

_MAGIC = b"ASGKMLP1"

JACOBI_KINDS = {"point": 0, "block": 1, "kron": 2, "line": 3}


class JacobiPreconditioner:
    """Point or cell-block Jacobi preconditioner of I - dt*K for a square
    kronmult_matrix (see asgk_jacobi_create in include/asgard_b200.h).
    kind "kron": the cell-block inverse through the eigendecompositions of
    its one-dimensional factors (global plans whose terms act in one
    dimension each; raises AsgkError otherwise).  kind "line": exact solves
    along the pencils of the dimensions with symmetric 1D operators, chained
    (ASGK_JACOBI_LINE; global plans)."""

    def __init__(self, mat, dt, kind="block"):
        if kind not in JACOBI_KINDS:
            raise ValueError(f"kind must be one of {sorted(JACOBI_KINDS)}")
        h = C.c_void_p()
        check(lib.asgk_jacobi_create(C.byref(h), mat.handle, float(dt),
                                     JACOBI_KINDS[kind]), "jacobi_create")
        self._h = h
        self.kind, self.dt = kind, float(dt)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.asgk_jacobi_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def device_bytes(self):
        b = C.c_int64()
        check(lib.asgk_jacobi_info(self._h, None, None, C.byref(b)))
        return b.value

    def apply(self, v, z, stream=None, precision="fp64"):
        """z = M v on CUDA float64 tensors; precision "fp32" applies it in
        the arithmetic of the FP32 inner solves."""
        from .kronmult import _precision, _ptr, _stream
        if precision == "fp64":
            check(lib.asgk_jacobi_apply(self._h, _ptr(v), _ptr(z), _stream(stream)),
                  "jacobi_apply")
        else:
            check(lib.asgk_jacobi_apply_precision(self._h, _precision(precision), _ptr(v),
                                                  _ptr(z), _stream(stream)),
                  "jacobi_apply")
        return z


class LearnedPreconditioner:
    def __init__(self, op=None, *, d=None, n=3, table=None, level=None,
                 hidden=256, seed=0):
        if op is not None:
            d, n, table, level = op.d, op.n, op.table, op.level
        table = np.ascontiguousarray(table, dtype=np.int32)
        self.d, self.n, self.level, self.hidden = d, n, level, hidden
        self.cells = table.shape[0]
        levels = np.ascontiguousarray(table[:, :d], dtype=np.int32)
        h = C.c_void_p()
        check(lib.asgk_mlp_create(C.byref(h), d, n, self.cells,
                                  levels.ctypes.data, level, hidden, seed),
              "mlp_create")
        self._h = h
        self.dims = [n ** d, hidden, hidden, hidden, n ** d]
        self.useful = None   # set by validate()
        self.base = None

    def set_base(self, base):
        """Preconditioner base(v) + network(v): the network learns a
        correction to a JacobiPreconditioner (None removes it)."""
        check(lib.asgk_mlp_set_base(self._h, base.handle if base is not None else None),
              "mlp_set_base")
        self.base = base      # kept alive with the network
        if base is not None:
            # start as the base itself: output layer W4 (hidden x n^d, after
            # W1 and two hidden x hidden layers in the flat parameters) zero
            ts, H = self.dims[0], self.hidden
            p = self.get_params()
            o = ts * H + 2 * H * H
            p[o:o + H * ts] = 0.0
            self.set_params(p)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.asgk_mlp_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    # -- parameters ------------------------------------------------------
    def num_params(self):
        c = C.c_int64()
        check(lib.asgk_mlp_num_params(self._h, C.byref(c)))
        return c.value

    def get_params(self):
        p = np.zeros(self.num_params(), np.float32)
        check(lib.asgk_mlp_get_params(self._h, p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.num_params():
            raise ValueError("parameter count mismatch")
        check(lib.asgk_mlp_set_params(self._h, p.ctypes.data))

    def save(self, path):
        """Plain binary: magic, header (d, n, level, hidden, cells), FP32 params."""
        p = self.get_params()
        with open(path, "wb") as f:
            f.write(_MAGIC)
            f.write(struct.pack("<5q", self.d, self.n, self.level, self.hidden,
                                self.cells))
            f.write(p.tobytes())

    def load(self, path):
        with open(path, "rb") as f:
            if f.read(8) != _MAGIC:
                raise ValueError("not a learned-preconditioner file")
            hdr = struct.unpack("<5q", f.read(40))
            if hdr != (self.d, self.n, self.level, self.hidden, self.cells):
                raise ValueError(f"shape mismatch: file {hdr}")
            self.set_params(np.frombuffer(f.read(), dtype=np.float32))

    # -- gradient check entry -------------------------------------------
    def forward_backward(self, X, T):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        rows = X.shape[0]
        Y = np.zeros((rows, self.dims[-1]), np.float32)
        g = np.zeros(self.num_params(), np.float32)
        loss = C.c_double()
        check(lib.asgk_mlp_forward_backward(self._h, rows, X.ctypes.data,
                                            T.ctypes.data, Y.ctypes.data,
                                            g.ctypes.data, C.byref(loss)),
              "mlp_forward_backward")
        return Y, loss.value, g

    # -- training ----------------------------------------------------------
    def generate(self, mat, dt, num_solves=5, restart=50, tol=1e-10, seed=0,
                 max_cycles=40, white_only=False):
        """(residual, GMRES-correction) pairs from plain FP64 GMRES solves of
        random right-hand sides: every restart cycle k of a solve gives the
        residual r_k = b - A x_k and the correction e_k = x* - x_k that solves
        A e_k = r_k exactly (x* the converged solution).  Device tensors."""
        import torch
        from .kronmult import simple_gmres_euler
        N = mat.output_size()
        g = torch.Generator(device="cuda").manual_seed(seed)
        Vs, Es, its = [], [], []
        for s in range(num_solves):
            b = torch.rand(N, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
            x = torch.zeros(N, dtype=torch.float64, device="cuda")
            iterates, total = [], 0
            for _ in range(max_cycles):
                iterates.append(x.clone())
                info = simple_gmres_euler(dt, mat, x, b, restart, 1, tol,
                                          tol_mode="rel")
                total += info.iterations
                if info.true_relres <= tol:
                    break
            its.append(total)
            if white_only:
                iterates = iterates[:1]   # only (b, x*): uncorrelated residuals
            for xk in iterates:
                r = b.clone()
                mat.apply_euler(dt, -1.0, xk, 1.0, r)   # r = b - A x_k
                Vs.append(r)
                Es.append(x - xk)
        return torch.stack(Vs), torch.stack(Es), its

    def train(self, mat, dt, num_solves=5, epochs=60, batch=1024, lr=1e-3,
              seed=0, samples=None, mat_T=None, residual_epochs=30,
              residual_lr=3e-4, precision="fp32"):
        """Generates the samples (unless given as (V, E)) and trains: first
        on the correction itself (mean squared error of e_c, cell rows), then,
        when mat_T (K^T) is given, on the preconditioned residual
        ||A M r - r|| / ||r|| of every sample (asgk_mlp_train_residual)."""
        import torch
        from .kronmult import _precision
        if samples is None:
            V, E, its = self.generate(mat, dt, num_solves, seed=seed)
        else:
            V, E = samples
            its = []
        if self.base is not None:
            # the network learns what the base misses: e - base(r)
            E = E.clone()
            z = torch.empty_like(E[0])
            for i in range(V.shape[0]):
                self.base.apply(V[i], z)
                E[i] -= z
        loss = C.c_double()
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        check(lib.asgk_mlp_train(self._h, C.c_void_p(V.data_ptr()),
                                 C.c_void_p(E.data_ptr()), V.shape[0], epochs,
                                 batch, lr, seed, C.byref(loss), stream),
              "mlp_train")
        out = {"loss": loss.value, "rows": V.shape[0] * self.cells,
               "samples": V.shape[0], "solve_iterations": its}
        if mat_T is not None and residual_epochs > 0:
            rl = C.c_double()
            check(lib.asgk_mlp_train_residual(
                self._h, mat.handle, mat_T.handle, dt, C.c_void_p(V.data_ptr()),
                C.c_void_p(E.data_ptr()), V.shape[0], residual_epochs,
                residual_lr, _precision(precision), seed, C.byref(rl), stream),
                "mlp_train_residual")
            out["residual_loss"] = rl.value
        out["validation"] = self.validate(mat, dt, seed=seed + 7919)
        return out

    def validate(self, mat, dt, seed=0, restart=50, tol=1e-10):
        """Solves one held-out right-hand side with and without the network
        (FP64, relative tolerance; "without" keeps the base preconditioner
        when one is set) and records whether it reduced the iteration count;
        ``useful`` is False when it did not, and callers then fall back to
        the method without it (the solver also drops a network that stalls a
        solve)."""
        import torch
        from .kronmult import simple_gmres_euler
        N = mat.output_size()
        g = torch.Generator(device="cuda").manual_seed(seed)
        b = torch.rand(N, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        plain = simple_gmres_euler(dt, mat, torch.zeros_like(b), b, restart,
                                   400, tol, tol_mode="rel", precond=self.base)
        learned = simple_gmres_euler(dt, mat, torch.zeros_like(b), b, restart,
                                     400, tol, tol_mode="rel", precond=self)
        self.useful = (learned.status == 0 and learned.fallback == 0 and
                       learned.iterations < plain.iterations)
        return {"baseline": "block-jacobi" if self.base is not None else "none",
                "plain_iterations": plain.iterations,
                "learned_iterations": learned.iterations,
                "learned_fallback": learned.fallback,
                "gain": plain.iterations / max(learned.iterations, 1),
                "useful": self.useful}

    def apply(self, mat, v, z):
        import torch
        check(lib.asgk_mlp_apply(self._h, mat.handle, C.c_void_p(v.data_ptr()),
                                 C.c_void_p(z.data_ptr()),
                                 C.c_void_p(torch.cuda.current_stream().cuda_stream)),
              "mlp_apply")
        return z
