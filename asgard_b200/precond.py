"""Learned preconditioner: a per-cell MLP trained on the GPU from plain GMRES
solves, used on the right inside flexible GMRES.

    pc = LearnedPreconditioner(op)                  # op: SparseGridOperator
    stats = pc.train(mat, dt, num_solves=5)         # 5 x cells training rows
    info = simple_gmres_euler(dt, mat, x, b, ..., precond=pc)

Training data follow BASELINE's recipe: random right-hand sides v, the plain
FP64 GMRES solution e of (I - dt K) e = v, and one (v_c, e_c) row per cell.
"""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np

from ._lib import check, lib

_MAGIC = b"ASGKMLP1"


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
        self.dims = [n ** d + d, hidden, hidden, hidden, n ** d]

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
    def generate(self, mat, dt, num_solves=5, restart=50, tol=1e-10, seed=0):
        """(v, e) sample pairs from plain FP64 GMRES solves (device tensors)."""
        import torch
        from .kronmult import simple_gmres_euler
        N = mat.output_size()
        g = torch.Generator(device="cuda").manual_seed(seed)
        V = torch.empty(num_solves, N, dtype=torch.float64, device="cuda")
        E = torch.zeros(num_solves, N, dtype=torch.float64, device="cuda")
        its = []
        for s in range(num_solves):
            V[s] = torch.rand(N, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
            info = simple_gmres_euler(dt, mat, E[s], V[s], restart, 400, tol,
                                      tol_mode="rel")
            its.append(info.iterations)
        return V, E, its

    def train(self, mat, dt, num_solves=5, epochs=60, batch=1024, lr=1e-3,
              seed=0, samples=None):
        """Generates the samples (unless given as (V, E)) and trains."""
        import torch
        if samples is None:
            V, E, its = self.generate(mat, dt, num_solves, seed=seed)
        else:
            V, E = samples
            its = []
        loss = C.c_double()
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        check(lib.asgk_mlp_train(self._h, C.c_void_p(V.data_ptr()),
                                 C.c_void_p(E.data_ptr()), V.shape[0], epochs,
                                 batch, lr, seed, C.byref(loss), stream),
              "mlp_train")
        return {"loss": loss.value, "rows": V.shape[0] * self.cells,
                "solve_iterations": its}

    def apply(self, mat, v, z):
        import torch
        check(lib.asgk_mlp_apply(self._h, mat.handle, C.c_void_p(v.data_ptr()),
                                 C.c_void_p(z.data_ptr()),
                                 C.c_void_p(torch.cuda.current_stream().cuda_stream)),
              "mlp_apply")
        return z
