"""Python mirror of the reference's kronmult_matrix / simple_gmres interfaces.

Mirrors ``asgard::kronmult_matrix<P>`` (src/asgard_kronmult_matrix.hpp:111-682)
and ``asgard::solver::simple_gmres_euler`` / ``simple_gmres``
(src/solver.hpp:17-41) over the C ABI.  Device vectors are CUDA tensors
(torch, float64 unless stated); host vectors are numpy arrays.  Errors raise
the reference's exception types: ``RuntimeError`` for unsupported shapes and
runtime failures, ``ValueError`` (std::invalid_argument) for a restart larger
than the system.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import IMEX_HOOK, AsgkError, GmresInfo, check, lib

FP64, FP32, BF16 = 0, 1, 2
TOL_ABS, TOL_REL = 0, 1
_PREC = {"fp64": FP64, "fp32": FP32, "bf16": BF16}


def _precision(p) -> int:
    return _PREC[p] if isinstance(p, str) else int(p)


def _host(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _ptr(t):
    """Device pointer of a CUDA tensor (or 0/None)."""
    if t is None:
        return None
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


@dataclass
class gmres_info:
    """``gmres_info<P>`` (src/pde/pde_base.hpp:93-97) plus solve diagnostics."""
    error: float
    iterations: int
    status: int = 0
    true_relres: float = float("nan")
    outer_steps: int = 0
    matvecs_low: int = 0
    matvecs_fp64: int = 0
    precond_calls: int = 0
    fallback: int = 0


class kronmult_matrix:
    """A batched-Kronecker operator held on the GPU (see module docstring)."""

    def __init__(self, handle, d, n, rows, cols, terms):
        self._h = handle
        self.num_dimensions = d
        self.kron_size = n
        self.num_rows = rows
        self.num_cols = cols
        self.num_terms = terms

    # -- constructors ------------------------------------------------------
    @classmethod
    def from_csr(cls, d, n, num_rows, num_cols, num_terms, pntr, indx, iA, vA):
        """Reference CPU sparse format: row pointers, column cells, iA, vA."""
        pntr = _host(pntr, np.int64)
        indx = _host(indx, np.int32)
        iA = _host(iA, np.int32)
        vA = _host(vA, np.float64)
        h = C.c_void_p()
        check(lib.asgk_plan_create(C.byref(h), d, n, num_rows, num_cols,
                                   num_terms, pntr.ctypes.data,
                                   indx.ctypes.data, iA.ctypes.data,
                                   vA.ctypes.data, len(vA)), "plan_create")
        return cls(h, d, n, num_rows, num_cols, num_terms)

    @classmethod
    def from_pairs(cls, d, n, num_rows, num_cols, num_terms, row_indx,
                   col_indx, iA, vA):
        """Reference GPU format: per pair the tensor offsets into y and x."""
        iy = _host(row_indx, np.int32)
        ix = _host(col_indx, np.int32)
        iA = _host(iA, np.int32)
        vA = _host(vA, np.float64)
        h = C.c_void_p()
        check(lib.asgk_plan_create_pairs(C.byref(h), d, n, num_rows, num_cols,
                                         num_terms, len(iy), iy.ctypes.data,
                                         ix.ctypes.data, iA.ctypes.data,
                                         vA.ctypes.data, len(vA)),
              "plan_create_pairs")
        return cls(h, d, n, num_rows, num_cols, num_terms)

    @classmethod
    def from_conn(cls, d, n, num_rows, num_cols, num_terms, row_ptr, col_indx,
                  conn, vA):
        """Sparse-grid format: per pair the d 1D connection indices."""
        rp = _host(row_ptr, np.int64)
        ci = _host(col_indx, np.int32)
        cn = _host(conn, np.int32)
        vA = _host(vA, np.float64)
        h = C.c_void_p()
        check(lib.asgk_plan_create_conn(C.byref(h), d, n, num_rows, num_cols,
                                        num_terms, rp.ctypes.data,
                                        ci.ctypes.data, cn.ctypes.data,
                                        vA.ctypes.data, len(vA)),
              "plan_create_conn")
        return cls(h, d, n, num_rows, num_cols, num_terms)

    @classmethod
    def from_grid(cls, d, n, level, num_terms, vA):
        """The sparse grid of dimension d and this level with its connected
        cell pairs found on the GPU (vA in the per-1D-connection layout):
        the plan from_conn makes from the host-built pair list."""
        vA = _host(vA, np.float64)
        h = C.c_void_p()
        check(lib.asgk_plan_create_grid(C.byref(h), d, n, level, num_terms,
                                        vA.ctypes.data, len(vA)), "plan_create_grid")
        cells = lib.asgk_sparse_grid(d, level, None)
        return cls(h, d, n, cells, cells, num_terms)

    @classmethod
    def from_global(cls, d, n, level, table, num_terms, vA):
        """Global Kronecker form of the sparse grid's operator: the element
        table (cells x 2d) and vA in the per-1D-connection layout.  Terms
        acting in one dimension are applied in one pass, terms acting in
        several as the reference's chains of upper/lower 1D passes."""
        tb = _host(table, np.int32)
        vA = _host(vA, np.float64)
        cells = tb.shape[0]
        h = C.c_void_p()
        check(lib.asgk_plan_create_global(C.byref(h), d, n, level, cells,
                                          tb.ctypes.data, num_terms,
                                          vA.ctypes.data, len(vA)),
              "plan_create_global")
        return cls(h, d, n, cells, cells, num_terms)

    @classmethod
    def from_dense(cls, d, n, num_rows, num_cols, num_terms, terms, elem,
                   row_offset=0, col_offset=0, num_1d_blocks=1):
        """Dense form (the reference's dense constructor): every output cell
        with every input cell; terms is a list of num_terms arrays of
        d*num_1d_blocks^2*n^2 values (per dimension the column-major n x n
        blocks ordered by column cell, then row cell), elem the 1D cell
        indices of every cell (cells x d), rows starting at row_offset and
        columns at col_offset."""
        tv = [_host(t, np.float64) for t in terms]
        if len(tv) != num_terms:
            raise ValueError("terms must hold num_terms arrays")
        el = _host(elem, np.int32).ravel()
        ptrs = (C.c_void_p * max(num_terms, 1))(*[t.ctypes.data for t in tv])
        h = C.c_void_p()
        check(lib.asgk_plan_create_dense(C.byref(h), d, n, num_rows, num_cols,
                                         num_terms, ptrs, el.ctypes.data,
                                         len(el), row_offset, col_offset,
                                         num_1d_blocks), "plan_create_dense")
        return cls(h, d, n, num_rows, num_cols, num_terms)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.asgk_plan_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    # -- accessors (src/asgard_kronmult_matrix.hpp:480-577) ---------------
    def _info(self):
        vals = [C.c_int64() for _ in range(5)]
        check(lib.asgk_plan_info(self._h, *[C.byref(v) for v in vals]))
        return [v.value for v in vals]

    def num_batch(self):
        """num_rows * num_cols, as the reference's num_batch()
        (src/asgard_kronmult_matrix.hpp:481) returns for every matrix."""
        return self.num_rows * self.num_cols

    def num_pairs(self):
        """The (row, col) products one apply computes: the stored pairs
        (rows*cols for a dense plan, the single-direction entries for the
        global form)."""
        return self._info()[0]

    def tensor_size(self):
        return self.kron_size ** self.num_dimensions

    def input_size(self):
        return self._info()[1]

    def output_size(self):
        return self._info()[2]

    def flops(self):
        """Flops of one apply, multiply and add counted apart:
        compute_flops(d, n, T, num_pairs()) = 2 * n^d * n * d * T * pairs
        (2 * n^(d+1) per entry for the global form)."""
        return self._info()[3]

    def device_bytes(self):
        return self._info()[4]

    @staticmethod
    def compute_tensor_size(num_dimensions, kron_size):
        return kron_size ** num_dimensions

    @staticmethod
    def compute_flops(num_dimensions, kron_size, num_terms, num_batch):
        return kron_size ** num_dimensions * kron_size * num_dimensions * num_terms * num_batch * 2

    def kind(self):
        """"sparse", "dense" or "global"."""
        return ("sparse", "dense", "global")[lib.asgk_plan_kind(self._h)]

    def is_dense(self):
        return lib.asgk_plan_kind(self._h) == 1

    def is_onecall(self):
        return True

    def __bool__(self):
        return self.num_dimensions > 0

    def update_stored_coefficients(self, vA):
        """New factor values in the layout the plan was made from: one vA
        array, or for a dense plan the list of per-term arrays."""
        if self.is_dense():
            tv = [_host(t, np.float64) for t in vA]
            ptrs = (C.c_void_p * max(len(tv), 1))(*[t.ctypes.data for t in tv])
            check(lib.asgk_plan_update_terms(self._h, ptrs, len(tv)),
                  "update_stored_coefficients")
            return
        vA = _host(vA, np.float64)
        check(lib.asgk_plan_update_values(self._h, vA.ctypes.data, len(vA)),
              "update_stored_coefficients")

    def set_workspace(self, x, y):
        """Device tensors (float64, at least input_size / output_size) that
        host applies stage x and y in (kronmult_matrix::set_workspace);
        the caller keeps them alive."""
        check(lib.asgk_plan_set_workspace(self._h, _ptr(x), x.numel(), _ptr(y),
                                          y.numel()), "set_workspace")
        self._workspace = (x, y)

    # -- apply -------------------------------------------------------------
    def apply(self, alpha, x, beta, y, resource="device", precision="fp64",
              stream=None):
        """y = beta*y + alpha*K*x.

        resource="device": x, y are CUDA tensors (float64, or float32 for a
        float32 apply); resource="host": numpy float64 arrays, copied to and
        from the GPU inside the call."""
        if resource == "host":
            xs = _host(x, np.float64)
            if not (y.flags["C_CONTIGUOUS"] and y.dtype == np.float64):
                raise ValueError("y must be a contiguous float64 array")
            check(lib.asgk_apply_host(self._h, alpha, xs.ctypes.data, beta,
                                      y.ctypes.data, _stream(stream)), "apply")
            return y
        import torch
        if x.dtype == torch.float32:
            check(lib.asgk_apply_f32(self._h, alpha, _ptr(x), beta, _ptr(y),
                                     _stream(stream)), "apply")
        else:
            check(lib.asgk_apply(self._h, _precision(precision), alpha,
                                 _ptr(x), beta, _ptr(y), _stream(stream)),
                  "apply")
        return y

    def apply_euler(self, dt, alpha, x, beta, y, precision="fp64", stream=None):
        """y = beta*y + alpha*(x - dt*K*x) on device tensors."""
        check(lib.asgk_apply_euler(self._h, _precision(precision), dt, alpha,
                                   _ptr(x), beta, _ptr(y), _stream(stream)),
              "apply_euler")
        return y


def simple_gmres_euler(dt, mat: kronmult_matrix, x, b, restart=-1,
                       max_iter=-1, tol=-1.0, tol_mode="abs",
                       precision="fp64", precond=None, stream=None):
    """Solves (I - dt*K) x = b in place on device tensors (x = initial guess).

    tol_mode="abs" is the reference criterion (estimated residual <= tol);
    "rel" stops at tol * ||b||.  precision "fp32"/"bf16" runs the Krylov
    operator in that arithmetic inside FP64 iterative refinement.  precond is
    a preconditioner of asgard_b200.precond (JacobiPreconditioner or
    LearnedPreconditioner) used on the right through flexible GMRES."""
    from .precond import JacobiPreconditioner
    n = mat.output_size()
    if restart is not None and restart > n:
        raise ValueError(f"Number of inner iterations {restart} must be less than {n}!")
    info = GmresInfo()
    pc = precond.handle if precond is not None else None
    entry = (lib.asgk_gmres_euler_jacobi if isinstance(precond, JacobiPreconditioner)
             else lib.asgk_gmres_euler)
    rc = entry(mat.handle, dt, _ptr(x), _ptr(b),
                              -1 if restart is None else restart,
                              -1 if max_iter is None else max_iter, tol,
                              TOL_REL if tol_mode == "rel" else TOL_ABS,
                              _precision(precision), pc, C.byref(info),
                              _stream(stream))
    if rc == 1 and restart is not None and restart > n:
        raise ValueError("restart larger than the system")
    check(rc, "simple_gmres_euler")
    return gmres_info(**info.as_dict())


def implicit_advance(dt, mat: kronmult_matrix, x, steps, forcing=None,
                     restart=-1, max_iter=-1, tol=-1.0, tol_mode="abs",
                     precision="fp64", precond=None, stream=None):
    """`steps` backward-Euler steps with x resident on the device (the GMRES
    branch of the reference's implicit_advance, src/time_advance.cpp:308-470):
    per step x += dt*f_k, then (I - dt*K) x_new = x from the initial guess x.
    forcing: None, one device vector (every step) or a (steps, N) device
    tensor (one per step).  Returns the per-step gmres_info list."""
    from .precond import JacobiPreconditioner
    n = mat.output_size()
    if restart is not None and restart > n:
        raise ValueError(f"Number of inner iterations {restart} must be less than {n}!")
    infos = (GmresInfo * max(steps, 1))()
    stride = 0
    if forcing is not None and forcing.dim() == 2:
        if forcing.shape[0] < steps:
            raise ValueError("forcing must hold one vector per step")
        stride = forcing.stride(0)
    kind = (0 if precond is None else
            1 if isinstance(precond, JacobiPreconditioner) else 2)
    rc = lib.asgk_implicit_advance(mat.handle, dt, _ptr(x), steps,
                                   _ptr(forcing), stride,
                                   -1 if restart is None else restart,
                                   -1 if max_iter is None else max_iter, tol,
                                   TOL_REL if tol_mode == "rel" else TOL_ABS,
                                   _precision(precision), kind,
                                   precond.handle if precond is not None else None,
                                   infos, _stream(stream))
    check(rc, "implicit_advance")
    return [gmres_info(**infos[k].as_dict()) for k in range(steps)]


IMEX_BEFORE_EXPLICIT, IMEX_BEFORE_IMPLICIT = 0, 1


def imex_advance(dt, explicit: kronmult_matrix, implicit, x, steps, restart=-1,
                 max_iter=-1, tol=-1.0, tol_mode="abs", precision="fp64",
                 precond=(None, None), hook=None, stream=None):
    """`steps` steps of the reference's two-stage IMEX scheme (imex_advance,
    src/time_advance.cpp:477-990) with x resident on the device:
    f_1s = f_0 + dt E f_0, f_1 = (I - dt I)^-1 f_1s; f_2s = (f_0 + f_1 +
    dt E f_1) / 2, f_2 = (I - dt/2 I)^-1 f_2s, E = explicit, I = implicit
    (None: no implicit part, f_1 = f_1s and the step ends with f_2s).
    precond: Jacobi preconditioners of `implicit` for dt and dt/2 (or None).
    hook(step, stage, event, f) is called with f a device tensor (read-only)
    at IMEX_BEFORE_EXPLICIT (the state the stage's explicit apply reads: the
    reference's Poisson update) and IMEX_BEFORE_IMPLICIT (the stage's explicit
    result: moments and coefficient regeneration; the hook may call
    update_stored_coefficients on the plans); a non-zero return or an
    exception stops the loop.  Returns per step the (stage 1, stage 2)
    gmres_info pair."""
    import torch
    n = explicit.output_size()
    if implicit is not None and restart is not None and restart > n:
        raise ValueError(f"Number of inner iterations {restart} must be less than {n}!")
    work = torch.empty((4, max(n, 1)), dtype=torch.float64, device=x.device)
    views = {x.data_ptr(): x}
    views.update({work[i].data_ptr(): work[i] for i in range(4)})
    errors = []

    def _call(ctx, step, stage, event, f, strm):
        try:
            r = hook(step, stage, event, views[f])
            return 0 if r is None else int(r)
        except Exception as e:  # reported after the call returns
            errors.append(e)
            return 1
    cb = IMEX_HOOK(_call) if hook is not None else None
    infos = (GmresInfo * max(2 * steps, 1))()
    pc1, pc2 = precond if precond is not None else (None, None)
    rc = lib.asgk_imex_advance(explicit.handle,
                               implicit.handle if implicit is not None else None,
                               dt, _ptr(x), steps,
                               -1 if restart is None else restart,
                               -1 if max_iter is None else max_iter, tol,
                               TOL_REL if tol_mode == "rel" else TOL_ABS,
                               _precision(precision),
                               pc1.handle if pc1 is not None else None,
                               pc2.handle if pc2 is not None else None,
                               C.cast(cb, C.c_void_p) if cb is not None else None,
                               None, work.data_ptr(), infos, _stream(stream))
    if errors:
        raise errors[0]
    check(rc, "imex_advance")
    return [(gmres_info(**infos[2 * k].as_dict()), gmres_info(**infos[2 * k + 1].as_dict()))
            for k in range(steps)]


def simple_gmres(A, x, b, M=None, restart=-1, max_iter=-1, tol=-1.0):
    """Dense test path of solver::simple_gmres (host arrays, solved on the
    GPU).  M: the reference's dense preconditioner (src/solver.cpp:11-38),
    LU-factored and applied on the left; None or an empty matrix for none."""
    A = np.asfortranarray(A, dtype=np.float64)
    n = A.shape[0]
    if restart is not None and restart > n:
        raise ValueError(f"Number of inner iterations {restart} must be less than {n}!")
    bb = _host(b, np.float64)
    if not (x.flags["C_CONTIGUOUS"] and x.dtype == np.float64):
        raise ValueError("x must be a contiguous float64 array")
    Mp = None
    if M is not None and np.size(M) > 0:
        Mf = np.asfortranarray(M, dtype=np.float64)
        if Mf.shape != (n, n):
            raise ValueError("M must be n x n")
        Mp = Mf.ctypes.data
    info = GmresInfo()
    check(lib.asgk_gmres_dense_precond(n, A.ctypes.data, x.ctypes.data,
                                       bb.ctypes.data, Mp, restart, max_iter,
                                       tol, C.byref(info)),
          "simple_gmres")
    return gmres_info(**info.as_dict())


def cgs_step(V, k, w, h=None, stream=None):
    """One classical Gram-Schmidt step of the device GMRES on CUDA tensors:
    h = V[:, :k]^T w, w -= V[:, :k] h (in place); returns (h, ||w||).
    V is (k_cols, n) row-major in torch terms, i.e. column-major n x k_cols
    with leading dimension n."""
    import torch
    n = w.numel()
    if h is None:
        h = torch.empty(k, dtype=torch.float64, device=w.device)
    nrm = C.c_double()
    check(lib.asgk_cgs_step(_ptr(V), V.stride(0), k, _ptr(w), n, _ptr(h),
                            C.byref(nrm), _stream(stream)), "cgs_step")
    return h, nrm.value


def default_gmres_restarts(n: int) -> int:
    return lib.asgk_default_gmres_restarts(n)


def launch_count() -> int:
    return lib.asgk_launch_count()


def gmres_settings(graphs=None, node_steps=None, fp32_basis=None,
                   bf16_inner_tol=None) -> dict:
    """Process-wide settings of the device GMRES (asgk_set_gmres_graphs,
    asgk_set_gmres_node_steps, asgk_set_gmres_basis,
    asgk_set_bf16_inner_tol): restart cycles recorded as CUDA graphs, Arnoldi
    steps per recorded graph node, whether the FP32 inner solves orthogonalise
    against an FP32 copy of the basis, and the inner tolerance of the BF16
    tensor-core solves.  The arguments given are set; returns the settings in
    force before the call (pass the dict back as keyword arguments to restore
    them).  None of them changes iterates except fp32_basis and
    bf16_inner_tol."""
    old_tol = lib.asgk_set_bf16_inner_tol(bf16_inner_tol if bf16_inner_tol is not None else 0.0)
    old_steps = lib.asgk_set_gmres_node_steps(node_steps if node_steps is not None else 0)
    if graphs is None:
        old_graphs = lib.asgk_set_gmres_graphs(1)
        lib.asgk_set_gmres_graphs(old_graphs)
    else:
        old_graphs = lib.asgk_set_gmres_graphs(1 if graphs else 0)
    if fp32_basis is None:
        old_basis = lib.asgk_set_gmres_basis(1)
        lib.asgk_set_gmres_basis(old_basis)
    else:
        old_basis = lib.asgk_set_gmres_basis(1 if fp32_basis else 0)
    return {"graphs": bool(old_graphs), "node_steps": old_steps,
            "fp32_basis": bool(old_basis), "bf16_inner_tol": old_tol}


__all__ = ["kronmult_matrix", "simple_gmres_euler", "simple_gmres", "cgs_step",
           "implicit_advance", "imex_advance", "gmres_settings",
           "gmres_info", "default_gmres_restarts", "launch_count", "AsgkError"]
