"""Test infrastructure: ctypes bindings to the two CPU checkers.

* ``liboracle.so`` -- the plain-C restatement in ``asgard_oracle.c`` of the
  reference's CPU kronmult, sparse-grid/pair-list builder and GMRES.
* ``_ref/libasgard_ref.so`` -- the reference itself, compiled from its own
  sources by ``Makefile`` (target ``ref``), reached through ``ref_shim.cpp``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may
import this package, and only as the checker or the CPU baseline; the product
(``asgard_b200``) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libasgard_ref.so")
REF_GLOBAL_SO = os.path.join(HERE, "_ref", "libasgard_ref_global.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")

_oracle = None
_ref = None
_ref_global = None


def build_oracle(force: bool = False) -> str:
    """Compiles liboracle.so (gcc is present wherever the tests run)."""
    if force or not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-C", HERE, "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return ORACLE_SO


def oracle():
    global _oracle
    if _oracle is None:
        build_oracle()
        lib = C.CDLL(ORACLE_SO)
        for name, T in (("f64", _f64p), ("f32", _f32p)):
            fn = getattr(lib, f"orc_kronmult_sparse_{name}")
            S = C.c_double if name == "f64" else C.c_float
            fn.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, C.c_int,
                           _i32p, T, S, T, S, T]
            fn.restype = C.c_int
        lib.orc_assemble_dense.argtypes = [C.c_int, C.c_int, C.c_int, _i32p,
                                           _i32p, C.c_int, _i32p, _f64p, _f64p]
        lib.orc_connect_1d.argtypes = [C.c_int, C.POINTER(C.c_int),
                                       C.POINTER(C.c_int), C.c_void_p,
                                       C.c_void_p]
        lib.orc_sparse_grid.argtypes = [C.c_int, C.c_int, C.c_void_p]
        lib.orc_sparse_grid.restype = C.c_int64
        lib.orc_build_pairs.argtypes = [C.c_int, C.c_int, C.c_int, _i32p,
                                        C.POINTER(C.c_int64), C.c_void_p,
                                        C.c_void_p, C.c_void_p]
        lib.orc_expand_iA.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int64,
                                      _i32p, _i32p]
        lib.orc_expand_iA.restype = None
        lib.orc_rotg.argtypes = [C.POINTER(C.c_double)] * 4
        lib.orc_rotg.restype = None
        lib.orc_gmres_euler.argtypes = [C.c_int, C.c_int, C.c_int, _i32p,
                                        _i32p, C.c_int, _i32p, _f64p,
                                        C.c_double, _f64p, _f64p, C.c_int,
                                        C.c_int, C.c_double,
                                        C.POINTER(C.c_double),
                                        C.POINTER(C.c_int)]
        lib.orc_gmres_dense.argtypes = [C.c_int, _f64p, _f64p, _f64p, C.c_int,
                                        C.c_int, C.c_double,
                                        C.POINTER(C.c_double),
                                        C.POINTER(C.c_int)]
        lib.orc_make_kronmult_data.argtypes = [C.c_int] * 6 + [
            _i32p, _i32p, _i32p, C.c_void_p, C.c_void_p, C.c_void_p]
        for name, T in (("f64", _f64p), ("f32", _f32p)):
            S = C.c_double if name == "f64" else C.c_float
            fn = getattr(lib, f"orc_kronmult_dense_{name}")
            fn.argtypes = [C.c_int] * 5 + [_i32p, C.c_int, C.c_int, C.c_void_p,
                                           C.c_int, S, T, S, T]
            fn.restype = C.c_int
        lib.orc_make_kronmult_welem.argtypes = [C.c_int] * 5 + [
            _i32p, C.c_void_p, C.c_void_p, C.c_void_p]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _load_blas_deps():
    # OpenBLAS (linked by the reference builds) finds its private
    # libgfortran only when that is loaded first from the same folder.
    import glob, site
    for sp in site.getsitepackages():
        deps = glob.glob(os.path.join(sp, "opencv_python_headless.libs", "lib*.so*"))
        for key in ("quadmath", "gfortran"):
            for dep in deps:
                if key in os.path.basename(dep):
                    C.CDLL(dep, mode=C.RTLD_GLOBAL)


def ref_global_available() -> bool:
    return os.path.exists(REF_GLOBAL_SO)


class RefGlobal:
    """The reference's global Kronecker product (global_cpu,
    src/device/asgard_glkronmult_cpu.cpp:150-188; built by `make -C oracle
    ref_global`) on a sparse-grid operator: build once, apply many times."""

    def __init__(self, d, n, level, table, terms, vA):
        global _ref_global
        if _ref_global is None:
            if not ref_global_available():
                raise FileNotFoundError(REF_GLOBAL_SO)
            _load_blas_deps()
            lib = C.CDLL(REF_GLOBAL_SO)
            lib.ref_global_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int,
                                              _i32p, C.c_int, _f64p]
            lib.ref_global_create.restype = C.c_void_p
            lib.ref_global_run.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p,
                                           C.POINTER(C.c_double)]
            lib.ref_global_run.restype = C.c_int
            lib.ref_global_destroy.argtypes = [C.c_void_p]
            _ref_global = lib
        self._lib = _ref_global
        table = np.ascontiguousarray(table, dtype=np.int32)
        self.N = table.shape[0] * n ** d
        self._h = self._lib.ref_global_create(d, n, level, table.shape[0], table,
                                              terms, np.ascontiguousarray(vA, dtype=np.float64))
        if not self._h:
            raise ValueError("ref_global_create rejected its input")

    def apply(self, x, reps=1):
        """y = K x; returns (y, best seconds of one product)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.N)
        sec = C.c_double()
        if self._lib.ref_global_run(self._h, reps, x, y, C.byref(sec)) != 0:
            raise ValueError("ref_global_run failed")
        return y, sec.value

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.ref_global_destroy(self._h)
            self._h = None


def ref_global_apply(d, n, level, table, terms, vA, x, reps=1):
    """One-shot RefGlobal(...).apply(x, reps)."""
    return RefGlobal(d, n, level, table, terms, vA).apply(x, reps)


REF_GSOLVE_SO = os.path.join(HERE, "_ref", "libasgard_ref_gsolve.so")
_ref_gsolve = None


def ref_gsolve_available() -> bool:
    return os.path.exists(REF_GSOLVE_SO)


def _gsolve_lib():
    global _ref_gsolve
    if _ref_gsolve is None:
        if not ref_gsolve_available():
            raise FileNotFoundError(REF_GSOLVE_SO)
        _load_blas_deps()
        lib = C.CDLL(REF_GSOLVE_SO)
        lib.ref_gsolve_create_synthetic.argtypes = [
            C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _i32p, _i32p,
            _f64p, _f64p]
        lib.ref_gsolve_create_synthetic.restype = C.c_void_p
        lib.ref_gsolve_create_builtin.argtypes = [C.c_char_p, C.c_int, C.c_int,
                                                  C.c_int]
        lib.ref_gsolve_create_builtin.restype = C.c_void_p
        lib.ref_gsolve_destroy.argtypes = [C.c_void_p]
        lib.ref_gsolve_destroy.restype = None
        lib.ref_gsolve_info.argtypes = [C.c_void_p, C.POINTER(C.c_int),
                                        C.POINTER(C.c_int), C.POINTER(C.c_int),
                                        C.POINTER(C.c_int64)]
        lib.ref_gsolve_table.argtypes = [C.c_void_p, _i32p]
        lib.ref_gsolve_precond.argtypes = [C.c_void_p, _f64p]
        lib.ref_gsolve_apply.argtypes = [C.c_void_p, C.c_double, _f64p,
                                         C.c_double, _f64p,
                                         C.POINTER(C.c_double)]
        lib.ref_gsolve_gmres_euler.argtypes = [
            C.c_void_p, C.c_double, _f64p, _f64p, C.c_int, C.c_int,
            C.c_double, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int),
            C.POINTER(C.c_double)]
        _ref_gsolve = lib
    return _ref_gsolve


def load_ops1d(path=None):
    """The level-7 1D blocks the synthetic advection/diffusion operators are
    made of (generated from the reference by tests/golden/make_golden.py):
    pntr/indx (level-7 1D connectivity), adv, dif (one column-major 3x3 block
    per connection)."""
    if path is None:
        path = os.path.join(os.path.dirname(HERE), "asgard_b200", "data",
                            "ops1d_L7.npz")
    z = np.load(path)
    return {k: np.ascontiguousarray(z[k]) for k in z.files}


class RefGlobalSolver:
    """The reference's implicit global-Kronecker path end to end
    (``oracle/ref_gsolve_shim.cpp``): its sparse grid, make_global_kron_matrix,
    set_specific_mode (values + diagonal preconditioner), the operator's CPU
    apply and solver::simple_gmres_euler (src/solver.cpp:93-117, left diagonal
    preconditioning, absolute tolerance on the estimated preconditioned
    residual), OpenMP on all host threads.

    ``RefGlobalSolver.synthetic(d, level, terms, nu)`` builds the benchmark's
    advection/diffusion operator; ``RefGlobalSolver.builtin(name, d, level,
    n)`` a built-in reference PDE."""

    def __init__(self, handle):
        self._lib = _gsolve_lib()
        if not handle:
            raise ValueError("the reference rejected the operator")
        self._h = handle
        d, n, cells, N = C.c_int(), C.c_int(), C.c_int(), C.c_int64()
        self._lib.ref_gsolve_info(self._h, C.byref(d), C.byref(n),
                                  C.byref(cells), C.byref(N))
        self.d, self.n, self.cells, self.N = d.value, n.value, cells.value, N.value

    @classmethod
    def synthetic(cls, d, level, terms, nu, ops=None):
        ops = ops if ops is not None else load_ops1d()
        lib = _gsolve_lib()
        h = lib.ref_gsolve_create_synthetic(
            d, level, terms, 3, nu, ops["pntr"].astype(np.int32),
            ops["indx"].astype(np.int32),
            ops["adv"].astype(np.float64).reshape(-1),
            ops["dif"].astype(np.float64).reshape(-1))
        return cls(h)

    @classmethod
    def builtin(cls, name, d, level, n):
        lib = _gsolve_lib()
        return cls(lib.ref_gsolve_create_builtin(name.encode(), d, level, n))

    def table(self):
        t = np.zeros((self.cells, 2 * self.d), np.int32)
        self._lib.ref_gsolve_table(self._h, t)
        return t

    def precond(self):
        """The reference's diagonal preconditioner values pc (its solve
        divides by 1 - dt*pc)."""
        pc = np.zeros(self.N)
        if self._lib.ref_gsolve_precond(self._h, pc) != 0:
            raise ValueError("no preconditioner built")
        return pc

    def apply(self, alpha, x, beta=0.0, y=None):
        """y <- beta*y + alpha*K*x; returns (y, seconds)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.N) if y is None else y
        sec = C.c_double()
        if self._lib.ref_gsolve_apply(self._h, alpha, x, beta, y,
                                      C.byref(sec)) != 0:
            raise ValueError("apply failed")
        return y, sec.value

    def gmres_euler(self, dt, x, b, restart, max_iter, tol, quiet=True):
        """solver::simple_gmres_euler in place on x; returns (error,
        iterations, seconds)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        err, its, sec = C.c_double(), C.c_int(), C.c_double()
        rc = self._lib.ref_gsolve_gmres_euler(
            self._h, dt, x, b, restart, max_iter, tol, int(quiet),
            C.byref(err), C.byref(its), C.byref(sec))
        if rc != 0:
            raise ValueError("simple_gmres_euler failed")
        return err.value, its.value, sec.value

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.ref_gsolve_destroy(self._h)
            self._h = None


def ref():
    """The reference compiled from source; raises if it was not built."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(REF_SO)
        # OpenBLAS (linked by the reference build) finds its private
        # libgfortran only when that is loaded first from the same folder.
        import glob, site
        for sp in site.getsitepackages():
            deps = glob.glob(os.path.join(sp, "opencv_python_headless.libs",
                                          "lib*.so*"))
            for key in ("quadmath", "gfortran"):
                for dep in deps:
                    if key in os.path.basename(dep):
                        C.CDLL(dep, mode=C.RTLD_GLOBAL)
        lib = C.CDLL(REF_SO)
        for name, T in (("f64", _f64p), ("f32", _f32p)):
            S = C.c_double if name == "f64" else C.c_float
            fn = getattr(lib, f"ref_cpu_sparse_{name}")
            fn.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, C.c_int,
                           _i32p, T, S, T, S, T]
            fn = getattr(lib, f"ref_make_kronmult_data_{name}")
            fn.argtypes = [C.c_int] * 5 + [_i32p, _i32p, _i32p, T, T, T, T]
            fn = getattr(lib, f"ref_make_welem_{name}")
            fn.argtypes = [C.c_int] * 5 + [_i32p, T, T, T, T]
            fn = getattr(lib, f"ref_dense_apply_{name}")
            fn.argtypes = [C.c_int] * 5 + [T, _i32p] + [C.c_int] * 4 + [S, T, S, T]
        lib.ref_gmres_euler_f64.argtypes = [
            C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _i32p, _f64p,
            C.c_int64, C.c_double, _f64p, _f64p, C.c_int, C.c_int, C.c_double,
            C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int)]
        lib.ref_gmres_dense_f64.argtypes = [
            C.c_int, _f64p, _f64p, _f64p, C.c_void_p, C.c_int, C.c_int,
            C.c_double, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int)]
        lib.ref_connect_1d.argtypes = [C.c_int, C.POINTER(C.c_int),
                                       C.POINTER(C.c_int), C.c_void_p,
                                       C.c_void_p, C.c_void_p]
        lib.ref_pde_create.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        lib.ref_pde_create.restype = C.c_void_p
        lib.ref_pde_destroy.argtypes = [C.c_void_p]
        lib.ref_pde_destroy.restype = None
        lib.ref_pde_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 5 + [
            C.POINTER(C.c_int64)] * 3 + [C.POINTER(C.c_double)]
        lib.ref_pde_export.argtypes = [C.c_void_p, _i32p, _i32p, _i32p, _f64p,
                                       _i32p]
        lib.ref_pde_coefficients.argtypes = [C.c_void_p, C.c_int, C.c_int,
                                             C.c_void_p, C.POINTER(C.c_int)]
        lib.ref_pde_apply.argtypes = [C.c_void_p, C.c_double, _f64p,
                                      C.c_double, _f64p]
        lib.ref_pde_gmres_euler.argtypes = [
            C.c_void_p, C.c_double, _f64p, _f64p, C.c_int, C.c_int,
            C.c_double, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int)]
        _ref = lib
    return _ref


# ----------------------------------------------------------------- helpers

def kronmult(d, n, pntr, indx, terms, iA, vA, alpha, x, beta, y, lib=None):
    """y <- beta*y + alpha*K*x in place (oracle restatement by default)."""
    f32 = vA.dtype == np.float32
    rows = len(pntr) - 1
    if lib is None:
        fn = getattr(oracle(), "orc_kronmult_sparse_" + ("f32" if f32 else "f64"))
    else:
        fn = getattr(lib, "ref_cpu_sparse_" + ("f32" if f32 else "f64"))
    rc = fn(d, n, rows, pntr, indx, terms, iA, vA, alpha, x, beta, y)
    if rc != 0:
        raise RuntimeError(f"kronmult checker returned {rc}")
    return y


def connect_1d(level, lib=None):
    rows, conn = C.c_int(), C.c_int()
    if lib is None:
        f = oracle().orc_connect_1d
        f(level, C.byref(rows), C.byref(conn), None, None)
        pntr = np.zeros(rows.value + 1, np.int32)
        indx = np.zeros(conn.value, np.int32)
        f(level, C.byref(rows), C.byref(conn), pntr.ctypes.data, indx.ctypes.data)
    else:
        f = lib.ref_connect_1d
        f(level, C.byref(rows), C.byref(conn), None, None, None)
        pntr = np.zeros(rows.value + 1, np.int32)
        indx = np.zeros(conn.value, np.int32)
        f(level, C.byref(rows), C.byref(conn), pntr.ctypes.data,
          indx.ctypes.data, None)
    return pntr, indx


def sparse_grid(d, L):
    lib = oracle()
    cells = lib.orc_sparse_grid(d, L, None)
    table = np.zeros((cells, 2 * d), np.int32)
    lib.orc_sparse_grid(d, L, table.ctypes.data)
    return table


def build_pairs(d, L, table):
    lib = oracle()
    nnz = C.c_int64()
    table = np.ascontiguousarray(table, dtype=np.int32)
    cells = table.shape[0]
    lib.orc_build_pairs(d, L, cells, table.ravel(), C.byref(nnz), None, None, None)
    pntr = np.zeros(cells + 1, np.int32)
    indx = np.zeros(nnz.value, np.int32)
    conn = np.zeros((nnz.value, d), np.int32)
    lib.orc_build_pairs(d, L, cells, table.ravel(), C.byref(nnz),
                        pntr.ctypes.data, indx.ctypes.data, conn.ctypes.data)
    return pntr, indx, conn


def expand_iA(d, n, terms, conn):
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    nnz = conn.shape[0]
    iA = np.zeros(nnz * terms * d, np.int32)
    oracle().orc_expand_iA(d, n, terms, nnz, conn.ravel(), iA)
    return iA


def gmres_euler(d, n, pntr, indx, terms, iA, vA, dt, x, b, restart, max_outer,
                tol, lib=None):
    err, it = C.c_double(), C.c_int()
    rows = len(pntr) - 1
    if lib is None:
        rc = oracle().orc_gmres_euler(d, n, rows, pntr, indx, terms, iA, vA,
                                      dt, x, b, restart, max_outer, tol,
                                      C.byref(err), C.byref(it))
    else:
        rc = lib.ref_gmres_euler_f64(d, n, rows, terms, pntr, indx, iA, vA,
                                     len(vA), dt, x, b, restart, max_outer,
                                     tol, 1, C.byref(err), C.byref(it))
    if rc != 0:
        raise RuntimeError(f"gmres checker returned {rc}")
    return err.value, it.value


def imex_advance(d, n, explicit, implicit, dt, x, steps, restart, max_outer,
                 tol, hook=None):
    """The reference's two-stage IMEX step (imex_advance,
    src/time_advance.cpp:477-990) restated over the oracle's kronmult and
    GMRES, x (FP64 numpy) updated in place.  explicit / implicit: operators
    as (pntr, indx, terms, iA, vA) tuples; implicit None is the reference
    without a collision operator (f_1 = f_1s, the step ends with f_2s).
    hook(step, stage, event, f) runs where the reference updates PDE state:
    event 0 before each explicit apply (f: its input, the Poisson update at
    :572-640, called at :792 and :891), event 1 before each implicit solve
    (f: the stage's explicit result, calculate_moments +
    generate_all_coefficients at :829-840 and :930-938); it may change the vA
    arrays in place.  Returns
    the per-step (stage 1, stage 2) GMRES iteration counts."""
    def apply(op, v):
        pntr, indx, terms, iA, vA = op
        y = np.zeros_like(v)
        return kronmult(d, n, pntr, indx, terms, iA, vA, 1.0, v, 0.0, y)

    def solve(h, x0, b):
        pntr, indx, terms, iA, vA = implicit
        _, it = gmres_euler(d, n, pntr, indx, terms, iA, vA, h, x0, b, restart,
                            max_outer, tol)
        return it

    call = hook if hook is not None else (lambda *a: None)
    its = []
    for k in range(steps):
        f0 = x.copy()                         # f_orig (:524-529)
        call(k, 0, 0, x)
        x += dt * apply(explicit, x)          # f_1s = f_0 + dt A f_0 (:800-822)
        call(k, 0, 1, x)
        f1 = x.copy()                         # initial guess f_1s (:849)
        it1 = solve(dt, f1, x.copy()) if implicit is not None else 0
        f1_out = f1.copy()                    # f_1_output (:873)
        x[:] = f0                             # (:887)
        call(k, 1, 0, f1)
        f1 += dt * apply(explicit, f1)        # f_2 = f_1 + dt T(f_1) (:897-918)
        x += f1
        x *= 0.5                              # f_2s (:921-922)
        call(k, 1, 1, x)
        if implicit is not None:
            it2 = solve(0.5 * dt, f1_out, x.copy())   # from f_1_output (:945-970)
            x[:] = f1_out
        else:
            it2 = 0
        its.append((it1, it2))
    return its


def gmres_dense(A, x, b, restart, max_outer, tol, lib=None, M=None):
    """solver::simple_gmres on a dense A (oracle restatement, or the compiled
    reference with lib=ref()); M: the reference's dense preconditioner
    (LU-factored and applied on the left, src/solver.cpp:11-38, 55-74),
    reference only."""
    n = len(b)
    At = np.asfortranarray(A).ravel(order="F").copy()
    err, it = C.c_double(), C.c_int()
    if lib is None:
        if M is not None:
            raise ValueError("the oracle restatement takes no preconditioner")
        rc = oracle().orc_gmres_dense(n, At, x, b, restart, max_outer, tol,
                                      C.byref(err), C.byref(it))
    else:
        Mt = None if M is None else np.asfortranarray(M).ravel(order="F").copy()
        rc = lib.ref_gmres_dense_f64(n, At, x, b,
                                     None if Mt is None else Mt.ctypes.data,
                                     restart, max_outer, tol, 1, C.byref(err),
                                     C.byref(it))
    if rc != 0:
        raise RuntimeError(f"gmres checker returned {rc}")
    return err.value, it.value


def make_kronmult_data(d, n, rows, terms, mats, dtype=np.float64):
    """The reference tests' random kronmult data (minstd_rand(42))."""
    nb = rows * rows
    pntr = np.zeros(rows + 1, np.int32)
    indx = np.zeros(nb, np.int32)
    iA = np.zeros(nb * terms * d, np.int32)
    ts = n ** d
    vA = np.zeros(n * n * mats, dtype)
    x = np.zeros(ts * rows, dtype)
    y = np.zeros(ts * rows, dtype)
    oracle().orc_make_kronmult_data(d, n, rows, terms, mats,
                                    8 if dtype == np.float64 else 4, pntr,
                                    indx, iA, vA.ctypes.data, x.ctypes.data,
                                    y.ctypes.data)
    return dict(pntr=pntr, indx=indx, iA=iA, vA=vA, x=x, y=y)


def _term_pointers(terms):
    return (C.c_void_p * max(len(terms), 1))(*[t.ctypes.data for t in terms])


def kronmult_dense(d, n, rows, cols, terms, elem, row_offset, col_offset, nb,
                   alpha, x, beta, y, lib=None):
    """Dense form y <- beta*y + alpha*K*x in place (kronmult::cpu_dense):
    terms is a list of per-term coefficient arrays (d*nb^2*n^2 each), elem
    the cells' 1D indices (d per cell).  lib=ref() runs the reference's own
    kronmult_matrix (dense constructor) instead of the restatement."""
    f32 = x.dtype == np.float32
    dt = np.float32 if f32 else np.float64
    tv = [np.ascontiguousarray(t, dtype=dt) for t in terms]
    el = np.ascontiguousarray(elem, dtype=np.int32).ravel()
    if lib is None:
        fn = getattr(oracle(), "orc_kronmult_dense_" + ("f32" if f32 else "f64"))
        rc = fn(d, n, rows, cols, len(tv), el, row_offset, col_offset,
                _term_pointers(tv), nb, alpha, x, beta, y)
    else:
        fn = getattr(lib, "ref_dense_apply_" + ("f32" if f32 else "f64"))
        rc = fn(d, n, rows, cols, len(tv), np.concatenate(tv) if tv else
                np.zeros(1, dt), el, len(el), row_offset, col_offset, nb,
                alpha, x, beta, y)
    if rc != 0:
        raise RuntimeError(f"dense kronmult checker returned {rc}")
    return y


def ref_make_kronmult_welem(d, n, terms, index_range, dtype=np.float64,
                            want_ref=True):
    """The reference's own make_kronmult_welem (compiled from its sources):
    the same fields as make_kronmult_welem plus ref_y, its explicit
    Kronecker-product answer of y + K x (when want_ref)."""
    rows = index_range ** d
    ts = n ** d
    per = d * index_range * index_range * n * n
    elem = np.zeros(rows * d, np.int32)
    coeff = np.zeros(max(terms * per, 1), dtype)
    x = np.zeros(rows * ts, dtype)
    y = np.zeros(rows * ts, dtype)
    ref_y = np.zeros(rows * ts, dtype)
    fn = getattr(ref(), "ref_make_welem_" + ("f64" if dtype == np.float64 else "f32"))
    fn(d, n, terms, index_range, int(want_ref), elem, coeff, x, y, ref_y)
    return dict(rows=rows, elem=elem.reshape(rows, d),
                terms=[coeff[t * per:(t + 1) * per] for t in range(terms)],
                x=x, y=y, ref_y=ref_y)


def make_kronmult_welem(d, n, terms, index_range, dtype=np.float64):
    """The reference's dense-test data (kronmult_intputs_welem,
    minstd_rand(42)): elem, the list of per-term coefficient arrays, x, y."""
    rows = index_range ** d
    ts = n ** d
    per = d * index_range * index_range * n * n
    elem = np.zeros(rows * d, np.int32)
    coeff = np.zeros(terms * per, dtype)
    x = np.zeros(rows * ts, dtype)
    y = np.zeros(rows * ts, dtype)
    rc = oracle().orc_make_kronmult_welem(d, n, terms, index_range,
                                          8 if dtype == np.float64 else 4,
                                          elem, coeff.ctypes.data,
                                          x.ctypes.data, y.ctypes.data)
    if rc != 0:
        raise RuntimeError("make_kronmult_welem failed")
    return dict(rows=rows, elem=elem.reshape(rows, d),
                terms=[coeff[t * per:(t + 1) * per] for t in range(terms)],
                x=x, y=y)


class RefPDE:
    """A built-in reference PDE with its sparse kronmult matrix (reference builder)."""

    def __init__(self, name: str, level: int, degree: int, dims: int):
        self.lib = ref()
        levels = " ".join([str(level)] * dims)
        self.h = self.lib.ref_pde_create(name.encode(), levels.encode(), degree)
        if not self.h:
            raise RuntimeError(f"reference could not build pde {name}")
        d, n, rows, terms, L = (C.c_int() for _ in range(5))
        nnz, ia, va = (C.c_int64() for _ in range(3))
        dt = C.c_double()
        rc = self.lib.ref_pde_info(self.h, C.byref(d), C.byref(n), C.byref(rows),
                                   C.byref(terms), C.byref(L), C.byref(nnz),
                                   C.byref(ia), C.byref(va), C.byref(dt))
        if rc != 0:
            raise RuntimeError("reference matrix is split into several calls")
        self.d, self.n, self.rows, self.terms = d.value, n.value, rows.value, terms.value
        self.max_level, self.nnz, self.dt = L.value, nnz.value, dt.value
        self.pntr = np.zeros(self.rows + 1, np.int32)
        self.indx = np.zeros(self.nnz, np.int32)
        self.iA = np.zeros(ia.value, np.int32)
        self.vA = np.zeros(va.value, np.float64)
        self.table = np.zeros(self.rows * 2 * self.d, np.int32)
        self.lib.ref_pde_export(self.h, self.pntr, self.indx, self.iA, self.vA,
                                self.table)
        self.table = self.table.reshape(self.rows, 2 * self.d)

    def coefficients(self, term, dim):
        lda = C.c_int()
        self.lib.ref_pde_coefficients(self.h, term, dim, None, C.byref(lda))
        out = np.zeros(lda.value * lda.value, np.float64)
        self.lib.ref_pde_coefficients(self.h, term, dim, out.ctypes.data,
                                      C.byref(lda))
        return out.reshape(lda.value, lda.value, order="F")

    def apply(self, alpha, x, beta, y):
        self.lib.ref_pde_apply(self.h, alpha, x, beta, y)
        return y

    def gmres_euler(self, dt, x, b, restart, max_outer, tol):
        err, it = C.c_double(), C.c_int()
        self.lib.ref_pde_gmres_euler(self.h, dt, x, b, restart, max_outer, tol,
                                     1, C.byref(err), C.byref(it))
        return err.value, it.value

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_pde_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------- Jacobi
# numpy restatements (small sizes only) of the diagonal preconditioner data


def _self_pair(pntr, indx, row):
    b, e = int(pntr[row]), int(pntr[row + 1])
    hit = np.nonzero(np.asarray(indx[b:e]) == row)[0]
    return b + int(hit[0]) if len(hit) else -1


def point_jacobi_diag(d, n, pntr, indx, terms, iA, vA):
    """pc_i = sum_t prod_k A_{t,k}(i_k, i_k) over each cell's own pair:
    build_preconditioner (src/asgard_kronmult_matrix.cpp:1015-1067, the loop
    at :1046-1063), with the factors addressed by the local-mode iA of the
    cell's diagonal pair instead of the global 1D coefficient matrices."""
    rows = len(pntr) - 1
    ts = n ** d
    pc = np.zeros(rows * ts)
    for r in range(rows):
        p = _self_pair(pntr, indx, r)
        if p < 0:
            continue
        for i in range(ts):
            s = 0.0
            for t in range(terms):
                a, ii = 1.0, i
                for k in range(d - 1, -1, -1):
                    ik = ii % n
                    ii //= n
                    a *= vA[iA[(p * terms + t) * d + k] + ik + ik * n]
                s += a
            pc[r * ts + i] = s
    return pc


def diagonal_blocks(d, n, pntr, indx, terms, iA, vA):
    """K_cc = sum_t (x)_k A_{t,k} over each cell's own pair (dimension 0
    slowest, column-major factors), rows x ts x ts."""
    rows = len(pntr) - 1
    ts = n ** d
    out = np.zeros((rows, ts, ts))
    for r in range(rows):
        p = _self_pair(pntr, indx, r)
        if p < 0:
            continue
        for t in range(terms):
            m = np.ones((1, 1))
            for k in range(d):
                off = int(iA[(p * terms + t) * d + k])
                A = np.asarray(vA[off:off + n * n]).reshape(n, n).T  # A(i, j)
                m = np.kron(m, A)
            out[r] += m
    return out


# ---------------------------------------------------------------- line Jacobi
# The definition of this library's line preconditioner (ASGK_JACOBI_LINE;
# no counterpart in the reference), stated with dense algebra at small sizes
# so that it checks the device's eigendecomposition-based apply
# independently.  Operators are sparse-grid operators in the global form
# (every term acts in one dimension or is the identity), factors in the
# per-1D-connection layout [conn][term][dim][n*n] of connect_1d(level).

def _global_1d_operators(d, level, terms, vA, n=3):
    """Per dimension the full 1D operator (n*2^level square) summed over the
    terms acting in that dimension, and the number of identity terms."""
    pntr, indx = connect_1d(level)
    R = len(pntr) - 1
    rows1 = np.repeat(np.arange(R), np.diff(pntr))
    blocks = np.asarray(vA, dtype=np.float64).reshape(len(indx), terms, d, n, n)
    blocks = blocks.transpose(0, 1, 2, 4, 3)  # [..., row i, col j]
    eye = np.eye(n)
    F = [np.zeros((n * R, n * R)) for _ in range(d)]
    n_id = 0
    for t in range(terms):
        act = []
        for k in range(d):
            b = blocks[:, t, k]
            ident = all(np.array_equal(b[j], eye if rows1[j] == indx[j] else 0 * eye)
                        for j in range(len(indx)))
            if not ident:
                act.append(k)
        if not act:
            n_id += 1
            continue
        if len(act) > 1:
            raise ValueError("terms acting in several dimensions are not supported")
        k = act[0]
        for j in range(len(indx)):
            r, c = rows1[j], indx[j]
            F[k][n * r:n * r + n, n * c:n * c + n] += blocks[j, t, k]
    return F, n_id


def line_dimensions(d, level, terms, vA, n=3):
    """Dimensions with a nonzero symmetric 1D operator: the ones the line
    preconditioner solves along (increasing order)."""
    F, _ = _global_1d_operators(d, level, terms, vA, n)
    out = []
    for k in range(d):
        s = np.abs(F[k]).max()
        if s > 0 and np.abs(F[k] - F[k].T).max() <= 1e-12 * s:
            out.append(k)
    return out


def line_jacobi_apply(d, level, table, terms, vA, dt, v, n=3):
    """z = M_{k_m}^-1 B ... B M_{k_2}^-1 B M_{k_1}^-1 v over the line
    dimensions k_1 < ... < k_m, with (s = 1 - dt * identity terms)
      M_k = s I - dt (K_k + sum_{j line, j != k} D_j),   B = s I - dt sum_{j line} D_j,
    K_k the operator of the terms acting in dimension k (block diagonal over
    the pencils of cells that agree outside k) and D_j its cell-diagonal
    part.  Each pencil system of M_k is assembled densely and solved."""
    F, n_id = _global_1d_operators(d, level, terms, vA, n)
    line = line_dimensions(d, level, terms, vA, n)
    if not line:
        raise ValueError("no dimension with a symmetric operator")
    s = 1.0 - dt * n_id
    table = np.asarray(table)
    lev, pos = table[:, :d].astype(np.int64), table[:, d:].astype(np.int64)
    c1 = np.where(lev == 0, 0, (1 << np.maximum(lev - 1, 0)) + pos)
    cells = table.shape[0]
    z = np.asarray(v, dtype=np.float64).reshape((cells,) + (n,) * d).copy()

    def selfblock(j, c):
        return F[j][n * c:n * c + n, n * c:n * c + n]

    def along(M, x, axis):
        return np.moveaxis(np.tensordot(M, x, axes=([1], [axis])), 0, axis)

    def bj(z):
        out = s * z
        for cell in range(cells):
            for j in line:
                out[cell] -= dt * along(selfblock(j, c1[cell, j]), z[cell], j)
        return out

    def solve_k(z, k):
        out = np.empty_like(z)
        others = [j for j in range(d) if j != k]
        keys = {}
        for cell in range(cells):
            keys.setdefault(tuple(c1[cell, others]), []).append(cell)
        rest = n ** (d - 1)
        for key, mem in keys.items():
            mem = sorted(mem, key=lambda c: c1[c, k])
            idx = np.concatenate([np.arange(n * c1[c, k], n * c1[c, k] + n) for c in mem])
            AP = F[k][np.ix_(idx, idx)]
            # the other line dimensions' self blocks, on the rest axes
            # (dimensions != k in increasing order, the first slowest)
            S = np.zeros((rest, rest))
            for j in line:
                if j == k:
                    continue
                m = np.ones((1, 1))
                for jj in others:
                    m = np.kron(m, selfblock(j, key[others.index(jj)]) if jj == j else np.eye(n))
                S += m
            M = s * np.eye(len(idx) * rest) - dt * (np.kron(AP, np.eye(rest)) +
                                                    np.kron(np.eye(len(idx)), S))
            # gather: rows (member, poly_k), columns the rest axes
            X = np.stack([np.moveaxis(z[c], k, 0).reshape(n, rest) for c in mem])
            U = np.linalg.solve(M, X.reshape(-1)).reshape(len(mem), n, rest)
            for i, c in enumerate(mem):
                out[c] = np.moveaxis(U[i].reshape((n,) + (n,) * (d - 1)), 0, k)
        return out

    for i, k in enumerate(line):
        if i > 0:
            z = bj(z)
        z = solve_k(z, k)
    return z.reshape(-1)
