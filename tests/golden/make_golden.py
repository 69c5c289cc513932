"""Regenerates the golden fixtures in this folder from the reference itself.

Run from the repository root, with the reference tree available and the
reference oracle built (``make -C oracle ref``):

    python tests/golden/make_golden.py [kron dense ops1d pde gmres]

Every fixture is produced by reference code compiled from the reference's own
sources (``oracle/_ref/libasgard_ref.so``), so the tests can pin the C
restatement (``oracle/asgard_oracle.c``) and the CUDA path on machines where
the reference tree is absent.

Fixtures:
  ../../asgard_b200/data/ops1d_L7.npz
                      1D operator blocks of the reference's continuity_1
                      (term 0, DG advection) and diffusion_1 (term 0, LDG
                      diffusion) at level 7, degree 3 (n = 3), one 3x3
                      column-major block per connect_1d connection (the
                      factors of the synthetic advection/diffusion
                      operators; stored with the package, which needs them).
  kronmult_data.npz   make_kronmult_data answers (explicit Kronecker products,
                      src/asgard_kronmult_tests.hpp) for the reference test
                      shapes of src/asgard_kronmult_matrix_tests.cpp.
  dense_data.npz      make_kronmult_welem answers of the dense tests
                      (src/asgard_kronmult_matrix_tests.cpp:118-176, 197-305)
                      for the shapes whose element table stays inside the
                      coefficient arrays: the explicit Kronecker answer and
                      the reference kronmult_matrix (dense, cpu_dense) answer,
                      plus one non-square case with row/column offsets.
  pde_*.npz           sparse kronmult matrices made by make_kronmult_sparse
                      for built-in PDEs, with an apply and a GMRES solve.
  gmres_3x3.json      the known-answer systems of src/solver_tests.cpp:141-213.
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# reference test shapes (d, n, rows, terms, matrices) with small answers
KRON_SHAPES = [
    (1, 2, 10, 2, 7), (1, 3, 11, 2, 7), (1, 6, 11, 2, 7),
    (2, 1, 12, 3, 7), (2, 2, 12, 3, 7), (2, 3, 12, 3, 7), (2, 5, 12, 3, 7),
    (2, 8, 13, 2, 7), (2, 17, 13, 2, 7), (2, 32, 13, 2, 7),
    (3, 2, 12, 2, 7), (3, 3, 17, 3, 7), (3, 5, 12, 2, 7),
    (4, 2, 9, 2, 7), (4, 3, 10, 3, 7), (4, 5, 9, 2, 7),
    (5, 2, 8, 2, 7), (5, 3, 10, 2, 7), (5, 4, 8, 2, 7),
    (6, 1, 6, 2, 7), (6, 2, 6, 2, 7), (6, 3, 8, 2, 7), (6, 4, 6, 2, 7),
]


# dense-test shapes (d, n, terms, index_range) of the reference whose
# element table stays inside the coefficient arrays: make_kronmult_welem
# writes the cells' 1D indices as base-d digits, so for (4, n, 2, 3) and
# (6, n, 2, 2) they reach index_range and the reference test reads past the
# blocks of each dimension (those shapes have no defined answer)
DENSE_SHAPES = ([(1, 2, 1, 1), (1, 2, 1, 5), (1, 2, 2, 5), (1, 2, 2, 7)]
                + [(1, n, 3, 7) for n in range(1, 7)]
                + [(2, n, 3, 5) for n in range(1, 6)]
                + [(3, n, 3, 3) for n in range(1, 6)]
                + [(5, n, 2, 1) for n in range(1, 6)]
                + [(6, 4, 2, 1)])
# non-square with offsets: cells [5, 15) against cells [9, 21) of a d = 2,
# n = 3, index_range 5 table (25 cells), alpha 0.7, beta -1.3
DENSE_OFFSET = dict(d=2, n=3, terms=2, index_range=5, rows=10, cols=12,
                    row_offset=5, col_offset=9, alpha=0.7, beta=-1.3)


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def kron_data():
    R = oracle.ref()
    out = {}
    for (d, n, rows, terms, mats) in KRON_SHAPES:
        for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
            nb = rows * rows
            ts = n ** d
            pntr = np.zeros(rows + 1, np.int32)
            indx = np.zeros(nb, np.int32)
            iA = np.zeros(nb * terms * d, np.int32)
            vA = np.zeros(n * n * mats, dt)
            x = np.zeros(ts * rows, dt)
            y = np.zeros(ts * rows, dt)
            ref_y = np.zeros(ts * rows, dt)
            getattr(R, "ref_make_kronmult_data_" + tag)(
                d, n, rows, terms, mats, pntr, indx, iA, vA, x, y, ref_y)
            key = f"{tag}_{d}_{n}_{rows}_{terms}_{mats}"
            out[key + "_ref_y"] = ref_y
            out[key + "_inputs_sha256"] = np.frombuffer(
                digest(iA, vA, x, y).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(OUT, "kronmult_data.npz"), **out)


def dense_data():
    R = oracle.ref()
    out = {}
    for (d, n, terms, rg) in DENSE_SHAPES:
        for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
            a = oracle.ref_make_kronmult_welem(d, n, terms, rg, dt)
            y = a["y"].copy()
            oracle.kronmult_dense(d, n, a["rows"], a["rows"], a["terms"],
                                  a["elem"], 0, 0, rg, dt(1.0), a["x"],
                                  dt(1.0), y, lib=R)
            key = f"{tag}_{d}_{n}_{terms}_{rg}"
            out[key + "_ref_y"] = a["ref_y"]
            out[key + "_cpu_dense_y"] = y
            out[key + "_inputs_sha256"] = np.frombuffer(
                digest(a["elem"], *a["terms"], a["x"], a["y"]).encode(),
                dtype=np.uint8)
    c = DENSE_OFFSET
    a = oracle.ref_make_kronmult_welem(c["d"], c["n"], c["terms"],
                                       c["index_range"], np.float64,
                                       want_ref=False)
    ts = c["n"] ** c["d"]
    x = a["x"][c["col_offset"] * ts:(c["col_offset"] + c["cols"]) * ts].copy()
    y = a["y"][c["row_offset"] * ts:(c["row_offset"] + c["rows"]) * ts].copy()
    oracle.kronmult_dense(c["d"], c["n"], c["rows"], c["cols"], a["terms"],
                          a["elem"], c["row_offset"], c["col_offset"],
                          c["index_range"], c["alpha"], x, c["beta"], y, lib=R)
    out["offset_y"] = y
    np.savez_compressed(os.path.join(OUT, "dense_data.npz"), **out)


def ops1d():
    L = 7
    adv = oracle.RefPDE("continuity_1", L, 3, 1).coefficients(0, 0)
    dif = oracle.RefPDE("diffusion_1", L, 3, 1).coefficients(0, 0)
    pntr, indx = oracle.connect_1d(L, lib=oracle.ref())
    n = 3
    blocks = {}
    for name, M in (("adv", adv), ("dif", dif)):
        b = np.zeros((len(indx), n * n))
        for r in range(len(pntr) - 1):
            for j in range(pntr[r], pntr[r + 1]):
                c = indx[j]
                b[j] = M[n * r:n * r + n, n * c:n * c + n].ravel(order="F")
        blocks[name] = b
    np.savez_compressed(os.path.join(ROOT, "asgard_b200", "data", "ops1d_L7.npz"), pntr=pntr,
                        indx=indx, adv=blocks["adv"], dif=blocks["dif"])


def pde_cases():
    for name, L, dims in (("continuity_2", 4, 2), ("continuity_3", 3, 3),
                          ("continuity_6", 2, 6), ("diffusion_2", 3, 2)):
        P = oracle.RefPDE(name, L, 3, dims)
        N = P.rows * P.n ** P.d
        rng = np.random.default_rng(7)
        x = rng.uniform(-1, 1, N)
        y0 = rng.uniform(-1, 1, N)
        y = P.apply(1.0, x, 0.0, np.zeros(N))
        y2 = P.apply(-0.5, x, 2.0, y0.copy())
        b = rng.uniform(-1, 1, N)
        sol = np.zeros(N)
        dt = P.dt
        err, its = P.gmres_euler(dt, sol, b, 20, 50, 1e-12)
        # x, y0 and b are regenerated by the tests from the same seeded
        # generator (numpy PCG64, seed 7, drawn in this order)
        np.savez_compressed(
            os.path.join(OUT, f"pde_{name}_L{L}.npz"), d=P.d, n=P.n,
            terms=P.terms, level=P.max_level, pntr=P.pntr, indx=P.indx,
            iA=P.iA, vA=P.vA, table=P.table, y=y, y_ab=y2, dt=dt,
            gmres_x=sol, gmres_err=err, gmres_iters=its)


def gmres_3x3():
    # values of src/solver_tests.cpp:143-161 (row-major A)
    case = dict(
        A=[[3.383861628748717e+00, 1.113343240310116e-02, 2.920740795411032e+00],
           [3.210305545769361e+00, 3.412141162288144e+00, 3.934494120167269e+00],
           [1.723479266939425e+00, 1.710451084172946e+00, 4.450671104482062e+00]],
        b1=[2.084406360034887e-01, 6.444769305362776e-01, 3.687335330031937e-01],
        x1=[4.715561567725287e-02, 1.257695999382253e-01, 1.625351700791827e-02],
        b2=[9.789303188021963e-01, 8.085725142873675e-01, 7.370498473207234e-01],
        x2=[1.812300946484165e-01, -7.824949213916167e-02, 1.254969087137521e-01])
    # the point-Jacobi preconditioner of the preconditioned cases (:149-151)
    case["M"] = [[3.383861628748717e+00, 0.0, 0.0],
                 [0.0, 3.412141162288144e+00, 0.0],
                 [0.0, 0.0, 4.450671104482062e+00]]
    A = np.array(case["A"])
    R = oracle.ref()
    for k in ("1", "2"):
        for tag, M in (("", None), ("pre_", np.array(case["M"]))):
            x = np.zeros(3)
            err, its = oracle.gmres_dense(A, x, np.array(case["b" + k]), 3, 3,
                                          np.finfo(np.float64).eps, lib=R, M=M)
            case[f"ref_{tag}x" + k] = x.tolist()
            case[f"ref_{tag}err" + k] = err
            case[f"ref_{tag}iters" + k] = its
    with open(os.path.join(OUT, "gmres_3x3.json"), "w") as f:
        json.dump(case, f, indent=1)


if __name__ == "__main__":
    # optional names restrict the run: kron dense ops1d pde gmres
    parts = {"kron": kron_data, "dense": dense_data, "ops1d": ops1d,
             "pde": pde_cases, "gmres": gmres_3x3}
    oracle.ref()
    for name in (sys.argv[1:] or list(parts)):
        parts[name]()
    for f in sorted(os.listdir(OUT)):
        print(f, os.path.getsize(os.path.join(OUT, f)))
