"""The C++ drop-in header, compiled and run as reference code would use it
(tests/cpp/dropin_main.cpp), checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT, rel_err, rmse_close

pytestmark = pytest.mark.gpu


def compile_dropin(exe):
    libdir = os.path.join(ROOT, "asgard_b200")
    cuda = "/usr/local/cuda"
    cmd = ["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp"),
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"),
           "-L", libdir, "-lasgard_b200", "-L", os.path.join(cuda, "lib64"),
           "-lcudart", f"-Wl,-rpath,{libdir}", f"-Wl,-rpath,{cuda}/lib64",
           "-o", str(exe)]
    return subprocess.run(cmd, capture_output=True, text=True)


def _read(path):
    out = []
    with open(path, "rb") as f:
        data = f.read()
    o = 0
    for dt in [np.int32] * 3 + [np.float64] * 10:
        n = int(np.frombuffer(data, np.int64, 1, o)[0])
        o += 8
        out.append(np.frombuffer(data, dt, n, o).copy())
        o += n * np.dtype(dt).itemsize
    return out


def test_cpp_dropin_header(cuda, tmp_path):
    exe = tmp_path / "dropin"
    r = compile_dropin(exe)
    assert r.returncode == 0, r.stderr
    out = tmp_path / "out.bin"
    subprocess.run([str(exe), str(out)], check=True)
    pntr, col, iA, vA, x, y0, y_host, y_dev, b, sol, x3, x3p, meta = _read(out)
    d, n, T = int(meta[0]), int(meta[1]), int(meta[2])
    expect = oracle.kronmult(d, n, pntr, col, T, iA, vA, 0.5, x, -2.0, y0.copy())
    assert rel_err(y_host, expect) < 1e-13
    assert rel_err(y_dev, expect) < 1e-13
    # implicit step: the oracle's GMRES on the same system
    xo = np.zeros_like(b)
    _, its_o = oracle.gmres_euler(d, n, pntr, col, T, iA, vA, 1e-2, xo, b,
                                  20, 50, 1e-12)
    assert meta[4] <= 1e-12
    assert abs(int(meta[5]) - its_o) <= 1
    assert rel_err(sol, xo) < 1e-10
    assert meta[6] == 1.0                         # std::invalid_argument thrown
    gold = [4.715561567725287e-02, 1.257695999382253e-01, 1.625351700791827e-02]
    assert rmse_close(x3, gold, 10 * np.finfo(np.float64).eps)
    # flops(): reference convention (multiply-add once), compute_flops() x2
    assert meta[10] == 2 * meta[9]
    # global form: equal to the pair form for terms acting in every
    # dimension (chains of masked 1D passes) and for single-direction ones
    assert meta[11] < 1e-13
    assert meta[12] < 1e-13
    # num_batch() is rows*cols for every matrix, as in the reference
    cells = int(meta[3])
    assert meta[13] == cells * cells and meta[14] == 0.0
    # dense form of the same operator: is_dense, rows*cols products, the
    # reference's flops_ (n^d * n * rows * cols * T * d), the sparse result,
    # and update_stored_coefficients with per-term arrays
    assert meta[15] == 1.0 and meta[16] == cells * cells
    assert meta[17] == n ** d * n * cells * cells * T * d
    assert meta[18] < 1e-13
    assert meta[19] < 1e-13
    # multi-call forms (CSR row blocks, GPU pair chunks): the same operator
    assert meta[20] < 1e-13 and meta[21] < 1e-13
    assert meta[22] == len(col)
    # set_workspace: host applies stage x in the caller's device buffer
    assert meta[23] < 1e-13 and meta[24] == 1.0
    # the preconditioned overload (point Jacobi, right-preconditioned): the
    # same solution to the tolerance the criterion allows
    assert meta[25] < 1e-8 and meta[26] >= 1 and meta[27] <= 1e-12
    # simple_gmres with the reference's dense preconditioner: the preconditioned
    # 3x3 known answer, the reference's iteration count (4)
    eps = np.finfo(np.float64).eps
    assert rmse_close(x3p, gold, 10 * eps) and meta[28] < eps and meta[29] == 4
    # a Jacobi preconditioner built for another dt: std::invalid_argument
    assert meta[30] == 1.0
    # kronmult_matrix<float>: FP32 applies on host and device vectors and
    # the FP32 implicit step agree with the FP64 results to FP32 accuracy
    assert meta[31] < 1e-6 and meta[32] < 1e-6
    assert meta[33] < 1e-5 and meta[34] >= 1
