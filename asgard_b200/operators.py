"""Sparse-grid operator structure and the synthetic operators of the benchmarks.

The structure (element table, 1D connectivity, connected cell pairs) comes
from the library's host builder (``asgk_sparse_grid``, ``asgk_connect_1d``,
``asgk_build_pairs``), which follows the reference's element table and
``make_kronmult_sparse`` exactly.  Factor values (``vA``) follow the
reference layout: per 1D connection a block of ``d*T`` column-major n x n
factors, factor (t, k) of a pair at ``conn_k*(d*T*n*n) + (t*d + k)*n*n``
(src/asgard_kronmult_matrix.cpp:369-393, 455-461).

Synthetic operators (seeded; no PDE setup involved):

* ``kind="random"``: every factor block uniform in [-1, 1].
* ``kind="advdiff"``: term t acts in dimension ``t % d``; even terms use the
  1D DG advection block of the reference's continuity_1 (term 0), odd terms
  ``nu`` times the 1D LDG diffusion block of the reference's diffusion_1
  (term 0), both at degree 3 (n = 3) on the hierarchical level-7 mesh; every
  other dimension of a term carries the identity (mass) block.  The blocks
  are read from ``data/ops1d_L7.npz`` (generated from the reference by
  ``tests/golden/make_golden.py``); a level L <= 7 operator uses the blocks
  of the cells that exist at level L.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import check, lib

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def sparse_grid(d: int, level: int) -> np.ndarray:
    """Element table: (cells, 2d) int32, levels then positions."""
    cells = lib.asgk_sparse_grid(d, level, None)
    if cells < 0:
        raise ValueError("unsupported sparse grid")
    table = np.zeros((cells, 2 * d), np.int32)
    lib.asgk_sparse_grid(d, level, table.ctypes.data)
    return table


def connect_1d(level: int):
    rows, conn = C.c_int(), C.c_int()
    check(lib.asgk_connect_1d(level, C.byref(rows), C.byref(conn), None, None))
    pntr = np.zeros(rows.value + 1, np.int32)
    indx = np.zeros(conn.value, np.int32)
    check(lib.asgk_connect_1d(level, C.byref(rows), C.byref(conn),
                              pntr.ctypes.data, indx.ctypes.data))
    return pntr, indx


def build_pairs(d: int, level: int, table: np.ndarray):
    """Connected cell pairs: row_ptr (int64), col (int32), conn (nnz, d)."""
    table = np.ascontiguousarray(table, dtype=np.int32)
    cells = table.shape[0]
    nnz = C.c_int64()
    check(lib.asgk_build_pairs(d, level, cells, table.ctypes.data,
                               C.byref(nnz), None, None, None), "build_pairs")
    row_ptr = np.zeros(cells + 1, np.int64)
    col = np.zeros(nnz.value, np.int32)
    conn = np.zeros((nnz.value, d), np.int32)
    check(lib.asgk_build_pairs(d, level, cells, table.ctypes.data,
                               C.byref(nnz), row_ptr.ctypes.data,
                               col.ctypes.data, conn.ctypes.data),
          "build_pairs")
    return row_ptr, col, conn


def expand_iA(conn: np.ndarray, d: int, n: int, terms: int) -> np.ndarray:
    """Reference iA (pair-major, then term, then dimension) from conn."""
    nnz = conn.shape[0]
    blk = d * terms * n * n
    tk = (np.arange(terms)[:, None] * d + np.arange(d)[None, :]) * n * n
    iA = conn[:, None, :].astype(np.int64) * blk + tk[None, :, :]
    return iA.reshape(nnz * terms * d).astype(np.int32)


_OPS = None


def ops1d():
    global _OPS
    if _OPS is None:
        z = np.load(os.path.join(DATA, "ops1d_L7.npz"))
        _OPS = {k: z[k] for k in z.files}
    return _OPS


def factor_values(d: int, level: int, terms: int, kind: str = "advdiff",
                  nu: float = 0.1, seed: int = 0, n: int = 3) -> np.ndarray:
    """vA for every 1D connection at this level (layout in module docstring)."""
    pntr, indx = connect_1d(level)
    nconn = len(indx)
    nn = n * n
    if kind == "random":
        rng = np.random.default_rng(seed)
        return rng.uniform(-1.0, 1.0, nconn * d * terms * nn)
    if kind != "advdiff":
        raise ValueError(kind)
    if n != 3 or level > 7:
        raise ValueError("advdiff factors exist for n = 3 and level <= 7")
    ops = ops1d()
    p7, i7 = ops["pntr"], ops["indx"]
    rows = np.repeat(np.arange(len(pntr) - 1), np.diff(pntr))
    # position of connection (r, c) in the level-7 connectivity
    pos7 = np.empty(nconn, np.int64)
    for j in range(nconn):
        r, c = rows[j], indx[j]
        seg = i7[p7[r]:p7[r + 1]]
        pos7[j] = p7[r] + int(np.searchsorted(seg, c))
    adv = ops["adv"][pos7]
    dif = ops["dif"][pos7] * nu
    eye = np.where((rows == indx)[:, None], np.eye(n).ravel(order="F")[None, :], 0.0)
    vA = np.zeros((nconn, terms, d, nn))
    for t in range(terms):
        for k in range(d):
            if k == t % d:
                vA[:, t, k] = adv if t % 2 == 0 else dif
            else:
                vA[:, t, k] = eye
    return vA.reshape(-1)


def transpose_factor_values(vA: np.ndarray, d: int, level: int, terms: int,
                            n: int = 3) -> np.ndarray:
    """Factor values of the transposed operator K^T on the same pair list.

    The connected-pair set is symmetric, so K^T has the same CSR structure;
    its pair (c, r) needs (A_{t,k} at the 1D connection (r_k, c_k))^T.  With
    factors addressed by the pair's own connection (c_k, r_k), block j of the
    result is the transposed block of the mirror connection of j."""
    pntr, indx = connect_1d(level)
    rows = np.repeat(np.arange(len(pntr) - 1), np.diff(pntr))
    R = len(pntr) - 1
    lut = np.full((R, R), -1, np.int64)
    lut[rows, indx] = np.arange(len(indx))
    mirror = lut[indx, rows]
    if (mirror < 0).any():
        raise ValueError("1D connectivity is not symmetric")
    blocks = vA.reshape(len(indx), terms, d, n, n)     # [..., col j, row i]
    return np.ascontiguousarray(blocks[mirror].transpose(0, 1, 2, 4, 3)).reshape(-1)


class SparseGridOperator:
    """Structure + values of a synthetic sparse-grid operator."""

    def __init__(self, d: int, level: int, terms: int, kind: str = "advdiff",
                 nu: float = 0.1, seed: int = 0, n: int = 3):
        self.d, self.level, self.terms, self.n = d, level, terms, n
        self.kind, self.nu, self.seed = kind, nu, seed
        self.table = sparse_grid(d, level)
        self.row_ptr, self.col, self.conn = build_pairs(d, level, self.table)
        self.vA = factor_values(d, level, terms, kind, nu, seed, n)
        self.rows = self.table.shape[0]
        self.tensor = n ** d
        self.N = self.rows * self.tensor
        self.nnz = len(self.col)

    def iA(self) -> np.ndarray:
        return expand_iA(self.conn, self.d, self.n, self.terms)

    def elem(self) -> np.ndarray:
        """1D cell index of every cell in every dimension (cells x d): 0 at
        level 0, else 2^(level-1) + position (the dense form's elem,
        src/asgard_kronmult_matrix.cpp:116-131)."""
        lev = self.table[:, :self.d].astype(np.int64)
        pos = self.table[:, self.d:].astype(np.int64)
        idx = np.where(lev == 0, 0, (1 << np.maximum(lev - 1, 0)) + pos)
        return np.ascontiguousarray(idx, dtype=np.int32)

    def dense_terms(self):
        """The factors as the dense form holds them: per term, per dimension
        the full 1D operator cut into 2^level x 2^level blocks of n x n,
        ordered by column cell then row cell, zero where two 1D cells are not
        connected (make_kronmult_dense, src/asgard_kronmult_matrix.cpp:95-113)."""
        pntr, indx = connect_1d(self.level)
        nb, d, T, nn = len(pntr) - 1, self.d, self.terms, self.n * self.n
        rows = np.repeat(np.arange(nb), np.diff(pntr))
        blocks = self.vA.reshape(len(indx), T, d, nn)
        out = []
        for t in range(T):
            a = np.zeros((d, nb * nb, nn))
            a[:, indx * nb + rows, :] = blocks[:, t].transpose(1, 0, 2)
            out.append(a.reshape(-1))
        return out, nb

    def kronmult_matrix(self, expanded: bool = False, mode: str = "pairs"):
        """mode "pairs": the connected-pair kronmult (expanded: the
        reference's iA offsets instead of connection indices); "global": the
        global Kronecker form (one pass per term acting in one dimension,
        upper/lower chains for terms acting in several); "dense":
        the reference's dense form (every cell pair, full 1D operators)."""
        from .kronmult import kronmult_matrix
        if mode == "global":
            return kronmult_matrix.from_global(self.d, self.n, self.level,
                                               self.table, self.terms, self.vA)
        if mode == "dense":
            terms, nb = self.dense_terms()
            return kronmult_matrix.from_dense(self.d, self.n, self.rows,
                                              self.rows, self.terms, terms,
                                              self.elem(), 0, 0, nb)
        if mode != "pairs":
            raise ValueError(mode)
        if expanded:
            return kronmult_matrix.from_csr(self.d, self.n, self.rows,
                                            self.rows, self.terms,
                                            self.row_ptr, self.col,
                                            self.iA(), self.vA)
        return kronmult_matrix.from_conn(self.d, self.n, self.rows, self.rows,
                                         self.terms, self.row_ptr, self.col,
                                         self.conn, self.vA)

    def kronmult_matrix_transposed(self):
        """K^T as a plan (same pair list, transposed mirror factors)."""
        from .kronmult import kronmult_matrix
        vT = transpose_factor_values(self.vA, self.d, self.level, self.terms,
                                     self.n)
        return kronmult_matrix.from_conn(self.d, self.n, self.rows, self.rows,
                                         self.terms, self.row_ptr, self.col,
                                         self.conn, vT)

    def flops(self) -> int:
        return 2 * self.d * self.terms * self.n ** (self.d + 1) * self.nnz
