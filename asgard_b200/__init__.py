"""asgard_b200: B200 (sm_100a) kronmult operator apply and implicit GMRES.

The compute path is the in-tree CUDA library ``libasgard_b200.so`` (C ABI in
``include/asgard_b200.h``); this package mirrors the reference's
``kronmult_matrix`` / ``simple_gmres_euler`` interfaces over it.  Importing
fails if the library is missing -- there is no CPU fallback.
"""
from ._lib import AsgkError, lib  # noqa: F401  (loads the CUDA library)
from .kronmult import (BF16, FP32, FP64, IMEX_BEFORE_EXPLICIT, IMEX_BEFORE_IMPLICIT,
                       cgs_step, default_gmres_restarts, gmres_info,
                       gmres_settings, imex_advance, implicit_advance, kronmult_matrix,
                       launch_count, simple_gmres, simple_gmres_euler)
from .operators import (SparseGridOperator, build_pairs, connect_1d,
                        expand_iA, factor_values, sparse_grid)
from .precond import JacobiPreconditioner, LearnedPreconditioner

__all__ = [
    "kronmult_matrix", "simple_gmres_euler", "simple_gmres", "gmres_info", "cgs_step",
    "implicit_advance", "imex_advance", "gmres_settings",
    "default_gmres_restarts", "launch_count", "SparseGridOperator",
    "sparse_grid", "connect_1d", "build_pairs", "expand_iA", "factor_values",
    "FP64", "FP32", "BF16", "IMEX_BEFORE_EXPLICIT", "IMEX_BEFORE_IMPLICIT",
    "AsgkError", "LearnedPreconditioner",
    "JacobiPreconditioner",
]
