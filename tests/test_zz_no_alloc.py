"""asgk_cgs_step_noalloc: the Gram-Schmidt step for callers that must not
allocate device memory while they solve (their device memory belongs to their
own pool, or they cannot take the device-wide synchronisation of
cudaMalloc/cudaFree).  Called through the C ABI and checked against
asgk_cgs_step, which allocates its scratch, on two calls in a row (the second
reuses the fixed scratch the first left behind).  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13  # the FP64 parity tolerance of the other GPU tests


def _call(fn, V, k, w, h):
    import asgard_b200 as ab
    import torch
    nrm = C.c_double()
    rc = fn(C.c_void_p(V.data_ptr()), V.stride(0), k, C.c_void_p(w.data_ptr()),
            w.numel(), C.c_void_p(h.data_ptr()), C.byref(nrm),
            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc, nrm.value


def _rel(a, b):
    import torch
    return (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()


def test_cgs_step_noalloc_matches_allocating_entry_point(cuda):
    import asgard_b200 as ab
    import torch
    lib = ab.lib
    g = torch.Generator(device="cuda").manual_seed(123)
    for n, k in ((327888, 17), (50001, 51)):  # two calls in a row
        V = torch.rand(k, n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        w0 = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        w_ref, w_na = w0.clone(), w0.clone()
        h_ref = torch.empty(k, dtype=torch.float64, device="cuda")
        h_na = torch.full((k,), float("nan"), dtype=torch.float64, device="cuda")
        rc_ref, nrm_ref = _call(lib.asgk_cgs_step, V, k, w_ref, h_ref)
        rc_na, nrm_na = _call(lib.asgk_cgs_step_noalloc, V, k, w_na, h_na)
        assert rc_ref == 0 and rc_na == 0
        assert _rel(h_na, h_ref) < TOL
        assert _rel(w_na, w_ref) < TOL
        assert abs(nrm_na - nrm_ref) <= TOL * nrm_ref


def test_cgs_step_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import asgard_b200 as ab
    import torch
    n, k = 1000, 257
    V = torch.ones(k, n, dtype=torch.float64, device="cuda")
    w = torch.ones(n, dtype=torch.float64, device="cuda")
    h = torch.zeros(k, dtype=torch.float64, device="cuda")
    rc, _ = _call(ab.lib.asgk_cgs_step_noalloc, V, k, w, h)
    assert rc == 8  # ASGK_ERR_NOALLOC_LIMIT
    assert torch.equal(w, torch.ones_like(w))
