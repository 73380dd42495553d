"""ecg_gemm_noalloc: the FP64 GEMM entry point that allocates no device memory.

It serves callers that must not allocate in their call path (code running
under another framework's memory manager, inside stream capture, or with all
device memory already handed out): they pass device pointers for A, B and C,
and the split-K partial products use a fixed scratch array inside the
library.  Its results are compared with the existing ecg_diag_gemm entry point
at the GEMM tests' tolerance, on two calls in a row.  This file is collected
last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NOALLOC_MAX_MN = 1 << 22


def _dev(torch, a):
    """Column-major device copy of a 2-D host array (returns tensor, pointer)."""
    t = torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)).cuda()
    return t, C.c_void_p(t.data_ptr())


def _noalloc(L, torch, ta, tb, alpha, A, B, beta, Cm):
    m, n = Cm.shape
    k = A.shape[0] if ta == "T" else A.shape[1]
    tA, pA = _dev(torch, A)
    tB, pB = _dev(torch, B)
    tC, pC = _dev(torch, Cm)
    ns = C.c_int32(0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = L.ecg_gemm_noalloc(ta.encode(), tb.encode(), m, n, k, float(alpha), pA, A.shape[0], pB,
                            B.shape[0], float(beta), pC, m, stream, C.byref(ns))
    assert st == 0, L.ecg_last_error(None).decode()
    torch.cuda.synchronize()
    return tC.cpu().numpy().T.copy(), ns.value


def test_noalloc_gemm_matches_existing_entry_point():
    import torch
    import ecgpu
    from ecgpu._lib import lib
    L = lib()
    ctx = ecgpu.Context(0)
    rng = np.random.default_rng(42)
    cases = [("N", "N", 120, 70, 3000), ("T", "N", 76, 16, 25536), ("N", "T", 300, 257, 700),
             ("T", "T", 33, 65, 129)]
    for ta, tb, m, n, k in cases:
        for call in range(2):  # two calls in a row share the scratch array
            A = rng.standard_normal((k, m) if ta == "T" else (m, k))
            B = rng.standard_normal((n, k) if tb == "T" else (k, n))
            C0 = rng.standard_normal((m, n))
            alpha, beta = (0.7, -0.3) if call == 0 else (-1.25, 0.0)
            ref = ctx.diag_gemm(ta, tb, alpha, A, B, beta, C0)
            out, nsplit = _noalloc(L, torch, ta, tb, alpha, A, B, beta, C0)
            assert nsplit >= 1
            assert np.abs(out - ref).max() < 1e-12 * max(1, k), (ta, tb, m, n, k, call)
    ctx.close()


def test_noalloc_gemm_rejects_oversized_output():
    import torch
    from ecgpu._lib import ECG_ERR_ARG, lib
    L = lib()
    t = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = C.c_void_p(t.data_ptr())
    m = n = 4096  # m*n = 2^24 > 2^22: rejected on the host before any device access
    st = L.ecg_gemm_noalloc(b"N", b"N", m, n, 4, 1.0, p, m, p, 4, 0.0, p, m, None, None)
    assert st == ECG_ERR_ARG
    assert "exceeds" in L.ecg_last_error(None).decode()
    assert m * n > NOALLOC_MAX_MN
