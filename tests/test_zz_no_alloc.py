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


def test_noalloc_gemm_at_the_size_limit():
    """m*n at the scratch limit (2^22 output elements), and a 1 x 4194300
    output whose column tiles exceed the grid's y extent (computed as the
    transposed product): both match ecg_diag_gemm."""
    import torch
    import ecgpu
    from ecgpu._lib import lib
    L = lib()
    ctx = ecgpu.Context(0)
    rng = np.random.default_rng(7)
    for ta, tb, m, n, k in [("N", "N", 2048, 2048, 64), ("T", "N", 1, 4194300, 8)]:
        A = rng.standard_normal((k, m) if ta == "T" else (m, k))
        B = rng.standard_normal((n, k) if tb == "T" else (k, n))
        C0 = rng.standard_normal((m, n))
        assert m * n <= NOALLOC_MAX_MN
        ref = ctx.diag_gemm(ta, tb, 0.5, A, B, 2.0, C0)
        out, nsplit = _noalloc(L, torch, ta, tb, 0.5, A, B, 2.0, C0)
        assert nsplit >= 1
        assert np.abs(out - ref).max() < 1e-12 * max(1, k), (m, n, k)
    ctx.close()


def test_noalloc_gemm_allocates_nothing_and_replays_in_a_graph():
    """After a first call on the device (which looks up the scratch array's
    address), further calls change no device-memory figure, and a call
    captured in a CUDA graph replays to the same result as ecg_diag_gemm."""
    import torch
    import ecgpu
    from ecgpu._lib import lib
    L = lib()
    ctx = ecgpu.Context(0)
    rng = np.random.default_rng(9)
    m, n, k = 200, 150, 5000
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n))
    tA, pA = _dev(torch, A)
    tB, pB = _dev(torch, B)
    tC = torch.zeros((n, m), dtype=torch.float64, device="cuda")
    pC = C.c_void_p(tC.data_ptr())

    def call():
        st = L.ecg_gemm_noalloc(b"N", b"N", m, n, k, 1.0, pA, m, pB, k, 0.0, pC, m,
                                C.c_void_p(torch.cuda.current_stream().cuda_stream), None)
        assert st == 0, L.ecg_last_error(None).decode()

    call()  # first call on this device: address look-up
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        call()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    ref = ctx.diag_gemm("N", "N", 1.0, A, B, 0.0, np.zeros((m, n)))
    tC.zero_()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            call()
    torch.cuda.current_stream().wait_stream(s)
    tC.zero_()
    g.replay()
    torch.cuda.synchronize()
    out = tC.cpu().numpy().T
    assert np.abs(out - ref).max() < 1e-12 * k
    del g
    ctx.close()
