"""Failure paths of the C ABI, injected on the host: every error is a status
code plus message and leaves the context usable.  Nothing here faults,
traps or hangs the GPU."""
import numpy as np
import pytest

import ecgpu
from ecgpu._lib import (ECG_ERR_ARG, ECG_ERR_NONFINITE, ECG_ERR_OOM, ECG_ERR_STATE,
                        ECG_ERR_TIMEOUT, ECG_OPT_TC_WAIT_NS, ECG_PREC_MIXED)

pytestmark = pytest.mark.gpu


def test_call_before_system_is_state_error():
    with ecgpu.Context(0) as c:
        c.no, c.nv, c.n = 2, 3, 5
        with pytest.raises(ecgpu.ECGError) as e:
            c.mp2()
        assert e.value.code == ECG_ERR_STATE


def test_nonfinite_inputs(h2o_df):
    B, S = h2o_df
    with ecgpu.Context(0) as c:
        Bbad = B.copy(order="F")
        Bbad[1, 2, 3] = np.nan
        with pytest.raises(ecgpu.ECGError) as e:
            c.set_system(Bbad, S.h, S.e0, S.no)
        assert e.value.code == ECG_ERR_NONFINITE
        c.set_system(B, S.h, S.e0, S.no)
        _, T1, T2 = c.mp2()
        T2[0, 0, 0, 0] = np.inf
        with pytest.raises(ecgpu.ECGError) as e:
            c.cc_residual(T1, T2)
        assert e.value.code == ECG_ERR_NONFINITE
        T2[0, 0, 0, 0] = 0.0
        R1, R2 = c.cc_residual(T1, T2)  # still usable
        assert np.isfinite(R2).all()


def test_memory_cap_is_oom(h2o_df):
    B, S = h2o_df
    with ecgpu.Context(0) as c:
        c.set_mem_cap(1 << 16)
        with pytest.raises(ecgpu.ECGError) as e:
            c.set_system(B, S.h, S.e0, S.no)
        assert e.value.code == ECG_ERR_OOM
        c.set_mem_cap(0)
        c.set_system(B, S.h, S.e0, S.no)
        assert np.isfinite(c.mp2()[0])


def test_bad_arguments(h2o_df):
    B, S = h2o_df
    with ecgpu.Context(0) as c:
        with pytest.raises(ecgpu.ECGError) as e:
            c.set_system(B, S.h, S.e0, 0)
        assert e.value.code == ECG_ERR_ARG
        c.set_system(B, S.h, S.e0, S.no)
        _, T1, T2 = c.mp2()
        with pytest.raises(ecgpu.ECGError) as e:
            c.cc_solve(T1, T2, opts=c.opts(maxdiis=0))
        assert e.value.code == ECG_ERR_ARG
        with pytest.raises(ecgpu.ECGError) as e:
            c.set_precision(7)
        assert e.value.code == ECG_ERR_ARG
        with pytest.raises(ecgpu.ECGError) as e:
            c.diag_permute(np.zeros((2, 2)), (0, 0))
        assert e.value.code == ECG_ERR_ARG


def test_resident_amplitudes(h2o_df):
    """(T) without amplitudes uses those the context holds (no upload) and
    gives the same energy as with the host copy; with none on the device
    (a fresh system, or after a rejected load) it is a state error.  A NaN in
    the last element of T2 is caught by the device-side check."""
    B, S = h2o_df
    with ecgpu.Context(0) as c:
        c.set_system(B, S.h, S.e0, S.no)
        with pytest.raises(ecgpu.ECGError) as e:
            c.pert_t()
        assert e.value.code == ECG_ERR_STATE
        _, T1, T2 = c.mp2()
        r = c.cc_solve(T1, T2)
        assert c.pert_t() == c.pert_t(r["T1"], r["T2"])
        T2bad = np.array(r["T2"], order="F")
        T2bad[-1, -1, -1, -1] = np.nan
        with pytest.raises(ecgpu.ECGError) as e:
            c.pert_t(r["T1"], T2bad)
        assert e.value.code == ECG_ERR_NONFINITE
        with pytest.raises(ecgpu.ECGError) as e:
            c.pert_t()
        assert e.value.code == ECG_ERR_STATE
        assert c.pert_t(r["T1"], r["T2"])[0] < 0.0  # still usable


def test_tensor_core_wait_timeout_is_reported():
    """A 1 ns bound on the tensor-core GEMM's main-loop waits makes the first
    wait for an accumulator run out: the kernel records the time-out, waits
    (with its full bound) for its own loads and MMAs in flight, frees its
    tensor memory and returns; the call reports ECG_ERR_TIMEOUT.  With the
    default bound restored the same GEMM is correct and the context works."""
    rng = np.random.default_rng(4)
    m, n, k = 1024, 1024, 8192
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n))
    C = np.zeros((m, n))
    ref = A @ B
    with ecgpu.Context(0) as c:
        c.set_precision(ECG_PREC_MIXED)
        c.set_option(ECG_OPT_TC_WAIT_NS, 1)
        with pytest.raises(ecgpu.ECGError) as e:
            c.diag_gemm("N", "N", 1.0, A, B, 0.0, C)
        assert e.value.code == ECG_ERR_TIMEOUT
        c.set_option(ECG_OPT_TC_WAIT_NS, 0)
        out = c.diag_gemm("N", "N", 1.0, A, B, 0.0, C)
        scale = np.abs(A) @ np.abs(B)
        assert (np.abs(out - ref) / scale).max() < 4.0 * (k / 16 + 16) * 2.0 ** -24
        with pytest.raises(ecgpu.ECGError) as e:
            c.set_option(99, 1)
        assert e.value.code == ECG_ERR_ARG


def test_concurrent_contexts_own_their_scratch():
    """Two contexts, each on its own host thread and stream, run split-K FP64
    GEMMs (output of fewer tiles than SMs, long K) and split-BF16 GEMMs at the
    same time: each stream owns its split-K and operand scratch, so every
    result matches numpy."""
    import threading
    errs = []

    def work(seed, prec):
        try:
            rng = np.random.default_rng(seed)
            with ecgpu.Context(0) as c:
                c.set_precision(prec)
                for it in range(6):
                    m, n, k = 96 + 8 * it, 80, 6000 + 512 * it
                    A = rng.standard_normal((m, k))
                    B = rng.standard_normal((k, n))
                    out = c.diag_gemm("N", "N", 1.0, A, B, 0.0, np.zeros((m, n)))
                    err = np.abs(out - A @ B).max() / (np.abs(A) @ np.abs(B)).max()
                    tol = 1e-13 if prec == 0 else 4.0 * (k / 16 + 16) * 2.0 ** -24
                    if not err < tol:
                        errs.append((seed, prec, it, err))
        except Exception as e:  # noqa: BLE001 - reported below
            errs.append((seed, prec, repr(e)))

    th = [threading.Thread(target=work, args=(s, p)) for s, p in
          ((1, 0), (2, 0), (3, ECG_PREC_MIXED), (4, ECG_PREC_MIXED))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
