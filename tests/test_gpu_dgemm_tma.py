"""The TMA-staged FP64 GEMM (csrc/dev_dgemm.cu) against numpy, through the C
ABI: every tile configuration, both memory orders of each operand, split-K,
ragged edges, alpha/beta; and its bounded waits' time-out.  A configuration
is forced through the GEMM tuning table, whose key for a plain FP64 GEMM is
"dgemmt m n k batch ab" (a = A stored k-fastest, b = B stored n-fastest) and
whose value is 8*S + 4 + cfg (S = K slices, cfg = TMA tile configuration).

Each forced call is first made with a 1 ns bound on the kernel's mbarrier
waits (ECG_OPT_TC_WAIT_NS): a bound below the timer's resolution makes the
first wait that finds its stage still loading give up, so the call must
report ECG_ERR_TIMEOUT.  That shows that the TMA kernel ran (the cp.async
kernel, which the library falls back to when TMA cannot address an operand,
has no waits); the same call with the default bound is then checked."""
import numpy as np
import pytest

import ecgpu
from ecgpu._lib import ECG_ERR_TIMEOUT, ECG_OPT_TC_WAIT_NS

pytestmark = pytest.mark.gpu


def _force(ctx, tmp_path, m, n, k, ta, tb, cfg, S):
    p = tmp_path / f"force_{m}_{n}_{k}_{ta}{tb}.txt"
    p.write_text(f"dgemmt {m} {n} {k} 1 {int(ta == 'T')}{int(tb == 'T')} {8 * S + 4 + cfg}\n")
    ctx.tune_load(p)


def _gemm_checked_tma(ctx, ta, tb, alpha, A, B, beta, C0):
    ctx.set_option(ECG_OPT_TC_WAIT_NS, 1)
    try:
        with pytest.raises(ecgpu.ECGError) as e:
            ctx.diag_gemm(ta, tb, alpha, A, B, beta, C0)
        assert e.value.code == ECG_ERR_TIMEOUT
    finally:
        ctx.set_option(ECG_OPT_TC_WAIT_NS, 0)
    return ctx.diag_gemm(ta, tb, alpha, A, B, beta, C0)


def _operands(rng, m, n, k, ta, tb):
    A = rng.standard_normal((k, m) if ta == "T" else (m, k))
    B = rng.standard_normal((n, k) if tb == "T" else (k, n))
    return A, B


@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("tb", ["N", "T"])
def test_tma_gemm_configs_match_numpy(ctx, tmp_path, ta, tb):
    """Ragged sizes (even leading dimensions, so TMA can address them) on
    every tile configuration, unsplit and split over K; alpha and beta."""
    rng = np.random.default_rng(11)
    for cfg in range(4):
        for S in (1, 3):
            m, n, k = 198 + 2 * cfg, 134 + 2 * S, 150 + 16 * cfg + 2 * S
            A, B = _operands(rng, m, n, k, ta, tb)
            C0 = rng.standard_normal((m, n))
            _force(ctx, tmp_path, m, n, k, ta, tb, cfg, S)
            out = _gemm_checked_tma(ctx, ta, tb, 0.7, A, B, -1.3, C0)
            opA = A.T if ta == "T" else A
            opB = B.T if tb == "T" else B
            ref = 0.7 * opA @ opB - 1.3 * C0
            scale = 0.7 * np.abs(opA) @ np.abs(opB) + 1.3 * np.abs(C0)
            err = (np.abs(out - ref) / scale).max()
            assert err < 1e-14, (cfg, S, ta, tb, err)


def test_tma_gemm_small_and_thin(ctx, tmp_path):
    """Shapes smaller than one box in every dimension, and a long thin K."""
    rng = np.random.default_rng(12)
    for (m, n, k) in ((6, 10, 4), (8, 2, 2), (2, 256, 1030), (300, 2, 64)):
        for ta, tb in (("N", "N"), ("T", "T")):
            A, B = _operands(rng, m, n, k, ta, tb)
            _force(ctx, tmp_path, m, n, k, ta, tb, 0, 1)
            out = _gemm_checked_tma(ctx, ta, tb, 1.0, A, B, 0.0, np.zeros((m, n)))
            ref = (A.T if ta == "T" else A) @ (B.T if tb == "T" else B)
            assert np.abs(out - ref).max() < 1e-12 * max(1.0, np.abs(ref).max()), (m, n, k, ta, tb)


def test_tma_gemm_time_out_leaves_context_usable(tmp_path):
    """After a timed-out TMA GEMM (its waits give up, it waits with its full
    bound for the copies it issued and returns) the context runs the next
    GEMMs, FP64 and tensor-core ones, correctly."""
    rng = np.random.default_rng(13)
    m, n, k = 512, 384, 2048
    A, B = _operands(rng, m, n, k, "N", "N")
    with ecgpu.Context(0) as c:
        _force(c, tmp_path, m, n, k, "N", "N", 0, 1)
        out = _gemm_checked_tma(c, "N", "N", 1.0, A, B, 0.0, np.zeros((m, n)))
        assert np.abs(out - A @ B).max() < 1e-12 * np.abs(A @ B).max()
        out = c.diag_gemm("T", "N", 1.0, A, A, 0.0, np.zeros((k, k)))
        assert np.abs(out - A.T @ A).max() < 1e-12 * np.abs(A.T @ A).max()
