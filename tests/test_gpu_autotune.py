"""The GEMM autotuner: tuning a shape leaves the call's result unchanged,
records an entry, and the table survives a save/load round trip."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_gemms_and_table(tmp_path):
    import ecgpu
    from ecgpu._lib import ECG_OPT_AUTOTUNE
    rng = np.random.default_rng(3)
    shapes = [(300, 200, 2000), (1000, 96, 6000), (640, 640, 256)]
    with ecgpu.Context(0) as c:
        ref = {}
        for prec in (ecgpu.ECG_PREC_FP64, ecgpu.ECG_PREC_MIXED):
            c.set_precision(prec)
            for m, n, k in shapes:
                A = rng.standard_normal((m, k))
                B = rng.standard_normal((k, n))
                C0 = rng.standard_normal((m, n))
                c.set_option(ECG_OPT_AUTOTUNE, 0)
                plain = c.diag_gemm("N", "N", 0.5, A, B, 1.5, C0)
                c.set_option(ECG_OPT_AUTOTUNE, 1)
                tuned = c.diag_gemm("N", "N", 0.5, A, B, 1.5, C0)
                again = c.diag_gemm("N", "N", 0.5, A, B, 1.5, C0)  # from the table
                scale = 0.5 * (np.abs(A) @ np.abs(B)) + 1.5 * np.abs(C0)
                tol = 1e-14 * k if prec == ecgpu.ECG_PREC_FP64 else 4.0 * (k / 16 + 16) * 2.0 ** -24
                exact = 0.5 * (A @ B) + 1.5 * C0
                for out in (plain, tuned, again):
                    assert (np.abs(out - exact) / scale).max() < tol
                ref[(prec, m)] = tuned
        c.set_option(ECG_OPT_AUTOTUNE, 0)
        p = tmp_path / "tune.txt"
        n = c.tune_save(p)
        assert n >= 6
        lines = p.read_text().splitlines()
        assert all(len(x.rsplit(" ", 1)) == 2 for x in lines)
        assert c.tune_load(p) == n
        bad = tmp_path / "bad.txt"
        bad.write_text("dgemm 1 2 3 1 00 notanumber\n")
        with pytest.raises(ecgpu.ECGError):
            c.tune_load(bad)


def test_autotuned_mixed_ccsd_matches():
    """A mixed-precision CCSD solve with every GEMM shape tuned on first use
    converges to the same energy as with the fixed rules (1e-8)."""
    import ecgpu
    from ecgpu._lib import ECG_OPT_AUTOTUNE
    from ecgpu.synthetic import make_system
    B, h1, e0, _ = make_system(10, 80, 200)
    E = []
    for tune in (0, 1):
        with ecgpu.Context(0) as c:
            c.set_option(ECG_OPT_AUTOTUNE, tune)
            c.set_precision(ecgpu.ECG_PREC_MIXED)
            c.set_system(B, h1, e0, 10)
            _, T1, T2 = c.mp2()
            r = c.cc_solve(T1, T2)
            assert r["converged"]
            E.append(r["E"])
            c.set_option(ECG_OPT_AUTOTUNE, 0)
    assert abs(E[0] - E[1]) < 1e-8, E
