"""Analytic CC energy gradients through the Lambda (adjoint) equations.

The reverse rule of the total CCSD/DCSD energy with respect to the MO
one-electron matrix h (orbitals fixed) returns G = dE/dh.  It is checked
(a) against the oracle's densities (calc_1RDM, src/cc/cc_lagrange.jl:786-848)
at the same converged amplitudes, and (b) against fourth-order central finite
differences of converged energies for a one-electron perturbation h + lambda P.
P is a seeded random symmetric matrix: the FCIDUMP fixture carries no dipole
integrals, and any symmetric one-electron operator tests the same rule.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# squared residual 1e-16: reachable in FP64 (the iteration floor sits near 1e-17);
# the Hylleraas energies are then stable to ~1e-15
TIGHT = dict(thr=1e-16, conven=1.0, maxit=200)


def _perturbation(n, seed=7):
    """Symmetric one-electron operator of unit spectral norm (a field-like
    strength, so that the finite-difference truncation stays ~1e-12)."""
    P = np.random.default_rng(seed).standard_normal((n, n))
    P = 0.5 * (P + P.T)
    return P / np.linalg.norm(P, 2)


def _energy(ctx, B, h, e0, no, dc, prec):
    import ecgpu
    ctx.set_precision(prec)
    ctx.set_system(B, h, e0, no)
    _, _, ehf = ctx.fock()
    _, T1, T2 = ctx.mp2()
    r = ctx.cc_solve(T1, T2, dc=dc, opts=ctx.opts(**TIGHT))
    assert r["converged"]
    ctx.set_precision(ecgpu.ECG_PREC_FP64)
    return ehf + r["E"], r


def _ec(B, h, e0, no, prec, conv=TIGHT):
    from ecgpu.driver import ECInfo, FDump
    EC = ECInfo()
    EC.fd = FDump(h, e0, 2 * no, B=B)
    EC.set("cc", **conv)
    EC.set("gpu", precision=prec)
    return EC


def test_gradient_matches_oracle_density(h2o_df, ctx):
    """G = dD1 + HF density equals the oracle's calc_1RDM at the same
    converged amplitudes and multipliers."""
    import oracle as O
    B, S = h2o_df
    _, r = _energy(ctx, B, S.h, S.e0, S.no, False, 0)
    lr = ctx.lambda_solve(r["T1"], r["T2"], opts=ctx.opts(**TIGHT))
    assert lr["converged"]
    G = ctx.energy_gradient(r["T1"], r["T2"], lr["U1"], lr["U2"])
    _, dD1 = O.one_rdm(S, lr["U1"], lr["U2"], r["T1"], r["T2"])
    ref = dD1.copy()
    ref[np.arange(S.no), np.arange(S.no)] += 2.0
    assert np.abs(G - ref).max() < 1e-10


@pytest.mark.parametrize("method", ["ccsd", "dcsd"])
def test_gradient_matches_finite_differences(h2o_df, ctx, method):
    """dE/dlambda from the rrule pullback agrees with the fourth-order central
    difference (step 1e-3, truncation ~1e-12) of converged FP64 energies."""
    from ecgpu.driver import rrule_cc_energy
    B, S = h2o_df
    P = _perturbation(S.h.shape[0])
    E0, pullback = rrule_cc_energy(_ec(B, S.h, S.e0, S.no, "fp64"), method)
    analytic = float(np.sum(pullback(1.0) * P))
    dc = method == "dcsd"
    d = 1e-3
    E = {k: _energy(ctx, B, S.h + k * d * P, S.e0, S.no, dc, 0)[0] for k in (-2, -1, 1, 2)}
    fd = (E[-2] - 8 * E[-1] + 8 * E[1] - E[2]) / (12 * d)
    assert abs(fd - analytic) < 1e-7, (fd, analytic)
    assert abs(E0 - _energy(ctx, B, S.h, S.e0, S.no, dc, 0)[0]) < 1e-11


def test_mixed_precision_gradient():
    """The rrule in ECG_PREC_MIXED (split-BF16 products, FP64 refinement of
    both the amplitude and the Lambda equations) reproduces the FP64 gradient
    on an (H2O)_3/cc-pVDZ-sized system, where the ring and ladder GEMMs take
    the tensor-core path."""
    from ecgpu.driver import rrule_cc_energy
    from ecgpu.synthetic import make_workload
    B, h, e0, no = make_workload("h2o3_vdz")
    P = _perturbation(h.shape[0])
    conv = dict(thr=1e-12, conven=1.0, maxit=100)
    E64, pb64 = rrule_cc_energy(_ec(B, h, e0, no, "fp64", conv), "ccsd")
    Emx, pbmx = rrule_cc_energy(_ec(B, h, e0, no, "mixed", conv), "ccsd")
    assert abs(Emx - E64) < 1e-6
    assert abs(float(np.sum((pbmx(1.0) - pb64(1.0)) * P))) < 1e-6


def test_lambda_buffers_reallocated_after_set_system(h2o_df):
    """A second set_system frees the first system's buffers; the Lambda
    buffers, allocated on first use, are allocated again (no stale pointers),
    and a DIIS object made for the earlier system is refused."""
    import ecgpu
    B, S = h2o_df
    rng = np.random.default_rng(3)
    with ecgpu.Context(0) as c:
        c.set_system(B, S.h, S.e0, S.no)
        _, T1, T2 = c.mp2()
        U1 = rng.standard_normal(T1.shape)
        Y = rng.standard_normal(T2.shape)
        U2 = Y + Y.transpose(1, 0, 3, 2)
        R1a, R2a = c.lambda_residual(T1, T2, U1, U2)
        d = ecgpu.Diis(c, 8)
        c.set_system(B, S.h, S.e0, S.no)
        R1b, R2b = c.lambda_residual(T1, T2, U1, U2)
        assert np.abs(R1a - R1b).max() < 1e-13 and np.abs(R2a - R2b).max() < 1e-13
        with pytest.raises(ecgpu.ECGError):
            d.perform(np.zeros(8), np.zeros(8))
