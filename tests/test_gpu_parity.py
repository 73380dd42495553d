"""Parity of the CUDA path (libecgpu through its C ABI) with the oracle.

FP64 throughout; tolerances: residuals and densities 1e-11 absolute
(summation-order differences only), energies 1e-10 Eh against the oracle on
the same trajectory, and the reference's pinned energies as in
tests/test_oracle_golden.py.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _perturbed(S, f, seed=0, amp=0.01):
    rng = np.random.default_rng(seed)
    _, T1, T2 = O.mp2(S, f)
    T1 = T1 + amp * rng.standard_normal(T1.shape)
    X = amp * rng.standard_normal(T2.shape)
    return T1, T2 + X + X.transpose(1, 0, 3, 2)


@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("tb", ["N", "T"])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (64, 64, 16), (129, 65, 33),
                                   (300, 200, 150), (520, 384, 96)])
def test_gemm_kernel(ctx, ta, tb, m, n, k):
    rng = np.random.default_rng(m * 1000 + n * 10 + k)
    A = rng.standard_normal((k, m) if ta == "T" else (m, k))
    B = rng.standard_normal((n, k) if tb == "T" else (k, n))
    C = rng.standard_normal((m, n))
    ref = 0.7 * ((A.T if ta == "T" else A) @ (B.T if tb == "T" else B)) - 0.3 * C
    out = ctx.diag_gemm(ta, tb, 0.7, A, B, -0.3, C)
    assert np.abs(out - ref).max() < 1e-12 * max(1, k)


@pytest.mark.parametrize("shape,perm", [((5, 7, 3, 4), (1, 0, 3, 2)), ((40, 33, 9), (2, 0, 1)),
                                        ((64, 64, 8, 8), (0, 3, 1, 2)), ((3, 70, 50), (0, 2, 1)),
                                        ((100,), (0,)), ((40, 6, 5, 7), (0, 2, 3, 1)),
                                        ((33, 8, 65), (2, 1, 0))])
def test_permute_kernel(ctx, shape, perm):
    rng = np.random.default_rng(1)
    x = np.asfortranarray(rng.standard_normal(shape))
    y = np.asfortranarray(rng.standard_normal(tuple(shape[p] for p in perm)))
    out = ctx.diag_permute(x, perm, 2.0, -1.0, y)
    assert np.abs(out - (2.0 * np.transpose(x, perm) - y)).max() < 1e-14


@pytest.fixture(scope="module")
def sys_h2o(ctx, h2o_df):
    B, S = h2o_df
    ctx.set_system(B, S.h, S.e0, S.no)
    return S, O.gen_fock(S)


def test_fock_hf_mp2(ctx, sys_h2o):
    S, f = sys_h2o
    fg, eps, ehf = ctx.fock()
    assert np.abs(fg - f).max() < 1e-13
    assert abs(ehf - O.hf_energy(S, f)) < 1e-12
    e, T1, T2 = ctx.mp2()
    eo, T1o, T2o = O.mp2(S, f)
    assert abs(e - eo) < 1e-13
    assert np.abs(T1 - T1o).max() < 1e-14 and np.abs(T2 - T2o).max() < 1e-14


@pytest.mark.parametrize("dc", [False, True])
def test_cc_residual(ctx, sys_h2o, dc):
    S, f = sys_h2o
    T1, T2 = _perturbed(S, f)
    R1, R2 = ctx.cc_residual(T1, T2, dc=dc)
    R1o, R2o = O.cc_resid(S, T1, T2, dc=dc)
    assert np.abs(R1 - R1o).max() < 1e-12
    assert np.abs(R2 - R2o).max() < 1e-12


@pytest.mark.parametrize("dc", [False, True])
def test_cc_solve_matches_oracle(ctx, sys_h2o, dc):
    S, f = sys_h2o
    e, T1, T2 = ctx.mp2()
    r = ctx.cc_solve(T1, T2, dc=dc)
    Eo, T1o, T2o, it, conv = O.cc_iterations(S, *O.mp2(S, f)[1:], f, dc=dc)
    assert r["converged"] and conv and r["iterations"] == it
    assert abs(r["E"] - Eo) < 1e-10
    assert np.abs(r["T2"] - T2o).max() < 1e-9


def test_pert_t(ctx, sys_h2o):
    S, f = sys_h2o
    e, T1, T2 = ctx.mp2()
    r = ctx.cc_solve(T1, T2)
    et, etb = ctx.pert_t(r["T1"], r["T2"])
    eto, etbo = O.pert_t(S, r["T1"], r["T2"], f)
    assert abs(et - eto) < 1e-12 and abs(etb - etbo) < 1e-12


@pytest.mark.parametrize("dc", [False, True])
def test_lambda_residual_and_rdm(ctx, sys_h2o, dc):
    S, f = sys_h2o
    T1, T2 = _perturbed(S, f, seed=5)
    rng = np.random.default_rng(7)
    U1 = rng.standard_normal(T1.shape)
    Y = rng.standard_normal(T2.shape)
    U2 = Y + Y.transpose(1, 0, 3, 2)
    R1, R2 = ctx.lambda_residual(T1, T2, U1, U2, dc=dc)
    dr = O.dressed_ints(S, T1)
    o, v = S.sl["o"], S.sl["v"]
    vT = np.einsum("bmdc,dcji->mbij", dr[0][v, o, v, v], T2)
    R1o, R2o = O.vector_times_jacobian(S, U1, U2, T1, T2, f, dr, vT, dc=dc)
    assert np.abs(R1 - R1o).max() < 1e-11 * max(1, np.abs(R1o).max())
    assert np.abs(R2 - R2o).max() < 1e-11 * max(1, np.abs(R2o).max())
    D1, dD1 = ctx.one_rdm(T1, T2, U1, U2)
    D1o, dD1o = O.one_rdm(S, U1, U2, T1, T2)
    assert np.abs(D1 - D1o).max() < 1e-12 and np.abs(dD1 - dD1o).max() < 1e-12


def test_lambda_solve_and_lambda_t(ctx, sys_h2o):
    S, f = sys_h2o
    e, T1, T2 = ctx.mp2()
    r = ctx.cc_solve(T1, T2)
    lr = ctx.lambda_solve(r["T1"], r["T2"])
    U1o, U2o, lit, lconv = O.lambda_iterations(S, r["T1"], r["T2"], f)
    assert lr["converged"] and lr["iterations"] == lit
    assert np.abs(lr["U2"] - U2o).max() < 1e-9 and np.abs(lr["U1"] - U1o).max() < 1e-9
    e1, e1b = ctx.lambda_pert_t(r["T1"], r["T2"], lr["U1"], lr["U2"])
    e1o, e1bo = O.lambda_pert_t(S, r["T1"], r["T2"], U1o, U2o, f)
    assert abs(e1 - e1o) < 1e-11 and abs(e1b - e1bo) < 1e-11


def test_driver_reproduces_reference_pins(h2o, gold, tmp_path):
    """ccdriver on the reference's H2O.FCIDUMP integrals (through Cholesky
    factors) against test/h2o.jl's pinned energies: HF, MP2 and CCSD(T) to
    1e-9 (CCSD(T) with the pre-0.13 DIIS dot that produced the pin, see
    tests/test_oracle_golden.py), DCSD converged tightly to 1e-9, ΛCCSD(T)
    to 3e-7; the current-DIIS trajectories equal the oracle's to 1e-9."""
    from ecgpu.driver import ECInfo, FDump, ccdriver
    g = gold["h2o"]
    EC = ECInfo(scr=str(tmp_path))
    EC.fd = FDump(h2o.h, h2o.e0, 2 * h2o.no, V=h2o.V)
    e = ccdriver(EC, "ccsd(t)")
    assert abs(e["HF"] - g["HF"]) < 1e-9
    assert abs(e["MP2c"] - g["MP2c"]) < 1e-9
    ref = O.ccdriver(h2o, "ccsd(t)")
    assert e["iterations"] == ref["iterations"]
    assert abs(e["CCSD(T)c"] - ref["CCSD(T)c"]) < 1e-9
    assert abs(e["CCSD(T)c"] - g["CCSD(T)c"]) < 3e-7
    EC.set("diis", dot="plain")
    e = ccdriver(EC, "ccsd(t)")
    assert e["iterations"] == 13
    assert abs(e["CCSD(T)c"] - g["CCSD(T)c"]) < 1e-9
    e = ccdriver(EC, "λccsd(t)")
    assert abs(e["ΛCCSD(T)c"] - g["LCCSD(T)c"]) < 3e-7
    EC.set("diis", dot="cs")
    e = ccdriver(EC, "λccsd(t)")
    ref = O.ccdriver(h2o, "λccsd(t)")
    assert abs(e["ΛCCSD(T)c"] - ref["ΛCCSD(T)c"]) < 1e-9
    assert abs(e["ΛCCSD(T)c"] - g["LCCSD(T)c"]) < 3e-7
    EC.set("cc", thr=1e-20, conven=1e-4, maxit=60)
    e = ccdriver(EC, "dcsd")
    assert abs(e["DCSDc"] - g["DCSDc"]) < 1e-9
    assert (tmp_path / "cc_amplitudes_2.bin").exists()


@pytest.mark.parametrize("batch", [1, 16])
def test_pert_t_multibatch_graph_sweep(batch):
    """The (T) sweep in many batches — the first run directly, the rest replayed
    from one CUDA graph — on the (H2O)_3/cc-pVDZ shape (o = 12: 352 triplets,
    352 or 22 batches), (T), [T] and Lambda-(T) against the oracle
    (cc_triples.jl:39-295) to 1e-11, and equal to the automatic batching."""
    import ecgpu
    from ecgpu._lib import ECG_OPT_TRIPLES_BATCH
    from ecgpu.synthetic import make_workload
    B, h1, e0, no = make_workload("h2o3_vdz")
    S = O.System.from_df(np.ascontiguousarray(B.transpose(2, 0, 1)), h1, e0, no)
    f = O.gen_fock(S)
    rng = np.random.default_rng(5)
    with ecgpu.Context(0) as c:
        c.set_system(B, h1, e0, no)
        _, T1, T2 = c.mp2()
        T1 = np.asfortranarray(T1 + 1e-3 * rng.standard_normal(T1.shape))
        U1 = np.asfortranarray(2.0 * T1)
        U2 = np.asfortranarray(2.0 * T2 - T2.transpose(0, 1, 3, 2))
        auto = c.pert_t(T1, T2), c.lambda_pert_t(T1, T2, U1, U2)
        c.set_option(ECG_OPT_TRIPLES_BATCH, batch)
        et, etb = c.pert_t(T1, T2)
        lt, ltb = c.lambda_pert_t(T1, T2, U1, U2)
    eto, etbo = O.pert_t(S, T1, T2, f)
    lto, ltbo = O.lambda_pert_t(S, T1, T2, U1, U2, f)
    assert et < -1e-4
    assert abs(et - eto) < 1e-11 and abs(etb - etbo) < 1e-11
    assert abs(lt - lto) < 1e-11 and abs(ltb - ltbo) < 1e-11
    assert abs(et - auto[0][0]) < 1e-12 and abs(lt - auto[1][0]) < 1e-12


def test_synthetic_water_dimer_ccsd_t(ctx):
    """(H2O)_2/cc-pVDZ-sized synthetic system: full CCSD(T) vs the oracle."""
    from ecgpu.synthetic import make_workload
    B, h1, e0, no = make_workload("h2o2_vdz")
    S = O.System.from_df(np.transpose(B, (2, 0, 1)), h1, e0, no)
    f = O.gen_fock(S)
    ctx.set_system(B, h1, e0, no)
    T1, T2 = _perturbed(S, f, seed=11)
    for dc in (False, True):
        R1, R2 = ctx.cc_residual(T1, T2, dc=dc)
        R1o, R2o = O.cc_resid(S, T1, T2, dc=dc)
        assert np.abs(R1 - R1o).max() < 1e-11 and np.abs(R2 - R2o).max() < 1e-11
    e, T1, T2 = ctx.mp2()
    r = ctx.cc_solve(T1, T2)
    Eo, T1o, T2o, it, conv = O.cc_iterations(S, *O.mp2(S, f)[1:], f)
    assert r["iterations"] == it and abs(r["E"] - Eo) < 1e-10
    et, _ = ctx.pert_t(r["T1"], r["T2"])
    eto, _ = O.pert_t(S, r["T1"], r["T2"], f)
    assert abs(et - eto) < 1e-11


def test_deterministic(ctx, h2o_df):
    B, S = h2o_df
    ctx.set_system(B, S.h, S.e0, S.no)
    out = []
    for _ in range(2):
        e, T1, T2 = ctx.mp2()
        r = ctx.cc_solve(T1, T2)
        out.append((r["E"], ctx.pert_t(r["T1"], r["T2"])))
    assert out[0] == out[1]


def test_diis_standalone(ctx, h2o_df):
    """ecg_diis_* against the oracle's DIIS on a linear fixed-point problem."""
    import ecgpu
    B, S = h2o_df
    ctx.set_system(B, S.h, S.e0, S.no)
    rng = np.random.default_rng(2)
    n = 50
    A = np.eye(n) + 0.1 * rng.standard_normal((n, n))
    b = rng.standard_normal(n)
    d = ecgpu.Diis(ctx, n, maxdiis=4)
    od = O.Diis(4, 10.0, dots=None)
    x = np.zeros(n)
    xo = np.zeros(n)
    for _ in range(8):
        r = A @ x - b
        x = d.perform(x - 0.5 * r, r)
        ro = A @ xo - b
        vec = [xo - 0.5 * ro]
        od.perform(vec, [ro])
        xo = vec[0]
        assert np.abs(x - xo).max() < 1e-10


@pytest.mark.parametrize("ta,tb,m,n,k", [("N", "N", 1, 1, 1), ("N", "N", 128, 128, 64),
                                         ("N", "T", 200, 130, 100), ("T", "N", 300, 257, 700),
                                         ("T", "T", 129, 65, 1000), ("N", "N", 1216, 1216, 1216),
                                         ("T", "N", 2926, 136, 2926), ("N", "T", 2000, 3000, 320)])
def test_mixed_gemm_kernel(ta, tb, m, n, k):
    """Split-BF16 tcgen05 GEMM: FP32-level error, below 4 (k/16 + 16) 2^-24 of
    sum |a||b| (the bound of FP32 accumulation over k/16 MMA steps)."""
    import ecgpu
    rng = np.random.default_rng(m + 7 * n + 13 * k)
    A = rng.standard_normal((k, m) if ta == "T" else (m, k))
    B = rng.standard_normal((n, k) if tb == "T" else (k, n))
    C = rng.standard_normal((m, n))
    opA = A.T if ta == "T" else A
    opB = B.T if tb == "T" else B
    ref = 0.7 * (opA @ opB) - 0.3 * C
    scale = 0.7 * (np.abs(opA) @ np.abs(opB)) + 0.3 * np.abs(C)
    with ecgpu.Context(0) as c:
        c.set_precision(ecgpu.ECG_PREC_MIXED)
        out = c.diag_gemm(ta, tb, 0.7, A, B, -0.3, C)
    err = np.abs(out - ref) / scale
    assert err.max() < 4.0 * (k / 16 + 16) * 2.0 ** -24, err.max()
    if k >= 64:
        # FP32 accumulation of BF16 slice products leaves errors far above an
        # FP64 GEMM's (~1e-16): the tensor-core kernel computed this result
        assert err.max() > 1e-11, err.max()


@pytest.mark.parametrize("dc", [False, True])
def test_mixed_precision_solve_within_1_uEh(dc):
    """ECG_PREC_MIXED (split-BF16 tensor-core products, then FP64 refinement)
    converges to the FP64 energy within 1 microhartree on an (H2O)_3/cc-pVDZ-
    sized system, where the ring and ladder GEMMs take the tensor-core path."""
    import ecgpu
    from ecgpu.synthetic import make_workload
    B, h1, e0, no = make_workload("h2o3_vdz")
    out = {}
    for prec in (ecgpu.ECG_PREC_FP64, ecgpu.ECG_PREC_MIXED):
        with ecgpu.Context(0) as c:
            c.set_precision(prec)
            c.set_system(B, h1, e0, no)
            _, T1, T2 = c.mp2()
            r = c.cc_solve(T1, T2, dc=dc)
            assert r["converged"]
            out[prec] = r
    dE = abs(out[ecgpu.ECG_PREC_MIXED]["E"] - out[ecgpu.ECG_PREC_FP64]["E"])
    assert dE < 1e-6, dE


@pytest.mark.parametrize("no,nq", [(24, 128), (13, 30)])
def test_mixed_precision_solve_wide_ladder_tiles(no, nq):
    """v = 64.  o = 24: the ladder contractions have N = o(o+1)/2 = 300 and
    o(o-1)/2 = 276 columns and run on 160-column tensor-core tiles, with V
    written in FP32 by the tensor cores and packed straight into BF16 slices.
    o = 13, nQ = 30: the V build is below the tensor-core size rule, so the
    FP64 V is packed into BF16 slices.  The mixed CCSD energy (after FP64
    refinement) is within 1 microhartree of FP64."""
    import ecgpu
    from ecgpu.synthetic import make_system
    B, h1, e0, _ = make_system(no, 64, nq)
    out = {}
    for prec in (ecgpu.ECG_PREC_FP64, ecgpu.ECG_PREC_MIXED):
        with ecgpu.Context(0) as c:
            c.set_precision(prec)
            c.set_system(B, h1, e0, no)
            _, T1, T2 = c.mp2()
            r = c.cc_solve(T1, T2)
            assert r["converged"]
            out[prec] = r["E"]
    dE = abs(out[ecgpu.ECG_PREC_MIXED] - out[ecgpu.ECG_PREC_FP64])
    assert dE < 1e-6, dE


def test_mixed_precision_triples():
    """(T) and Lambda-(T) with split-BF16 tensor-core W products agree with FP64
    to 1e-8 Eh on the (H2O)_3/cc-pVDZ-sized system."""
    import ecgpu
    from ecgpu.synthetic import make_workload
    B, h1, e0, no = make_workload("h2o3_vdz")
    with ecgpu.Context(0) as c:
        c.set_system(B, h1, e0, no)
        _, T1, T2 = c.mp2()
        r = c.cc_solve(T1, T2)
        lr = c.lambda_solve(r["T1"], r["T2"])
        e64 = c.pert_t(r["T1"], r["T2"])
        l64 = c.lambda_pert_t(r["T1"], r["T2"], lr["U1"], lr["U2"])
        c.set_precision(ecgpu.ECG_PREC_MIXED)
        emx = c.pert_t(r["T1"], r["T2"])
        lmx = c.lambda_pert_t(r["T1"], r["T2"], lr["U1"], lr["U2"])
    assert abs(emx[0] - e64[0]) < 1e-8 and abs(emx[1] - e64[1]) < 1e-8
    assert abs(lmx[0] - l64[0]) < 1e-8


def test_mixed_precision_triples_wide_tiles():
    """v = 300: the (T) GEMMs whose columns run over v use 160-column
    tensor-core tiles (N = 300 in 320 columns instead of 384); (T), [T] and
    Lambda-(T) from MP2 amplitudes agree with FP64 to 2e-5 relative, the
    precision of the two-slice BF16 products (~2^-16; a tile that dropped or
    misplaced columns would be off by O(1))."""
    import ecgpu
    from ecgpu.synthetic import make_system
    no = 3
    B, h1, e0, _ = make_system(no, 300, 400)
    with ecgpu.Context(0) as c:
        c.set_system(B, h1, e0, no)
        _, T1, T2 = c.mp2()
        U1, U2 = 2.0 * T1, 2.0 * T2
        e64 = c.pert_t(T1, T2)
        l64 = c.lambda_pert_t(T1, T2, U1, U2)
        c.set_precision(ecgpu.ECG_PREC_MIXED)
        emx = c.pert_t(T1, T2)
        lmx = c.lambda_pert_t(T1, T2, U1, U2)
    assert e64[0] < -1e-6
    for x, ref in ((emx[0], e64[0]), (emx[1], e64[1]), (lmx[0], l64[0])):
        assert abs(x - ref) < 2e-5 * abs(ref), (x, ref)


@pytest.mark.parametrize("no", [1, 2])
def test_pert_t_few_occupied(no):
    """(T), [T] and Lambda-(T) with one and two occupied orbitals (no triplet
    at all, or only i = j < k and i < j = k) on a synthetic system with
    v = 20 (ragged 8^3 cubes), FP64 against the oracle (cc_triples.jl:39-295),
    mixed against FP64; with one occupied orbital every energy is 0."""
    import ecgpu
    from ecgpu.synthetic import make_system
    B, h1, e0, _ = make_system(no, 20, 30)
    S = O.System.from_df(np.ascontiguousarray(B.transpose(2, 0, 1)), h1, e0, no)
    f = O.gen_fock(S)
    rng = np.random.default_rng(11)
    with ecgpu.Context(0) as c:
        c.set_system(B, h1, e0, no)
        _, T1, T2 = c.mp2()
        U1 = T1 + 0.01 * rng.standard_normal(T1.shape)
        Y = 0.01 * rng.standard_normal(T2.shape)
        U2 = np.asfortranarray(T2 + Y + Y.transpose(1, 0, 3, 2))
        et, etb = c.pert_t(T1, T2)
        lt, ltb = c.lambda_pert_t(T1, T2, U1, U2)
        c.set_precision(ecgpu.ECG_PREC_MIXED)
        mt, mtb = c.pert_t(T1, T2)
    eto, etbo = O.pert_t(S, T1, T2, f)
    lto, ltbo = O.lambda_pert_t(S, T1, T2, U1, U2, f)
    if no == 1:
        assert et == etb == lt == ltb == mt == mtb == 0.0
        assert eto == etbo == lto == ltbo == 0.0
        return
    assert et < -1e-8
    assert abs(et - eto) < 1e-13 and abs(etb - etbo) < 1e-13
    assert abs(lt - lto) < 1e-13 and abs(ltb - ltbo) < 1e-13
    assert abs(mt - et) < 2e-5 * abs(et) and abs(mtb - etb) < 2e-5 * abs(etb)


def test_mixed_ccsd_t_vtz_shape():
    """The (H2O)_6/cc-pVTZ virtual and auxiliary space (v = 318, nQ = 846) with
    o = 6: mixed CCSD (FP64 refinement) and mixed (T) within 1 microhartree of
    FP64.  The mixed GEMMs run with the tile widths of that shape (160 columns
    for N = v = 318, 256 for the (T) GEMM over v^2 columns)."""
    import ecgpu
    from ecgpu.synthetic import make_system
    no = 6
    B, h1, e0, _ = make_system(no, 318, 846)
    out = {}
    for prec in (ecgpu.ECG_PREC_FP64, ecgpu.ECG_PREC_MIXED):
        with ecgpu.Context(0) as c:
            c.set_precision(prec)
            c.set_system(B, h1, e0, no)
            _, T1, T2 = c.mp2()
            r = c.cc_solve(T1, T2)
            assert r["converged"]
            out[prec] = (r["E"], c.pert_t()[0])
    e64, emx = out[ecgpu.ECG_PREC_FP64], out[ecgpu.ECG_PREC_MIXED]
    assert out[ecgpu.ECG_PREC_FP64][1] < -1e-5
    assert abs(emx[0] - e64[0]) < 1e-6, (emx[0], e64[0])
    assert abs(emx[1] - e64[1]) < 1e-6, (emx[1], e64[1])


def test_driver_from_fcidump_text(h2o_fcidump_text, gold, tmp_path):
    """ccdriver(EC, "ccsd(t)"; fcidump) as test/h2o.jl calls it, on the
    reference's H2O.FCIDUMP text (pre-0.13 DIIS dot, see test_oracle_golden)."""
    from ecgpu.driver import ECInfo, ccdriver
    g = gold["h2o"]
    EC = ECInfo(scr=str(tmp_path))
    EC.set("diis", dot="plain")
    e = ccdriver(EC, "ccsd(t)", fcidump=h2o_fcidump_text)
    assert abs(e["HF"] - g["HF"]) < 1e-9 and abs(e["MP2c"] - g["MP2c"]) < 1e-9
    assert abs(e["CCSD(T)c"] - g["CCSD(T)c"]) < 1e-9
