"""Coupled cluster on real molecules: integrals from the GPU integral engine
(DF-HF + dfdump on the seeded water-cluster geometries), the CC path checked
against the oracle on the same factors (FP64) and mixed precision against
FP64 (1 microhartree)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def test_water_dimer_ccsd_t_matches_oracle():
    import ecgpu
    from ecgpu.molecular import molecular_workload
    with ecgpu.Context(0) as c:
        B, h1, e0, no, info = molecular_workload(c, "h2o2_vdz")
        assert B.shape == (46, 46, 168) and no == 8
        S = O.System.from_df(np.ascontiguousarray(np.transpose(B, (2, 0, 1))), h1, e0, no)
        f = O.gen_fock(S)
        c.set_system(B, h1, e0, no)
        _, _, ehf = c.fock()
        assert abs(ehf - info["E_HF"]) < 1e-10
        assert abs(ehf - O.hf_energy(S, f)) < 1e-10
        _, T1, T2 = c.mp2()
        r = c.cc_solve(T1, T2)
        Eo, T1o, T2o, it, conv = O.cc_iterations(S, *O.mp2(S, f)[1:], f)
        assert r["converged"] and conv and r["iterations"] == it
        assert abs(r["E"] - Eo) < 1e-10
        et, etb = c.pert_t()
        eto, etbo = O.pert_t(S, r["T1"], r["T2"], f)
        assert abs(et - eto) < 1e-11 and abs(etb - etbo) < 1e-11


@pytest.mark.parametrize("dc", [False, True])
def test_water_trimer_mixed_within_1_uEh(dc):
    """(H2O)_3/cc-pVDZ (configuration 2): mixed-precision CCSD/DCSD and (T)
    within 1 microhartree of FP64."""
    import ecgpu
    from ecgpu.molecular import molecular_workload
    with ecgpu.Context(0) as c:
        B, h1, e0, no, _ = molecular_workload(c, "h2o3_vdz")
    out = {}
    for prec in (ecgpu.ECG_PREC_FP64, ecgpu.ECG_PREC_MIXED):
        with ecgpu.Context(0) as c:
            c.set_precision(prec)
            c.set_system(B, h1, e0, no)
            _, T1, T2 = c.mp2()
            r = c.cc_solve(T1, T2, dc=dc)
            assert r["converged"]
            out[prec] = (r["E"], c.pert_t()[0])
    (e64, t64), (emx, tmx) = out[ecgpu.ECG_PREC_FP64], out[ecgpu.ECG_PREC_MIXED]
    assert abs(emx - e64) < 1e-6 and abs(tmx - t64) < 1e-6, (emx - e64, tmx - t64)
