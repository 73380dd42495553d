"""The density-fitted CPU restatement (oracle/dfcc.py) against the 4-index
oracle (oracle/ccref.py) on the same factors — CPU only.  The DF form is the
CPU baseline at sizes where the 4-index integrals do not fit in memory."""
import numpy as np
import pytest

import oracle as O
from oracle.dfcc import DFCC


def _df_system(no, nv, nq, seed=3):
    from ecgpu.synthetic import make_system
    B, h1, e0, _ = make_system(no, nv, nq, seed=seed)
    S = O.System.from_df(np.ascontiguousarray(np.transpose(B, (2, 0, 1))), h1, e0, no)
    return B, h1, e0, S


@pytest.mark.parametrize("dc", [False, True])
def test_df_residual_matches_4index(dc):
    B, h1, e0, S = _df_system(3, 11, 20)
    f = O.gen_fock(S)
    rng = np.random.default_rng(1)
    _, T1, T2 = O.mp2(S, f)
    T1 = T1 + 0.01 * rng.standard_normal(T1.shape)
    X = 0.01 * rng.standard_normal(T2.shape)
    T2 = T2 + X + X.transpose(1, 0, 3, 2)
    d = DFCC(B, h1, e0, 3, dc=dc, ablock=4)
    assert np.abs(d.fock - f).max() < 1e-13
    d.start(T1, T2)
    for name, _, fn in d._tasks[:-1]:  # everything but the update
        fn()
    R1o, R2o = O.cc_resid(S, T1, T2, dc=dc)
    assert np.abs(d.R1 - R1o).max() < 1e-12
    assert np.abs(d.R2 - R2o).max() < 1e-12


def test_df_iterations_and_pert_t_match_4index(h2o_df):
    Bf, S = h2o_df
    f = O.gen_fock(S)
    d = DFCC(np.asarray(Bf), S.h, S.e0, S.no)
    e_mp2 = d.mp2()
    assert abs(e_mp2 - O.mp2(S, f)[0]) < 1e-12
    d.start()
    E, it, conv = d.solve()
    Eo, T1o, T2o, ito, convo = O.cc_iterations(S, *O.mp2(S, f)[1:], f)
    assert conv and convo and it == ito
    assert abs(E - Eo) < 1e-10 and np.abs(d.T2 - T2o).max() < 1e-9
    et, etb = d.pert_t(d.T1, d.T2)
    eto, etbo = O.pert_t(S, d.T1, d.T2, f)
    assert abs(et - eto) < 1e-12 and abs(etb - etbo) < 1e-12
    # a subset of triplets: the partial sums add up to the whole
    trip = list(O.ccref._triplets(S.no))
    p1 = d.pert_t(d.T1, d.T2, trip[:5])
    p2 = d.pert_t(d.T1, d.T2, trip[5:])
    assert abs(p1[0] + p2[0] - et) < 1e-13
