"""The numpy checker of the device DF factors (oracle/dfhf.py) against the
textbook definitions on CPU: with 4-index integrals (mn|ls) = sum_L AAL[m,n,L]
AAL[l,s,L] and the density D = C C^T of the occupied orbitals, the closed-shell
Fock matrix of gen_dffock (src/scf/fockfactory.jl:202-245) is
F = h + 2 sum_ls (mn|ls) D_ls - sum_ls (ml|ns) D_ls, and the MO factors of
generate_3idx_integrals (src/integrals/dftools.jl:92-136) reproduce the MO
integrals (pq|rs) = sum_mnls C_mp C_nq (mn|ls) C_lr C_ss."""
import numpy as np

from oracle import dfhf as O


def _factors(rng, n, naux, nL):
    B3 = rng.standard_normal((n, n, naux))
    B3 = B3 + B3.transpose(1, 0, 2)  # (mn|P) = (nm|P)
    M = rng.standard_normal((naux, nL))
    return B3, M


def test_df_fock_matches_four_index_definition():
    rng = np.random.default_rng(21)
    n, naux, nL, nocc = 9, 14, 11, 3
    B3, M = _factors(rng, n, naux, nL)
    AAL = O.df_factors(B3, M)
    assert np.allclose(AAL, np.einsum("mnP,PL->mnL", B3, M))
    eri = np.einsum("mnL,lsL->mnls", AAL, AAL)
    h = rng.standard_normal((n, n))
    h = h + h.T
    C = rng.standard_normal((n, nocc))
    D = C @ C.T
    F = h + 2.0 * np.einsum("mnls,ls->mn", eri, D) - np.einsum("mlns,ls->mn", eri, D)
    Fo = O.df_fock(h, AAL, C)
    assert np.abs(Fo - F).max() < 1e-12 * np.abs(F).max()
    assert np.abs(Fo - Fo.T).max() < 1e-12 * np.abs(F).max()
    assert np.array_equal(O.df_fock(h, AAL, np.zeros((n, 0))), h)


def test_df_mo_matches_four_index_transform():
    rng = np.random.default_rng(22)
    n, naux, nL, nmo = 8, 12, 10, 6
    B3, M = _factors(rng, n, naux, nL)
    AAL = O.df_factors(B3, M)
    C = rng.standard_normal((n, nmo))
    B = O.df_mo(AAL, C)
    assert B.shape == (nmo, nmo, nL)
    eri_ao = np.einsum("mnL,lsL->mnls", AAL, AAL)
    eri_mo = np.einsum("mp,nq,mnls,lr,st->pqrt", C, C, eri_ao, C, C, optimize=True)
    assert np.abs(np.einsum("pqL,rtL->pqrt", B, B) - eri_mo).max() < 1e-11 * np.abs(eri_mo).max()
