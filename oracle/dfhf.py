"""Density-fitted Fock build and MO transform in numpy — the checker for the
device DF factors (ecg_df_create / ecg_df_fock / ecg_df_mo).

TEST INFRASTRUCTURE ONLY.  Restates, on full in-memory arrays:

* generate_AO_DF_integrals (ElemCo.jl src/integrals/dftools.jl:28-84):
  AAL[m,n,L] = sum_P (mn|P) M[P,L];
* gen_dffock, closed shell (src/scf/fockfactory.jl:202-245):
  LoA[L,j,n] = sum_m AAL[m,n,L] C[m,j], cL[L] = sum_{j,n} LoA[L,j,n] C[n,j],
  F = h - sum_{L,j} LoA[L,j,m] LoA[L,j,n] + 2 sum_L AAL[m,n,L] cL[L];
* generate_3idx_integrals (src/integrals/dftools.jl:92-136):
  mmL[p,q,L] = sum_{m,n} C[m,p] AAL[m,n,L] C[n,q].
"""
import numpy as np

__all__ = ["df_factors", "df_fock", "df_mo"]


def df_factors(B3, M):
    """AAL from (mn|P) (n, n, naux) and M (naux, nL)."""
    return np.einsum("mnP,PL->mnL", B3, M, optimize=True)


def df_fock(h, AAL, Cocc):
    LoA = np.einsum("mnL,mj->Ljn", AAL, Cocc, optimize=True)
    cL = np.einsum("Ljn,nj->L", LoA, Cocc, optimize=True)
    F = h - np.einsum("Ljm,Ljn->mn", LoA, LoA, optimize=True)
    F += 2.0 * np.einsum("mnL,L->mn", AAL, cL, optimize=True)
    return F


def df_mo(AAL, C):
    mAL = np.einsum("mp,mnL->pnL", C, AAL, optimize=True)
    return np.einsum("pnL,nq->pqL", mAL, C, optimize=True)
