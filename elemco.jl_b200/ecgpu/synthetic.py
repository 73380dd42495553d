"""Seeded synthetic closed-shell systems with molecule-like DF spectra.

Stands in for the density-fitted integrals of a real molecule when no integral
engine is available: ``B[p,q,Q]`` is symmetric in (p,q) with a geometric
decay of the auxiliary weights (1 -> 1e-6 over Q), orbital energies are drawn
uniformly from [-1.4, -0.4] Eh (occupied) and [0.1, 4.0] Eh (virtual), and the
one-electron matrix is chosen so that the Fock matrix built from B is exactly
diag(eps) — a canonical Hartree-Fock reference.  B is scaled so that the MP2
correlation energy is -0.05 Eh per occupied orbital (water: -0.2 Eh for four
valence pairs), which keeps CCSD well conditioned at every size.

Shapes of the named workloads (active orbitals after freezing O/C 1s):
  (H2O)_2/cc-pVDZ  o=8  v=38  nQ=168
  (H2O)_3/cc-pVDZ  o=12 v=57  nQ=252
  (H2O)_4/cc-pVDZ  o=16 v=76  nQ=336
  (H2O)_6/cc-pVTZ  o=24 v=318 nQ=846
  C_nH_2n+2/cc-pVDZ, n=6..10: 14n+5(2n+2) basis functions, o=3n+1 (C 1s
  frozen), v = nbf-(4n+1), nQ ~ 3.46 nbf (cc-pVDZ-RI)
"""
import numpy as np

WORKLOADS = {
    "h2o_vdz": (5, 19, 84),
    "h2o2_vdz": (8, 38, 168),
    "h2o3_vdz": (12, 57, 252),
    "h2o4_vdz": (16, 76, 336),
    "h2o6_vtz": (24, 318, 846),
    "c6h14_vdz": (19, 129, 532),
    "c7h16_vdz": (22, 149, 616),
    "c8h18_vdz": (25, 169, 700),
    "c9h20_vdz": (28, 189, 784),
    "c10h22_vdz": (31, 209, 868),
}


def _mp2(B, eps, no):
    o, v = slice(0, no), slice(no, None)
    ovov = np.einsum("iaQ,jbQ->iajb", B[o, v, :], B[o, v, :], optimize=True)
    D = (eps[o][:, None, None, None] - eps[v][None, :, None, None]
         + eps[o][None, None, :, None] - eps[v][None, None, None, :])
    return float(np.sum(ovov * (2.0 * ovov - ovov.transpose(0, 3, 2, 1)) / D))


def make_system(no, nv, nq, seed=1234, emp2_per_occ=-0.05):
    """Return (B[p,q,Q] Fortran-ordered, h1, e0, eps)."""
    rng = np.random.default_rng(seed)
    n = no + nv
    eps = np.concatenate([np.sort(rng.uniform(-1.4, -0.4, no)),
                          np.sort(rng.uniform(0.1, 4.0, nv))])
    w = 10.0 ** (-6.0 * np.arange(nq) / max(nq - 1, 1))
    B = np.empty((n, n, nq), order="F")
    for q in range(nq):
        G = rng.standard_normal((n, n))
        B[:, :, q] = w[q] * (G + G.T) / np.sqrt(2.0 * n)
    # MP2 energy scales with the 4th power of B
    B *= (emp2_per_occ * no / _mp2(B, eps, no)) ** 0.25
    # Fock from B:  f = h + 2 J - K  with the occupied block; choose h so f = diag(eps)
    o = slice(0, no)
    Jq = np.einsum("kkQ->Q", B[o, o, :])
    J = np.einsum("pqQ,Q->pq", B, Jq)
    K = np.einsum("pkQ,kqQ->pq", B[:, o, :], B[o, :, :])
    h1 = np.asfortranarray(np.diag(eps) - 2.0 * J + K)
    return B, h1, 0.0, eps


def make_workload(name, seed=1234, no=None):
    """(B, h1, e0, no) of a named workload; `no` overrides its occupied count."""
    no0, nv, nq = WORKLOADS[name]
    no = no or no0
    B, h1, e0, eps = make_system(no, nv, nq, seed=seed)
    return B, h1, e0, no
