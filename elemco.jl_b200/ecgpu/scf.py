"""Closed-shell DF-HF and the density-fitted integrals of the CC path.

* :func:`dfhf` restates ``dfhf`` (src/scf/dfhf.jl:24-94): the Fock matrix is
  built with a ``jkfit`` auxiliary basis as ``gen_dffock`` does
  (src/scf/fockfactory.jl:202-245), DIIS on the Fock matrix with the
  commutator ``S D F - F D S`` as residual (plain dot, src/solvers/diis.jl),
  convergence on its squared norm (``scf.thr`` 1e-10) and on the energy change
  (``scf.thren``, default sqrt(thr)/10), the generalized eigenproblem
  ``F C = S C eps`` each iteration.  Start orbitals: a superposition of
  atomic densities (the reference's default ``guess = :SAD``; here the atoms'
  spherically averaged DF-HF densities in the molecule's own basis), or the
  core Hamiltonian (``guess = :HCORE``).
* :func:`dfints` restates the closed-shell ``generate_integrals`` of
  ``dfdump`` (src/integrals/dfdump.jl:29-119): the frozen core
  (``core = :large``, first-row 1s), the three-index factors of the active
  orbitals with the ``mpfit`` basis (the two-electron integrals of the CC
  path), and the one-electron part corrected so that the Fock matrix built
  from them equals the ``jkfit`` DF-HF Fock matrix:
  ``int1 = F_jkfit - F_mpfit`` and
  ``int0 = E_nuc + sum_occ h_ii + sum_core F_ii - sum_active-occ int1_ii``.

The Gaussian integrals (overlap, kinetic, nuclear attraction, (P|Q), (mn|P))
come from libecgpu's GPU integral engine.  The fitted factors
AAL[m,n,L] = sum_P (mn|P) M[P,L] stay on the device (``ecg_df_*``), where the
Fock builds and the MO transform run; the host keeps the n x n matrices
(the generalized eigenproblem, DIIS on the Fock matrix).  The fitting
metric's inverse square root is the pivoted Cholesky of ``sqrtinvchol``
(src/tools/tensortools.jl:377-389, tolerance ``cholesky.thred`` 1e-6).
"""
import math

import numpy as np

from . import basis as Bm
from ._lib import ECG_INT_DIPOLE, ECG_INT_KINETIC, ECG_INT_NUCLEAR, ECG_INT_OVERLAP

__all__ = ["sqrtinvchol", "AOIntegrals", "dfhf", "dfints", "DFHFResult"]


def sqrtinvchol(A, tol=1e-6):
    """M with M M^T = A^{-1} (on the span kept): pivoted Cholesky with the
    largest remaining diagonal as pivot, stopping below `tol`; M = P U^{-1}
    (minimum-norm solve when columns were dropped)."""
    A = np.array(A, dtype=float)
    n = A.shape[0]
    piv = np.arange(n)
    U = np.zeros((n, n))
    d = np.diag(A).copy()
    r = 0
    W = A.copy()
    for k in range(n):
        j = k + int(np.argmax(d[piv[k:]]))
        if d[piv[j]] <= tol:
            break
        piv[[k, j]] = piv[[j, k]]
        p = piv[k]
        U[k, p] = math.sqrt(d[p])
        rest = piv[k + 1:]
        U[k, rest] = (W[p, rest] - U[:k, p] @ U[:k, rest]) / U[k, p]
        d[rest] -= U[k, rest] ** 2
        r = k + 1
    Ur = U[:r][:, piv]  # r x n in pivoted column order (upper triangular in its first r)
    if r == n:
        Minv = np.linalg.solve(Ur, np.eye(n))
    else:
        Minv = np.linalg.lstsq(Ur, np.eye(r), rcond=None)[0]
    M = np.zeros((n, r))
    M[piv] = Minv
    return M


class AOIntegrals:
    """AO integrals of a molecule in a basis, computed on the GPU."""

    def __init__(self, ctx, mol, ao="cc-pvdz", library=None):
        self.ctx, self.mol = ctx, mol
        self.ao = Bm.shells(Bm.load(ao, library), mol.symbols, mol.xyz)
        self.library = library
        self.S = ctx.int1e(ECG_INT_OVERLAP, self.ao)
        self.h = (ctx.int1e(ECG_INT_KINETIC, self.ao)
                  + ctx.int1e(ECG_INT_NUCLEAR, self.ao, mol.charges, mol.xyz))
        self.enuc = mol.nuclear_repulsion()

    def fitted(self, fit, thred=1e-6):
        """Device factors (:class:`ecgpu.context.DFFactors`)
        AAL[m, n, L] = sum_P (mn|P) M[P, L] with M M^T = (P|Q)^{-1}
        (generate_AO_DF_integrals, src/integrals/dftools.jl:28-84)."""
        fb = Bm.shells(Bm.load(fit, self.library), self.mol.symbols, self.mol.xyz)
        M = sqrtinvchol(self.ctx.int2c2e(fb), thred)
        return self.ctx.df_factors(self.ao, fb, M)

    def dipole(self, origin=(0.0, 0.0, 0.0)):
        return self.ctx.int1e(ECG_INT_DIPOLE, self.ao, origin=origin)


def df_fock(h, AAL, Cocc):
    """gen_dffock closed shell (src/scf/fockfactory.jl:202-245):
    F = h + 2 J - K with the device DF factors AAL (ecg_df_fock)."""
    return AAL.fock(h, Cocc)


class _Diis:
    """DIIS on the Fock matrix (src/solvers/diis.jl:246-305, plain dot, SVD
    solve with singular values below eps*smax dropped)."""

    def __init__(self, maxdiis=6, resthr=10.0):
        self.maxdiis, self.resthr = maxdiis, resthr
        self.v, self.r = [None] * maxdiis, [None] * maxdiis
        self.next, self.ndim = 0, 0
        self.B = np.zeros((maxdiis + 1, maxdiis + 1))

    def perform(self, vec, res):
        if self.ndim < self.maxdiis:
            self.ndim += 1
        ith, nd = self.next, self.ndim
        self.v[ith], self.r[ith] = vec.copy(), res.copy()
        this = float(np.sum(res * res))
        for i in range(nd):
            self.B[i, ith] = self.B[ith, i] = this if i == ith else float(np.sum(res * self.r[i]))
            self.B[i, nd] = self.B[nd, i] = -1.0
        self.B[nd, nd] = 0.0
        rhs = np.zeros(nd + 1)
        rhs[nd] = -1.0
        U, s, Vt = np.linalg.svd(self.B[:nd + 1, :nd + 1])
        k = int(np.sum(s >= np.finfo(float).eps * s[0]))
        c = Vt[:k].T @ ((U[:, :k].T @ rhs) / s[:k])
        if nd == 1 and self.next == 0 and this > self.resthr:
            self.ndim = 0
            return vec
        if nd < self.maxdiis:
            self.next = nd
        else:
            cmin = 1e10
            for i in range(nd):
                if abs(c[i]) < cmin and (i != ith or nd == 1):
                    cmin, self.next = abs(c[i]), i
        return sum(c[i] * self.v[i] for i in range(nd))


class DFHFResult:
    def __init__(self, E, C, eps, nocc, iterations, converged, F, ints, AAL):
        self.E, self.C, self.eps, self.nocc = E, C, eps, nocc
        self.iterations, self.converged = iterations, converged
        self.F, self.ints, self.AAL = F, ints, AAL


# Spherically averaged ground-state occupations of the atoms' lowest orbitals
# (1s; 2s; 2p x 3) for the atomic-density guess.
_ATOM_OCC = {"H": [1.0], "C": [2.0, 2.0] + [2.0 / 3.0] * 3, "N": [2.0, 2.0, 1.0, 1.0, 1.0],
             "O": [2.0, 2.0] + [4.0 / 3.0] * 3}


def _atomic_density(ctx, sym, ao, jkfit, thred, library, maxit=100):
    """Spin-restricted, spherically averaged DF-HF density of an isolated atom
    in its basis (fractional occupations of the 2p shell)."""
    from .molecules import Molecule
    atom = Molecule([sym], [[0.0, 0.0, 0.0]])
    ints = AOIntegrals(ctx, atom, ao, library)
    AAL = ints.fitted(jkfit, thred)
    occ = np.array(_ATOM_OCC[sym])
    eps, C = _geneig(ints.h, ints.S)
    diis = _Diis()
    D = None
    for _ in range(maxit):
        X = C[:, :len(occ)] * np.sqrt(occ / 2.0)
        Dn = 2.0 * X @ X.T
        if D is not None and np.abs(Dn - D).max() < 1e-10:
            break
        D = Dn
        F = df_fock(ints.h, AAL, X)
        SDF = ints.S @ D @ F
        F = diis.perform(F, SDF - SDF.T)
        eps, C = _geneig(F, ints.S)
    AAL.close()
    return D


def sad_guess(ctx, mol, ao, jkfit, thred=1e-6, library=None):
    """Superposition of atomic densities (the reference's default start,
    ``scf.guess = :SAD``, src/scf/orbtools.jl), each atom's density computed
    in the molecule's basis; returns the block-diagonal AO density."""
    shells = Bm.shells(Bm.load(ao, library), mol.symbols, mol.xyz)
    fa = shells.function_atoms()
    D = np.zeros((shells.nbf, shells.nbf))
    cache = {}
    for a, sym in enumerate(mol.symbols):
        if sym not in cache:
            cache[sym] = _atomic_density(ctx, sym, ao, jkfit, thred, library)
        idx = np.where(fa == a)[0]
        D[np.ix_(idx, idx)] = cache[sym]
    return D


def _density_factor(D):
    """X with D = 2 X X^T for a positive semidefinite density D."""
    w, V = np.linalg.eigh(0.5 * (D + D.T))
    keep = w > 1e-12
    return V[:, keep] * np.sqrt(w[keep] / 2.0)


def dfhf(ctx, mol, ao="cc-pvdz", jkfit="cc-pvtz-jkfit", thr=1e-10, thren=-1.0, maxit=50,
         thred=1e-6, library=None, log=None, guess="sad"):
    """Closed-shell DF-HF (src/scf/dfhf.jl:24-94); guess "sad" (atomic
    densities) or "hcore" (core Hamiltonian)."""
    if mol.nelec % 2:
        raise ValueError("closed-shell DF-HF needs an even number of electrons")
    ints = AOIntegrals(ctx, mol, ao, library)
    AAL = ints.fitted(jkfit, thred)
    S, h = ints.S, ints.h
    nocc = mol.nelec // 2
    if thren < 0.0:
        thren = math.sqrt(thr) * 0.1
    if guess == "sad":
        X = _density_factor(sad_guess(ctx, mol, ao, jkfit, thred, library))
        eps, C = _geneig(df_fock(h, AAL, X), S)
    elif guess == "hcore":
        eps, C = _geneig(h, S)
    else:
        raise ValueError("guess must be 'sad' or 'hcore'")
    diis = _Diis()
    E = prev = 0.0
    conv = False
    it = 0
    F = h
    for it in range(1, maxit + 1):
        Co = C[:, :nocc]
        F = df_fock(h, AAL, Co)
        E = float(np.einsum("pi,pq,qi->", Co, F + h, Co)) + ints.enuc
        dE = E - prev
        prev = E
        D = Co @ Co.T
        SDF = S @ D @ F
        dF = SDF - SDF.T
        var = float(np.sum(dF * dF))
        if log:
            log(it, E, dE, var)
        if abs(dE) < thren and var < thr:
            conv = True
            break
        Fx = diis.perform(F, dF)
        eps, C = _geneig(Fx, S)
    return DFHFResult(E, C, eps, nocc, it, conv, F, ints, AAL)


def _geneig(F, S):
    """F C = S C eps with S-orthonormal C (symmetric-orthogonalised)."""
    s, U = np.linalg.eigh(S)
    X = U / np.sqrt(s)
    e, V = np.linalg.eigh(X.T @ F @ X)
    return e, X @ V


def dfints(hf, mpfit="cc-pvdz-mpfit", jkfit="cc-pvtz-jkfit", ncore=None, thred=1e-6):
    """The CC path's integrals from converged DF-HF orbitals (dfdump.jl:29-119).

    Returns (B[p,q,L] over the active orbitals (F-ordered), int1, int0, nocc
    active, reference energy), ready for ``Context.set_system``."""
    ints, C, nocc = hf.ints, hf.C, hf.nocc
    mol = ints.mol
    nc = mol.ncore() if ncore is None else int(ncore)
    act = C[:, nc:]
    n = act.shape[1]
    # mpfit factors of the active orbitals (generate_3idx_integrals,
    # src/integrals/dftools.jl:92-136), on the device
    AAL = ints.fitted(mpfit, thred)
    try:
        B = AAL.mo(act)
        # Fock matrix of the active space from the mpfit integrals,
        # 2 J - K over the active occupied orbitals, in the AO basis on the
        # device, then transformed
        no = nocc - nc
        f_mp = act.T @ AAL.fock(np.zeros_like(ints.h), act[:, :no]) @ act
    finally:
        AAL.close()
    # jkfit DF-HF Fock matrix of the orbitals (all occupied, core included)
    Fjk = C.T @ df_fock(ints.h, hf.AAL, C[:, :nocc]) @ C
    int1 = Fjk[nc:, nc:] - f_mp
    hmo = C.T @ ints.h @ C
    hii = float(np.sum(np.diag(hmo)[:nocc]))
    int0 = ints.enuc + hii + float(np.sum(np.diag(Fjk)[:nc])) - float(np.sum(np.diag(int1)[:no]))
    eref = ints.enuc + hii + float(np.sum(np.diag(Fjk)[:nocc]))
    return B, np.asfortranarray(int1), int0, no, eref
