"""numpy restatement of ElemCo.jl's closed-shell coupled-cluster path.

TEST INFRASTRUCTURE ONLY (the checker for the CUDA library; see package
docstring). Every function cites the reference file:line it restates; paths
are relative to the ElemCo.jl project root.

Conventions (as in the reference):
  * ``V[p,q,r,s] = <pq|rs> = (pr|qs)`` physicists' notation, all orbitals
    (``src/integrals/dump.jl:100``).  From DF factors ``B[Q,p,q]`` with
    ``(pq|rs) = sum_Q B[Q,p,q] B[Q,r,s]``: ``V = einsum('Qpr,Qqs->pqrs')``
    (``src/integrals/dfdump.jl:65-81``).
  * ``T1[a,i]``, ``T2[a,b,i,j]``; occupied orbitals first (``o``), then
    virtuals (``v``).  Arrays use the reference's index order; numpy storage
    order is irrelevant here.
"""
import math

import numpy as np

__all__ = [
    "System", "Options", "read_fixture", "gen_fock", "hf_energy", "mp2",
    "dressed_ints", "calc_D2", "cc_resid", "hylleraas", "doubles_energy",
    "singles_energy", "doubles_norm", "singles_norm", "cs_doubles_dot",
    "cs_singles_dot", "update_singles", "update_doubles", "Diis",
    "cc_iterations", "pert_t", "lambda_pert_t", "vector_times_jacobian",
    "one_rdm", "lambda_iterations", "correlation_norm", "ccdriver",
    "cholesky_df", "contra2covariant",
]


def _es(sub, *ops):
    return np.einsum(sub, *ops, optimize=True)


class Options:
    """Defaults of ``CcOptions``/``DiisOptions`` (``src/infos/options.jl:128-282``)."""

    def __init__(self, **kw):
        self.thr = 1.0e-10      # options.jl:130 (squared residual norm)
        self.conven = 0.1       # :132
        self.maxit = 50         # :134
        self.shifts = 0.15      # :136
        self.shiftp = 0.2       # :138
        self.maxdiis = 6        # options.jl:274
        self.resthr = 10.0      # :276
        # dot product of the CC DIIS: "cs" = the closed-shell custom dots
        # passed to perform! (cc.jl:2498-2499,2598; ElemCo.jl >= 0.13.0,
        # CHANGELOG.md:76); "plain" = the unweighted dot weighted_dot falls back
        # to (diis.jl:155-167), which closed-shell CC used before 0.13.0
        self.diis_dot = "cs"
        for k, v in kw.items():
            if not hasattr(self, k):
                raise KeyError(k)
            setattr(self, k, v)


class System:
    """Closed-shell integrals in the MO basis (the reference's ``EC.fd``)."""

    def __init__(self, h, V, e0, nocc, st=False):
        self.h = np.asarray(h, dtype=np.float64)
        self.V = np.asarray(V, dtype=np.float64)
        self.e0 = float(e0)
        self.n = self.h.shape[0]
        self.no = int(nocc)
        self.nv = self.n - self.no
        self.st = bool(st)
        self.sl = {"o": slice(0, self.no), "v": slice(self.no, self.n),
                   "m": slice(0, self.n), ":": slice(0, self.n)}

    @classmethod
    def from_df(cls, B, h, e0, nocc):
        B = np.asarray(B, dtype=np.float64)
        V = _es("Qpr,Qqs->pqrs", B, B)
        return cls(h, V, e0, nocc)

    def ints2(self, spaces):
        """Block ``<s1 s2|s3 s4>`` (``src/tools/tensortools.jl:295-310``)."""
        return self.V[tuple(self.sl[c] for c in spaces)]

    def ints1(self, spaces):
        return self.h[self.sl[spaces[0]], self.sl[spaces[1]]]


def read_fixture(path):
    """Build a :class:`System` from a golden ``.npz`` integral list.

    Integral semantics of ``set_int2!``/``set_int1!``
    (``src/integrals/dump.jl:473-560``): line ``(i1 i2|i3 i4)`` is stored as
    ``<i1 i3|i2 i4>`` with 8-fold symmetry, or only particle symmetry when
    the dump is similarity transformed (``ST>0``).
    """
    z = np.load(path)
    n = int(z["norb"])
    st = int(z["st"]) > 0
    V = np.zeros((n, n, n, n))
    h = np.zeros((n, n))
    for (i1, i2, i3, i4), x in zip(z["idx"].astype(int) - 1, z["val"]):
        if i4 >= 0:
            V[i1, i3, i2, i4] = x
            V[i3, i1, i4, i2] = x
            if not st:
                V[i1, i4, i2, i3] = x
                V[i2, i3, i1, i4] = x
                V[i2, i4, i1, i3] = x
                V[i4, i1, i3, i2] = x
                V[i3, i2, i4, i1] = x
                V[i4, i2, i3, i1] = x
        elif i2 >= 0:
            h[i1, i2] = x
            if not st:
                h[i2, i1] = x
    nelec = int(z["nelec"])
    return System(h, V, float(z["e0"]), nelec // 2, st=st)


def cholesky_df(V, tol=1e-12):
    """Pivoted Cholesky of the (pr|qs) supermatrix -> ``B[Q,p,r]``.

    Restates ``calc_integrals_decomposition`` (``src/integrals/decomptools.jl:22-52``,
    Cholesky with row-maximum pivoting and tolerance ``tol``).
    """
    n = V.shape[0]
    M = V.transpose(0, 2, 1, 3).reshape(n * n, n * n).copy()   # (pr|qs)
    d = np.diag(M).copy()
    L = []
    while True:
        k = int(np.argmax(d))
        if d[k] <= tol:
            break
        col = M[:, k].copy()
        for l in L:
            col -= l * l[k]
        col /= math.sqrt(d[k])
        L.append(col)
        d -= col * col
        d[k] = 0.0
    return np.array(L).reshape(len(L), n, n)


# ---------------------------------------------------------------- Fock / HF


def gen_fock(S):
    """``gen_fock`` (``src/scf/fockfactory.jl:27-30``)."""
    o = S.sl["o"]
    return (S.h + 2.0 * _es("piqi->pq", S.V[:, o, :, o])
            - _es("piiq->pq", S.V[:, o, o, :]))


def hf_energy(S, fock):
    """``calc_HF_energy`` closed shell (``src/cc/cctools.jl:65-72``)."""
    eps = np.diag(fock)
    return float(np.sum(eps[S.sl["o"]]) + np.trace(S.ints1("oo")) + S.e0)


# ---------------------------------------------------------------- updates


def update_singles(R1, eo, ev, shift):
    """``update_singles`` (``src/cc/cctools.jl:198-207``)."""
    return -R1 / (ev[:, None] - eo[None, :] + shift)


def update_doubles(R2, eo, ev, shift):
    """``update_doubles`` (``src/cc/cctools.jl:228-240``)."""
    D = (ev[:, None, None, None] + ev[None, :, None, None]
         - eo[None, None, :, None] - eo[None, None, None, :] + shift)
    return -R2 / D


def singles_norm(T1):
    """``calc_singles_norm`` (``cctools.jl:410-413``)."""
    return 2.0 * float(np.sum(T1 * T1))


def doubles_norm(T2):
    """``calc_doubles_norm`` (``cctools.jl:477-480``)."""
    return float(np.sum((2.0 * T2 - T2.transpose(1, 0, 2, 3)) * T2))


def contra_singles_norm(T1):
    """``calc_contra_singles_norm`` (``cctools.jl:420-423``)."""
    return 0.5 * float(np.sum(T1 * T1))


def contra_doubles_norm(T2):
    """``calc_contra_doubles_norm`` (``cctools.jl:487-490``)."""
    return float(np.sum((2.0 * T2 + T2.transpose(1, 0, 2, 3)) * T2)) / 3.0


def cs_singles_dot(A, B):
    """``calc_cs_singles_dot`` (``cctools.jl:453-456``)."""
    return 2.0 * float(np.sum(A * B))


def cs_doubles_dot(A, B):
    """``calc_cs_doubles_dot`` (``cctools.jl:511-515``)."""
    return float(np.sum((2.0 * A - A.transpose(1, 0, 2, 3)) * B))


def contra2covariant(U2):
    """``contra2covariant`` (``cctools.jl:935-938``)."""
    return (2.0 * U2 + U2.transpose(1, 0, 2, 3)) / 3.0


# ---------------------------------------------------------------- energies


def singles_energy(S, T1, fock, fock_only=False):
    """``calc_singles_energy`` (``src/cc/cc.jl:97-115``)."""
    E = 0.0
    if not fock_only:
        oovv = S.ints2("oovv")
        d = _es("ai,bj,ijab->", T1, T1, oovv)
        ex = _es("bi,aj,ijab->", T1, T1, oovv)
        E = (d - ex) + d
    o, v = S.sl["o"], S.sl["v"]
    E += 2.0 * float(np.sum(T1 * fock[o, v].T))
    return float(E)


def doubles_energy(S, T2):
    """``calc_doubles_energy`` (``cc.jl:157-168``)."""
    oovv = S.ints2("oovv")
    d = _es("abij,ijab->", T2, oovv)
    ex = _es("baij,ijab->", T2, oovv)
    return float((d - ex) + d)


def hylleraas(S, T1, T2, R1, R2, fock):
    """``calc_hylleraas`` (``cc.jl:195-249``); returns (E, projected E)."""
    oovv = S.ints2("oovv")
    o, v = S.sl["o"], S.sl["v"]
    d = _es("ai,bj,ijab->", T1, T1, oovv)
    ex = _es("bi,aj,ijab->", T1, T1, oovv)
    ET1 = 2.0 * d - ex
    pd = _es("abij,ijab->", T2, oovv)
    pex = _es("baij,ijab->", T2, oovv)
    rd = float(np.sum(T2 * R2))
    rex = _es("baij,abij->", T2, R2)
    ET2 = 2.0 * (pd + rd) - (pex + rex)
    pET2 = 2.0 * pd - pex
    pET1 = 2.0 * float(np.sum(fock[o, v].T * T1))
    rET1 = 2.0 * float(np.sum(R1 * T1))
    ET1 += pET1 + rET1
    E = ET2 + ET1
    pE = pET2 + pET1 + (2.0 * d - ex)
    return float(E), float(pE)


def mp2(S, fock):
    """``calc_MP2`` (``cc.jl:1011-1024``): start amplitudes and energy."""
    eps = np.diag(fock)
    eo, ev = eps[S.sl["o"]], eps[S.sl["v"]]
    T2 = update_doubles(S.ints2("vvoo"), eo, ev, 0.0)
    E = doubles_energy(S, T2)
    T1 = update_singles(fock[S.sl["v"], S.sl["o"]], eo, ev, 0.0)
    E += singles_energy(S, T1, fock, fock_only=True)
    return E, T1, T2


# ---------------------------------------------------------------- residual


def dressed_ints(S, T1):
    """T1-dressed integrals and Fock matrix.

    ``calc_dressed_ints`` (``src/cc/cc.jl:453-774``) builds each dressed block
    from half-dressed ones; the blocks it produces equal one similarity
    transform of all four indices, bra indices with ``(1 - t)`` and ket
    indices with ``(1 + t)``, where ``t[v,o] = T1`` (zero elsewhere):
    ``d_pqrs = sum L[p,p'] L[q,q'] <p'q'|r's'> R[r',r] R[s',s]``.  The
    one-electron part ``dh`` is ``dress_fock_closedshell`` (``cc.jl:777-795``)
    and the dressed Fock matrix ``df`` follows ``cc.jl:797-815``.
    """
    n = S.n
    t = np.zeros((n, n))
    t[S.sl["v"], S.sl["o"]] = T1
    L = np.eye(n) - t
    R = np.eye(n) + t
    Vd = _es("pP,qQ,PQRS,Rr,Ss->pqrs", L, L, S.V, R, R)
    dh = L @ S.h @ R
    o = S.sl["o"]
    df = dh + 2.0 * _es("pkqk->pq", Vd[:, o, :, o]) - _es("pkkq->pq", Vd[:, o, o, :])
    return Vd, dh, df


def calc_D2(S, T1, T2):
    """``calc_D2`` (``cc.jl:1085-1113``) without the diagonal scaling."""
    n, no = S.n, S.no
    o, v = S.sl["o"], S.sl["v"]
    D2 = np.zeros((n, n, no, no))
    D2[v, v] = T2 + _es("ai,bj->abij", T1, T1)
    I = np.eye(no)
    D2[o, o] = _es("ij,lk->ikjl", I, I)
    D2[o, v] = _es("ij,ak->jaik", I, T1)
    D2[v, o] = _es("ij,ak->ajki", I, T1)
    return D2


def cc_resid(S, T1, T2, dc=False, dressed=None):
    """Closed-shell CCSD (``dc=False``) / DCSD residual, kext variant.

    Restates ``calc_cc_resid`` (``src/cc/cc.jl:1343-1489``) with
    ``use_kext=true`` (default, ``options.jl:149``).  The kext block
    (``cc.jl:1400-1425``) contracts the undressed integrals with ``D2`` over all
    orbitals; summing the triangle plus its transpose (``cc.jl:1410``) equals
    the full ``sum_{qs} <pr|qs> D2[q,s,i,j]`` used here.
    """
    o, v = S.sl["o"], S.sl["v"]
    Vd, dh, df = dressed if dressed is not None else dressed_ints(S, T1)
    T2t = 2.0 * T2 - T2.transpose(1, 0, 2, 3)
    # singles (cc.jl:1357-1375)
    R1 = dh[v, o].copy()
    R1 += _es("abij,jb->ai", T2t, df[o, v])
    R1 -= _es("kjci,cakj->ai", Vd[o, o, v, o], T2t)
    # I_klij (cc.jl:1387-1398)
    klcd = S.ints2("oovv")
    I = Vd[o, o, o, o].copy()
    if not dc:
        I += _es("klcd,cdij->klij", klcd, T2)
    R2 = _es("klij,abkl->abij", I, T2)
    # kext (cc.jl:1400-1425)
    K2 = _es("prqs,qsij->prij", S.V, calc_D2(S, T1, T2))
    R2 += K2[v, v]
    R2 -= _es("kbij,ak->abij", K2[o, v], T1)
    R2 -= _es("akij,bk->abij", K2[v, o], T1)
    R2 += _es("klij,ak,bl->abij", K2[o, o], T1, T1)
    R1 += 2.0 * _es("akik->ai", K2[v, o]) - _es("akki->ai", K2[v, o])
    x1 = 2.0 * _es("klil->ki", K2[o, o]) - _es("klli->ki", K2[o, o])
    R1 -= _es("ki,ak->ai", x1, T1)
    # quadratic term (cc.jl:1433-1437)
    if not dc:
        R2 += _es("lcaj,cbil->abij", _es("klcd,adkj->lcaj", klcd, T2), T2)
    # xad, xki (cc.jl:1440-1450)
    fac = 0.5 if dc else 1.0
    xad = df[v, v] - fac * _es("klcd,cakl->ad", klcd, T2t)
    xki = df[o, o] + fac * _es("klcd,cdil->ki", klcd, T2t)
    # P(ia;jb) terms (cc.jl:1453-1484)
    R2r = _es("ad,dbij->abij", xad, T2) - _es("ki,abkj->abij", xki, T2)
    W = Vd[v, o, o, v] + 0.5 * _es("klcd,adil->akic", klcd, T2t)
    R2r += _es("akic,cbkj->abij", W, T2t)
    if not dc:
        T2m = T2t - T2
        R2r -= _es("lcai,cblj->abij", _es("klcd,daki->lcai", klcd, T2), T2m)
    d_vovo = Vd[v, o, v, o]
    R2r -= _es("akci,cbkj->abij", d_vovo, T2)
    R2r -= _es("bkci,ackj->abij", d_vovo, T2)
    R2 += R2r + R2r.transpose(1, 0, 3, 2)
    return R1, R2


# ---------------------------------------------------------------- DIIS


class Diis:
    """DIIS (``src/solvers/diis.jl:34-305``), vectors held in memory.

    ``dots`` are per-component dot functions (``custom_dot``, diis.jl:174-189);
    ``None`` means the plain dot (``weighted_dot`` with no weights, :155-167).
    """

    def __init__(self, maxdiis=6, resthr=10.0, dots=None):
        self.maxdiis = maxdiis
        self.resthr = resthr
        self.dots = dots
        self.amps = [None] * maxdiis
        self.res = [None] * maxdiis
        self.next = 0
        self.ndim = 0
        self.bmat = np.zeros((maxdiis + 1, maxdiis + 1))

    def _dot(self, A, B):
        if self.dots is None:
            return float(sum(np.sum(a * b) for a, b in zip(A, B)))
        return float(sum(f(a, b) for f, a, b in zip(self.dots, A, B)))

    def perform(self, amps, res):
        if self.ndim < self.maxdiis:
            self.ndim += 1
        ithis, nd = self.next, self.ndim
        self.amps[ithis] = [a.copy() for a in amps]
        self.res[ithis] = [r.copy() for r in res]
        # update_Bmat (diis.jl:210-234)
        this = self._dot(res, res)
        for i in range(nd):
            if i != ithis:
                d = self._dot(res, self.res[i])
                self.bmat[i, ithis] = self.bmat[ithis, i] = d
            else:
                self.bmat[ithis, ithis] = this
            self.bmat[i, nd] = self.bmat[nd, i] = -1.0
        self.bmat[nd, nd] = 0.0
        rhs = np.zeros(nd + 1)
        rhs[nd] = -1.0
        B = self.bmat[: nd + 1, : nd + 1]
        # svd(bmat)\rhs (diis.jl:261): pseudo-inverse, singular values
        # below eps*smax dropped (Julia LinearAlgebra ldiv! for SVD)
        U, s, Vt = np.linalg.svd(B)
        k = int(np.sum(s >= np.finfo(float).eps * s[0]))
        coeffs = Vt[:k].T @ ((U[:, :k].T @ rhs) / s[:k])
        # replacement policy (diis.jl:265-286)
        if nd == 1 and self.next == 0 and this > self.resthr:
            self.ndim = 0
            return amps
        elif nd < self.maxdiis:
            self.next = nd
        else:
            cmin = 1.0e10
            for i in range(nd):
                if abs(coeffs[i]) < cmin and (i != ithis or nd == 1):
                    cmin = abs(coeffs[i])
                    self.next = i
        # combine (diis.jl:135-148)
        out = [c * coeffs[0] for c in self.amps[0]]
        for i in range(1, nd):
            for j, a in enumerate(self.amps[i]):
                out[j] = out[j] + coeffs[i] * a
        for a, x in zip(amps, out):
            a[...] = x
        return amps


# ---------------------------------------------------------------- CC loop


def cc_iterations(S, T1, T2, fock, dc=False, opts=None, log=None):
    """``cc_iterations!`` closed shell (``src/cc/cc.jl:2518-2656``).

    Returns (E_hylleraas, T1, T2, n_iterations, converged).
    """
    opts = opts or Options()
    eps = np.diag(fock)
    eo, ev = eps[S.sl["o"]], eps[S.sl["v"]]
    if opts.diis_dot not in ("cs", "plain"):
        raise ValueError(f"diis_dot must be 'cs' or 'plain', not {opts.diis_dot!r}")
    dots = (cs_singles_dot, cs_doubles_dot) if opts.diis_dot == "cs" else None
    diis = Diis(opts.maxdiis, opts.resthr, dots=dots)
    thren = math.sqrt(opts.thr) * opts.conven
    T1 = T1.copy()
    T2 = T2.copy()
    E = 0.0
    converged = False
    it = 0
    for it in range(1, opts.maxit + 1):
        R1, R2 = cc_resid(S, T1, T2, dc=dc)
        NormR2 = doubles_norm(R2)
        E, _ = hylleraas(S, T1, T2, R1, R2, fock)
        T2 += update_doubles(R2, eo, ev, opts.shiftp)
        NormR1 = singles_norm(R1)
        T1 += update_singles(R1, eo, ev, opts.shifts)
        diis.perform([T1, T2], [R1, R2])
        En = doubles_energy(S, T2) + singles_energy(S, T1, fock)
        dE = En - E
        NormR = NormR1 + NormR2
        if log is not None:
            log(it, NormR, E, dE)
        if NormR < opts.thr and abs(dE) < thren:
            converged = True
            break
    return E, T1, T2, it, converged


# ---------------------------------------------------------------- (T)


def _triplets(no):
    """Triplet order and weights of ``cc_triples.jl:62-72``."""
    for k in range(no):
        for j in range(k + 1):
            prefac = 1.0 if j == k else 2.0
            for i in range(j + 1):
                fac = prefac
                if i == j:
                    if j == k:
                        continue
                    fac = 1.0
                yield i, j, k, fac


def _kijk(T2, vvvo, ovoo, i, j, k):
    """The 12 contractions of ``cc_triples.jl:89-104``."""
    K = _es("ad,bcd->abc", T2[:, :, i, j], vvvo[:, :, :, k])
    K += _es("db,acd->abc", T2[:, :, i, j], vvvo[:, :, :, k])
    K += _es("ad,cbd->abc", T2[:, :, i, k], vvvo[:, :, :, j])
    K += _es("dc,abd->abc", T2[:, :, i, k], vvvo[:, :, :, j])
    K += _es("bd,cad->abc", T2[:, :, j, k], vvvo[:, :, :, i])
    K += _es("dc,bad->abc", T2[:, :, j, k], vvvo[:, :, :, i])
    K -= _es("bal,lc->abc", T2[:, :, :, i], ovoo[:, :, j, k])
    K -= _es("abl,lc->abc", T2[:, :, :, j], ovoo[:, :, i, k])
    K -= _es("cal,lb->abc", T2[:, :, :, i], ovoo[:, :, k, j])
    K -= _es("acl,lb->abc", T2[:, :, :, k], ovoo[:, :, i, j])
    K -= _es("cbl,la->abc", T2[:, :, :, j], ovoo[:, :, k, i])
    K -= _es("bcl,la->abc", T2[:, :, :, k], ovoo[:, :, j, i])
    return K


def _xijk(K, eo, ev, i, j, k):
    X = (4.0 * K - 2.0 * K.transpose(0, 2, 1) - 2.0 * K.transpose(2, 1, 0)
         - 2.0 * K.transpose(1, 0, 2) + K.transpose(2, 0, 1) + K.transpose(1, 2, 0))
    D = (eo[i] + eo[j] + eo[k] - ev[:, None, None] - ev[None, :, None]
         - ev[None, None, :])
    return X / D


def pert_t(S, T1, T2, fock):
    """Closed-shell (T) (``src/cc/cc_triples.jl:39-157``); returns ((T), [T])."""
    vv_oo = S.ints2("oovv").transpose(2, 3, 0, 1)
    vvvo = S.ints2("vvvo")
    ovoo = S.ints2("ovoo")
    eps = np.diag(fock)
    eo, ev = eps[S.sl["o"]], eps[S.sl["v"]]
    IntX = np.zeros((S.nv, S.no))
    IntY = np.zeros((S.nv, S.no))
    Enb3 = 0.0
    for i, j, k, fac in _triplets(S.no):
        K = _kijk(T2, vvvo, ovoo, i, j, k)
        X = _xijk(K, eo, ev, i, j, k)
        Enb3 += fac * float(np.sum(K * X))
        IntX[:, i] += fac * _es("abc,bc->a", X, vv_oo[:, :, j, k])
        IntX[:, j] += fac * _es("abc,ac->b", X, vv_oo[:, :, i, k])
        IntX[:, k] += fac * _es("abc,ab->c", X, vv_oo[:, :, i, j])
        IntY[:, i] += fac * _es("abc,bc->a", X, T2[:, :, j, k])
        IntY[:, j] += fac * _es("abc,ac->b", X, T2[:, :, i, k])
        IntY[:, k] += fac * _es("abc,ab->c", X, T2[:, :, i, j])
    fov = fock[S.sl["o"], S.sl["v"]]
    En3 = float(np.sum(T1 * IntX)) + float(np.sum(fov.T * IntY)) + Enb3
    return En3, Enb3


def lambda_pert_t(S, T1, T2, U1, U2c, fock):
    """Closed-shell Lambda-(T) (``cc_triples.jl:159-295``); ``U2c`` contravariant."""
    U2 = contra2covariant(U2c)
    vv_oo = S.ints2("oovv").transpose(2, 3, 0, 1)
    vvvo = S.ints2("vvvo")
    ovoo = S.ints2("ovoo")
    vv_vo = S.ints2("vovv").transpose(2, 3, 0, 1)
    ov_oo = S.ints2("ooov").transpose(2, 3, 0, 1)
    eps = np.diag(fock)
    eo, ev = eps[S.sl["o"]], eps[S.sl["v"]]
    IntX = np.zeros((S.nv, S.no))
    IntY = np.zeros((S.nv, S.no))
    Enb3 = 0.0
    for i, j, k, fac in _triplets(S.no):
        X = _xijk(_kijk(T2, vvvo, ovoo, i, j, k), eo, ev, i, j, k)
        K = _kijk(U2, vv_vo, ov_oo, i, j, k)
        Enb3 += fac * float(np.sum(K * X))
        IntX[:, i] += fac * _es("abc,bc->a", X, vv_oo[:, :, j, k])
        IntX[:, j] += fac * _es("abc,ac->b", X, vv_oo[:, :, i, k])
        IntX[:, k] += fac * _es("abc,ab->c", X, vv_oo[:, :, i, j])
        IntY[:, i] += fac * _es("abc,bc->a", X, U2[:, :, j, k])
        IntY[:, j] += fac * _es("abc,ac->b", X, U2[:, :, i, k])
        IntY[:, k] += fac * _es("abc,ab->c", X, U2[:, :, i, j])
    fov = fock[S.sl["o"], S.sl["v"]]
    En3 = 0.5 * float(np.sum(U1 * IntX)) + float(np.sum(fov.T * IntY)) + Enb3
    return En3, Enb3


# ---------------------------------------------------------------- Lambda


def one_rdm(S, U1, U2, T1, T2):
    """``calc_1RDM`` closed shell (``src/cc/cc_lagrange.jl:793-848``)."""
    Doo = -2.0 * _es("cdik,cdjk->ij", U2, T2)
    Dvv = 2.0 * _es("bckl,ackl->ab", U2, T2)
    Dov = U1.T.copy()
    Dvo = 2.0 * _es("ck,acik->ai", U1, T2) - _es("ck,acki->ai", U1, T2)
    dDoo = Doo - Dov @ T1
    dDvv = Dvv + T1 @ Dov
    dDvo = Dvo + 2.0 * T1 - Dvv @ T1 + T1 @ dDoo
    o, v = S.sl["o"], S.sl["v"]
    D1 = np.zeros((S.n, S.n))
    dD1 = np.zeros((S.n, S.n))
    D1[o, o], D1[v, v], D1[o, v], D1[v, o] = Doo, Dvv, Dov, Dvo
    dD1[o, o], dD1[v, v], dD1[o, v], dD1[v, o] = dDoo, dDvv, Dov, dDvo
    return D1, dD1


def vector_times_jacobian(S, U1, U2, T1, T2, fock, dressed, vT_ovoo, dc=False):
    """``calc_ccsd_vector_times_Jacobian`` closed shell (``cc_lagrange.jl:9-220``)."""
    o, v = S.sl["o"], S.sl["v"]
    Vd, dh, dfock = dressed
    D1, dD1 = one_rdm(S, U1, U2, T1, T2)
    fov = fock[o, v]
    dfov = dfock[o, v]
    R1 = 2.0 * fov.T.copy()
    oovv = S.ints2("oovv")
    R2 = 2.0 * oovv.transpose(2, 3, 0, 1) - oovv.transpose(2, 3, 1, 0)
    I = Vd[o, o, o, o].copy()
    if not dc:
        I += _es("mncd,cdij->mnij", oovv, T2)
    R2 += _es("mnij,efij->efmn", I, U2)
    # kext (cc_lagrange.jl:39-75): K[r,s,m,n] = sum_pq <pq|rs> dU2[p,q,m,n]
    n = S.n
    dU2 = np.zeros((n, n, S.no, S.no))
    dU2[v, v] = U2
    dUovoo = _es("abmn,ai->ibmn", U2, T1)
    dU2[v, o] = -_es("abmn,bj->ajmn", U2, T1)
    dU2[o, o] = _es("ibmn,bj->ijmn", dUovoo, T1)
    dU2[o, v] = -dUovoo
    K = _es("pqrs,pqmn->rsmn", S.V, dU2)
    R2 += K[v, v]
    R1 += 2.0 * _es("ejmj->em", K[v, o])
    R1 += 2.0 * _es("ebmj,bj->em", K[v, v], T1)
    fac = 0.25 if dc else 0.5
    tR2 = fac * _es("mk,knef->efmn", D1[o, o], oovv)
    tR2 -= fac * _es("ce,mncf->efmn", D1[v, v], oovv)
    tT2 = 2.0 * T2 - T2.transpose(0, 1, 3, 2)
    xoo = _es("cdil,mlcd->mi", tT2, oovv)
    xvv = _es("ackl,klec->ae", tT2, oovv)
    W = Vd[v, o, o, v] + _es("kmce,acik->amie", oovv, tT2)
    tR2 += _es("afin,amie->efmn", U2, W)
    tR2 += 0.5 * _es("em,nf->efmn", U1, dfov)
    d_vovv = Vd[v, o, v, v]
    tR2 += 0.5 * _es("an,amfe->efmn", U1, d_vovv)
    d_oovo = Vd[o, o, v, o]
    tR2 -= 0.5 * _es("fi,mnei->efmn", U1, d_oovo)
    pR2 = 2.0 * tR2 - tR2.transpose(0, 1, 3, 2)
    D2 = _es("acik,cbkj->abij", U2, tT2)
    R1 += 2.0 * _es("adml,aled->em", D2, d_vovv)
    R1 -= 2.0 * _es("edil,lmdi->em", D2, d_oovo)
    if not dc:
        pR2 -= _es("fcnl,mlce->efmn", D2, oovv)
    D2 = _es("acik,cbkj->abij", U2, T2) + _es("caik,bckj->abij", U2, T2)
    if not dc:
        pR2 += _es("ednk,kmfd->efmn", D2, oovv)
    R1 -= 2.0 * _es("acmk,akce->em", D2, d_vovv)
    R1 += 2.0 * _es("ecik,mkci->em", D2, d_oovo)
    D2 = _es("cdij,cdkl->ijkl", U2, T2)
    R1 += 2.0 * _es("mjkl,klej->em", D2, d_oovo)
    if not dc:
        R2 += _es("mnkl,klef->efmn", D2, oovv)
    R1 -= 2.0 * _es("ebij,mbij->em", U2, vT_ovoo)
    fac = 0.5 if dc else 1.0
    pR2 += _es("afmn,ae->efmn", U2, dfock[v, v] - fac * xvv)
    pR2 -= _es("efin,mi->efmn", U2, dfock[o, o] + fac * xoo)
    d_vovo = Vd[v, o, v, o]
    pR2 -= _es("afin,amei->efmn", U2, d_vovo)
    pR2 -= _es("ebin,bmfi->efmn", U2, d_vovo)
    R2 += pR2 + pR2.transpose(1, 0, 3, 2)
    # singles (cc_lagrange.jl:205-218)
    momm = S.V[:, o, :, :]
    R1 += _es("pq,qmpe->em", dD1, 2.0 * momm[:, :, :, v] - momm[:, :, v, :].transpose(0, 1, 3, 2))
    R1 -= 2.0 * _es("ebij,bmji->em", U2, Vd[v, o, o, o])
    R1 += _es("mk,ke->em", D1[o, o], dfov)
    R1 -= _es("de,md->em", D1[v, v], dfov)
    R1 += _es("am,ae->em", U1, dfock[v, v] - xvv)
    R1 -= _es("ei,mi->em", U1, dfock[o, o] + xoo)
    return R1, R2


def correlation_norm(U1, U2, T1, T2):
    """``calc_correlation_norm`` closed shell (``cc_lagrange.jl:1065-1078``)."""
    N = float(np.sum(U2 * T2))
    N += _es("abij,ai,bj->", U2, T1, T1)
    N += float(np.sum(U1 * T1))
    return float(N)


def lambda_iterations(S, T1, T2, fock, dc=False, opts=None, log=None):
    """``lm_cc_iterations!`` closed shell (``cc_lagrange.jl:1155-1223``).

    Returns (U1, U2 contravariant, n_iterations, converged).
    """
    opts = opts or Options()
    eps = np.diag(fock)
    eo, ev = eps[S.sl["o"]], eps[S.sl["v"]]
    dressed = dressed_ints(S, T1)
    Vd = dressed[0]
    o, v = S.sl["o"], S.sl["v"]
    vT_ovoo = _es("bmdc,dcji->mbij", Vd[v, o, v, v], T2)
    # transform_amplitudes2lagrange_multipliers! (cctools.jl:887-930)
    U2 = T2 + _es("ai,bj->abij", T1, T1)
    U2 = U2 + (U2 - U2.transpose(0, 1, 3, 2))
    U1 = 2.0 * T1
    diis = Diis(opts.maxdiis, opts.resthr, dots=None)
    thren = math.sqrt(opts.thr) * opts.conven
    norm = 0.0
    converged = False
    it = 0
    for it in range(1, opts.maxit + 1):
        R1, R2 = vector_times_jacobian(S, U1, U2, T1, T2, fock, dressed, vT_ovoo, dc=dc)
        U2 = U2 + update_doubles(R2, eo, ev, opts.shiftp)
        NormR2 = contra_doubles_norm(R2)
        NormR1 = contra_singles_norm(R1)
        U1 = U1 + update_singles(R1, eo, ev, opts.shifts)
        diis.perform([U1, U2], [R1, R2])
        prev = norm
        norm = correlation_norm(U1, U2, T1, T2)
        NormR = NormR1 + NormR2
        if log is not None:
            log(it, NormR, norm, norm - prev)
        if NormR < opts.thr and abs(norm - prev) < thren:
            converged = True
            break
    return U1, U2, it, converged


# ---------------------------------------------------------------- driver


def _parse_method(method):
    m = method.strip().lower().replace("λ", "l").replace("Λ", "l")
    lam = m.startswith("l")
    if lam:
        m = m[1:]
    pert = m.endswith("(t)")
    if pert:
        m = m[:-3]
    if m not in ("ccsd", "dcsd"):
        raise ValueError(f"unsupported closed-shell method {method!r}")
    return m.upper(), m == "dcsd", lam, pert


def ccdriver(S, method, opts=None, log=None):
    """``ccdriver`` + ``eval_cc_groundstate`` (``src/cc/ccdriver.jl:37-76,348-393``).

    Returns a dict with the reference's OutDict keys (``HF``, ``MP2c``,
    ``MP2``, ``<M>c``, ``<M>``, ``[T]``, ``(T)``, ``<M>(T)c``, ``<M>(T)``, where
    ``<M>`` is ``CCSD``/``DCSD`` or ``ΛCCSD``/``ΛDCSD``) plus the amplitudes.
    """
    name, dc, lam, pert = _parse_method(method)
    main = ("Λ" if lam else "") + name
    fock = gen_fock(S)
    out = {}
    EHF = hf_energy(S, fock)
    out["HF"] = EHF
    Emp2, T1, T2 = mp2(S, fock)
    out["MP2c"] = Emp2
    out["MP2"] = Emp2 + EHF
    E, T1, T2, nit, conv = cc_iterations(S, T1, T2, fock, dc=dc, opts=opts, log=log)
    out[main + "c"] = E
    out[main] = E + EHF
    out["Ec"] = E
    out["E"] = E + EHF
    out["iterations"] = nit
    out["converged"] = conv
    out["T1"], out["T2"] = T1, T2
    if lam:
        U1, U2, lit, lconv = lambda_iterations(S, T1, T2, fock, dc=dc, opts=opts)
        out["U1"], out["U2"] = U1, U2
        out["lambda_iterations"] = lit
        out["lambda_converged"] = lconv
    if pert:
        if lam:
            ET3, ET3b = lambda_pert_t(S, T1, T2, out["U1"], out["U2"], fock)
        else:
            ET3, ET3b = pert_t(S, T1, T2, fock)
        out["[T]"] = ET3b
        out["(T)"] = ET3
        out[main + "(T)c"] = E + ET3
        out[main + "(T)"] = E + ET3 + EHF
    return out
