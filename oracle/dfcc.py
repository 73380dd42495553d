"""Density-fitted numpy restatement of the closed-shell CCSD/DCSD iteration
and (T), for systems whose 4-index integrals do not fit in memory.

TEST INFRASTRUCTURE ONLY (a CPU checker and the timed CPU baseline; never
called by the product path).  The math is ElemCo.jl's closed-shell path
restated with density-fitting factors ``(pq|rs) = sum_Q B[Q,p,q] B[Q,r,s]``
in place of the 4-index ``int2`` (ElemCo.jl keeps int2 whole: 55 GB at
(H2O)_6/cc-pVTZ):

* T1 dressing ``calc_dressed_ints`` / ``dress_fock_closedshell``
  (src/cc/cc.jl:453-815): every dressed block is a product of two dressed
  factors ``dB = (1 - t) B (1 + t)``, t[v,o] = T1;
* the residual ``calc_cc_resid`` (src/cc/cc.jl:1343-1489): the kext term
  (cc.jl:1400-1425) becomes the dressed particle-particle ladder
  ``sum_cd (ac|bd)^ T2[c,d,i,j]`` plus ``(ai|bj)^`` and the three-index
  singles intermediate ``W[c,i,Q] = sum_ld T2t[c,d,i,l] B[Q,l,d]``;
* the iteration ``cc_iterations!`` (cc.jl:2518-2656), updates
  (src/cc/cctools.jl:198-300), DIIS (src/solvers/diis.jl:246-305, via
  :class:`oracle.ccref.Diis`) and energies (cc.jl:97-249);
* (T) ``calc_pertT_closed_shell`` (src/cc/cc_triples.jl:39-157), with the
  vvvo and ovoo blocks built from the factors.

The iteration is a list of tasks (:meth:`DFCC.iteration_tasks`) so that a
timed sample can run a stated part of it; the ladder is one task per block
of the virtual index a.  ``tests/test_oracle_df.py`` checks this module
against the 4-index oracle (oracle/ccref.py).
"""
import math

import numpy as np

from . import ccref as O

__all__ = ["DFCC", "iteration_flops"]


def _dot(a, b, axes):
    return np.tensordot(a, b, axes=axes)


def iteration_flops(no, nv, nq, dc=False):
    """Algorithmic flops of one iteration: ladder 2o^2v^4 + its DF rebuild
    2nQv^4 + ring 16o^3v^3 (8 for DCSD) + 4o^4v^2."""
    o, v = float(no), float(nv)
    return 2 * o**2 * v**4 + 2 * nq * v**4 + (8.0 if dc else 16.0) * o**3 * v**3 \
        + 4 * o**4 * v**2


class DFCC:
    """Closed-shell CC state in density-fitted form.

    ``B`` is ``B[p,q,Q]`` (n x n x nQ, any memory order), ``h1`` the MO
    one-electron matrix, ``e0`` the core energy, ``no`` the occupied count.
    """

    def __init__(self, B, h1, e0, no, dc=False, opts=None, ablock=4):
        B = np.asarray(B, dtype=np.float64)
        n = B.shape[0]
        self.n, self.no, self.nv, self.nq = n, int(no), n - int(no), B.shape[2]
        o = slice(0, self.no)
        v = slice(self.no, n)
        Bq = np.ascontiguousarray(B.transpose(2, 0, 1))  # [Q,p,q]
        self.bvv = np.ascontiguousarray(Bq[:, v, v])
        self.bov = np.ascontiguousarray(Bq[:, o, v])
        self.bvo = np.ascontiguousarray(Bq[:, v, o])
        self.boo = np.ascontiguousarray(Bq[:, o, o])
        self.h = np.asarray(h1, dtype=np.float64)
        self.e0 = float(e0)
        self.dc = bool(dc)
        self.opts = opts or O.Options()
        self.ablock = int(ablock)
        # <kl|cd> = (kc|ld), undressed (ints2 "oovv")
        self.klcd = _dot(self.bov, self.bov, ([0], [0])).transpose(0, 2, 1, 3).copy()
        self.T1 = np.zeros((self.nv, self.no))
        self.dress()
        self.fock = self.df.copy()
        self.eps = np.diag(self.fock).copy()

    # ------------------------------------------------------------ dressing
    def dress(self, T1=None):
        """dB = (1 - t) B (1 + t), dh, dressed Fock (cc.jl:453-815)."""
        T1 = self.T1 if T1 is None else T1
        no = self.no
        # dB_vv = B_vv - T1 B_ov
        self.dbvv = self.bvv - np.einsum("ai,Qib->Qab", T1, self.bov, optimize=True)
        # dB_oo = B_oo + B_ov T1
        self.dboo = self.boo + np.einsum("Qib,bj->Qij", self.bov, T1, optimize=True)
        # dB_vo = B_vo - T1 B_oo + dB_vv T1
        self.dbvo = (self.bvo - np.einsum("ai,Qij->Qaj", T1, self.boo, optimize=True)
                     + np.einsum("Qab,bj->Qaj", self.dbvv, T1, optimize=True))
        t = np.zeros((self.n, self.n))
        t[no:, :no] = T1
        self.dh = (np.eye(self.n) - t) @ self.h @ (np.eye(self.n) + t)
        J = np.einsum("Qkk->Q", self.dboo)
        n = self.n
        df = self.dh.copy()
        dB = np.empty((self.nq, n, n))
        dB[:, :no, :no] = self.dboo
        dB[:, :no, no:] = self.bov
        dB[:, no:, :no] = self.dbvo
        dB[:, no:, no:] = self.dbvv
        df += 2.0 * np.einsum("Qpq,Q->pq", dB, J, optimize=True)
        df -= np.einsum("Qpk,Qkq->pq", dB[:, :, :no], dB[:, :no, :], optimize=True)
        self.df = df

    # ------------------------------------------------------------ residual
    def iteration_tasks(self):
        """One ``cc_iterations!`` pass as [(name, flops, fn)]: dressing, the
        residual terms (the ladder as one task per a-block), norms and
        Hylleraas energy, update, DIIS and the energy of the new amplitudes.
        Running all tasks in order is one iteration; afterwards ``self.E``,
        ``self.NormR`` and ``self.dE`` hold its results."""
        o, v, Q = self.no, self.nv, self.nq
        dc = self.dc
        tasks = []

        def t_dress():
            self.dress()
            T2 = self.T2
            self.Tt = 2.0 * T2 - T2.transpose(1, 0, 2, 3)
        tasks.append(("dress", 4.0 * Q * v * v * o + 2.0 * Q * (o + v) ** 2 * o, t_dress))

        def t_singles():
            Tt, df = self.Tt, self.df
            R1 = df[o:, :o].copy()
            # W[c,i,Q] = sum_{ld} Tt[c,d,i,l] B[Q,l,d]
            W3 = np.einsum("cdil,Qld->ciQ", Tt, self.bov, optimize=True)
            R1 += np.einsum("Qac,ciQ->ai", self.dbvv, W3, optimize=True)
            R1 -= np.einsum("ajQ,Qji->ai", W3, self.dboo, optimize=True)
            R1 += np.einsum("abij,jb->ai", Tt, df[:o, o:], optimize=True)
            self.R1 = R1
        tasks.append(("singles", 4.0 * v * v * o * o * Q, t_singles))

        def t_iklij():
            T2 = self.T2
            I = np.einsum("Qki,Qlj->klij", self.dboo, self.dboo, optimize=True)
            if not dc:
                I += np.einsum("klcd,cdij->klij", self.klcd, T2, optimize=True)
            self.R2 = np.einsum("abkl,klij->abij", T2, I, optimize=True)
            # (ai|bj)^ of the kext term
            self.R2 += np.einsum("Qai,Qbj->abij", self.dbvo, self.dbvo, optimize=True)
        tasks.append(("I_klij", 4.0 * o**4 * v * v + 2.0 * o * o * v * v * Q, t_iklij))

        # ladder sum_cd (ac|bd)^ T2[c,d,i,j], (ac|bd)^ = sum_Q dB[Q,a,c] dB[Q,b,d]
        for a0 in range(0, v, self.ablock):
            a1 = min(v, a0 + self.ablock)

            def t_ladder(a0=a0, a1=a1):
                na = a1 - a0
                Vb = _dot(self.dbvv[:, a0:a1, :], self.dbvv, ([0], [0]))  # [a,c,b,d]
                Vb = Vb.transpose(0, 2, 1, 3).reshape(na * v, v * v)       # [(a,b),(c,d)]
                L = Vb @ self.T2.reshape(v * v, o * o)
                self.R2[a0:a1] += L.reshape(na, v, o, o)
            tasks.append((f"ladder a{a0}", 2.0 * (a1 - a0) * v * v * v * (Q + o * o), t_ladder))

        def t_quad_x():
            T2, Tt, kl = self.T2, self.Tt, self.klcd
            if not dc:
                Y = np.einsum("klcd,adkj->lcaj", kl, T2, optimize=True)
                self.R2 += np.einsum("lcaj,cbil->abij", Y, T2, optimize=True)
            fac = 0.5 if dc else 1.0
            self.xad = self.df[o:, o:] - fac * np.einsum("klcd,cakl->ad", kl, Tt, optimize=True)
            self.xki = self.df[:o, :o] + fac * np.einsum("klcd,cdil->ki", kl, Tt, optimize=True)
        tasks.append(("quadratic, x_ad, x_ki", (0.0 if dc else 4.0) * o**3 * v**3, t_quad_x))

        def t_ring1():
            T2, Tt = self.T2, self.Tt
            R2r = np.einsum("ad,dbij->abij", self.xad, T2, optimize=True)
            R2r -= np.einsum("abkj,ki->abij", T2, self.xki, optimize=True)
            W = np.einsum("Qai,Qkc->akic", self.dbvo, self.bov, optimize=True)
            W += 0.5 * np.einsum("klcd,adil->akic", self.klcd, Tt, optimize=True)
            R2r += np.einsum("akic,cbkj->abij", W, Tt, optimize=True)
            self.R2r = R2r
        tasks.append(("ring d_voov", 4.0 * o**3 * v**3 + 2.0 * o * o * v * v * Q, t_ring1))

        def t_ring2():
            T2 = self.T2
            if not dc:
                Tm = self.Tt - T2
                Y = np.einsum("klcd,daki->lcai", self.klcd, T2, optimize=True)
                self.R2r -= np.einsum("lcai,cblj->abij", Y, Tm, optimize=True)
            Wv = np.einsum("Qac,Qki->akci", self.dbvv, self.dboo, optimize=True)
            self.R2r -= np.einsum("akci,cbkj->abij", Wv, T2, optimize=True)
            self.R2r -= np.einsum("bkci,ackj->abij", Wv, T2, optimize=True)
            self.R2 += self.R2r + self.R2r.transpose(1, 0, 3, 2)
            self.R2r = None
        tasks.append(("ring d_vovo", (8.0 if dc else 12.0) * o**3 * v**3
                      + 2.0 * o * o * v * v * Q, t_ring2))

        def t_update():
            T1, T2, R1, R2 = self.T1, self.T2, self.R1, self.R2
            eo, ev = self.eps[:o], self.eps[o:]
            NormR2 = O.doubles_norm(R2)
            self.E = self._hylleraas(T1, T2, R1, R2)
            T2 += O.update_doubles(R2, eo, ev, self.opts.shiftp)
            NormR1 = O.singles_norm(R1)
            T1 += O.update_singles(R1, eo, ev, self.opts.shifts)
            self.diis.perform([T1, T2], [R1, R2])
            En = self._energy(T1, T2)
            self.dE = En - self.E
            self.NormR = NormR1 + NormR2
        tasks.append(("update, DIIS, energies", 20.0 * o * o * v * v, t_update))
        return tasks

    # ------------------------------------------------------------ energies
    def _oovv_dots(self, X):
        """(sum X[a,b,i,j] <ij|ab>, sum X[b,a,i,j] <ij|ab>)."""
        kl = self.klcd  # [i,j,a,b]
        d = float(np.einsum("abij,ijab->", X, kl, optimize=True))
        ex = float(np.einsum("baij,ijab->", X, kl, optimize=True))
        return d, ex

    def _energy(self, T1, T2):
        """calc_doubles_energy + calc_singles_energy (cc.jl:97-168)."""
        d, ex = self._oovv_dots(T2)
        E = 2.0 * d - ex
        TT = np.einsum("ai,bj->abij", T1, T1)
        d1, ex1 = self._oovv_dots(TT)
        E += 2.0 * d1 - ex1 + 2.0 * float(np.sum(T1 * self.fock[:self.no, self.no:].T))
        return E

    def _hylleraas(self, T1, T2, R1, R2):
        """calc_hylleraas (cc.jl:195-249)."""
        pd, pex = self._oovv_dots(T2)
        rd = float(np.sum(T2 * R2))
        rex = float(np.einsum("baij,abij->", T2, R2, optimize=True))
        TT = np.einsum("ai,bj->abij", T1, T1)
        d1, ex1 = self._oovv_dots(TT)
        ET1 = 2.0 * d1 - ex1 + 2.0 * float(np.sum(self.fock[:self.no, self.no:].T * T1)) \
            + 2.0 * float(np.sum(R1 * T1))
        return 2.0 * (pd + rd) - (pex + rex) + ET1

    # ------------------------------------------------------------ driver
    def mp2(self):
        """calc_MP2 (cc.jl:1011-1024): start amplitudes; returns the energy."""
        o = self.no
        eo, ev = self.eps[:o], self.eps[o:]
        vvoo = np.einsum("Qai,Qbj->abij", self.bvo, self.bvo, optimize=True)
        self.T2 = O.update_doubles(vvoo, eo, ev, 0.0)
        self.T1 = O.update_singles(self.fock[o:, :o], eo, ev, 0.0)
        d, ex = self._oovv_dots(self.T2)
        return 2.0 * d - ex + 2.0 * float(np.sum(self.T1 * self.fock[:o, o:].T))

    def start(self, T1=None, T2=None):
        """Start (or restart) the iterations from T1/T2 (default: MP2)."""
        if T1 is None:
            self.mp2()
        else:
            self.T1 = np.array(T1, dtype=np.float64)
            self.T2 = np.array(T2, dtype=np.float64)
        dots = (O.cs_singles_dot, O.cs_doubles_dot) if self.opts.diis_dot == "cs" else None
        self.diis = O.Diis(self.opts.maxdiis, self.opts.resthr, dots=dots)
        self._tasks = self.iteration_tasks()

    def iterate(self):
        """One full iteration; returns (E, NormR, dE)."""
        for _, _, fn in self._tasks:
            fn()
        return self.E, self.NormR, self.dE

    def solve(self):
        """cc_iterations! to the reference's convergence test (cc.jl:2625)."""
        thren = math.sqrt(self.opts.thr) * self.opts.conven
        for it in range(1, self.opts.maxit + 1):
            E, NormR, dE = self.iterate()
            if NormR < self.opts.thr and abs(dE) < thren:
                return E, it, True
        return self.E, self.opts.maxit, False

    # ------------------------------------------------------------ (T)
    def vvvo_k(self, k):
        """vvvo[:,:,:,k] with vvvo[b,c,d,k] = <bc|dk> = (bd|ck)."""
        return np.einsum("Qbd,Qc->bcd", self.bvv, self.bvo[:, :, k], optimize=True)

    def pert_t(self, T1, T2, triplets=None):
        """calc_pertT_closed_shell (cc_triples.jl:39-157) over all triplets, or
        over the given (i, j, k, weight) subset (returns the partial [T] sum
        and the partial IntX/IntY contribution of those triplets)."""
        o = self.no
        eo, ev = self.eps[:o], self.eps[o:]
        vv_oo = self.klcd.transpose(2, 3, 0, 1)
        # ovoo[i,a,j,k] = <ia|jk> = (ij|ak)
        ovoo = np.einsum("Qij,Qak->iajk", self.boo, self.bvo, optimize=True)
        cache = {}

        def vvvo_x(x):
            if x not in cache:
                cache[x] = self.vvvo_k(x)
            return cache[x]

        IntX = np.zeros((self.nv, o))
        IntY = np.zeros((self.nv, o))
        Enb3 = 0.0
        for i, j, k, fac in (triplets if triplets is not None else O._triplets(o)):
            vv = {x: vvvo_x(x) for x in {i, j, k}}
            K = _kijk_cols(T2, vv, ovoo, i, j, k)
            X = O._xijk(K, eo, ev, i, j, k)
            Enb3 += fac * float(np.sum(K * X))
            IntX[:, i] += fac * np.einsum("abc,bc->a", X, vv_oo[:, :, j, k])
            IntX[:, j] += fac * np.einsum("abc,ac->b", X, vv_oo[:, :, i, k])
            IntX[:, k] += fac * np.einsum("abc,ab->c", X, vv_oo[:, :, i, j])
            IntY[:, i] += fac * np.einsum("abc,bc->a", X, T2[:, :, j, k])
            IntY[:, j] += fac * np.einsum("abc,ac->b", X, T2[:, :, i, k])
            IntY[:, k] += fac * np.einsum("abc,ab->c", X, T2[:, :, i, j])
        fov = self.fock[:o, o:]
        return float(np.sum(T1 * IntX)) + float(np.sum(fov.T * IntY)) + Enb3, Enb3


def _kijk_cols(T2, vv, ovoo, i, j, k):
    """The 12 contractions of cc_triples.jl:89-104 with vvvo columns vv[x] =
    vvvo[:,:,:,x] (the same terms as oracle.ccref._kijk)."""
    es = lambda s, a, b: np.einsum(s, a, b, optimize=True)  # noqa: E731
    K = es("ad,bcd->abc", T2[:, :, i, j], vv[k])
    K += es("db,acd->abc", T2[:, :, i, j], vv[k])
    K += es("ad,cbd->abc", T2[:, :, i, k], vv[j])
    K += es("dc,abd->abc", T2[:, :, i, k], vv[j])
    K += es("bd,cad->abc", T2[:, :, j, k], vv[i])
    K += es("dc,bad->abc", T2[:, :, j, k], vv[i])
    K -= es("bal,lc->abc", T2[:, :, :, i], ovoo[:, :, j, k])
    K -= es("abl,lc->abc", T2[:, :, :, j], ovoo[:, :, i, k])
    K -= es("cal,lb->abc", T2[:, :, :, i], ovoo[:, :, k, j])
    K -= es("acl,lb->abc", T2[:, :, :, k], ovoo[:, :, i, j])
    K -= es("cbl,la->abc", T2[:, :, :, j], ovoo[:, :, k, i])
    K -= es("bcl,la->abc", T2[:, :, :, k], ovoo[:, :, j, i])
    return K
