"""Gaussian integrals in numpy by Obara-Saika recurrences — a checker for the
GPU integral engine (which uses McMurchie-Davidson).

TEST INFRASTRUCTURE ONLY (small shells, slow pure Python).  Restates the
published Obara-Saika vertical/horizontal recurrences (Obara and Saika, J.
Chem. Phys. 84, 3963 (1986); Head-Gordon and Pople, J. Chem. Phys. 89, 5777
(1988)), the Boys function through the confluent hypergeometric function
F_m(T) = 1F1(m+1/2; m+3/2; -T) / (2m+1), and real solid harmonics by their
recursion in l (Helgaker, Jorgensen, Olsen, Molecular Electronic-Structure
Theory, eqs. 6.4.70-6.4.72).  The integrals are those ElemCo.jl takes from
libcint (src/system/libcint5.jl:25-81): overlap, kinetic, nuclear attraction,
dipole, (P|Q) and (mn|P), over shells given as in include/ecgpu.h
(contraction coefficients of normalised primitives, spherical functions
m = -l..l normalised to unit self-overlap).
"""
import math
from functools import lru_cache

import numpy as np
from scipy.special import hyp1f1

__all__ = ["boys", "cart_list", "solid_harmonics", "Shells", "overlap", "kinetic", "nuclear",
           "dipole", "int2c2e", "int3c2e"]


def boys(m, T):
    return hyp1f1(m + 0.5, m + 1.5, -T) / (2 * m + 1)


def cart_list(l):
    return [(i, j, l - i - j) for i in range(l, -1, -1) for j in range(l - i, -1, -1)]


@lru_cache(None)
def _poly_sh(l, m):
    """S_lm as a dict {(i,j,k): coefficient} (recursion in l)."""
    if l == 0:
        return {(0, 0, 0): 1.0}

    def add(acc, poly, f, shift):
        for (i, j, k), c in poly.items():
            key = (i + shift[0], j + shift[1], k + shift[2])
            acc[key] = acc.get(key, 0.0) + f * c

    L = l - 1
    out = {}
    if m == l or m == -l:
        f = math.sqrt((2.0 if L == 0 else 1.0) * (2 * L + 1) / (2 * L + 2))
        if m == l:
            add(out, _poly_sh(L, L), f, (1, 0, 0))
            if L > 0:
                add(out, _poly_sh(L, -L), -f, (0, 1, 0))
        else:
            add(out, _poly_sh(L, L), f, (0, 1, 0))
            if L > 0:
                add(out, _poly_sh(L, -L), f, (1, 0, 0))
        return out
    d = math.sqrt((L + m + 1) * (L - m + 1))
    add(out, _poly_sh(L, m), (2 * L + 1) / d, (0, 0, 1))
    if abs(m) <= L - 1:
        g = math.sqrt((L + m) * (L - m)) / d
        prev = _poly_sh(L - 1, m)
        for sh in ((2, 0, 0), (0, 2, 0), (0, 0, 2)):
            add(out, prev, -g, sh)
    return out


def solid_harmonics(l):
    """(2l+1) x ncart matrix, rows m = -l..l, columns in cart_list(l) order."""
    cl = cart_list(l)
    M = np.zeros((2 * l + 1, len(cl)))
    for r, m in enumerate(range(-l, l + 1)):
        for key, c in _poly_sh(l, m).items():
            M[r, cl.index(key)] += c
    return M


class Shells:
    """Contracted shells: list of (l, centre(3), exps, coefs)."""

    def __init__(self, shells):
        self.shells = [(int(l), np.asarray(c, float), np.asarray(e, float),
                        np.asarray(k, float) * np.asarray(e, float) ** ((2 * l + 3) / 4.0))
                       for l, c, e, k in shells]

    def nbf(self):
        return sum(2 * l + 1 for l, *_ in self.shells)


# ------------------------------------------------------------------ 1e


def _s1d(i, j, a, b, A, B):
    """1D overlap of (x-A)^i e^{-a(x-A)^2} (x-B)^j e^{-b(x-B)^2} (OS recursion)."""
    p = a + b
    P = (a * A + b * B) / p
    S = {}

    def s(i_, j_):
        if i_ < 0 or j_ < 0:
            return 0.0
        if (i_, j_) in S:
            return S[(i_, j_)]
        if i_ == 0 and j_ == 0:
            v = math.sqrt(math.pi / p) * math.exp(-a * b / p * (A - B) ** 2)
        elif i_ > 0:
            v = (P - A) * s(i_ - 1, j_) + ((i_ - 1) * s(i_ - 2, j_) + j_ * s(i_ - 1, j_ - 1)) / (2 * p)
        else:
            v = (P - B) * s(i_, j_ - 1) + (i_ * s(i_ - 1, j_ - 1) + (j_ - 1) * s(i_, j_ - 2)) / (2 * p)
        S[(i_, j_)] = v
        return v
    return s(i, j)


def _prim1e(kind, la, A, a, lb, B, b, extra):
    out = np.zeros((len(cart_list(la)), len(cart_list(lb))))
    for x, ca in enumerate(cart_list(la)):
        for y, cb in enumerate(cart_list(lb)):
            if kind == "S":
                out[x, y] = np.prod([_s1d(ca[d], cb[d], a, b, A[d], B[d]) for d in range(3)])
            elif kind == "T":
                Sd = [_s1d(ca[d], cb[d], a, b, A[d], B[d]) for d in range(3)]
                tot = 0.0
                for d in range(3):
                    j = cb[d]
                    t = (b * (2 * j + 1) * _s1d(ca[d], j, a, b, A[d], B[d])
                         - 2 * b * b * _s1d(ca[d], j + 2, a, b, A[d], B[d]))
                    if j >= 2:
                        t -= 0.5 * j * (j - 1) * _s1d(ca[d], j - 2, a, b, A[d], B[d])
                    tot += t * np.prod([Sd[e] for e in range(3) if e != d])
                out[x, y] = tot
            elif kind == "D":
                comp, O = extra
                Sd = [_s1d(ca[d], cb[d], a, b, A[d], B[d]) for d in range(3)]
                d = comp
                m = _s1d(ca[d] + 1, cb[d], a, b, A[d], B[d]) + (A[d] - O[d]) * Sd[d]
                out[x, y] = m * np.prod([Sd[e] for e in range(3) if e != d])
    return out


def _prim_nuc(la, A, a, lb, B, b, C, Z):
    """-Z <a|1/|r-C||b> by OS vertical (on a) and horizontal recursion."""
    p = a + b
    P = (a * A + b * B) / p
    K = math.exp(-a * b / p * np.sum((A - B) ** 2))
    T = p * np.sum((P - C) ** 2)
    L = la + lb
    F = [boys(m, T) for m in range(L + 1)]
    memo = {}

    def v(ax, m):
        if min(ax) < 0:
            return 0.0
        key = (ax, m)
        if key in memo:
            return memo[key]
        if ax == (0, 0, 0):
            r = 2 * math.pi / p * K * F[m]
        else:
            i = next(d for d in range(3) if ax[d] > 0)
            am = list(ax)
            am[i] -= 1
            am = tuple(am)
            amm = list(am)
            amm[i] -= 1
            amm = tuple(amm)
            r = (P[i] - A[i]) * v(am, m) - (P[i] - C[i]) * v(am, m + 1)
            if am[i] > 0:
                r += am[i] / (2 * p) * (v(amm, m) - v(amm, m + 1))
        memo[key] = r
        return r

    def hrr(ax, bx):
        if min(bx) < 0:
            return 0.0
        if bx == (0, 0, 0):
            return v(ax, 0)
        i = next(d for d in range(3) if bx[d] > 0)
        bm = list(bx)
        bm[i] -= 1
        ap = list(ax)
        ap[i] += 1
        return hrr(tuple(ap), tuple(bm)) + (A[i] - B[i]) * hrr(ax, tuple(bm))

    out = np.zeros((len(cart_list(la)), len(cart_list(lb))))
    for x, ca in enumerate(cart_list(la)):
        for y, cb in enumerate(cart_list(lb)):
            out[x, y] = -Z * hrr(ca, cb)
    return out


def _contract2(sh1, sh2, prim):
    l1, A, e1, c1 = sh1
    l2, B, e2, c2 = sh2
    out = 0.0
    for a, ca in zip(e1, c1):
        for b, cb in zip(e2, c2):
            out = out + ca * cb * prim(l1, A, a, l2, B, b)
    return solid_harmonics(l1) @ out @ solid_harmonics(l2).T


def _assemble1e(bs, prim):
    n = bs.nbf()
    M = np.zeros((n, n))
    off = np.cumsum([0] + [2 * s[0] + 1 for s in bs.shells])
    for i, s1 in enumerate(bs.shells):
        for j, s2 in enumerate(bs.shells):
            M[off[i]:off[i + 1], off[j]:off[j + 1]] = _contract2(s1, s2, prim)
    return M


def _norms(bs):
    S = _assemble1e(bs, lambda *q: _prim1e("S", *q, None))
    return 1.0 / np.sqrt(np.diag(S))


def overlap(bs):
    d = _norms(bs)
    return _assemble1e(bs, lambda *q: _prim1e("S", *q, None)) * np.outer(d, d)


def kinetic(bs):
    d = _norms(bs)
    return _assemble1e(bs, lambda *q: _prim1e("T", *q, None)) * np.outer(d, d)


def nuclear(bs, Z, xyz):
    d = _norms(bs)
    M = 0.0
    for z, C in zip(Z, np.asarray(xyz, float).reshape(-1, 3)):
        M = M + _assemble1e(bs, lambda l1, A, a, l2, B, b, C=C, z=z: _prim_nuc(l1, A, a, l2, B, b, C, z))
    return M * np.outer(d, d)


def dipole(bs, origin=(0.0, 0.0, 0.0)):
    d = _norms(bs)
    O = np.asarray(origin, float)
    return [_assemble1e(bs, lambda *q, c=c: _prim1e("D", *q, (c, O))) * np.outer(d, d)
            for c in range(3)]


# ------------------------------------------------------------------ 2e


def _prim_eri3(la, A, a, lb, B, b, lc, C, g):
    """(ab|c) primitive Cartesian block by OS VRR on (e0|c0) and HRR a -> b."""
    zeta, eta = a + b, g
    P = (a * A + b * B) / zeta
    Q = C
    rho = zeta * eta / (zeta + eta)
    W = (zeta * P + eta * Q) / (zeta + eta)
    K = math.exp(-a * b / zeta * np.sum((A - B) ** 2))
    T = rho * np.sum((P - Q) ** 2)
    L = la + lb + lc
    F = [boys(m, T) for m in range(L + 1)]
    base = 2 * math.pi ** 2.5 / (zeta * eta * math.sqrt(zeta + eta)) * K
    memo = {}

    def vrr(ex, cx, m):
        if min(ex) < 0 or min(cx) < 0:
            return 0.0
        key = (ex, cx, m)
        if key in memo:
            return memo[key]
        if ex == (0, 0, 0) and cx == (0, 0, 0):
            r = base * F[m]
        elif ex != (0, 0, 0):
            i = next(d for d in range(3) if ex[d] > 0)
            e1 = list(ex)
            e1[i] -= 1
            e1 = tuple(e1)
            e2 = list(e1)
            e2[i] -= 1
            e2 = tuple(e2)
            c1 = list(cx)
            c1[i] -= 1
            c1 = tuple(c1)
            r = (P[i] - A[i]) * vrr(e1, cx, m) + (W[i] - P[i]) * vrr(e1, cx, m + 1)
            if e1[i] > 0:
                r += e1[i] / (2 * zeta) * (vrr(e2, cx, m) - rho / zeta * vrr(e2, cx, m + 1))
            if cx[i] > 0:
                r += cx[i] / (2 * (zeta + eta)) * vrr(e1, c1, m + 1)
        else:
            i = next(d for d in range(3) if cx[d] > 0)
            c1 = list(cx)
            c1[i] -= 1
            c1 = tuple(c1)
            c2 = list(c1)
            c2[i] -= 1
            c2 = tuple(c2)
            r = (Q[i] - C[i]) * vrr(ex, c1, m) + (W[i] - Q[i]) * vrr(ex, c1, m + 1)
            if c1[i] > 0:
                r += c1[i] / (2 * eta) * (vrr(ex, c2, m) - rho / eta * vrr(ex, c2, m + 1))
        memo[key] = r
        return r

    def hrr(ax, bx, cx):
        if min(bx) < 0:
            return 0.0
        if bx == (0, 0, 0):
            return vrr(ax, cx, 0)
        i = next(d for d in range(3) if bx[d] > 0)
        bm = list(bx)
        bm[i] -= 1
        ap = list(ax)
        ap[i] += 1
        return hrr(tuple(ap), tuple(bm), cx) + (A[i] - B[i]) * hrr(ax, tuple(bm), cx)

    out = np.zeros((len(cart_list(la)), len(cart_list(lb)), len(cart_list(lc))))
    for x, ca in enumerate(cart_list(la)):
        for y, cb in enumerate(cart_list(lb)):
            for z, cc in enumerate(cart_list(lc)):
                out[x, y, z] = hrr(ca, cb, cc)
    return out


def int3c2e(ao, fit):
    """(mn|P), array [m, n, P]."""
    da, dp = _norms(ao), _norms(fit)
    offa = np.cumsum([0] + [2 * s[0] + 1 for s in ao.shells])
    offp = np.cumsum([0] + [2 * s[0] + 1 for s in fit.shells])
    out = np.zeros((ao.nbf(), ao.nbf(), fit.nbf()))
    for i, (la, A, ea, ca) in enumerate(ao.shells):
        for j, (lb, B, eb, cb) in enumerate(ao.shells):
            for k, (lc, C, ec, cc) in enumerate(fit.shells):
                blk = 0.0
                for a, xa in zip(ea, ca):
                    for b, xb in zip(eb, cb):
                        for g, xc in zip(ec, cc):
                            blk = blk + xa * xb * xc * _prim_eri3(la, A, a, lb, B, b, lc, C, g)
                blk = np.einsum("xyz,ax,by,cz->abc", blk, solid_harmonics(la), solid_harmonics(lb),
                                solid_harmonics(lc))
                out[offa[i]:offa[i + 1], offa[j]:offa[j + 1], offp[k]:offp[k + 1]] = blk
    return out * da[:, None, None] * da[None, :, None] * dp[None, None, :]


def int2c2e(fit):
    """(P|Q): the three-centre case with an s function of exponent 0 in place of n."""
    dp = _norms(fit)
    off = np.cumsum([0] + [2 * s[0] + 1 for s in fit.shells])
    out = np.zeros((fit.nbf(), fit.nbf()))
    for i, (la, A, ea, ca) in enumerate(fit.shells):
        for k, (lc, C, ec, cc) in enumerate(fit.shells):
            blk = 0.0
            for a, xa in zip(ea, ca):
                for g, xc in zip(ec, cc):
                    blk = blk + xa * xc * _prim_eri3(la, A, a, 0, A, 0.0, lc, C, g)[:, 0, :]
            out[off[i]:off[i + 1], off[k]:off[k + 1]] = solid_harmonics(la) @ blk @ solid_harmonics(lc).T
    return out * np.outer(dp, dp)
