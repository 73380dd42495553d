"""Gaussian basis sets in the Molpro library format and their shell arrays.

The reference reads its basis sets from ``lib/basis_sets/mpro/<name>.<v>.mpro``
(src/system/parse_basis.jl:35-58, highest version first; ``mpfit`` names map
to ``rifit`` files, ``*`` to ``_st_``).  A block for an element starts with
``! <element name>`` and holds lines ``s, O , exp1, exp2, ...`` (angular
momentum, element symbol, exponents) followed by contraction lines
``c, i.j, c1, c2, ...`` (coefficients of the normalised primitives i..j,
1-based) (parse_basis.jl:90-240).

:func:`read_mpro` parses such files; the package ships the H, C, N, O entries
of the sets the coupled-cluster workloads use in ``basis_data/`` (made by
``basis_data/make_basis_data.py``), and :func:`load` reads either.
:func:`shells` turns a basis and a molecule into the plain shell arrays of
the C ABI (``ecg_shells``), one segmented shell per contraction.
"""
import ctypes as C
import json
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "basis_data", "basis_hcno.json")

L_OF = {"s": 0, "p": 1, "d": 2, "f": 3, "g": 4, "h": 5, "i": 6}
ELEMENTS = {"H": ("hydrogen", 1), "C": ("carbon", 6), "N": ("nitrogen", 7),
            "O": ("oxygen", 8)}


def canonical_name(name):
    """Library file stem of a basis name (mpfit -> rifit, * -> _st_)."""
    return name.strip().lower().replace("*", "_st_").replace("mpfit", "rifit")


def read_mpro(text, elements=None):
    """{symbol: [(l, exponents, [(first, last, coefficients), ...]), ...]} of
    the element blocks in Molpro-format text (first/last 1-based)."""
    names = {v[0]: k for k, v in ELEMENTS.items()}
    out = {}
    cur = None
    for raw in text.splitlines():
        m = re.match(r"^!\s+([a-z]+)\s+", raw)
        if m and m.group(1) in names:
            sym = names[m.group(1)]
            cur = None if (elements and sym not in elements) else out.setdefault(sym, [])
            continue
        if re.match(r"^\s*[!}]", raw):
            cur = None
            continue
        if cur is None:
            continue
        line = re.sub(r"!.*", "", raw).strip().lower()
        if not line:
            continue
        parts = [p.strip() for p in line.split(",")]
        if parts[0] in L_OF and len(parts) >= 3:
            cur.append((L_OF[parts[0]], [float(x) for x in parts[2:] if x], []))
        elif parts[0] == "c" and cur:
            a, b = parts[1].split(".")
            cur[-1][2].append((int(a), int(b), [float(x) for x in parts[2:] if x]))
    return out


def load(name, library=None):
    """Basis `name` as {symbol: shells} from a Molpro library directory
    (``library``/mpro, or $ECGPU_BASIS_LIB) or the packaged data."""
    stem = canonical_name(name)
    lib = library or os.environ.get("ECGPU_BASIS_LIB")
    if lib:
        for v in (2, 1, 0):
            f = os.path.join(lib, "mpro", f"{stem}.{v}.mpro")
            if os.path.exists(f):
                with open(f) as fh:
                    return read_mpro(fh.read())
        raise FileNotFoundError(f"basis {name} not in {lib}")
    with open(DATA) as fh:
        data = json.load(fh)
    if stem not in data:
        raise KeyError(f"basis {name} ({stem}) is not in the packaged data {sorted(data)}")
    return {sym: [(l, e, [tuple(c) for c in cons]) for l, e, cons in sh]
            for sym, sh in data[stem].items()}


class ShellArrays:
    """Plain arrays of one basis on one molecule, and the ctypes struct."""

    def __init__(self, l, nprim, centre, exps, coefs, atom_of_shell):
        self.l = np.asarray(l, dtype=np.int32)
        self.nprim = np.asarray(nprim, dtype=np.int32)
        self.centre = np.ascontiguousarray(centre, dtype=np.float64)
        self.exps = np.ascontiguousarray(exps, dtype=np.float64)
        self.coefs = np.ascontiguousarray(coefs, dtype=np.float64)
        self.atom = np.asarray(atom_of_shell, dtype=np.int32)
        self.nbf = int(np.sum(2 * self.l + 1))

    def struct(self):
        from ._lib import Shells
        P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
        return Shells(len(self.l), P(self.l, C.c_int32), P(self.nprim, C.c_int32),
                      P(self.centre, C.c_double), P(self.exps, C.c_double),
                      P(self.coefs, C.c_double))

    def function_atoms(self):
        return np.repeat(self.atom, 2 * self.l + 1)

    def as_list(self):
        """[(l, centre, exps, coefs)] per shell (the oracle's input form)."""
        out, o = [], 0
        for s, l in enumerate(self.l):
            n = self.nprim[s]
            out.append((int(l), self.centre[3 * s:3 * s + 3], self.exps[o:o + n],
                        self.coefs[o:o + n]))
            o += n
        return out


def shells(basis, symbols, xyz):
    """Segmented shells of `basis` ({symbol: shells}) on atoms `symbols` at
    `xyz` (bohr, n x 3): one shell per contraction line, over its primitives."""
    l, nprim, centre, exps, coefs, atom = [], [], [], [], [], []
    for a, (sym, pos) in enumerate(zip(symbols, np.asarray(xyz, float).reshape(-1, 3))):
        if sym not in basis:
            raise KeyError(f"no {sym} in the basis")
        for lv, ex, cons in basis[sym]:
            for first, last, cf in cons:
                e = ex[first - 1:last]
                if len(cf) != len(e):
                    raise ValueError(f"contraction {first}.{last} of {sym} has {len(cf)} "
                                     f"coefficients for {len(e)} exponents")
                l.append(lv)
                nprim.append(len(e))
                centre.extend(pos)
                exps.extend(e)
                coefs.extend(cf)
                atom.append(a)
    return ShellArrays(l, nprim, centre, exps, coefs, atom)
