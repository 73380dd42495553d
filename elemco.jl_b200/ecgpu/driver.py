"""Host driver mirroring ElemCo.jl's closed-shell CC entry points.

    EC = ECInfo()
    EC.set("cc", thr=1e-12)                    # @set cc thr=1e-12
    energies = ccdriver(EC, "ccsd(t)", fcidump="H2O.FCIDUMP")
    energies["CCSD(T)"], energies["MP2c"], ...

Keys of the returned dict follow the reference's OutDict
(src/cc/ccdriver.jl:226-281, :387-390): ``HF``, ``MP2c``, ``MP2``,
``<M>c``, ``<M>``, ``Ec``, ``E`` and, with (T), ``[T]``, ``(T)``,
``<M>(T)c``, ``<M>(T)`` where ``<M>`` is ``CCSD``/``DCSD`` or
``ΛCCSD``/``ΛDCSD``.  All coupled-cluster work runs in libecgpu on the GPU;
this module only prepares inputs (FCIDUMP parsing, Cholesky factorisation of
4-index integrals) and writes the amplitude files.
"""
import math
import os
import re

import numpy as np

from ._lib import ECG_DIIS_CS, ECG_DIIS_PLAIN, ECG_PREC_FP64, ECG_PREC_MIXED
from .context import Context

# ---------------------------------------------------------------- options


class _Group(dict):
    def __getattr__(self, k):
        try:
            return self[k]
        except KeyError as e:
            raise AttributeError(k) from e


def _default_options():
    """Fields of CcOptions/DiisOptions the path reads (src/infos/options.jl:128-282)
    plus a ``gpu`` group (precision, device).  ``diis.dot`` selects the dot
    product of the CC DIIS: "cs", the closed-shell custom dots of the current
    reference (src/cc/cc.jl:2498-2499,2598), or "plain", the unweighted dot
    closed-shell CC used before ElemCo.jl 0.13 (src/solvers/diis.jl:155-167),
    which replays the trajectories behind older pinned energies."""
    return {
        "cc": _Group(thr=1.0e-10, conven=0.1, maxit=50, shifts=0.15, shiftp=0.2,
                     properties=False, save="cc_amplitudes", save_lm="cc_multipliers",
                     nomp2=0),
        "diis": _Group(maxdiis=6, resthr=10.0, crop=False, maxcrop=3, dot="cs"),
        "cholesky": _Group(thr=1.0e-12, thred=1.0e-6),
        "scf": _Group(thr=1.0e-10, thren=-1.0, maxit=50),
        "wf": _Group(core="large"),
        "gpu": _Group(precision="fp64", device=0),
    }


class ECInfo:
    """Subset of the reference's ECInfo (src/infos/ecinfos.jl:103-155)."""

    def __init__(self, scr=None):
        self.options = _default_options()
        self.scr = scr or os.getcwd()
        self.ext = ".bin"
        self.fd = None
        self._ctx = None
        self.system = None
        self.hf = None
        self._ncore = 0

    def set(self, group, **kw):
        """``@set group key=val`` (src/ElemCo.jl:331-357)."""
        g = self.options[group]
        for k, v in kw.items():
            if k not in g:
                raise KeyError(f"unknown option {group}.{k}")
            g[k] = v

    def set_system(self, mol, basis):
        """The molecule (:class:`ecgpu.molecules.Molecule`, bohr) and its basis
        sets {"ao": ..., "jkfit": ..., "mpfit": ...}, as
        ``ECInfo(system=parse_geometry(xyz, basis))`` (src/infos/ecinfos.jl)."""
        self.system = (mol, {k.lower(): v for k, v in basis.items()})
        self.hf = None

    def mo_dipole(self, origin=(0.0, 0.0, 0.0)):
        """<p|r - origin|q> over the active orbitals of the last dfints (3, n, n)."""
        hf, nc = self.hf, self._ncore
        C = hf.C[:, nc:]
        return np.array([C.T @ D @ C for D in hf.ints.dipole(origin)])

    def context(self):
        """The GPU context; the packaged GEMM tuning table for B200
        (``tuning/b200.txt``, written by the autotuner) is loaded on creation."""
        if self._ctx is None:
            self._ctx = Context(self.options["gpu"].device)
            table = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning", "b200.txt")
            if os.path.exists(table):
                self._ctx.tune_load(table)
        return self._ctx


# ---------------------------------------------------------------- FCIDUMP


class FDump:
    """MO integrals of a closed-shell system.

    ``V[p,q,r,s] = <pq|rs>`` (physicists' notation, as FDump{4} in
    src/integrals/dump.jl:100-128), ``h`` one-electron, ``e0`` core energy;
    or, instead of ``V``, DF factors ``B[p,q,Q]``.
    """

    def __init__(self, h, e0, nelec, V=None, B=None, st=False, head=None):
        self.h = np.asarray(h, dtype=np.float64)
        self.e0 = float(e0)
        self.nelec = int(nelec)
        self.V = V
        self.B = B
        self.st = bool(st)
        self.head = head or {}

    @property
    def norb(self):
        return self.h.shape[0]


def _parse_header(txt):
    head = {}
    toks = [t for t in re.split(r"[\s,]+", txt.replace("&FCI", " ").replace("=", " = ")) if t]
    key = None
    for i, t in enumerate(toks):
        if i + 1 < len(toks) and toks[i + 1] == "=":
            key = t.upper()
            head[key] = []
        elif t != "=" and key is not None:
            head[key].append(t)
    return head


def read_fcidump(path):
    """Read an FCIDUMP text file (src/integrals/dump.jl:326-348, :600-631).

    Integral lines ``x i j k l`` are (ij|kl); 8-fold symmetry is applied unless
    the header has ``ST>0`` (non-Hermitian: particle symmetry only).
    """
    with open(path) as f:
        text = f.read()
    m = re.search(r"^\s*(/|&END)\s*$", text, re.M)
    if not m:
        raise ValueError("FCIDUMP header not terminated")
    head = _parse_header(text[: m.start()])
    if "NORB" not in head:
        raise ValueError("NORB option not found in fcidump")
    n = int(head["NORB"][0])
    st = int(head.get("ST", ["0"])[0]) > 0
    if int(head.get("IUHF", ["0"])[0]) > 0:
        raise ValueError("unrestricted FCIDUMP: only closed-shell integrals are supported")
    rows = [r for r in (l.split() for l in text[m.end():].splitlines()) if len(r) == 5]
    vals = np.array([float(r[0].replace("D", "E")) for r in rows])
    idx = np.array([[int(x) for x in r[1:]] for r in rows], dtype=np.int64).reshape(-1, 4)
    if (idx > n).any():
        raise ValueError("Index larger than norb")
    V = np.zeros((n, n, n, n))
    h = np.zeros((n, n))
    e0 = None
    i1, i2, i3, i4 = (idx[:, c] - 1 for c in range(4))
    two = idx[:, 3] > 0
    one = (~two) & (idx[:, 1] > 0)
    core = (idx[:, 3] <= 0) & (idx[:, 1] <= 0) & (idx[:, 0] <= 0)
    a, b, c, d, x = i1[two], i2[two], i3[two], i4[two], vals[two]
    V[a, c, b, d] = x
    V[c, a, d, b] = x
    if not st:
        V[a, d, b, c] = x
        V[b, c, a, d] = x
        V[b, d, a, c] = x
        V[d, a, c, b] = x
        V[c, b, d, a] = x
        V[d, b, c, a] = x
    h[i1[one], i2[one]] = vals[one]
    if not st:
        h[i2[one], i1[one]] = vals[one]
    if core.any():
        e0 = float(vals[core][-1])
    if e0 is None:
        raise ValueError("No core energy found in fcidump. Incomplete file?")
    nelec = int(head.get("NELEC", ["0"])[0])
    return FDump(h, e0, nelec, V=V, st=st, head=head)


def write_fcidump(path, fd, tol=1e-14):
    """Write a closed-shell FCIDUMP (src/integrals/dump.jl:752) from ``fd.V``."""
    n = fd.norb
    lines = [f" &FCI NORB={n},NELEC={fd.nelec},MS2=0,", "  ORBSYM=" + "1," * n,
             "  ISYM=1," + (" ST=1," if fd.st else ""), " /"]
    V = fd.V
    for i in range(n):
        for j in range(i + 1):
            for k in range(n):
                for l in range(k + 1):
                    if (i * (i + 1) // 2 + j) < (k * (k + 1) // 2 + l):
                        continue
                    x = V[i, k, j, l]  # (ij|kl)
                    if abs(x) > tol:
                        lines.append(f" {x:.16E} {i + 1:3d} {j + 1:3d} {k + 1:3d} {l + 1:3d}")
    for i in range(n):
        for j in range(i + 1):
            if abs(fd.h[i, j]) > tol:
                lines.append(f" {fd.h[i, j]:.16E} {i + 1:3d} {j + 1:3d}   0   0")
    lines.append(f" {fd.e0:.16E}   0   0   0   0")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def cholesky_df(V, tol=1e-12):
    """Pivoted Cholesky of the (pr|qs) supermatrix: ``B[p,q,Q]``, Fortran order.

    Same decomposition as calc_integrals_decomposition
    (src/integrals/decomptools.jl:22-52): row-maximum pivoting, stop when the
    largest remaining diagonal is below ``tol``.
    """
    n = V.shape[0]
    M = np.ascontiguousarray(V.transpose(0, 2, 1, 3).reshape(n * n, n * n))
    d = np.diag(M).copy()
    L = np.zeros((n * n, n * n))
    r = 0
    while r < n * n:
        k = int(np.argmax(d))
        if d[k] <= tol:
            break
        col = M[:, k] - L[:, :r] @ L[k, :r]
        col /= math.sqrt(d[k])
        L[:, r] = col
        d -= col * col
        d[k] = 0.0
        r += 1
    return np.asfortranarray(L[:, :r].reshape(n, n, r))


# ---------------------------------------------------------------- amplitude files


def miosave(fname, *arrs):
    """Binary array file of src/tools/myio.jl:42-66 (type id, count, dims, data)."""
    with open(fname, "wb") as f:
        np.array([12, len(arrs)], dtype=np.int64).tofile(f)  # 12 = Float64
        for a in arrs:
            np.array([a.ndim, *a.shape], dtype=np.int64).tofile(f)
        for a in arrs:
            np.asfortranarray(a, dtype=np.float64).T.tofile(f)  # column-major bytes


def mioload(fname):
    with open(fname, "rb") as f:
        itype, narr = np.fromfile(f, dtype=np.int64, count=2)
        if itype != 12:
            raise ValueError("only Float64 arrays supported")
        shapes = []
        for _ in range(narr):
            nd = int(np.fromfile(f, dtype=np.int64, count=1)[0])
            shapes.append(tuple(int(x) for x in np.fromfile(f, dtype=np.int64, count=nd)))
        out = []
        for s in shapes:
            cnt = int(np.prod(s)) if s else 1
            out.append(np.fromfile(f, dtype=np.float64, count=cnt).reshape(s[::-1]).T.copy(order="F"))
    return out


# ---------------------------------------------------------------- driver


def parse_method(method):
    """Closed-shell methods of the kept API: ccsd, dcsd, ccsd(t), λccsd, λccsd(t), λdcsd.

    Returns (name, dc, lambda, pert).  Follows ECMethod's prefix/suffix rules
    (src/infos/ecmethods.jl:23-128) for these names.
    """
    m = method.strip().lower().replace("λ", "l").replace("Λ", "l")
    if m.startswith("lambda-"):
        m = "l" + m[7:]
    lam = m.startswith("l") and m[1:3] in ("cc", "dc")
    if lam:
        m = m[1:]
    pert = m.endswith("(t)")
    if pert:
        m = m[:-3]
    if m not in ("ccsd", "dcsd"):
        raise ValueError(f"unsupported closed-shell method {method!r} "
                         "(supported: ccsd, dcsd, ccsd(t), λccsd, λccsd(t), λdcsd)")
    return m.upper(), m == "dcsd", lam, pert


def _system_from(EC, fcidump):
    if fcidump:
        EC.fd = read_fcidump(fcidump)
    fd = EC.fd
    if fd is None:
        raise ValueError("no integrals: pass fcidump= or set EC.fd")
    if fd.st:
        raise ValueError("similarity-transformed (non-Hermitian) integrals are not supported "
                         "by the DF GPU path")
    if fd.B is None:
        fd.B = cholesky_df(fd.V, EC.options["cholesky"].thr)
    if fd.nelec % 2:
        raise ValueError("closed-shell path needs an even number of electrons")
    return fd.B, fd.h, fd.e0, fd.nelec // 2


def _solver_opts(ctx, o):
    dots = {"cs": ECG_DIIS_CS, "plain": ECG_DIIS_PLAIN}
    if o["diis"].dot not in dots:
        raise ValueError(f"diis.dot must be 'cs' or 'plain', not {o['diis'].dot!r}")
    return ctx.opts(thr=o["cc"].thr, conven=o["cc"].conven, maxit=o["cc"].maxit,
                    shifts=o["cc"].shifts, shiftp=o["cc"].shiftp, maxdiis=o["diis"].maxdiis,
                    resthr=o["diis"].resthr, diis_dot=dots[o["diis"].dot])


def ccdriver(EC, method, fcidump=""):
    """``ccdriver`` (src/cc/ccdriver.jl:37-76) for closed-shell methods on the GPU."""
    name, dc, lam, pert = parse_method(method)
    main = ("Λ" if lam else "") + name
    B, h, e0, nocc = _system_from(EC, fcidump)
    ctx = EC.context()
    o = EC.options
    ctx.set_precision(ECG_PREC_MIXED if o["gpu"].precision == "mixed" else ECG_PREC_FP64)
    ctx.set_system(B, h, e0, nocc)
    out = {}
    _, _, EHF = ctx.fock()
    out["HF"] = EHF
    emp2, T1, T2 = ctx.mp2()
    out["MP2c"] = emp2
    out["MP2"] = emp2 + EHF
    opts = _solver_opts(ctx, o)
    r = ctx.cc_solve(T1, T2, dc=dc, opts=opts)
    if not r["converged"]:
        print("WARNING: CC iterations did not converge!")
    E = r["E"]
    out[main + "c"] = E
    out[main] = E + EHF
    out["Ec"] = E
    out["E"] = E + EHF
    out["iterations"] = r["iterations"]
    T1, T2 = r["T1"], r["T2"]
    if o["cc"].save:
        miosave(os.path.join(EC.scr, o["cc"].save + "_1" + EC.ext), T1)
        miosave(os.path.join(EC.scr, o["cc"].save + "_2" + EC.ext), T2)
    if lam or o["cc"].properties:
        lr = ctx.lambda_solve(T1, T2, dc=dc, opts=opts)
        if not lr["converged"]:
            print("WARNING: CC-LM iterations did not converge!")
        U1, U2 = lr["U1"], lr["U2"]
        out["lambda_iterations"] = lr["iterations"]
        if o["cc"].save_lm:
            miosave(os.path.join(EC.scr, o["cc"].save_lm + "_1" + EC.ext), U1)
            miosave(os.path.join(EC.scr, o["cc"].save_lm + "_2" + EC.ext), U2)
    if pert:
        # the context still holds the converged amplitudes: no re-upload
        if lam:
            ET3, ET3b = ctx.lambda_pert_t(None, None, U1, U2)
        else:
            ET3, ET3b = ctx.pert_t()
        out["[T]"] = ET3b
        out["(T)"] = ET3
        out[main + "(T)c"] = E + ET3
        out[main + "(T)"] = E + ET3 + EHF
    return out


def rrule_cc_energy(EC, method, h=None, fcidump=""):
    """Reverse rule of the total closed-shell CCSD/DCSD energy E(h).

    `h` is the MO-basis one-electron matrix (default: that of the integrals);
    orbitals are held fixed.  Returns (E, pullback) with pullback(dE) = dE * G,
    G = dE/dh from the Lambda (adjoint) equations: the T1-dressed 1RDM plus the
    HF density (ecg_energy_gradient).  For a field term h + lambda P (e.g. a
    dipole operator P) dE/dlambda = sum(G * P).  This is the rule a Julia
    ChainRules.rrule for the @cc energy returns; the reference itself has no
    analytic property path (it computes the densities, src/cc/cc_lagrange.jl:786-791).
    """
    name, dc, lam, pert = parse_method(method)
    if pert or name not in ("CCSD", "DCSD"):
        raise ValueError("energy gradients are available for ccsd, dcsd, λccsd and λdcsd")
    B, h0, e0, nocc = _system_from(EC, fcidump)
    h = h0 if h is None else np.asarray(h, dtype=float)
    ctx = EC.context()
    o = EC.options
    ctx.set_precision(ECG_PREC_MIXED if o["gpu"].precision == "mixed" else ECG_PREC_FP64)
    ctx.set_system(B, h, e0, nocc)
    _, _, EHF = ctx.fock()
    _, T1, T2 = ctx.mp2()
    opts = _solver_opts(ctx, o)
    r = ctx.cc_solve(T1, T2, dc=dc, opts=opts)
    if not r["converged"]:
        raise RuntimeError("CC iterations did not converge")
    lr = ctx.lambda_solve(r["T1"], r["T2"], dc=dc, opts=opts)
    if not lr["converged"]:
        raise RuntimeError("CC-LM iterations did not converge")
    G = ctx.energy_gradient(r["T1"], r["T2"], lr["U1"], lr["U2"])
    E = EHF + r["E"]

    def pullback(dE):
        return dE * G

    return E, pullback


def dfhf(EC):
    """``@dfhf`` (src/scf/dfhf.jl:24-94): closed-shell DF-HF with the system's
    ``ao`` and ``jkfit`` bases; returns {"HF": E, "E": E}."""
    from .scf import dfhf as _dfhf
    mol, basis = EC.system
    o = EC.options["scf"]
    EC.hf = _dfhf(EC.context(), mol, basis["ao"], basis.get("jkfit", "cc-pvtz-jkfit"),
                  thr=o.thr, thren=o.thren, maxit=o.maxit, thred=EC.options["cholesky"].thred)
    if not EC.hf.converged:
        print("WARNING: DF-HF did not converge!")
    return {"HF": EC.hf.E, "E": EC.hf.E}


def dfints(EC):
    """``@dfints`` / ``dfdump`` (src/integrals/dfdump.jl:263-301): the active
    orbitals' DF integrals (``mpfit``) with the ``jkfit``-corrected one-electron
    part, stored in ``EC.fd`` (DF factors) for ccdriver."""
    from .scf import dfints as _dfints
    if EC.hf is None:
        raise ValueError("run dfhf first")
    mol, basis = EC.system
    core = EC.options["wf"].core
    nc = mol.ncore() if core == "large" else 0 if core == "none" else None
    if nc is None:
        raise ValueError("wf.core must be 'large' or 'none'")
    B, h1, e0, no, eref = _dfints(EC.hf, basis.get("mpfit", "cc-pvdz-mpfit"),
                                  basis.get("jkfit", "cc-pvtz-jkfit"), ncore=nc,
                                  thred=EC.options["cholesky"].thred)
    EC._ncore = nc
    EC.fd = FDump(h1, e0, 2 * no, B=B)
    return eref


def cc(EC, method, fcidump=""):
    """``@cc method`` (src/ElemCo.jl:523-548)."""
    return ccdriver(EC, method, fcidump=fcidump)
