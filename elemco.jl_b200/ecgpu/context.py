"""Context object over the libecgpu C ABI (one GPU, one CUDA stream).

Arrays are numpy float64 in the reference's index order and Fortran (column-
major) layout, exactly what the Julia ``ccall`` glue passes.
"""
import ctypes as C
import weakref

import numpy as np

from ._lib import (CcOpts, ECGError, ECG_PREC_FP64, as_f, dptr, fvec, lib)


class Context:
    """Device-resident closed-shell CC problem (``ecg_ctx``)."""

    def __init__(self, device=0):
        self._L = lib()
        h = C.c_void_p()
        st = self._L.ecg_create(int(device), C.byref(h))
        if st:
            raise ECGError(st, self._L.ecg_last_error(None).decode())
        self._h = h
        self._handles = weakref.WeakSet()  # device handles to release before the context
        self.no = self.nv = self.nq = 0

    def close(self):
        if getattr(self, "_h", None):
            for obj in list(self._handles):
                obj.close()
            self._L.ecg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, st):
        if st:
            raise ECGError(st, self._L.ecg_last_error(self._h).decode())

    # ------------------------------------------------------------ setup
    def set_mem_cap(self, nbytes):
        self._chk(self._L.ecg_set_mem_cap(self._h, int(nbytes)))

    def set_precision(self, prec=ECG_PREC_FP64):
        self._chk(self._L.ecg_set_precision(self._h, int(prec)))

    def tune_save(self, path):
        """Write the GEMM tuning table; returns its number of entries."""
        n = C.c_int64()
        self._chk(self._L.ecg_tune_save(self._h, str(path).encode(), C.byref(n)))
        return n.value

    def tune_load(self, path):
        """Merge a tuning file into the table; returns its number of entries."""
        n = C.c_int64()
        self._chk(self._L.ecg_tune_load(self._h, str(path).encode(), C.byref(n)))
        return n.value

    def set_option(self, key, value):
        """``ecg_set_option``: ECG_OPT_TRIPLES_BATCH, ECG_OPT_TC_WAIT_NS,
        ECG_OPT_AUTOTUNE (0 = automatic / off)."""
        self._chk(self._L.ecg_set_option(self._h, int(key), int(value)))

    def set_system(self, B, h1, e0, nocc):
        """B[p,q,Q] (n x n x nQ) DF factors, h1 (n x n), core energy e0."""
        B = as_f(B)
        h1 = as_f(h1)
        n, n2, nq = B.shape
        if n != n2 or h1.shape != (n, n):
            raise ValueError("shape mismatch between B and h1")
        self.no, self.nv, self.nq, self.n = int(nocc), n - int(nocc), nq, n
        self._chk(self._L.ecg_set_system(self._h, self.no, self.nv, self.nq, dptr(B), dptr(h1),
                                         float(e0)))

    @staticmethod
    def opts(**kw):
        o = CcOpts()
        lib().ecg_default_opts(C.byref(o))
        for k, v in kw.items():
            setattr(o, k, v)
        return o

    def _t(self):
        return fvec((self.nv, self.no)), fvec((self.nv, self.nv, self.no, self.no))

    # ------------------------------------------------------------ calls
    def fock(self):
        f = fvec((self.n, self.n))
        eps = fvec(self.n)
        e = C.c_double()
        self._chk(self._L.ecg_fock(self._h, dptr(f), dptr(eps), C.byref(e)))
        return f, eps, e.value

    def mp2(self):
        T1, T2 = self._t()
        e = C.c_double()
        self._chk(self._L.ecg_mp2(self._h, dptr(T1), dptr(T2), C.byref(e)))
        return e.value, T1, T2

    def cc_residual(self, T1, T2, dc=False):
        T1, T2 = as_f(T1), as_f(T2)
        R1, R2 = self._t()
        self._chk(self._L.ecg_cc_residual(self._h, int(dc), dptr(T1), dptr(T2), dptr(R1),
                                          dptr(R2)))
        return R1, R2

    def cc_solve(self, T1, T2, dc=False, opts=None):
        T1, T2 = as_f(T1).copy(order="F"), as_f(T2).copy(order="F")
        out = fvec(5)
        it, conv = C.c_int32(), C.c_int32()
        o = opts or self.opts()
        self._chk(self._L.ecg_cc_solve(self._h, int(dc), C.byref(o), dptr(T1), dptr(T2),
                                       dptr(out), C.byref(it), C.byref(conv)))
        return {"E": out[0], "ESS": out[1], "EOS": out[2], "NormR": out[3], "dE": out[4],
                "iterations": it.value, "converged": bool(conv.value), "T1": T1, "T2": T2}

    def cc_load(self, T1=None, T2=None, opts=None):
        o = opts or self.opts()
        T1 = None if T1 is None else as_f(T1)
        T2 = None if T2 is None else as_f(T2)
        self._chk(self._L.ecg_cc_load(self._h, dptr(T1), dptr(T2), C.byref(o)))

    def cc_step(self, dc=False, nsteps=1):
        out = fvec(5)
        self._chk(self._L.ecg_cc_step(self._h, int(dc), int(nsteps), dptr(out)))
        return out

    def cc_store(self, T1=None, T2=None):
        if T1 is None:
            T1, T2 = self._t()
        self._chk(self._L.ecg_cc_store(self._h, dptr(T1), dptr(T2)))
        return T1, T2

    def pert_t(self, T1=None, T2=None):
        """(T) and [T] energies; T1 = T2 = None uses the amplitudes the context
        holds (from the last mp2 / cc_solve on this system) without an upload."""
        if T1 is not None or T2 is not None:
            T1, T2 = as_f(T1), as_f(T2)
        e, eb = C.c_double(), C.c_double()
        self._chk(self._L.ecg_pert_t(self._h, dptr(T1), dptr(T2), C.byref(e), C.byref(eb)))
        return e.value, eb.value

    def lambda_residual(self, T1, T2, U1, U2, dc=False):
        R1, R2 = self._t()
        self._chk(self._L.ecg_lambda_residual(self._h, int(dc), dptr(as_f(T1)), dptr(as_f(T2)),
                                              dptr(as_f(U1)), dptr(as_f(U2)), dptr(R1),
                                              dptr(R2)))
        return R1, R2

    def lambda_solve(self, T1, T2, dc=False, opts=None):
        U1, U2 = self._t()
        out = fvec(3)
        it, conv = C.c_int32(), C.c_int32()
        o = opts or self.opts()
        self._chk(self._L.ecg_lambda_solve(self._h, int(dc), C.byref(o), dptr(as_f(T1)),
                                           dptr(as_f(T2)), dptr(U1), dptr(U2), dptr(out),
                                           C.byref(it), C.byref(conv)))
        return {"U1": U1, "U2": U2, "norm": out[0], "NormR": out[1], "dnorm": out[2],
                "iterations": it.value, "converged": bool(conv.value)}

    def lambda_pert_t(self, T1, T2, U1, U2):
        """Lambda-(T); T1 = T2 = None uses the amplitudes the context holds."""
        if T1 is not None or T2 is not None:
            T1, T2 = as_f(T1), as_f(T2)
        e, eb = C.c_double(), C.c_double()
        self._chk(self._L.ecg_lambda_pert_t(self._h, dptr(T1), dptr(T2),
                                            dptr(as_f(U1)), dptr(as_f(U2)), C.byref(e),
                                            C.byref(eb)))
        return e.value, eb.value

    def one_rdm(self, T1, T2, U1, U2):
        D1 = fvec((self.n, self.n))
        dD1 = fvec((self.n, self.n))
        self._chk(self._L.ecg_one_rdm(self._h, dptr(as_f(T1)), dptr(as_f(T2)), dptr(as_f(U1)),
                                      dptr(as_f(U2)), dptr(D1), dptr(dD1)))
        return D1, dD1

    def energy_gradient(self, T1, T2, U1, U2):
        """dE/dh (n x n, MO basis, orbitals fixed) of the converged CC energy:
        the T1-dressed 1RDM plus the HF density."""
        G = fvec((self.n, self.n))
        self._chk(self._L.ecg_energy_gradient(self._h, dptr(as_f(T1)), dptr(as_f(T2)),
                                              dptr(as_f(U1)), dptr(as_f(U2)), dptr(G)))
        return G

    def cc_step_host(self, T1, T2, dc=False):
        """One iteration with host amplitudes (updated in place)."""
        out = fvec(5)
        self._chk(self._L.ecg_cc_step_host(self._h, int(dc), dptr(T1), dptr(T2), dptr(out)))
        return out

    def stream(self):
        p = C.c_void_p()
        self._chk(self._L.ecg_get_stream(self._h, C.byref(p)))
        return p.value

    def kernel_launches(self):
        return int(self._L.ecg_kernel_launches(self._h))

    def set_gemm_timing(self, enable=True):
        self._chk(self._L.ecg_set_gemm_timing(self._h, int(enable)))

    def gemm_time(self):
        ms, fl = C.c_double(), C.c_double()
        n = C.c_int64()
        self._chk(self._L.ecg_gemm_time(self._h, C.byref(ms), C.byref(n), C.byref(fl)))
        return ms.value, n.value, fl.value

    def kernel_time(self, family):
        """(ms, launches, work) of a kernel family (ECG_KT_*) since the last read."""
        ms, w = C.c_double(), C.c_double()
        n = C.c_int64()
        self._chk(self._L.ecg_kernel_time(self._h, int(family), C.byref(ms), C.byref(n),
                                          C.byref(w)))
        return ms.value, n.value, w.value

    # ------------------------------------------------------------ integrals
    def int1e(self, kind, shells, charges=None, xyz=None, origin=None):
        """ecg_int1e over a :class:`ecgpu.basis.ShellArrays` basis: (n, n), or
        (3, n, n) for the dipole, column-major values in numpy's (m, n) order."""
        from ._lib import ECG_INT_DIPOLE
        n = shells.nbf
        ncomp = 3 if kind == ECG_INT_DIPOLE else 1
        out = np.zeros(ncomp * n * n)
        st = shells.struct()
        Z = None if charges is None else np.ascontiguousarray(charges, dtype=np.float64)
        X = None if xyz is None else np.ascontiguousarray(xyz, dtype=np.float64).ravel()
        O = None if origin is None else np.ascontiguousarray(origin, dtype=np.float64).ravel()
        self._chk(self._L.ecg_int1e(self._h, int(kind), C.byref(st), 0 if Z is None else len(Z),
                                    dptr(Z), dptr(X), dptr(O), dptr(out)))
        out = out.reshape(ncomp, n, n).transpose(0, 2, 1)
        return out if ncomp == 3 else out[0]

    def int2c2e(self, fit):
        n = fit.nbf
        out = np.zeros(n * n)
        st = fit.struct()
        self._chk(self._L.ecg_int2c2e(self._h, C.byref(st), dptr(out)))
        return out.reshape(n, n).T

    def int3c2e(self, ao, fit):
        """(mn|P) as an F-ordered (nao, nao, naux) array."""
        n, m = ao.nbf, fit.nbf
        out = np.zeros((n, n, m), order="F")
        sa, sf = ao.struct(), fit.struct()
        self._chk(self._L.ecg_int3c2e(self._h, C.byref(sa), C.byref(sf), dptr(out)))
        return out

    def df_factors(self, ao, fit, M):
        """:class:`DFFactors` AAL[m,n,L] = sum_P (mn|P) M[P,L] held on the device."""
        return DFFactors(self, ao, fit, M)

    def diag_gemm(self, ta, tb, alpha, A, B, beta, Cm):
        A, B = as_f(A), as_f(B)
        Cm = as_f(Cm).copy(order="F")
        m, n = Cm.shape
        k = A.shape[0] if ta == "T" else A.shape[1]
        self._chk(self._L.ecg_diag_gemm(self._h, ta.encode(), tb.encode(), m, n, k, float(alpha),
                                        dptr(A), A.shape[0], dptr(B), B.shape[0], float(beta),
                                        dptr(Cm), m))
        return Cm

    def diag_permute(self, x, perm, alpha=1.0, beta=0.0, out=None):
        x = as_f(x)
        dims = (C.c_int64 * x.ndim)(*x.shape)
        pm = (C.c_int * x.ndim)(*perm)
        oshape = tuple(x.shape[p] for p in perm)
        out = fvec(oshape) if out is None else as_f(out).copy(order="F")
        self._chk(self._L.ecg_diag_permute(self._h, x.ndim, dims, pm, float(alpha), dptr(x),
                                           float(beta), dptr(out)))
        return out


class Diis:
    """Stand-alone device DIIS (``ecg_diis_*``, plain dot products)."""

    def __init__(self, ctx, length, maxdiis=6, resthr=10.0):
        h = C.c_void_p()
        ctx._chk(ctx._L.ecg_diis_create(ctx._h, int(maxdiis), float(resthr), int(length),
                                        C.byref(h)))
        self._ctx, self._h, self.length = ctx, h, int(length)

    def perform(self, vec, res):
        vec = np.ascontiguousarray(vec, dtype=np.float64).copy()
        res = np.ascontiguousarray(res, dtype=np.float64)
        self._ctx._chk(self._ctx._L.ecg_diis_perform(self._h, dptr(vec), dptr(res)))
        return vec

    def close(self):
        if self._h:
            self._ctx._L.ecg_diis_destroy(self._h)
            self._h = None


class DFFactors:
    """Density-fitted three-index factors on the device (``ecg_df_*``):
    AAL[m,n,L] = sum_P (mn|P) M[P,L] for an AO basis and a fitting basis
    (:class:`ecgpu.basis.ShellArrays`), M (naux x nL) with M M^T = (P|Q)^-1."""

    def __init__(self, ctx, ao, fit, M):
        M = as_f(M)
        if M.shape[0] != fit.nbf:
            raise ValueError("M must have one row per fitting function")
        h = C.c_void_p()
        sa, sf = ao.struct(), fit.struct()
        ctx._chk(ctx._L.ecg_df_create(ctx._h, C.byref(sa), C.byref(sf), dptr(M), M.shape[1],
                                      C.byref(h)))
        self._ctx, self._h = ctx, h
        self.nao, self.nL = ao.nbf, M.shape[1]
        ctx._handles.add(self)

    def _handle(self):
        if not self._h:
            raise ValueError("DF factors already released")
        return self._h

    def fock(self, h, Cocc):
        """F = h + 2 J - K (closed shell) from the occupied orbitals Cocc (n x nocc)."""
        n = self.nao
        h = as_f(h)
        Cocc = as_f(np.reshape(Cocc, (n, -1)))
        F = fvec((n, n))
        self._ctx._chk(self._ctx._L.ecg_df_fock(self._handle(), dptr(h), dptr(Cocc),
                                                Cocc.shape[1], dptr(F)))
        return F

    def mo(self, Cmo):
        """B[p,q,L] = sum_{m,n} C[m,p] AAL[m,n,L] C[n,q], F-ordered (nmo, nmo, nL)."""
        Cmo = as_f(Cmo)
        nmo = Cmo.shape[1]
        B = fvec((nmo, nmo, self.nL))
        self._ctx._chk(self._ctx._L.ecg_df_mo(self._handle(), dptr(Cmo), nmo, dptr(B)))
        return B

    def close(self):
        if self._h:
            self._ctx._L.ecg_df_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
