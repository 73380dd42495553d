"""ctypes binding of libecgpu.so (declarations in include/ecgpu.h).

The library is loaded from this directory (built by elemco.jl_b200/build.py);
``ECGPU_LIB`` may name another build of the same C ABI.  There is no Python
compute path behind these calls: if the library is missing, loading fails.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

ECG_OK = 0
ECG_ERR_ARG = 1
ECG_ERR_CUDA = 2
ECG_ERR_OOM = 3
ECG_ERR_NONFINITE = 4
ECG_ERR_TIMEOUT = 5
ECG_ERR_STATE = 6
ECG_PREC_FP64 = 0
ECG_PREC_MIXED = 1
ECG_DIIS_CS = 0
ECG_DIIS_PLAIN = 1
ECG_OPT_TRIPLES_BATCH = 1
ECG_OPT_TC_WAIT_NS = 2
ECG_OPT_AUTOTUNE = 3
ECG_KT_DGEMM = 0
ECG_KT_TCGEMM = 1
ECG_KT_TRIPLES = 2
ECG_INT_OVERLAP = 0
ECG_INT_KINETIC = 1
ECG_INT_NUCLEAR = 2
ECG_INT_DIPOLE = 3

_NAMES = {1: "ECG_ERR_ARG", 2: "ECG_ERR_CUDA", 3: "ECG_ERR_OOM", 4: "ECG_ERR_NONFINITE",
          5: "ECG_ERR_TIMEOUT", 6: "ECG_ERR_STATE"}


class ECGError(RuntimeError):
    """A nonzero status from libecgpu; ``code`` is the ECG_ERR_* value."""

    def __init__(self, code, msg):
        super().__init__(f"{_NAMES.get(code, code)}: {msg}")
        self.code = code


class CcOpts(C.Structure):
    _fields_ = [("thr", C.c_double), ("conven", C.c_double), ("maxit", C.c_int32),
                ("shifts", C.c_double), ("shiftp", C.c_double), ("maxdiis", C.c_int32),
                ("resthr", C.c_double), ("diis_dot", C.c_int32)]


class Shells(C.Structure):
    """``ecg_shells``: a basis as plain arrays (include/ecgpu.h)."""
    _fields_ = [("nshell", C.c_int32), ("l", C.POINTER(C.c_int32)),
                ("nprim", C.POINTER(C.c_int32)), ("centre", C.POINTER(C.c_double)),
                ("exps", C.POINTER(C.c_double)), ("coefs", C.POINTER(C.c_double))]


_D = C.POINTER(C.c_double)
_P = C.c_void_p
_S = C.POINTER(Shells)
_lib = None

# name -> (restype, argtypes)
SIGNATURES = {
    "ecg_default_opts": (None, [C.POINTER(CcOpts)]),
    "ecg_create": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "ecg_destroy": (C.c_int, [_P]),
    "ecg_last_error": (C.c_char_p, [_P]),
    "ecg_set_mem_cap": (C.c_int, [_P, C.c_uint64]),
    "ecg_set_precision": (C.c_int, [_P, C.c_int]),
    "ecg_set_option": (C.c_int, [_P, C.c_int32, C.c_int64]),
    "ecg_tune_save": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_int64)]),
    "ecg_tune_load": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_int64)]),
    "ecg_set_system": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, _D, _D, C.c_double]),
    "ecg_fock": (C.c_int, [_P, _D, _D, _D]),
    "ecg_mp2": (C.c_int, [_P, _D, _D, _D]),
    "ecg_cc_residual": (C.c_int, [_P, C.c_int, _D, _D, _D, _D]),
    "ecg_cc_solve": (C.c_int, [_P, C.c_int, C.POINTER(CcOpts), _D, _D, _D,
                               C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "ecg_cc_load": (C.c_int, [_P, _D, _D, C.POINTER(CcOpts)]),
    "ecg_cc_step": (C.c_int, [_P, C.c_int, C.c_int32, _D]),
    "ecg_cc_store": (C.c_int, [_P, _D, _D]),
    "ecg_pert_t": (C.c_int, [_P, _D, _D, _D, _D]),
    "ecg_lambda_residual": (C.c_int, [_P, C.c_int, _D, _D, _D, _D, _D, _D]),
    "ecg_lambda_solve": (C.c_int, [_P, C.c_int, C.POINTER(CcOpts), _D, _D, _D, _D, _D,
                                   C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "ecg_lambda_pert_t": (C.c_int, [_P, _D, _D, _D, _D, _D, _D]),
    "ecg_one_rdm": (C.c_int, [_P, _D, _D, _D, _D, _D, _D]),
    "ecg_energy_gradient": (C.c_int, [_P, _D, _D, _D, _D, _D]),
    "ecg_diis_create": (C.c_int, [_P, C.c_int32, C.c_double, C.c_int64, C.POINTER(_P)]),
    "ecg_diis_perform": (C.c_int, [_P, _D, _D]),
    "ecg_diis_destroy": (C.c_int, [_P]),
    "ecg_kernel_launches": (C.c_int64, [_P]),
    "ecg_cc_step_host": (C.c_int, [_P, C.c_int, _D, _D, _D]),
    "ecg_get_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "ecg_set_gemm_timing": (C.c_int, [_P, C.c_int]),
    "ecg_gemm_time": (C.c_int, [_P, _D, C.POINTER(C.c_int64), _D]),
    "ecg_kernel_time": (C.c_int, [_P, C.c_int32, _D, C.POINTER(C.c_int64), _D]),
    "ecg_diag_gemm": (C.c_int, [_P, C.c_char, C.c_char, C.c_int64, C.c_int64, C.c_int64,
                                C.c_double, _D, C.c_int64, _D, C.c_int64, C.c_double, _D,
                                C.c_int64]),
    "ecg_diag_permute": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int),
                                   C.c_double, _D, C.c_double, _D]),
    "ecg_shells_nbf": (C.c_int, [_S, C.POINTER(C.c_int32)]),
    "ecg_int1e": (C.c_int, [_P, C.c_int32, _S, C.c_int32, _D, _D, _D, _D]),
    "ecg_int2c2e": (C.c_int, [_P, _S, _D]),
    "ecg_int3c2e": (C.c_int, [_P, _S, _S, _D]),
    "ecg_df_create": (C.c_int, [_P, _S, _S, _D, C.c_int64, C.POINTER(_P)]),
    "ecg_df_fock": (C.c_int, [_P, _D, _D, C.c_int64, _D]),
    "ecg_df_mo": (C.c_int, [_P, _D, C.c_int64, _D]),
    "ecg_df_destroy": (C.c_int, [_P]),
    "ecg_gemm_noalloc": (C.c_int, [C.c_char, C.c_char, C.c_int64, C.c_int64, C.c_int64,
                                   C.c_double, _P, C.c_int64, _P, C.c_int64, C.c_double, _P,
                                   C.c_int64, _P, C.POINTER(C.c_int32)]),
}


def library_path():
    return os.environ.get("ECGPU_LIB") or os.path.join(HERE, "libecgpu.so")


def lib():
    """Load libecgpu.so once; raises OSError if it is missing."""
    global _lib
    if _lib is None:
        path = library_path()
        if not os.path.exists(path):
            raise OSError(f"libecgpu not built: {path} (run python elemco.jl_b200/build.py)")
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def dptr(a):
    """Pointer to a Fortran-ordered float64 array (None passes NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim <= 1), "need F-ordered f64"
    return a.ctypes.data_as(_D)


def fvec(shape):
    return np.zeros(shape, dtype=np.float64, order="F")


def as_f(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))
