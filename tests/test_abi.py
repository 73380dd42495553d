"""The C-ABI library loads and exports every function include/*.h declares
(no compute calls, no GPU needed)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(ecg_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("ecg_create", "ecg_set_system", "ecg_cc_solve", "ecg_pert_t",
                 "ecg_lambda_solve", "ecg_diis_perform"):
        assert must in names


def test_library_exports_all_declared_symbols():
    import ecgpu
    path = ecgpu.library_path()
    if not os.path.exists(path):
        pytest.skip("libecgpu.so not built (run python elemco.jl_b200/build.py)")
    lib = ctypes.CDLL(path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from ecgpu._lib import SIGNATURES
    missing = [n for n in declared_functions() if n not in SIGNATURES]
    assert not missing, missing
