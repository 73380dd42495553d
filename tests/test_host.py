"""Host-side logic of the ecgpu package (no GPU): FCIDUMP IO, Cholesky
factors, amplitude files, method parsing, options, synthetic systems."""
import os

import numpy as np
import pytest

import oracle as O
from ecgpu import driver as D
from ecgpu.synthetic import WORKLOADS, make_system


def _fd_from_oracle(S, nelec):
    return D.FDump(S.h, S.e0, nelec, V=S.V.copy())


def test_fcidump_roundtrip(tmp_path, h2o):
    fd = _fd_from_oracle(h2o, 2 * h2o.no)
    p = tmp_path / "X.FCIDUMP"
    D.write_fcidump(str(p), fd, tol=0.0)
    back = D.read_fcidump(str(p))
    assert back.norb == h2o.n and back.nelec == 2 * h2o.no and not back.st
    assert np.abs(back.V - h2o.V).max() < 1e-15
    assert np.abs(back.h - h2o.h).max() < 1e-15
    assert back.e0 == pytest.approx(h2o.e0, abs=1e-15)


def test_fcidump_errors(tmp_path):
    p = tmp_path / "bad.FCIDUMP"
    p.write_text(" &FCI NORB=2,NELEC=2,\n /\n 1.0 1 1 1 1\n")
    with pytest.raises(ValueError, match="core energy"):
        D.read_fcidump(str(p))
    p.write_text(" &FCI NORB=2,NELEC=2,\n /\n 1.0 3 1 1 1\n 0.0 0 0 0 0\n")
    with pytest.raises(ValueError, match="larger than norb"):
        D.read_fcidump(str(p))
    p.write_text(" &FCI NELEC=2,\n /\n 0.0 0 0 0 0\n")
    with pytest.raises(ValueError, match="NORB"):
        D.read_fcidump(str(p))


def test_cholesky_df_matches_oracle(h2o):
    B = D.cholesky_df(h2o.V, 1e-12)
    assert B.flags.f_contiguous
    Vb = np.einsum("prQ,qsQ->pqrs", B, B)
    assert np.abs(Vb - h2o.V).max() < 1e-11
    Bo = O.cholesky_df(h2o.V, 1e-12)
    assert B.shape[2] == Bo.shape[0]


def test_mio_roundtrip(tmp_path):
    a = np.asfortranarray(np.random.default_rng(0).standard_normal((3, 4, 2, 5)))
    b = np.asfortranarray(np.arange(6.0).reshape(2, 3))
    f = str(tmp_path / "x.bin")
    D.miosave(f, a, b)
    a2, b2 = D.mioload(f)
    assert np.array_equal(a, a2) and np.array_equal(b, b2)
    raw = np.fromfile(f, dtype=np.int64, count=4)
    assert list(raw) == [12, 2, 4, 3]  # Float64 type id, 2 arrays, rank 4, first dim


@pytest.mark.parametrize("m,exp", [
    ("ccsd", ("CCSD", False, False, False)), ("dcsd", ("DCSD", True, False, False)),
    ("ccsd(t)", ("CCSD", False, False, True)), ("λccsd", ("CCSD", False, True, False)),
    ("λccsd(t)", ("CCSD", False, True, True)), ("ΛDCSD", ("DCSD", True, True, False)),
])
def test_parse_method(m, exp):
    assert D.parse_method(m) == exp


def test_parse_method_rejects():
    for m in ("uccsd", "ccsdt", "mp2", "ldcsdx"):
        with pytest.raises(ValueError):
            D.parse_method(m)


def test_options_set():
    EC = D.ECInfo()
    EC.set("cc", thr=1e-12, maxit=7)
    assert EC.options["cc"].thr == 1e-12 and EC.options["cc"].maxit == 7
    with pytest.raises(KeyError):
        EC.set("cc", nonsense=1)


def test_synthetic_system_is_canonical():
    no, nv, nq = WORKLOADS["h2o_vdz"]
    B, h1, e0, eps = make_system(no, nv, nq)
    assert B.flags.f_contiguous and np.allclose(B, B.transpose(1, 0, 2))
    S = O.System.from_df(np.transpose(B, (2, 0, 1)), h1, e0, no)
    f = O.gen_fock(S)
    assert np.abs(f - np.diag(eps)).max() < 1e-13


def test_oracle_synthetic_ccsd_converges():
    B, h1, e0, eps = make_system(5, 19, 84)
    S = O.System.from_df(np.transpose(B, (2, 0, 1)), h1, e0, 5)
    r = O.ccdriver(S, "ccsd(t)")
    assert r["converged"] and r["iterations"] < 20
    assert -1.0 < r["CCSDc"] < 0.0 and r["(T)"] < 0.0


def test_read_reference_fcidump_text(h2o_fcidump_text, h2o):
    """read_fcidump on the reference's H2O.FCIDUMP header (multi-line ORBSYM,
    OCC, CLOSED and FOCK values) and its integral lines."""
    fd = D.read_fcidump(h2o_fcidump_text)
    assert fd.norb == 23 and fd.nelec == 8 and not fd.st
    assert len(fd.head["FOCK"]) == 23 and fd.head["OCC"][0] == "4"
    assert np.abs(fd.V - h2o.V).max() < 1e-15 and np.abs(fd.h - h2o.h).max() < 1e-15
    assert fd.e0 == h2o.e0
