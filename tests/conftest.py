"""Shared fixtures.  GPU tests are marked ``gpu`` and call libecgpu through
its C ABI; everything else runs on the CPU."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "elemco.jl_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libecgpu.so")


@pytest.fixture(scope="session")
def gold():
    with open(os.path.join(GOLDEN, "reference_energies.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def h2o():
    import oracle as O
    return O.read_fixture(os.path.join(GOLDEN, "h2o_fcidump.npz"))


@pytest.fixture(scope="session")
def h2o_st1():
    import oracle as O
    return O.read_fixture(os.path.join(GOLDEN, "h2o_st1_fcidump.npz"))


@pytest.fixture(scope="session")
def h2o_df(h2o):
    """H2O.FCIDUMP integrals as Cholesky DF factors (tol 1e-12) and the
    System the oracle builds from the same factors."""
    import oracle as O
    B = O.cholesky_df(h2o.V, 1e-12)
    S = O.System.from_df(B, h2o.h, h2o.e0, h2o.no)
    return np.asfortranarray(B.transpose(1, 2, 0)), S


@pytest.fixture(scope="session")
def ctx():
    import ecgpu
    c = ecgpu.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def h2o_fcidump_text(tmp_path_factory):
    """The reference's test/files/H2O.FCIDUMP reassembled as text: its own
    header (tests/golden/h2o_fcidump_header.txt) and the integral lines of the
    committed fixture in the file's "value i j k l" form (Fortran E format)."""
    z = np.load(os.path.join(GOLDEN, "h2o_fcidump.npz"))
    with open(os.path.join(GOLDEN, "h2o_fcidump_header.txt")) as f:
        head = f.read()
    lines = [head.rstrip("\n")]
    for (i, j, k, l), x in zip(z["idx"].astype(int), z["val"]):
        m, e = f"{x:.15E}".split("E")
        lines.append(f" {float(m) / 10:.16f}E{int(e) + 1:+03d} {i:3d} {j:3d} {k:3d} {l:3d}")
    lines.append(f" {float(z['e0']):.16E}   0   0   0   0")
    p = tmp_path_factory.mktemp("fcidump") / "H2O.FCIDUMP"
    p.write_text("\n".join(lines) + "\n")
    return str(p)
