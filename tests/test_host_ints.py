"""Host-side pieces of the integral and DF-HF path (CPU only): the integral
oracle on textbook values, basis-set parsing, the fitting metric's inverse
square root, and the molecule generators."""
import numpy as np

from oracle import ints as I


def test_oracle_h2_sto3g():
    """H2, STO-3G (zeta 1.24), R = 1.4 bohr: Szabo and Ostlund, Modern Quantum
    Chemistry, section 3.5.2 (S12 0.6593, T11 0.7600, T12 0.2365, V11 from
    nucleus A -1.2266, from B -0.6538, V12 -0.5974)."""
    e = [3.42525091, 0.62391373, 0.16885540]
    c = [0.15432897, 0.53532814, 0.44463454]
    bs = I.Shells([(0, [0, 0, 0], e, c), (0, [0, 0, 1.4], e, c)])
    S, T = I.overlap(bs), I.kinetic(bs)
    VA = I.nuclear(bs, [1.0], [[0, 0, 0]])
    VB = I.nuclear(bs, [1.0], [[0, 0, 1.4]])
    assert abs(S[0, 1] - 0.6593) < 1e-4 and abs(T[0, 0] - 0.7600) < 1e-4
    assert abs(T[0, 1] - 0.2365) < 1e-4
    assert abs(VA[0, 0] + 1.2266) < 1e-4 and abs(VB[0, 0] + 0.6538) < 1e-4
    assert abs(VA[0, 1] + 0.5974) < 1e-4


def test_oracle_solid_harmonics_orthonormal():
    for l in range(5):
        S = I.overlap(I.Shells([(l, [0, 0, 0], [1.3], [1.0])]))
        assert np.abs(S - np.eye(2 * l + 1)).max() < 1e-14


def test_basis_parsing_water():
    from ecgpu import basis as Bm
    from ecgpu.molecules import water
    w = water()
    assert Bm.shells(Bm.load("cc-pvdz"), w.symbols, w.xyz).nbf == 24
    assert Bm.shells(Bm.load("cc-pvdz-mpfit"), w.symbols, w.xyz).nbf == 84
    assert Bm.shells(Bm.load("cc-pvtz"), w.symbols, w.xyz).nbf == 58
    text = """
! hydrogen             (4s,1p) -> [2s,1p]
s, H , 1.301000E+01, 1.962000E+00, 4.446000E-01, 1.220000E-01
c, 1.4, 1.968500E-02, 1.379770E-01, 4.781480E-01, 5.012400E-01
c, 4.4, 1.000000E+00
p, H , .7270000
c, 1.1, 1.0000000
!
"""
    b = Bm.read_mpro(text)
    assert b["H"][0][0] == 0 and b["H"][1][1] == [0.727]
    assert b["H"][0][2][1] == (4, 4, [1.0])


def test_sqrtinvchol():
    from ecgpu.scf import sqrtinvchol
    rng = np.random.default_rng(0)
    X = rng.standard_normal((12, 12))
    A = X @ X.T + 0.1 * np.eye(12)
    M = sqrtinvchol(A, 1e-10)
    assert np.abs(M @ M.T - np.linalg.inv(A)).max() < 1e-10
    Y = rng.standard_normal((12, 7))
    Ar = Y @ Y.T  # rank 7: redundant directions dropped
    M = sqrtinvchol(Ar, 1e-8)
    assert M.shape == (12, 7)
    assert np.abs(M.T @ Ar @ M - np.eye(7)).max() < 1e-8


def test_molecule_generators():
    from ecgpu import molecules as Mo
    w = Mo.water()
    assert w.nelec == 10 and w.ncore() == 1
    for n in (2, 3, 4, 6):
        c = Mo.water_cluster(n)
        O = c.xyz[0::3]
        d = np.linalg.norm(O[:, None] - O[None], axis=2) + 10 * np.eye(n)
        assert d.min() >= 4.8 and len(c.symbols) == 3 * n
        # every monomer keeps its internal geometry
        for k in range(n):
            m = c.xyz[3 * k:3 * k + 3]
            assert abs(np.linalg.norm(m[1] - m[0]) - np.linalg.norm(w.xyz[1] - w.xyz[0])) < 1e-12
        assert np.allclose(c.xyz, Mo.water_cluster(n).xyz)
    a = Mo.alkane(6)
    assert a.symbols.count("C") == 6 and a.symbols.count("H") == 14
    C = a.xyz[:6]
    assert np.all(np.abs(np.linalg.norm(C[1:] - C[:-1], axis=1) - 2.91) < 0.08)
