"""Molecular geometries of the benchmark configurations (bohr).

* :func:`water`: the water molecule of the DF-HF test and configuration 1,
  O (0, 0, -0.130186067), H (0, +-1.489124508, 1.033245507)
  (ElemCo.jl test/df_hf.jl).
* :func:`water_cluster`: (H2O)_n by seeded random rigid placement of that
  monomer — each new molecule at a centre-of-mass distance drawn uniformly
  from [5.2, 5.8] bohr from a randomly chosen placed molecule, in a uniformly
  random (Haar) orientation, rejected if any O-O distance falls below
  4.8 bohr or any other pair of atoms below 2.5 bohr; seed 1234 + n.
* :func:`alkane`: staggered zig-zag C_nH_{2n+2} with C-C 2.91 bohr, C-H 2.06
  bohr and tetrahedral angles, plus seeded uniform +-0.02 bohr jitter.
"""
import math

import numpy as np

ZNUC = {"H": 1.0, "C": 6.0, "N": 7.0, "O": 8.0}
MASS = {"H": 1.008, "C": 12.011, "N": 14.007, "O": 15.999}


class Molecule:
    def __init__(self, symbols, xyz):
        self.symbols = list(symbols)
        self.xyz = np.asarray(xyz, dtype=float).reshape(-1, 3)

    @property
    def charges(self):
        return np.array([ZNUC[s] for s in self.symbols])

    @property
    def nelec(self):
        return int(round(self.charges.sum()))

    def nuclear_repulsion(self):
        """sum_{A<B} Z_A Z_B / |R_A - R_B| (src/system/msystems.jl)."""
        Z, X = self.charges, self.xyz
        e = 0.0
        for a in range(len(Z)):
            for b in range(a):
                e += Z[a] * Z[b] / np.linalg.norm(X[a] - X[b])
        return e

    def ncore(self):
        """Frozen core of the reference's default (`core = :large`): the 1s
        shell of first-row atoms (src/system/msystems.jl:545)."""
        return sum(1 for s in self.symbols if ZNUC[s] > 2.0)


WATER_XYZ = np.array([[0.0, 0.0, -0.130186067],
                      [0.0, 1.489124508, 1.033245507],
                      [0.0, -1.489124508, 1.033245507]])


def water():
    return Molecule(["O", "H", "H"], WATER_XYZ)


def _haar_rotation(rng):
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def water_cluster(n, seed=None):
    rng = np.random.default_rng(1234 + n if seed is None else seed)
    m = np.array([MASS[s] for s in ("O", "H", "H")])
    mono = WATER_XYZ - (m[:, None] * WATER_XYZ).sum(0) / m.sum()
    mols = [mono.copy()]
    coms = [np.zeros(3)]
    tries = 0
    while len(mols) < n:
        tries += 1
        if tries > 100000:
            raise RuntimeError("cluster placement failed")
        base = coms[rng.integers(len(coms))]
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        com = base + rng.uniform(5.2, 5.8) * d
        new = com + mono @ _haar_rotation(rng).T
        ok = True
        for old in mols:
            if np.linalg.norm(new[0] - old[0]) < 4.8:
                ok = False
                break
            dist = np.linalg.norm(new[:, None, :] - old[None, :, :], axis=2)
            if dist.min() < 2.5:
                ok = False
                break
        if ok:
            mols.append(new)
            coms.append(com)
    return Molecule(["O", "H", "H"] * n, np.concatenate(mols))


def alkane(n, seed=None):
    """C_nH_{2n+2}: carbons on a planar zig-zag, hydrogens completing the
    tetrahedra (two per CH2, three per CH3), staggered."""
    rng = np.random.default_rng(4321 + n if seed is None else seed)
    cc, ch = 2.91, 2.06
    half = math.radians(109.4712206) / 2.0
    dx, dy = cc * math.sin(half), cc * math.cos(half)
    C = np.array([[i * dx, (i % 2) * dy, 0.0] for i in range(n)])
    sym, xyz = ["C"] * n, [c for c in C]
    tdir = lambda v: v / np.linalg.norm(v)  # noqa: E731
    for i in range(n):
        nb = [C[j] - C[i] for j in (i - 1, i + 1) if 0 <= j < n]
        if n == 1:
            dirs = [np.array([1, 1, 1]), np.array([1, -1, -1]), np.array([-1, 1, -1]),
                    np.array([-1, -1, 1])]
            dirs = [tdir(d.astype(float)) for d in dirs]
        else:
            # bisector away from the carbon neighbours, tetrahedral opening in z
            s = -tdir(sum(tdir(v) for v in nb)) if len(nb) == 2 else None
            if len(nb) == 2:
                dirs = [math.cos(half) * s + math.sin(half) * np.array([0, 0, 1.0]),
                        math.cos(half) * s - math.sin(half) * np.array([0, 0, 1.0])]
            else:
                u = tdir(nb[0])
                # three hydrogens around -u at the tetrahedral angle
                perp = np.cross(u, [0, 0, 1.0])
                perp = tdir(perp) if np.linalg.norm(perp) > 1e-8 else np.array([1.0, 0, 0])
                perp2 = np.cross(u, perp)
                ct = math.cos(math.pi - 2 * half)
                st = math.sin(math.pi - 2 * half)
                dirs = [tdir(-ct * u + st * (math.cos(ph) * perp + math.sin(ph) * perp2))
                        for ph in (math.pi / 2, math.pi / 2 + 2 * math.pi / 3,
                                   math.pi / 2 + 4 * math.pi / 3)]
        for d in dirs:
            sym.append("H")
            xyz.append(C[i] + ch * d)
    X = np.array(xyz) + rng.uniform(-0.02, 0.02, (len(xyz), 3))
    return Molecule(sym, X)
