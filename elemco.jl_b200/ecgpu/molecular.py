"""Benchmark workloads built from real molecules: geometry (ecgpu.molecules),
DF-HF on the GPU integral engine, and the dfdump integrals of the CC path.

  h2o_vdz      water, cc-pVDZ, cc-pVDZ-RI for both DF-HF and CC, no frozen
               core (o=5, v=19, nQ=84)
  h2oN_vdz     (H2O)_N, N = 2, 3, 4: cc-pVDZ, DF-HF with cc-pVDZ-JKFIT, CC with
               cc-pVDZ-RI, frozen O 1s
  h2o6_vtz     (H2O)_6: cc-pVTZ, cc-pVTZ-JKFIT, cc-pVTZ-RI, frozen O 1s
               (o=24, v=318, nQ=846)
  cNh2N+2_vdz  alkanes C_nH_2n+2, n = 6..10: cc-pVDZ, cc-pVDZ-JKFIT, cc-pVDZ-RI,
               frozen C 1s
"""
import re

from .molecules import alkane, water, water_cluster
from .scf import dfhf, dfints

_SPEC = {"vdz": ("cc-pvdz", "cc-pvdz-jkfit", "cc-pvdz-mpfit"),
         "vtz": ("cc-pvtz", "cc-pvtz-jkfit", "cc-pvtz-mpfit")}


def molecule_of(name):
    m = re.fullmatch(r"h2o(\d*)_(vdz|vtz)", name)
    if m:
        n = int(m.group(1) or 1)
        return (water() if n == 1 else water_cluster(n)), m.group(2)
    m = re.fullmatch(r"c(\d+)h(\d+)_(vdz|vtz)", name)
    if m:
        return alkane(int(m.group(1))), m.group(3)
    raise KeyError(f"unknown molecular workload {name!r}")


def molecular_workload(ctx, name, log=None):
    """(B[p,q,Q], h1, e0, no, info) of a named workload, computed on the GPU."""
    mol, b = molecule_of(name)
    ao, jk, mp = _SPEC[b]
    if name == "h2o_vdz":
        jk, ncore = mp, 0  # configuration 1: RI basis for HF and CC, all electrons
    else:
        ncore = None
    hf = dfhf(ctx, mol, ao, jk, log=log)
    if not hf.converged:
        raise RuntimeError(f"DF-HF of {name} did not converge")
    B, h1, e0, no, eref = dfints(hf, mp, jk, ncore=ncore)
    info = {"molecule": name, "atoms": len(mol.symbols), "nbf": hf.C.shape[0],
            "E_HF": hf.E, "scf_iterations": hf.iterations, "ao": ao, "jkfit": jk, "mpfit": mp}
    return B, h1, e0, no, info
