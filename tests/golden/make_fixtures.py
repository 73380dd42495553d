"""Generate the golden fixtures used by the parity tests.

Reads the reference's FCIDUMP test fixtures as text and stores their integral
lists in compact ``.npz`` files, plus the reference's pinned energies as JSON.
Only this script reads the reference checkout; the tests and the GPU box use
the committed outputs.

Run from the repo root:  python tests/golden/make_fixtures.py REFERENCE_ROOT
(the ElemCo.jl checkout; or set ELEMCO_REF to it)

Sources (paths inside the ElemCo.jl project):
  test/files/H2O.FCIDUMP      closed shell, NORB=23, NELEC=8   (test/h2o.jl:16)
  test/files/H2O_ST1.FCIDUMP  non-Hermitian (ST=1), NORB=24    (test/h2o_st1.jl:15)
  energies pinned in test/h2o.jl:6-10, test/h2o_st1.jl:6-9 and test/df_hf.jl:5-7
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_fcidump_text(path):
    """Minimal FCIDUMP text parser (header keys + five-column integral lines).

    Follows the reader in src/integrals/dump.jl:326-348 (header) and
    :600-631 (integral lines: value i1 i2 i3 i4; i4>0 two-electron,
    i2>0 one-electron, i1<=0 core energy).
    """
    with open(path) as f:
        text = f.read()
    end = re.search(r"^\s*(/|&END)\s*$", text, re.M)
    head_txt, body = text[: end.start()], text[end.end():]
    head_txt = head_txt.replace("&FCI", " ")
    head = {}
    toks = re.split(r"[\s,]+", head_txt.replace("=", " = "))
    toks = [t for t in toks if t]
    key = None
    for i, t in enumerate(toks):
        if i + 1 < len(toks) and toks[i + 1] == "=":
            key = t.upper()
            head[key] = []
        elif t == "=":
            continue
        elif key is not None:
            head[key].append(t)
    vals, idx = [], []
    e0 = None
    for line in body.splitlines():
        p = line.split()
        if len(p) != 5:
            continue
        v = float(p[0].replace("D", "E"))
        i1, i2, i3, i4 = (int(x) for x in p[1:])
        if i1 <= 0 and i2 <= 0 and i3 <= 0 and i4 <= 0:
            e0 = v
            continue
        vals.append(v)
        idx.append((i1, i2, i3, i4))
    return head, np.array(idx, dtype=np.int16), np.array(vals), e0


def main(refroot):
    files = {
        "h2o_fcidump.npz": "test/files/H2O.FCIDUMP",
        "h2o_st1_fcidump.npz": "test/files/H2O_ST1.FCIDUMP",
    }
    # the header of H2O.FCIDUMP as it stands (multi-line ORBSYM/OCC/CLOSED/FOCK
    # values): the FCIDUMP reader is tested on it with the fixture's integrals
    with open(os.path.join(refroot, files["h2o_fcidump.npz"])) as f:
        hdr = []
        for line in f:
            hdr.append(line)
            if line.strip() in ("/", "&END"):
                break
    with open(os.path.join(HERE, "h2o_fcidump_header.txt"), "w") as f:
        f.writelines(hdr)
    for out, rel in files.items():
        head, idx, val, e0 = parse_fcidump_text(os.path.join(refroot, rel))
        np.savez_compressed(
            os.path.join(HERE, out),
            norb=int(head["NORB"][0]),
            nelec=int(head["NELEC"][0]),
            ms2=int(head.get("MS2", ["0"])[0]),
            st=int(head.get("ST", ["0"])[0]),
            idx=idx,
            val=val,
            e0=e0,
            source=rel,
        )
        print(f"{out}: {len(val)} integrals, NORB={head['NORB'][0]}, e0={e0}")

    energies = {
        "_source": "ElemCo.jl test/h2o.jl:6-10, test/h2o_st1.jl:6-9 (asserted there at 1e-6 Eh)",
        "h2o": {
            "fixture": "h2o_fcidump.npz",
            "HF": -75.6457645933,
            "MP2c": -0.287815830908,
            "CCSD(T)c": -0.329259440500,
            "LCCSD(T)c": -0.326915143863,
            "DCSDc": -0.328754956597,
        },
        "df_hf": {
            "_source": "test/df_hf.jl:5-7: water (bohr, :12-15), cc-pVDZ, jkfit "
                       "cc-pVTZ-JKFIT, mpfit cc-pVDZ-MPFIT, frozen O 1s",
            "HF": -76.02145513971418,
            "MP2c": -0.204723138509385,
            "DCSDc": -0.219150244853825,
        },
        "h2o_st1": {
            "fixture": "h2o_st1_fcidump.npz",
            "HF": -76.298014304953,
            "MP2c": -0.069545740864,
            "CCSDc": -0.082041632192,
            "DCSDc": -0.082498102641,
        },
    }
    with open(os.path.join(HERE, "reference_energies.json"), "w") as f:
        json.dump(energies, f, indent=1)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ELEMCO_REF")
    if not root:
        sys.exit("usage: make_fixtures.py REFERENCE_ROOT  (or set ELEMCO_REF)")
    main(root)
