"""Extract the H, C, N, O entries of the basis sets the coupled-cluster
workloads use from a Molpro-format basis library (ElemCo.jl's
lib/basis_sets, highest file version first, as src/system/parse_basis.jl:35-58
chooses) into basis_hcno.json next to this script.

    python elemco.jl_b200/ecgpu/basis_data/make_basis_data.py LIBRARY_DIR
(LIBRARY_DIR holds mpro/*.mpro; or set ECGPU_BASIS_LIB)
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from ecgpu.basis import canonical_name, read_mpro  # noqa: E402

SETS = ["cc-pvdz", "cc-pvtz", "cc-pvdz-rifit", "cc-pvtz-rifit", "cc-pvdz-jkfit",
        "cc-pvtz-jkfit"]


def main(lib):
    out = {}
    for name in SETS:
        stem = canonical_name(name)
        for v in (2, 1, 0):
            f = os.path.join(lib, "mpro", f"{stem}.{v}.mpro")
            if os.path.exists(f):
                break
        else:
            raise FileNotFoundError(stem)
        with open(f) as fh:
            out[stem] = read_mpro(fh.read(), elements=("H", "C", "N", "O"))
        print(f"{name}: {os.path.basename(f)} {sorted(out[stem])}")
    with open(os.path.join(HERE, "basis_hcno.json"), "w") as fh:
        json.dump(out, fh, separators=(",", ":"))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ECGPU_BASIS_LIB")
    if not root:
        sys.exit("usage: make_basis_data.py LIBRARY_DIR  (or set ECGPU_BASIS_LIB)")
    main(root)
