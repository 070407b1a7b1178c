"""Extract the basis sets this package ships from a Tonto basis library directory.

The GPU host has no copy of Tonto, so the contracted-Gaussian data for the elements
the synthetic workloads and the fixture molecules use are stored here as JSON, in the
same form ``tonto_b200.basis.parse_tonto_basis_text`` returns (coefficients as written
in the library, i.e. relative to normalised primitives).

Usage:  python extract_basis.py <tonto basis_sets directory>
"""

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from tonto_b200.basis import parse_tonto_basis_text  # noqa: E402

SETS = ["STO-3G", "6-31G(d)", "6-311G(d,p)", "DZP", "cc-pVDZ", "cc-pVTZ", "def2-SVP"]
ELEMENTS = ["H", "C", "N", "O"]


def main(libdir: str) -> None:
    for name in SETS:
        with open(os.path.join(libdir, name)) as fh:
            parsed = parse_tonto_basis_text(fh.read())
        keep = {k: v for k, v in parsed.items() if k.split(":")[0] in ELEMENTS}
        missing = [e for e in ELEMENTS if not any(k.split(":")[0] == e for k in keep)]
        with open(os.path.join(HERE, name + ".json"), "w") as fh:
            json.dump(keep, fh, indent=1)
        print(name, sorted(keep), "missing:", missing)


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TONTO_BASIS_DIR")
    if not src:
        sys.exit("usage: python extract_basis.py <the basis_sets directory of a Tonto checkout> (or set TONTO_BASIS_DIR)")
    main(src)
