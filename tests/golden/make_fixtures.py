"""Extract the energy fixtures that pin the J/K path from Tonto's own blessed tests.

Reads ``tests/short/h2o_rhf_*/{stdin,stdout}`` and
``tests/short/h2o_rhf_cc-pVDZ_electron_density_plot`` of a Tonto checkout: the atoms
(labels are atomic numbers, positions in angstrom), the basis name, whether a
spherical basis is requested, and the printed SCF results with the number of
decimals printed.  Writes ``tonto_fixtures.json`` next to this script.

Usage:  python make_fixtures.py <tonto checkout>
"""

import json
import os
import re
import sys

ELEMENT_Z = {"H": 1, "C": 6, "N": 7, "O": 8}

CASES = [
    "h2o_rhf_cc-pVDZ_electron_density_plot",
    "h2o_rhf_cc-pVDZ",
    "h2o_rhf_STO-3G",
    "h2o_rhf_6-31G(d)",
    "h2o_rhf_DZP",
    "h2o_rhf_6-311G(d,p)",
    "h2o_rhf_cc-pVTZ_spherical_harmonic_basis",
]

KEYS = {
    "E": r"Total energy \(E_e\+V_NN\)\s+E \.+\s+(-?\d+\.\d+)",
    "V_NN": r"Nuclear repulsion energy\s+V_NN \.+\s+(-?\d+\.\d+)",
    "V_ee": r"Electron repulsion energy V_ee \.+\s+(-?\d+\.\d+)",
    "V_eN": r"Nuclear attraction energy V_eN \.+\s+(-?\d+\.\d+)",
    "T": r"Kinetic energy\s+T \.+\s+(-?\d+\.\d+)",
}


def main(root: str) -> None:
    out = []
    for case in CASES:
        d = os.path.join(root, "tests", "short", case)
        stdin = open(os.path.join(d, "stdin")).read()
        stdout = open(os.path.join(d, "stdout")).read()
        stdin_nc = re.sub(r"!.*", "", stdin)
        basis = re.search(r"basis_name=\s*(\S+)", stdin_nc).group(1)
        spherical = bool(re.search(r"use_spherical_basis=\s*TRUE", stdin_nc))
        data = re.search(r"data=\s*\{([^}]*)\}", stdin_nc).group(1)
        atoms = []
        for line in data.strip().splitlines():
            t = line.split()
            if len(t) == 4:
                label = re.sub(r"\d+$", "", t[0]) if not t[0].isdigit() else t[0]
                z = int(label) if label.isdigit() else ELEMENT_Z[label]
                atoms.append([z, float(t[1]), float(t[2]), float(t[3])])
        conv = float(re.search(r"convergence=\s*([0-9.eEdD+-]+)", stdin_nc).group(1))
        res = {}
        for k, pat in KEYS.items():
            m = re.search(pat, stdout)
            if m:
                s = m.group(1)
                res[k] = {"value": float(s), "decimals": len(s.split(".")[1])}
        nbf = int(re.search(r"No\. of basis functions \.+\s+(\d+)", stdout).group(1))
        out.append({"case": case, "basis": basis, "spherical": spherical, "atoms_angstrom": atoms,
                    "scf_convergence": conv, "n_bf": nbf, "results": res,
                    "source": f"tests/short/{case}/stdout"})
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tonto_fixtures.json")
    with open(path, "w") as fh:
        json.dump({"generator": "tests/golden/make_fixtures.py", "cases": out}, fh, indent=1)
    print("wrote", path, len(out), "cases")


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TONTO_ROOT")
    if not src:
        sys.exit("usage: python make_fixtures.py <the root of a Tonto checkout> (or set TONTO_ROOT)")
    main(src)
