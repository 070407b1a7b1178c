"""Basis sets and molecules in Tonto's conventions.

This module is the host-side description of what Tonto's MOLECULE hands to its J/K
builder: atoms with positions in bohr, and per atom an ordered list of contracted
shells.  It restates these Tonto conventions:

* Basis-library text format (``basis_sets/*``): blocks ``Label:basis { ... }`` with
  either ``gamess-us`` shell records (``S 3`` then ``i exponent coefficient`` lines) or
  ``turbomole`` records (``3 s`` then ``exponent coefficient`` lines).
* Library contraction coefficients refer to normalised primitives; Tonto stores them
  "unnormalised" (molecule.main.foo:795-810, shell.foo:459-507): every primitive
  carries the normalisation of the x^l component and the contraction is scaled so
  that the contracted x^l function has unit norm.
* Basis-function order: atoms in input order, shells in library order, components
  within a shell in Tonto's Cartesian order (gaussian_data.foo:295-479) or, for l >= 2
  in a spherical basis, real solid harmonics ordered m = 0, +1, -1, +2, -2, ...
  (gaussian_data.foo:1143-1350).  p shells stay Cartesian (x, y, z) in both.
* Angstrom to bohr: 1 / 0.5291772108 (include/macros.in:508-509).
"""

from __future__ import annotations

import json
import math
import os
import re
from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import numpy as np

ANGSTROM_PER_BOHR = 0.5291772108
BOHR_PER_ANGSTROM = 1.0 / ANGSTROM_PER_BOHR

L_OF = {"s": 0, "p": 1, "d": 2, "f": 3, "g": 4, "h": 5}
ELEMENT_Z = {"H": 1, "He": 2, "Li": 3, "Be": 4, "B": 5, "C": 6, "N": 7, "O": 8, "F": 9, "Ne": 10,
             "Na": 11, "Mg": 12, "Al": 13, "Si": 14, "P": 15, "S": 16, "Cl": 17, "Ar": 18}
Z_ELEMENT = {v: k for k, v in ELEMENT_Z.items()}

BASIS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis")


def double_factorial_odd(n: int) -> float:
    """(2n-1)!! with (-1)!! = 1: Tonto's INT.double_factorial (int.foo:192-212)."""
    r = 1.0
    for k in range(1, 2 * n, 2):
        r *= k
    return r


def n_cart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def n_sph(l: int) -> int:
    return 2 * l + 1


# ---------------------------------------------------------------------------
# Basis library text
# ---------------------------------------------------------------------------

def parse_tonto_basis_text(text: str) -> Dict[str, List[Tuple[int, List[float], List[float]]]]:
    """Parse a Tonto basis-library file into {"O:cc-pVDZ": [(l, exps, coefs), ...]}.

    Handles the ``gamess-us`` and ``turbomole`` record layouts used by the files in
    Tonto's ``basis_sets/`` directory, including ``L`` (shared s/p exponent) shells.
    Coefficients are returned as written (relative to normalised primitives).
    """
    text = re.sub(r"!.*", "", text)
    out: Dict[str, List[Tuple[int, List[float], List[float]]]] = {}
    for m in re.finditer(r"([A-Z][a-z]?:[^\s{}]+)\s*\{([^{}]*)\}", text):
        label, body = m.group(1), m.group(2)
        toks = body.replace("D+", "E+").replace("D-", "E-").split()
        shells: List[Tuple[int, List[float], List[float]]] = []
        i = 0
        try:
            while i < len(toks):
                t = toks[i]
                if t[0].isalpha():          # gamess-us: "S 3" then "k exp coef"
                    lch = t.lower()
                    n = int(toks[i + 1])
                    i += 2
                    if lch == "l":
                        e, cs, cp = [], [], []
                        for _ in range(n):
                            e.append(float(toks[i + 1]))
                            cs.append(float(toks[i + 2]))
                            cp.append(float(toks[i + 3]))
                            i += 4
                        shells.append((0, e, cs))
                        shells.append((1, list(e), cp))
                    else:
                        e, c = [], []
                        for _ in range(n):
                            e.append(float(toks[i + 1]))
                            c.append(float(toks[i + 2]))
                            i += 3
                        shells.append((L_OF[lch], e, c))
                else:                       # turbomole: "3 s" then "exp coef"
                    n = int(t)
                    lch = toks[i + 1].lower()
                    i += 2
                    e, c = [], []
                    for _ in range(n):
                        e.append(float(toks[i]))
                        c.append(float(toks[i + 1]))
                        i += 2
                    shells.append((L_OF[lch], e, c))
        except (ValueError, KeyError, IndexError):
            continue                        # not a contracted-gaussian block (e.g. Slater sets)
        if shells:
            out[label] = shells
    return out


def load_basis_library(name: str) -> Dict[str, List[Tuple[int, List[float], List[float]]]]:
    """Load a basis set shipped with this package (JSON extracted from Tonto's library)."""
    path = os.path.join(BASIS_DIR, name + ".json")
    if not os.path.exists(path):
        raise FileNotFoundError(f"basis set {name!r} is not packaged ({path})")
    with open(path) as fh:
        raw = json.load(fh)
    return {k: [(int(l), list(map(float, e)), list(map(float, c))) for l, e, c in v] for k, v in raw.items()}


# ---------------------------------------------------------------------------
# Normalisation (shell.foo:459-507)
# ---------------------------------------------------------------------------

def unnormalize(l: int, exps: Sequence[float], coefs: Sequence[float]) -> List[float]:
    """Tonto's SHELL:unnormalize: fold the x^l primitive normalisation into the
    contraction coefficients and normalise the contracted x^l function."""
    sm = 0.0
    for i, a in enumerate(exps):
        for j in range(i):
            b = exps[j]
            ab = 2.0 * math.sqrt(a * b) / (a + b)
            sm += 2.0 * coefs[i] * coefs[j] * ab ** (l + 1.5)
        sm += coefs[i] * coefs[i]
    norm = math.sqrt(sm) * (2.0 * math.pi) ** 0.75
    df = double_factorial_odd(l)
    return [c * (4.0 * a) ** (0.5 * l + 0.75) / (norm * math.sqrt(df)) for a, c in zip(exps, coefs)]


# ---------------------------------------------------------------------------
# Molecule
# ---------------------------------------------------------------------------

@dataclass
class Shell:
    atom: int
    l: int
    exps: List[float]
    coefs: List[float]          # Tonto "unnormalised" contraction coefficients
    first_bf: int = 0


@dataclass
class Molecule:
    """Atoms (Z, bohr) plus shells in Tonto order.  ``spherical`` selects Tonto's
    ``use_spherical_basis`` (make_r_JK_direct) against Cartesian (make_r_JK_engine)."""
    Z: np.ndarray                       # (n_atom,) int
    xyz: np.ndarray                     # (n_atom, 3) bohr
    shells: List[Shell] = field(default_factory=list)
    spherical: bool = True
    basis_name: str = ""
    charge: int = 0

    @property
    def n_atom(self) -> int:
        return int(len(self.Z))

    @property
    def n_shell(self) -> int:
        return len(self.shells)

    def shell_nbf(self, l: int) -> int:
        return n_sph(l) if (self.spherical and l >= 2) else n_cart(l)

    @property
    def n_bf(self) -> int:
        return sum(self.shell_nbf(s.l) for s in self.shells)

    @property
    def n_electrons(self) -> int:
        return int(np.sum(self.Z)) - self.charge

    def nuclear_repulsion(self) -> float:
        Z = np.asarray(self.Z, dtype=np.float64)
        d = np.sqrt(((self.xyz[:, None, :] - self.xyz[None, :, :]) ** 2).sum(-1))
        i, j = np.tril_indices(self.n_atom, -1)
        return float(np.sum(Z[i] * Z[j] / d[i, j]))

    def flat_arrays(self):
        """Flattened shell data in the C-ABI layout (see include/tontofock.h)."""
        shell_atom = np.array([s.atom for s in self.shells], dtype=np.int32)
        shell_l = np.array([s.l for s in self.shells], dtype=np.int32)
        shell_nprim = np.array([len(s.exps) for s in self.shells], dtype=np.int32)
        shell_first_bf = np.array([s.first_bf for s in self.shells], dtype=np.int32)
        exps = np.array([e for s in self.shells for e in s.exps], dtype=np.float64)
        coefs = np.array([c for s in self.shells for c in s.coefs], dtype=np.float64)
        return shell_atom, shell_l, shell_nprim, shell_first_bf, exps, coefs


def build_molecule(Z: Sequence[int], xyz_bohr: np.ndarray, basis: str | Dict, spherical: bool = True,
                   charge: int = 0) -> Molecule:
    """Attach ``basis`` (a packaged basis name, or a parsed library dict) to the atoms."""
    lib = load_basis_library(basis) if isinstance(basis, str) else basis
    bname = basis if isinstance(basis, str) else ""
    mol = Molecule(Z=np.asarray(Z, dtype=np.int32), xyz=np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3),
                   spherical=spherical, basis_name=bname, charge=charge)
    bf = 0
    for ia, z in enumerate(mol.Z):
        key = None
        for k in lib:
            if k.split(":")[0] == Z_ELEMENT[int(z)]:
                key = k
                break
        if key is None:
            raise KeyError(f"no basis for element {Z_ELEMENT[int(z)]} in {bname or 'library'}")
        for l, e, c in lib[key]:
            sh = Shell(atom=ia, l=l, exps=list(e), coefs=unnormalize(l, e, c), first_bf=bf)
            mol.shells.append(sh)
            bf += mol.shell_nbf(l)
    return mol
