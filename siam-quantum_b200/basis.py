"""Contracted Cartesian Gaussian basis in the reference's layout.

Builds, for a molecule, the same ordered list of contracted basis functions as the reference's
genBasis (src/basis.c:529-623): atoms in input order; per atom the basis records of that
element in file order; per record the Cartesian components in the order read_GAMESS_BasisSet
creates them (src/basis.c:459-499):  S: s;  L: s, x, y, z;  P: x, y, z;
D: xx, yy, zz, xy, xz, yz;  F: xxx, yyy, zzz, xxy, xyy, xxz, xzz, yyz, yzz, xyz.
Each primitive gets norm = 1/sqrt(<g|g>) for g = x^l y^m z^n exp(-a r^2) (src/basis.c:597-615).

The result is a flat structure-of-arrays (`Basis`) that is what the C ABI takes.
"""
import json
import math
import os

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "basis_sets.json")
_CACHE = {}

COMPONENTS = {
    "S": [[(0, 0, 0), 0]],
    "L": [[(0, 0, 0), 0], [(1, 0, 0), 1], [(0, 1, 0), 1], [(0, 0, 1), 1]],
    "P": [[(1, 0, 0), 0], [(0, 1, 0), 0], [(0, 0, 1), 0]],
    "D": [[(2, 0, 0), 0], [(0, 2, 0), 0], [(0, 0, 2), 0], [(1, 1, 0), 0], [(1, 0, 1), 0],
          [(0, 1, 1), 0]],
    "F": [[(3, 0, 0), 0], [(0, 3, 0), 0], [(0, 0, 3), 0], [(2, 1, 0), 0], [(1, 2, 0), 0],
          [(2, 0, 1), 0], [(1, 0, 2), 0], [(0, 2, 1), 0], [(0, 1, 2), 0], [(1, 1, 1), 0]],
}

BASIS_NAMES = {"sto3g": "sto3g", "sto-3g": "sto3g", "321g": "321g", "3-21g": "321g",
               "631g": "631g", "6-31g": "631g", "631g*": "631g_star", "631g_star": "631g_star",
               "6-31g*": "631g_star", "dzp": "dzp", "qzp": "qzp_gh", "qzp-gh": "qzp_gh", "qzp_gh": "qzp_gh"}


def _dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def prim_norm(a, l, m, n):
    """1/sqrt of the self-overlap of x^l y^m z^n exp(-a r^2)."""
    s = (math.pi / (2.0 * a)) ** 1.5
    for k in (l, m, n):
        s *= _dfact(2 * k - 1) / (4.0 * a) ** k
    return 1.0 / math.sqrt(s)


def basis_table(name):
    key = BASIS_NAMES[name.lower()]
    if key not in _CACHE:
        with open(_DATA) as f:
            _CACHE.update(json.load(f))
    return _CACHE[key]


class Basis:
    """Flat basis arrays: per function nprim, lmn, center; concatenated exps/coefs/norms."""

    def __init__(self, nprim, lmn, center, exps, coefs, norms):
        self.nprim = np.ascontiguousarray(nprim, dtype=np.int32)
        self.lmn = np.ascontiguousarray(lmn, dtype=np.int32).reshape(-1, 3)
        self.center = np.ascontiguousarray(center, dtype=np.float64).reshape(-1, 3)
        self.exps = np.ascontiguousarray(exps, dtype=np.float64)
        self.coefs = np.ascontiguousarray(coefs, dtype=np.float64)
        self.norms = np.ascontiguousarray(norms, dtype=np.float64)
        self.offset = np.zeros(len(self.nprim), dtype=np.int64)
        self.offset[1:] = np.cumsum(self.nprim)[:-1]

    @property
    def nbf(self):
        return len(self.nprim)

    @property
    def ncoef(self):
        """norm*coef per primitive: the contraction weight the J/K engine uses."""
        return self.norms * self.coefs


def build_basis(atoms_bohr, name):
    """atoms_bohr: [(Z, x, y, z)] in bohr.  Returns a Basis in genBasis order."""
    tab = basis_table(name)
    nprim, lmn, center, exps, coefs, norms = [], [], [], [], [], []
    for z, x, y, w in atoms_bohr:
        z = int(round(z))
        recs = tab.get(str(z))
        if recs is None:
            raise ValueError("element Z=%d not in basis %s" % (z, name))
        for kind, prims in recs:
            for (l, m, n), col in COMPONENTS[kind]:
                nprim.append(len(prims))
                lmn.append((l, m, n))
                center.append((x, y, w))
                for p in prims:
                    a = p[0]
                    exps.append(a)
                    coefs.append(p[1 + col])
                    norms.append(prim_norm(a, l, m, n))
    return Basis(nprim, lmn, center, exps, coefs, norms)


def n_primitive_functions(b):
    return int(b.nprim.sum())


_ELEMENT_NAMES = ["", "HYDROGEN", "HELIUM", "LITHIUM", "BERYLLIUM", "BORON", "CARBON", "NITROGEN",
                  "OXYGEN", "FLUORINE", "NEON", "SODIUM", "MAGNESIUM", "ALUMINUM", "SILICON",
                  "PHOSPHORUS", "SULFUR", "CHLORINE", "ARGON"]


def gamess_text(name, elements):
    """GAMESS-US basis text for the given atomic numbers (the format read_GAMESS_BasisSet,
    src/basis.c:316, parses), so a CPU run of the reference can read the same tables."""
    tab = basis_table(name)
    lines = ["$DATA"]
    for z in sorted(set(elements)):
        lines.append(_ELEMENT_NAMES[z])
        for kind, prims in tab[str(z)]:
            lines.append("%s %d" % (kind, len(prims)))
            for k, p in enumerate(prims):
                lines.append("  %d " % (k + 1) + " ".join("%.10E" % v for v in p))
    lines.append("$END")
    return "\n".join(lines) + "\n"
