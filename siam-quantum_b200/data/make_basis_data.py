"""Extract Gaussian basis-set tables from GAMESS-US format files into basis_sets.json.

The published Pople basis sets (STO-3G, 3-21G, 6-31G, 6-31G*) and the DZP and QZP sets of the
Jorge group (with f shells: QZP on every heavy atom, DZP from potassium on) ship with the reference as
GAMESS-format text (basis/*.txt; parsed by read_GAMESS_BasisSet, src/basis.c:316-514).  The
GPU host has no reference tree, so the tables the workloads need are converted once into a
JSON data file that travels with this package.  Only exponents and contraction coefficients
are kept, per element and per shell keyword (S, L, P, D, F), in file order.

Usage:  python make_basis_data.py [<basis dir>]   (default: the reference's basis/ dir)
"""
import json
import os
import sys

FILES = {"sto3g": "sto3g.txt", "321g": "321g.txt", "631g": "631g.txt",
         "631g_star": "631g_star.txt", "dzp": "DZP.txt", "qzp_gh": "QZP-gh.txt"}

ELEMENTS = ["HYDROGEN", "HELIUM", "LITHIUM", "BERYLLIUM", "BORON", "CARBON", "NITROGEN",
            "OXYGEN", "FLUORINE", "NEON", "SODIUM", "MAGNESIUM", "ALUMINUM", "SILICON",
            "PHOSPHORUS", "SULFUR", "CHLORINE", "ARGON", "POTASSIUM", "CALCIUM", "SCANDIUM",
            "TITANIUM", "VANADIUM", "CHROMIUM", "MANGANESE", "IRON", "COBALT", "NICKEL",
            "COPPER", "ZINC"]


def _num(tok):
    return float(tok.replace("D", "E").replace("d", "e"))


def parse_gamess(path):
    """Return {Z: [[kind, [[exp, c1(, c2)], ...]], ...]} for the elements of ELEMENTS."""
    lines = open(path).read().splitlines()
    out = {}
    i = 0
    # skip to $DATA
    while i < len(lines) and "$DATA" not in lines[i].upper():
        i += 1
    i += 1
    z = None
    while i < len(lines):
        s = lines[i].strip()
        i += 1
        if not s or s.startswith("!"):
            continue
        if s.upper().startswith("$END"):
            break
        toks = s.split()
        if len(toks) == 1 and toks[0].isalpha() and toks[0].upper() not in ("S", "L", "P", "D", "F"):
            if toks[0].upper() not in ELEMENTS:
                z = None
                continue
            z = ELEMENTS.index(toks[0].upper()) + 1
            out[z] = []
            continue
        kind = toks[0].upper()
        if z is None or kind not in ("S", "L", "P", "D", "F") or len(toks) < 2:
            continue
        nprim = int(toks[1])
        prims = []
        for _ in range(nprim):
            t = lines[i].split()
            i += 1
            prims.append([_num(x) for x in t[1:]])
        out[z].append([kind, prims])
    return out


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: make_basis_data.py <reference basis directory>")
    bdir = sys.argv[1]
    data = {name: parse_gamess(os.path.join(bdir, fn)) for name, fn in FILES.items()}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis_sets.json")
    with open(dst, "w") as f:
        json.dump(data, f, separators=(",", ":"))
    print("wrote", dst, {k: len(v) for k, v in data.items()})


if __name__ == "__main__":
    main()
