"""Molecular geometries for the J/K workloads (all generated, seeded; no external data).

Coordinates are returned in bohr, converted from angstrom with the reference's factor
(ANGSTROM2BOHR, src/util.h:21), as readMolecule_XYZ does (src/mol.c:92-166).
"""
import math

import numpy as np

ANGSTROM2BOHR = 1.889725988579
SYMBOLS = ["X", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si",
           "P", "S", "Cl", "Ar"]


def water():
    """RHF/3-21G water workload: O (0,0,0.1173), H (0,+-0.7572,-0.4692) angstrom."""
    return [(8, 0.0, 0.0, 0.1173), (1, 0.0, 0.7572, -0.4692), (1, 0.0, -0.7572, -0.4692)]


def benzene(cc=1.39, ch=1.09):
    """Planar D6h benzene: C on a ring of radius cc, H at radius cc+ch, angles 60*k deg."""
    atoms = []
    for k in range(6):
        a = math.radians(60.0 * k)
        atoms.append((6, cc * math.cos(a), cc * math.sin(a), 0.0))
    for k in range(6):
        a = math.radians(60.0 * k)
        atoms.append((1, (cc + ch) * math.cos(a), (cc + ch) * math.sin(a), 0.0))
    return atoms


def c60(b66=1.40, b65=1.45):
    """Ih C60 with 6:6 bonds b66 and 6:5 bonds b65 (angstrom).

    Each carbon sits on an icosahedron edge V->W at fraction t from V: pentagon edges are
    t*a and hexagon-hexagon edges (1-2t)*a for icosahedron edge a, so t = b65/(b66+2*b65)
    and a = b65/t.
    """
    phi = (1.0 + math.sqrt(5.0)) / 2.0
    verts = []
    for s1 in (-1.0, 1.0):
        for s2 in (-1.0, 1.0):
            verts += [(0.0, s1, s2 * phi), (s1, s2 * phi, 0.0), (s2 * phi, 0.0, s1)]
    verts = np.array(verts)
    d = np.linalg.norm(verts[:, None, :] - verts[None, :, :], axis=-1)
    edge = d[d > 1e-9].min()
    t = b65 / (b66 + 2.0 * b65)
    a = b65 / t
    verts *= a / edge
    atoms = []
    for i in range(12):
        for j in range(12):
            if i != j and abs(d[i, j] - edge) < 1e-9:
                p = verts[i] + t * (verts[j] - verts[i])
                atoms.append((6, float(p[0]), float(p[1]), float(p[2])))
    return atoms


def random_organic(rng, n_heavy, bond=(1.0, 1.5), min_dist=2.0, ch=1.09, max_tries=2000):
    """Random closed-shell C/N/O tree saturated with H (batched-SCF workload generator).

    Heavy atoms are attached one by one to a random earlier atom with a free valence, at a
    uniform bond length in `bond`, rejecting placements closer than `min_dist` to any
    non-bonded heavy atom.  Remaining valences (C4, N3, O2) are filled with H at `ch`.
    """
    valence = {6: 4, 7: 3, 8: 2}
    for _ in range(max_tries):
        z0 = int(rng.choice([6, 7, 8]))
        pos = [np.zeros(3)]
        zs = [z0]
        used = [0]
        nbr = [[]]
        ok = True
        while len(zs) < n_heavy and ok:
            cand = [i for i in range(len(zs)) if used[i] < valence[zs[i]]]
            placed = False
            for _try in range(50):
                if not cand:
                    break
                parent = int(rng.choice(cand))
                znew = int(rng.choice([6, 7, 8]))
                if used[parent] >= valence[zs[parent]]:
                    continue
                v = rng.normal(size=3)
                v /= np.linalg.norm(v)
                p = pos[parent] + v * rng.uniform(*bond)
                if all(np.linalg.norm(p - q) >= min_dist for k, q in enumerate(pos) if k != parent):
                    pos.append(p)
                    zs.append(znew)
                    used.append(1)
                    nbr.append([parent])
                    used[parent] += 1
                    nbr[parent].append(len(zs) - 1)
                    placed = True
                    break
            ok = placed
        if not ok:
            continue
        atoms = [(z, *map(float, p)) for z, p in zip(zs, pos)]
        # saturate with hydrogens, pointing away from existing neighbours
        hs = []
        for i, z in enumerate(zs):
            for _h in range(valence[z] - used[i]):
                for _try in range(100):
                    v = rng.normal(size=3)
                    v /= np.linalg.norm(v)
                    away = sum((pos[i] - pos[k]) for k in nbr[i]) if nbr[i] else np.zeros(3)
                    if np.linalg.norm(away) > 0:
                        v = v + 0.8 * away / np.linalg.norm(away)
                        v /= np.linalg.norm(v)
                    p = pos[i] + ch * v
                    others = [np.array(a[1:]) for a in atoms if True] + [np.array(h[1:]) for h in hs]
                    if all(np.linalg.norm(p - q) >= 0.9 for q in others if np.linalg.norm(q - pos[i]) > 1e-9):
                        hs.append((1, *map(float, p)))
                        break
                else:
                    hs.append((1, *map(float, pos[i] + ch * v)))
        return atoms + hs
    raise RuntimeError("random_organic: could not place atoms")


def to_bohr(atoms):
    return [(z, x * ANGSTROM2BOHR, y * ANGSTROM2BOHR, w * ANGSTROM2BOHR) for z, x, y, w in atoms]


def xyz_text(atoms, comment="generated"):
    """XYZ file text (angstrom) in the layout readMolecule_XYZ expects (src/mol.c:92)."""
    lines = [str(len(atoms)), comment]
    for z, x, y, w in atoms:
        lines.append("%-2s %20.12f %20.12f %20.12f" % (SYMBOLS[int(round(z))], x, y, w))
    return "\n".join(lines) + "\n"


def n_electrons(atoms, charge=0):
    return sum(a[0] for a in atoms) - charge


def organic_set(seed, count, heavy=(2, 20)):
    """`count` seeded random closed-shell organics (random_organic) with a uniform number of
    heavy atoms in [heavy[0], heavy[1]]: the batched-SCF workload."""
    rng = np.random.default_rng(seed)
    return [random_organic(rng, int(rng.integers(heavy[0], heavy[1] + 1))) for _ in range(count)]


def remove_one_h(atoms, rng):
    """The doublet radical of a closed-shell molecule: one hydrogen removed at random."""
    hs = [i for i, a in enumerate(atoms) if a[0] == 1]
    if not hs:
        raise ValueError("no hydrogen to remove")
    k = hs[int(rng.integers(len(hs)))]
    return atoms[:k] + atoms[k + 1:]
