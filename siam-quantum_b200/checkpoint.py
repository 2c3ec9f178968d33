"""Checkpoint files in the reference's text format (save_checkpoint, src/check.c:432-566; read
by load_checkpoint_molecule / _multiplicity / _basis / _orbital, src/check.c:37-295), and the
reference's checkpoint guess (guess_checkpoint_orbital, src/check.c:306-425): the checkpoint's
orbitals projected onto the current basis through the cross overlap, C_new = S^-1 Y C_chk^T.

Layout: SIAM_QUANTUM_CHECKPOINT, FORMAT_VERSION, TIME; the molecule (TOTAL_CHARGE, XYZ_FORMAT
with Z and bohr coordinates); the basis functions as printGTOBasis writes them
(src/basis.c:37-76: `nBasis: n`, then per function `l m n x y z nContract` and `exp coef`
lines, coefficients unnormalised); SPIN_MULTIPLICITY, SCF_METHOD, TOTAL_ENERGY,
ENERGY_CONVERGENCE, DENSITY_CONVERGENCE, the eigenvalues and orbitals of both spins (orbital i
is row i, n*n values, five per line)."""
import math
import time

import numpy as np

from . import basis as B

FORMAT_VERSION = "1.2.5"


def _rows(values, fmt=" %16.8E "):
    out = []
    for i, v in enumerate(values):
        if i % 5 == 0:
            out.append("\n")
        out.append(fmt % v)
    out.append("\n")
    return "".join(out)


def write_checkpoint(path, atoms_bohr, charge, mult, basis, energy, dE, rms_dp, CA, CB, eA, eB):
    """Write a checkpoint the reference's -LCHECK / -GUESS=CHECK can read.  `basis` is a
    basis.Basis (genBasis order); CA, CB are n x n with orbital i in row i."""
    n = basis.nbf
    lines = ["SIAM_QUANTUM_CHECKPOINT\n", "FORMAT_VERSION    %s\n" % FORMAT_VERSION,
             "TIME %s\n" % time.strftime("%a %b %d %H:%M:%S %Y"),
             "SECTION_MOLECULAR_SPECIFICATION_BEGIN\n", "TOTAL_CHARGE   %d\n" % charge, "XYZ_FORMAT\n",
             "%d\n\n" % len(atoms_bohr)]
    for z, x, y, w in atoms_bohr:
        lines.append("%3d %16.8E %16.8E %16.8E\n" % (int(round(z)), x, y, w))
    lines += ["SECTION_MOLECULAR_SPECIFICATION_END\n", "SECTION_BASIS_FUNCTION_BEGIN\n",
              "nBasis: %6d\n" % n]
    off = 0
    for i in range(n):
        k = int(basis.nprim[i])
        l, m, nn = (int(v) for v in basis.lmn[i])
        x, y, w = basis.center[i]
        lines.append("%2d%2d%2d %15.8E %15.8E %15.8E %6d\n" % (l, m, nn, x, y, w, k))
        for j in range(k):
            lines.append("                       %15.8E %15.8E\n" % (basis.exps[off + j], basis.coefs[off + j]))
        off += k
    lines += ["SECTION_BASIS_FUNCTION_END\n", "SECTION_ELECTRONIC_STRUCTURE_BEGIN\n",
              "SPIN_MULTIPLICITY   %d\n" % mult, "SCF_METHOD   HF\n", "TOTAL_ENERGY   %20.8f\n" % energy,
              "ENERGY_CONVERGENCE   %15.3E\n" % dE, "DENSITY_CONVERGENCE   %15.3E\n" % rms_dp,
              "EIGEN_VALUE_ALPHA" + _rows(eA), "EIGEN_VALUE_BETA" + _rows(eB),
              "ORBITAL_ALPHA" + _rows(np.asarray(CA).reshape(-1)),
              "ORBITAL_BETA" + _rows(np.asarray(CB).reshape(-1)),
              "SECTION_ELECTRONIC_STRUCTURE_END\n"]
    with open(path, "w") as f:
        f.write("".join(lines))


def read_checkpoint(path):
    """Parse a checkpoint (written by the reference or by write_checkpoint).  Returns a dict:
    charge, atoms (Z, x, y, z in bohr), mult, energy, basis (basis.Basis, normalised as
    readGTOInput does), eA, eB, CA, CB (orbital i in row i)."""
    tok = open(path).read().split()
    pos = {}
    for i, t in enumerate(tok):
        pos.setdefault(t, i)

    def after(key):
        if key not in pos:
            raise ValueError("checkpoint: keyword %s not found" % key)
        return pos[key] + 1

    q = int(tok[after("TOTAL_CHARGE")])
    i = after("XYZ_FORMAT")
    nat = int(tok[i])
    atoms = []
    for a in range(nat):
        z, x, y, w = tok[i + 1 + 4 * a:i + 5 + 4 * a]
        atoms.append((int(z), float(x), float(y), float(w)))
    i = after("SECTION_BASIS_FUNCTION_BEGIN")
    n = int(tok[i + 1])                  # "nBasis:" then the count
    i += 2
    nprim, lmn, center, exps, coefs = [], [], [], [], []
    for _f in range(n):
        l, m, nn = (int(v) for v in tok[i:i + 3])
        x, y, w = (float(v) for v in tok[i + 3:i + 6])
        k = int(tok[i + 6])
        i += 7
        nprim.append(k)
        lmn.append((l, m, nn))
        center.append((x, y, w))
        for _j in range(k):
            exps.append(float(tok[i]))
            coefs.append(float(tok[i + 1]))
            i += 2
    norms = []
    o = 0
    for f in range(n):
        for j in range(nprim[f]):
            norms.append(B.prim_norm(exps[o + j], *lmn[f]))
        o += nprim[f]
    bas = B.Basis(np.array(nprim, np.int32), np.array(lmn, np.int32), np.array(center), np.array(exps),
                  np.array(coefs), np.array(norms))

    def vec(key, count):
        j = after(key)
        return np.array([float(v) for v in tok[j:j + count]])

    return {"charge": q, "atoms": atoms, "mult": int(tok[after("SPIN_MULTIPLICITY")]),
            "energy": float(tok[after("TOTAL_ENERGY")]), "basis": bas,
            "eA": vec("EIGEN_VALUE_ALPHA", n), "eB": vec("EIGEN_VALUE_BETA", n),
            "CA": vec("ORBITAL_ALPHA", n * n).reshape(n, n), "CB": vec("ORBITAL_BETA", n * n).reshape(n, n)}


def _prims(b):
    """Flat primitive arrays of a basis: function index, exponent, weight (norm * coef),
    angular indices and centre per primitive."""
    f = np.repeat(np.arange(b.nbf), b.nprim)
    return (f, np.asarray(b.exps, float), np.asarray(b.coefs, float) * np.asarray(b.norms, float),
            np.asarray(b.lmn)[f], np.asarray(b.center, float)[f])


def _overlap_1d(la, lb, a, b, xa, xb):
    """1-D Cartesian overlap factors E^{la lb}_0 (McMurchie-Davidson) for arrays of primitive
    pairs; la, lb <= 4."""
    p = a + b
    xab = xa - xb
    xpa = -b / p * xab
    xpb = a / p * xab
    h = 0.5 / p
    L = int(max(la.max(), lb.max()))
    E = {(0, 0, 0): np.ones_like(p)}

    def get(i, j, t):
        if t < 0 or t > i + j or i < 0 or j < 0:
            return 0.0
        key = (i, j, t)
        if key not in E:
            if i > 0:
                E[key] = h * get(i - 1, j, t - 1) + xpa * get(i - 1, j, t) + (t + 1) * get(i - 1, j, t + 1)
            else:
                E[key] = h * get(i, j - 1, t - 1) + xpb * get(i, j - 1, t) + (t + 1) * get(i, j - 1, t + 1)
        return E[key]

    out = np.zeros_like(p)
    for i in range(L + 1):
        for j in range(L + 1):
            sel = (la == i) & (lb == j)
            if sel.any():
                out = np.where(sel, get(i, j, 0), out)
    return out


def overlap_matrix(bA, bB):
    """Contracted overlap <a|b> between the functions of two bases (n_A x n_B)."""
    fa, ea, wa, la, ca = _prims(bA)
    fb, eb, wb, lb, cb = _prims(bB)
    shape = (len(ea), len(eb))
    a = np.broadcast_to(ea[:, None], shape)
    b = np.broadcast_to(eb[None, :], shape)
    p = a + b
    r2 = ((ca[:, None, :] - cb[None, :, :]) ** 2).sum(-1)
    s = np.outer(wa, wb) * np.exp(-a * b / p * r2) * (math.pi / p) ** 1.5
    for d in range(3):
        s = s * _overlap_1d(np.broadcast_to(la[:, d][:, None], shape), np.broadcast_to(lb[:, d][None, :], shape),
                            a, b, np.broadcast_to(ca[:, None, d], shape), np.broadcast_to(cb[None, :, d], shape))
    # primitives of one function are contiguous: sum them
    sa = np.concatenate([[0], np.cumsum(bA.nprim)[:-1]])
    sb = np.concatenate([[0], np.cumsum(bB.nprim)[:-1]])
    return np.add.reduceat(np.add.reduceat(s, sa, axis=0), sb, axis=1)


def project_orbitals(chk, basis, S):
    """The reference's checkpoint guess: orbitals of `chk` (read_checkpoint) expressed in
    `basis` by solving S C_new^T = Y C_chk^T with Y = <basis|chk basis>; then each orbital is
    normalised with S (normalizeC).  Returns (CA, CB), orbital i in row i (n_chk rows)."""
    if basis.nbf < chk["basis"].nbf:
        raise ValueError("cannot use a larger checkpoint basis as guess")
    Y = overlap_matrix(basis, chk["basis"])
    out = []
    for C in (chk["CA"], chk["CB"]):
        X = np.linalg.solve(S, Y @ C.T).T
        nrm = np.sqrt(np.einsum("ij,jk,ik->i", X, S, X))
        out.append(X / nrm[:, None])
    return out[0], out[1]
