"""Generate the golden fixtures of the J/K parity tests by running the REFERENCE itself.

Runs oracle/_ref/sqref (the unmodified Siam Quantum 2 sources compiled by oracle/Makefile) on
seeded synthetic molecules and stores, per case, in <case>.npz:
  atoms (Z, x, y, z in angstrom), basis name,
  the reference's own genBasis arrays (nprim, lmn, xyz in bohr, exps, coefs, norms),
  the reference's basis-level Schwarz matrix (create_Schwarz),
  the converged SCF energy and densities PA, PB (uhf(), -SCFACC=1STEP -SCFCONV=1e-8) and the
  number of SCF iterations uhf() took (scf_iters),
  the reference's one-electron matrices S, T, V (GTO_overlap, GTO_kinetic, GTO_nuclei),
  fresh reference J/K builds from the converged density at cutoff 1e-10:
    *_mem  : -MAXMEM=250 (first visit computes every Schwarz survivor, no density screen)
    *_dir  : -MAXMEM=0   (density screen on every quartet)
Usage:  make -C oracle && python tests/golden/make_golden.py
        python tests/golden/make_golden.py --oneint   (add S, T, V to existing fixtures only)
        python tests/golden/make_golden.py --iters    (add the reference's SCF iteration count)
        python tests/golden/make_golden.py --forces   (add the reference's forces, uhf_force)
        python tests/golden/make_golden.py --fshells  (the f-shell cases, FSHELL_CASES)
        python tests/golden/make_golden.py --forces --fshells   (their forces)
        python tests/golden/make_golden.py --fd       (finite-difference gradients of the f cases)
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import port  # noqa: E402

import importlib.util  # noqa: E402
import types  # noqa: E402

_pkg = types.ModuleType("sqb200")
_pkg.__path__ = [os.path.join(ROOT, "siam-quantum_b200")]
sys.modules.setdefault("sqb200", _pkg)
from sqb200 import molecules as M  # noqa: E402

# the reference tree (environment variable SQ_REFERENCE): its basis-set files
if not os.environ.get("SQ_REFERENCE"):
    sys.exit("make_golden.py: set SQ_REFERENCE to the reference source tree")
BASIS_DIR = os.path.join(os.environ["SQ_REFERENCE"], "basis")
OUT = os.path.dirname(os.path.abspath(__file__))


def hydroxyl():
    """OH radical (doublet, UHF): O-H 0.97 angstrom along z."""
    return [(8, 0.0, 0.0, 0.0), (1, 0.0, 0.0, 0.97)]


def formaldehyde():
    """H2CO, planar: C-O 1.21, C-H 1.10 angstrom, H-C-H 116.5 degrees."""
    import math
    a = math.radians(116.5 / 2)
    return [(6, 0.0, 0.0, 0.0), (8, 0.0, 0.0, 1.21),
            (1, 0.0, 1.10 * math.sin(a), -1.10 * math.cos(a)),
            (1, 0.0, -1.10 * math.sin(a), -1.10 * math.cos(a))]


CASES = [
    ("water_321g", M.water, "321g", ()),
    ("oh_321g_uhf", hydroxyl, "321g", ()),
    ("h2co_631gs", formaldehyde, "631g_star", ()),
    ("benzene_631gs", M.benzene, "631g_star", ()),
]

# bases with f shells (QZP: two f shells on every heavy atom, one on hydrogen), for the
# generic quartet path; made by `--fshells`
FSHELL_CASES = [
    ("water_qzp", M.water, "QZP-gh", ()),
    ("oh_qzp_uhf", hydroxyl, "QZP-gh", ()),
]


def ref_basis(xyz, bas):
    r = subprocess.run([port.REF_BIN, "basis", xyz, bas], capture_output=True, text=True, check=True)
    lines = r.stdout.splitlines()
    i = 0
    while True:   # the reference prints chatter first; the dump starts with a lone count
        t = lines[i].split()
        if len(t) == 1 and t[0].isdigit() and len(lines[i + 1].split()) == 7:
            break
        i += 1
    n = int(lines[i]); i += 1
    nprim, lmn, xyzs, exps, coefs, norms = [], [], [], [], [], []
    for _ in range(n):
        t = lines[i].split(); i += 1
        nc = int(t[0])
        nprim.append(nc); lmn.append([int(x) for x in t[1:4]]); xyzs.append([float(x) for x in t[4:7]])
        for _k in range(nc):
            e, c, nm = (float(x) for x in lines[i].split()); i += 1
            exps.append(e); coefs.append(c); norms.append(nm)
    return (np.array(nprim, np.int32), np.array(lmn, np.int32), np.array(xyzs), np.array(exps),
            np.array(coefs), np.array(norms))


def add_oneint():
    for name, geom, bas, opts in CASES:
        path = os.path.join(OUT, name + ".npz")
        rec = dict(np.load(path, allow_pickle=True))
        with tempfile.TemporaryDirectory() as d:
            xyz = os.path.join(d, "m.xyz")
            with open(xyz, "w") as f:
                f.write(M.xyz_text(geom(), name))
            n = len(rec["nprim"])
            rec["S"], rec["T"], rec["V"] = port.ref_oneint(xyz, os.path.join(BASIS_DIR, bas + ".txt"), n)
        np.savez_compressed(path, **rec)
        print(name, "S/T/V added, nbf", n)


def add_scf_iters():
    """Store the reference's SCF iteration count (1STEP, SCFConv 1e-8) in existing fixtures."""
    for name, geom, bas, opts in CASES:
        path = os.path.join(OUT, name + ".npz")
        rec = dict(np.load(path, allow_pickle=True))
        with tempfile.TemporaryDirectory() as d:
            xyz = os.path.join(d, "m.xyz")
            with open(xyz, "w") as f:
                f.write(M.xyz_text(geom(), name))
            res, _, _ = port.ref_scf(xyz, os.path.join(BASIS_DIR, bas + ".txt"),
                                     ["-SCFACC=1STEP", "-SCFCONV=1e-8"] + list(opts))
        rec["scf_iters"] = np.int64(res["iters"])
        np.savez_compressed(path, **rec)
        print(name, "reference SCF iterations", res["iters"])


def add_forces(cases=CASES):
    """Store the reference's forces (uhf_force after uhf(), 1STEP, SCFConv 1e-8)."""
    for name, geom, bas, opts in cases:
        path = os.path.join(OUT, name + ".npz")
        rec = dict(np.load(path, allow_pickle=True))
        with tempfile.TemporaryDirectory() as d:
            xyz = os.path.join(d, "m.xyz")
            with open(xyz, "w") as f:
                f.write(M.xyz_text(geom(), name))
            F, res = port.ref_force(xyz, os.path.join(BASIS_DIR, bas + ".txt"),
                                    ["-SCFACC=1STEP", "-SCFCONV=1e-8"] + list(opts))
        rec["force"] = F
        np.savez_compressed(path, **rec)
        print(name, "reference forces", F.tolist())


def add_fd_gradients(cases=FSHELL_CASES, h=2.5e-4):
    """Store central finite differences of the reference's own SCF energy (uhf(), 1STEP,
    SCFConv 1e-11) with respect to every nuclear coordinate, step h angstrom, as fd_grad
    (hartree/bohr).  With f functions the reference's analytic forces (uhf_force) depart from
    these, so the device gradient of the f cases is checked against them."""
    from concurrent.futures import ThreadPoolExecutor
    bohr = 0.52917721092

    def energy(atoms, bas, opts):
        with tempfile.TemporaryDirectory() as d:
            xyz = os.path.join(d, "m.xyz")
            with open(xyz, "w") as f:
                f.write(M.xyz_text(atoms, "fd"))
            res, _, _ = port.ref_scf(xyz, os.path.join(BASIS_DIR, bas + ".txt"),
                                     ["-SCFACC=1STEP", "-SCFCONV=1e-11"] + list(opts))
        return float(res["energy"])

    for name, geom, bas, opts in cases:
        atoms = geom()
        jobs = []
        for a in range(len(atoms)):
            for x in range(3):
                for sgn in (1, -1):
                    at = [list(t) for t in atoms]
                    at[a][1 + x] += sgn * h
                    jobs.append([tuple(t) for t in at])
        with ThreadPoolExecutor(max_workers=8) as ex:
            E = list(ex.map(lambda at: energy(at, bas, opts), jobs))
        fd = np.array([(E[2 * k] - E[2 * k + 1]) / (2 * h / bohr) for k in range(3 * len(atoms))]).reshape(-1, 3)
        path = os.path.join(OUT, name + ".npz")
        rec = dict(np.load(path, allow_pickle=True))
        rec["fd_grad"] = fd
        np.savez_compressed(path, **rec)
        print(name, "finite-difference gradient", fd.tolist())


def main(cases=CASES):
    for name, geom, bas, opts in cases:
        atoms = geom()
        with tempfile.TemporaryDirectory() as d:
            xyz = os.path.join(d, "m.xyz")
            with open(xyz, "w") as f:
                f.write(M.xyz_text(atoms, name))
            bp = os.path.join(BASIS_DIR, bas + ".txt")
            nprim, lmn, xyzs, exps, coefs, norms = ref_basis(xyz, bp)
            n = len(nprim)
            S = port.ref_schwarz(xyz, bp, n)
            S1, T1, V1 = port.ref_oneint(xyz, bp, n)
            res, PA, PB = port.ref_scf(xyz, bp, ["-SCFACC=1STEP", "-SCFCONV=1e-8"] + list(opts))
            restricted = bool(np.array_equal(PA, PB))
            rec = dict(atoms=np.array(atoms), basis=bas, nprim=nprim, lmn=lmn, xyz=xyzs, exps=exps,
                       coefs=coefs, norms=norms, schwarz=S, energy=res["energy"], PA=PA, PB=PB,
                       restricted=restricted, cutoff=1e-10, S=S1, T=T1, V=V1,
                       scf_iters=np.int64(res["iters"]))
            for tag, mm in (("mem", 250), ("dir", 0)):
                JT, KA, KB, _ = port.ref_jk(xyz, bp, PA, None if restricted else PB,
                                            restricted=restricted, cutoff=1e-10, max_mem=mm)
                rec["JT_" + tag] = JT; rec["KA_" + tag] = KA; rec["KB_" + tag] = KB
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **rec)
        print(name, "nbf", n, "E", res["energy"], "restricted", restricted)


if __name__ == "__main__":
    if "--oneint" in sys.argv[1:]:
        add_oneint()
    elif "--iters" in sys.argv[1:]:
        add_scf_iters()
    elif "--fd" in sys.argv[1:]:
        add_fd_gradients()
    elif "--forces" in sys.argv[1:]:
        add_forces(FSHELL_CASES if "--fshells" in sys.argv[1:] else CASES)
    elif "--fshells" in sys.argv[1:]:
        main(FSHELL_CASES)
    else:
        main()
