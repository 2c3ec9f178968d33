"""Generate the C60/6-31G J/K fixture (c60_631g.npz) by running the REFERENCE itself.

C60 (Ih truncated icosahedron, 6:6 bonds 1.40, 6:5 bonds 1.45 angstrom; 540 basis functions),
RHF/6-31G:
  1. the reference program (oracle/_ref/sq, -NCPU=8 -MAXMEM=1000 -SCFCONV=1e-6 -SCHECK) writes a
     checkpoint of its converged orbitals; PA = sum over the 180 occupied orbitals C C^T (the
     density uhf_getDMatrix forms, src/uhf.c) from the orbitals as printed there;
  2. one fresh reference J/K build from that PA at Schwarz cutoff 1e-10 in the direct mode
     (-MAXMEM=0: density screen on every quartet), split over NCPU processes exactly as
     uhf_getGMatrix runs it (oracle/_ref/sqref jkpart: child c takes the bra shell pairs with
     PQ % NCPU == c, src/matrix.c:3909-3910); the children's JT/KA/KB are summed in the
     reference's order (src/uhf.c:179-186).
Stored (upper triangles of the symmetric matrices, row-major np.triu_indices order): the
reference's genBasis arrays, its Schwarz matrix, PA, JT, KA; plus ncpu and the SCF energy.

Usage:  make -C oracle REF_SRC=<reference>/src
        SQ_REFERENCE=<reference> python tests/golden/make_c60_golden.py [existing checkpoint]
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import port  # noqa: E402
from make_golden import M, ref_basis  # noqa: E402

if not os.environ.get("SQ_REFERENCE"):
    sys.exit("make_c60_golden.py: set SQ_REFERENCE to the reference source tree")
BASIS = os.path.join(os.environ["SQ_REFERENCE"], "basis", "631g.txt")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c60_631g.npz")
NCPU = 8
SQ = os.path.join(ROOT, "oracle", "_ref", "sq")


def load_checkpoint(path):
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "sqb200.checkpoint", os.path.join(ROOT, "siam-quantum_b200", "checkpoint.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.read_checkpoint(path)


def main():
    atoms = M.c60()
    with tempfile.TemporaryDirectory() as d:
        xyz = os.path.join(d, "c60.xyz")
        with open(xyz, "w") as f:
            f.write(M.xyz_text(atoms, "C60"))
        chk = sys.argv[1] if len(sys.argv) > 1 else os.path.join(d, "c60chk.txt")
        if len(sys.argv) <= 1:
            env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
            subprocess.run([SQ, xyz, BASIS, "-NCPU=8", "-MAXMEM=1000", "-SCFCONV=1e-6", "-SCHECK",
                            "-FCHECK=" + chk], cwd=d, env=env, check=True, capture_output=True)
        c = load_checkpoint(chk)
        nprim, lmn, bxyz, exps, coefs, norms = ref_basis(xyz, BASIS)
        n = len(nprim)
        nocc = sum(a[0] for a in atoms) // 2
        C = c["CA"][:nocc]
        PA = C.T @ C
        PA = 0.5 * (PA + PA.T)
        pa = os.path.join(d, "pa.bin")
        np.ascontiguousarray(PA).tofile(pa)
        sch = port.ref_schwarz(xyz, BASIS, n)
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
        procs = [subprocess.Popen([port.REF_BIN, "jkpart", xyz, BASIS, pa, "-", "1", "1e-10", "0", str(NCPU),
                                   str(k), os.path.join(d, "part%d.bin" % k)],
                                  stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, env=env)
                 for k in range(NCPU)]
        for p in procs:
            _, err = p.communicate()
            if p.returncode:
                sys.exit("jkpart failed: " + err.decode()[-2000:])
        JT = np.zeros((n, n)); KA = np.zeros((n, n))
        for k in range(NCPU - 1, -1, -1):        # uhf_getGMatrix's summation order
            m = np.fromfile(os.path.join(d, "part%d.bin" % k)).reshape(3, n, n)
            JT += m[0]
            KA += m[1]
    iu = np.triu_indices(n)
    np.savez_compressed(OUT, atoms=np.array(atoms), basis="631g", nprim=nprim, lmn=lmn, xyz=bxyz, exps=exps,
                        coefs=coefs, norms=norms, schwarz_u=sch[iu], PA_u=PA[iu], JT_u=JT[iu], KA_u=KA[iu],
                        ncpu=np.int64(NCPU), energy=np.float64(c["energy"]), cutoff=np.float64(1e-10))
    print("wrote", OUT, "nbf", n, "energy", c["energy"], "max|JT|", np.abs(JT).max())


if __name__ == "__main__":
    main()
