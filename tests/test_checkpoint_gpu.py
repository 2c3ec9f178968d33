"""The device SCF restarted from a checkpoint the reference itself wrote (-SCHECK): the
reference's orbitals, projected onto the job's basis as -GUESS=CHECK does (checkpoint.py),
start scf.SCFJob on the GPU.  It must land on the energy of the reference's own restart from
that checkpoint (-GUESS=CHECK) within 1e-8 Eh (the plain-FP64 bar) in the same number of
iterations (+-1), fewer than from the diagonal guess.  (Both restarts stop at |dE| <= 1e-8, so
against the diagonal-guess energy they agree only to about that convergence threshold.)"""
import os
import subprocess
import tempfile

import pytest

from conftest import GOLDEN_CASES, golden, load_oracle, load_sqb200

port = load_oracle()


@pytest.mark.gpu
@pytest.mark.skipif(not port.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_device_scf_restarts_from_reference_checkpoint(case):
    sqb = load_sqb200()
    g = golden(case)
    atoms = [(int(a[0]), float(a[1]), float(a[2]), float(a[3])) for a in g["atoms"]]
    with tempfile.TemporaryDirectory() as d:
        xyz = os.path.join(d, "m.xyz")
        with open(xyz, "w") as f:
            f.write(sqb.molecules.xyz_text(atoms))
        bas = os.path.join(d, "basis.txt")
        with open(bas, "w") as f:
            f.write(sqb.basis.gamess_text(str(g["basis"]), [a[0] for a in atoms]))
        chk = os.path.join(d, "ref_checkpoint.txt")
        r = subprocess.run([port.REF_BIN, "scf", xyz, bas, "-", "-SCFACC=1STEP", "-SCFCONV=1e-8", "-SCHECK",
                            "-FCHECK=" + chk], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0 and os.path.exists(chk), r.stderr[-2000:]
        res = port.ref_run(["scf", xyz, bas, "-", "-SCFACC=1STEP", "-SCFCONV=1e-8", "-GUESS=CHECK",
                            "-FCHECK=" + chk], timeout=600)
        e_ref, it_ref = res["energy"], int(res["iters"])
        job = sqb.scf.SCFJob(atoms, str(g["basis"]), mult=1 if g["restricted"] else 2, device=0, guess=chk)
        e = job.run()
        iters = job.iters
        job.close()
    assert abs(e - e_ref) <= 1e-8, (case, e, e_ref)
    assert abs(iters - it_ref) <= 1, (case, iters, it_ref)
    assert iters < int(g["scf_iters"]), (case, iters, int(g["scf_iters"]))
    assert abs(e - float(g["energy"])) <= 5e-8
