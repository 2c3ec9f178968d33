"""Checkpoint files in the reference's format (checkpoint.py): round trip, a checkpoint written
by the reference itself (sq -SCHECK) read here, an SCF restarted from it (-GUESS=CHECK
semantics), and the reference restarting from a checkpoint written here.  CPU only: the SCF
runs the device driver's host logic with the stand-in engine of test_scf_host."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import REFERENCE, ROOT, golden, golden_basis, load_oracle, load_sqb200
from test_scf_host import OracleJK

BASIS_DIR = os.path.join(REFERENCE, "basis") if REFERENCE else ""


def _ref_available():
    return os.path.exists(os.path.join(ROOT, "oracle", "_ref", "sqref")) and bool(BASIS_DIR) and os.path.isdir(BASIS_DIR)


def _ref_scf(xyz, bas, *opts):
    port = load_oracle()
    r = subprocess.run([port.REF_BIN, "scf", xyz, bas, "-", "-SCFACC=1STEP", "-SCFCONV=1e-8"] + list(opts),
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    res = [ln for ln in r.stderr.splitlines() if ln.startswith("RESULT")][0]
    its = [t for t in (ln.split() for ln in r.stdout.splitlines()) if len(t) == 3 and t[0].isdigit() and "E" in t[2]]
    return float(res.split()[1].split("=")[1]), int(its[-1][0])


def test_round_trip():
    sqb = load_sqb200()
    ck = sqb.checkpoint
    g = golden("h2co_631gs")
    b = golden_basis(g)
    rng = np.random.default_rng(3)
    n = b.nbf
    CA, CB = rng.normal(size=(n, n)), rng.normal(size=(n, n))
    eA, eB = np.sort(rng.normal(size=n)), np.sort(rng.normal(size=n))
    atoms = sqb.molecules.to_bohr([tuple(a) for a in g["atoms"]])
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "c.txt")
        ck.write_checkpoint(p, atoms, 0, 1, b, -113.8649828467, 1e-9, 2e-9, CA, CB, eA, eB)
        c = ck.read_checkpoint(p)
    assert c["charge"] == 0 and c["mult"] == 1 and abs(c["energy"] + 113.8649828467) < 1e-8
    assert [a[0] for a in c["atoms"]] == [int(a[0]) for a in atoms]
    assert np.array_equal(c["basis"].nprim, b.nprim) and np.array_equal(c["basis"].lmn, b.lmn)
    assert np.allclose(c["basis"].exps, b.exps, rtol=1e-8) and np.allclose(c["basis"].norms, b.norms, rtol=1e-7)
    assert np.allclose(c["CA"], CA, rtol=1e-8, atol=1e-15) and np.allclose(c["eB"], eB, rtol=1e-8)


@pytest.mark.skipif(not _ref_available(), reason="needs the reference build and its basis files")
def test_reference_checkpoint_read_and_restart():
    import torch
    sqb = load_sqb200()
    ck = sqb.checkpoint
    g = golden("water_321g")
    atoms = [tuple(a) for a in g["atoms"]]
    bas = os.path.join(BASIS_DIR, "321g.txt")
    with tempfile.TemporaryDirectory() as d:
        xyz = os.path.join(d, "w.xyz")
        with open(xyz, "w") as f:
            f.write(sqb.molecules.xyz_text(atoms))
        refchk = os.path.join(d, "ref.txt")
        e_ref, it_ref = _ref_scf(xyz, bas, "-SCHECK", "-FCHECK=" + refchk)
        c = ck.read_checkpoint(refchk)
        # the reference's checkpoint holds its basis (genBasis) and energy
        gb = golden_basis(g)
        assert np.allclose(c["basis"].exps, gb.exps, rtol=1e-8) and np.allclose(c["basis"].norms, gb.norms, rtol=1e-7)
        assert abs(c["energy"] - float(g["energy"])) < 1e-7
        # restart here from the reference's checkpoint
        job = sqb.scf.SCFJob(atoms, "321g", device=torch.device("cpu"), engine=OracleJK(g), guess=refchk)
        e = job.run()
        assert job.converged and abs(e - float(g["energy"])) < 1e-8 and job.iters < it_ref
        # and the reference restarting from a checkpoint written here
        ours = os.path.join(d, "ours.txt")
        job.save_checkpoint(ours)
        e2, it2 = _ref_scf(xyz, bas, "-GUESS=CHECK", "-FCHECK=" + ours)
        assert abs(e2 - float(g["energy"])) < 1e-8 and it2 < it_ref
