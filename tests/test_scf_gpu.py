"""Device SCF tail: one-electron matrices from the GPU against the reference's own S, T, V
(GTO_overlap/GTO_kinetic/GTO_nuclei, stored in the golden fixtures), and whole RHF/UHF SCF runs
on the device (GPU J/K of difference densities, the reference's density DIIS, cuSOLVER
eigensolves) against the reference's converged energies and iteration counts (uhf(),
-SCFACC=1STEP -SCFCONV=1e-8)."""
import json

import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden, golden_basis, load_sqb200, results_path

E_TOL = 1e-8     # Eh, total energy against the reference's uhf() (same loop, same test)


def test_electron_counts_follow_multiplicity():
    sqb = load_sqb200()
    water = sqb.molecules.water()
    assert sqb.scf.electrons(water) == (5, 5, 1)
    assert sqb.scf.electrons([(8, 0, 0, 0), (1, 0, 0, 0.97)]) == (5, 4, 2)
    assert sqb.scf.electrons(water, mult=3) == (6, 4, 3)
    with pytest.raises(ValueError):
        sqb.scf.electrons(water, mult=2)


def test_nuclear_repulsion_of_h2():
    sqb = load_sqb200()
    assert abs(sqb.scf.nuclear_repulsion([(1, 0, 0, 0), (1, 0, 0, 1.4)]) - 1 / 1.4) < 1e-15


@pytest.mark.gpu
@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_oneint_matches_reference(case):
    sqb = load_sqb200()
    g = golden(case)
    eng = sqb.JKEngine(golden_basis(g), schwarz=g["schwarz"])
    atoms = sqb.molecules.to_bohr([tuple(a) for a in g["atoms"]])
    S, T, V = eng.oneint([a[0] for a in atoms], [a[1:] for a in atoms])
    eng.close()
    assert np.abs(S - g["S"]).max() <= 1e-12
    assert np.abs(T - g["T"]).max() <= 1e-11
    assert np.abs(V - g["V"]).max() <= 1e-10 * max(1.0, np.abs(g["V"]).max())


@pytest.mark.gpu
@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_device_scf_energy(case):
    sqb = load_sqb200()
    g = golden(case)
    job = sqb.scf.SCFJob([tuple(a) for a in g["atoms"]], str(g["basis"]),
                         restricted=bool(g["restricted"]))
    e = job.run()
    iters, secs = job.iters, job.seconds
    job.close()
    err = abs(e - float(g["energy"]))
    with open(results_path("device_scf_%s.json" % case), "w") as f:
        json.dump({"energy": e, "reference": float(g["energy"]), "abs_err": err, "iters": iters,
                   "seconds": secs}, f)
    assert job.converged
    assert err <= E_TOL, err
    assert abs(iters - int(g["scf_iters"])) <= 1
