"""Nuclear gradient on the device (sqb200_gradient: two-electron derivative integrals, one-electron
derivative terms with the energy-weighted density, nuclear repulsion) after the device SCF,
against the reference's own forces (uhf_force after uhf(), stored in the fixtures; force =
-gradient).  Same screening as the reference (shell quartets and, per primitive quartet, function
quartets at 1e-10), same densities up to the SCF's convergence: tolerance 1e-9 hartree/bohr
(measured 1e-13 .. 3e-12).  The test runs several molecules in one process on purpose: a
kernel that read stack memory it had not written gave right answers only on a fresh context."""
import json

import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden, load_sqb200, results_path

TOL = 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_gradient_matches_reference_forces(case):
    sqb = load_sqb200()
    g = golden(case)
    job = sqb.scf.SCFJob([tuple(a) for a in g["atoms"]], str(g["basis"]), restricted=bool(g["restricted"]))
    job.run()
    G = job.gradient()
    job.close()
    F = g["force"]
    err = np.abs(G + F).max()
    with open(results_path("grad_%s.json" % case), "w") as f:
        json.dump({"grad": G.tolist(), "ref_force": F.tolist(), "max_abs_err": float(err)}, f)
    assert np.abs(G.sum(axis=0)).max() < 1e-8          # translational invariance
    assert err <= TOL, err
