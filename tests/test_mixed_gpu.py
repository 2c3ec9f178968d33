"""Mixed precision: quartets whose Schwarz bound is below tau use the FP32 kernel form (FP64
Boys function, screening and accumulation).  Errors are stated against the plain-FP64 build
and, through the relinked reference program (which builds with difference densities each
SCF iteration), against the reference's FP64 SCF energy: the bar is 1e-6 Eh."""
import json

import numpy as np
import pytest

from conftest import golden, golden_basis, load_sqb200, results_path
from test_dropin_scf import SQREF_GPU, _run

TAUS = [1e-3, 1e-4, 1e-5, 1e-6]


def _engine(g):
    sqb = load_sqb200()
    return sqb.JKEngine(golden_basis(g), schwarz=g["schwarz"])


@pytest.mark.gpu
def test_tau_zero_is_plain_fp64():
    g = golden("h2co_631gs")
    eng = _engine(g)
    J0, K0, _ = eng.build(g["PA"], scf_cutoff=1e-10)
    eng.set_precision(0.0)
    J1, K1, _ = eng.build(g["PA"], scf_cutoff=1e-10)
    # FP64 atomics accumulate in a varying order: equal up to rounding, not bit for bit
    assert np.abs(J0 - J1).max() < 1e-12 and np.abs(K0 - K1).max() < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["benzene_631gs", "oh_321g_uhf"])
def test_mixed_error_shrinks_with_tau(case, monkeypatch):
    # every class with quartets below tau takes its FP32 form, however few its FP32 work items
    # (by default a class with few of them stays in FP64)
    monkeypatch.setenv("SQB200_F32_MIN_ITEMS", "0")
    g = golden(case)
    restricted = bool(g["restricted"])
    eng = _engine(g)
    PB = None if restricted else g["PB"]
    J0, K0, KB0 = eng.build(g["PA"], PB, restricted=restricted, scf_cutoff=1e-10)
    q0 = eng.stats()["quartets"]
    errs = []
    for tau in TAUS:
        eng.set_precision(tau)
        J, K, KB = eng.build(g["PA"], PB, restricted=restricted, scf_cutoff=1e-10)
        assert eng.stats()["quartets"] == q0          # same screening, only precision moves
        errs.append(max(np.abs(J - J0).max(), np.abs(K - K0).max(), np.abs(KB - KB0).max()))
    with open(results_path("mixed_jk_err_%s.json" % case), "w") as f:
        json.dump(dict(zip(map(str, TAUS), errs)), f)
    assert errs[0] < 1e-4
    # monotone above FP64 rounding (1e-13 here); a molecule whose FP32 share is negligible at
    # every tau sits at rounding level throughout
    assert errs[-1] <= max(errs[0], 1e-13)
    assert errs[-1] < 1e-8
    if case == "benzene_631gs":
        assert errs[0] > 1e-12          # the FP32 forms did run


@pytest.mark.gpu
@pytest.mark.parametrize("tau", [1e-4, 1e-6])
def test_mixed_scf_energy_within_1e6(tau, monkeypatch):
    """Whole SCF through the reference's own uhf() (1STEP), GPU Fock build in mixed precision."""
    g = golden("benzene_631gs")
    monkeypatch.setenv("SQB200_FP32_BELOW", str(tau))
    e = _run(SQREF_GPU, g["atoms"], str(g["basis"]), ["-SCFACC=1STEP", "-SCFCONV=1e-8"])
    err = abs(e - float(g["energy"]))
    with open(results_path("mixed_scf_err_%g.json" % tau), "w") as f:
        json.dump({"tau": tau, "energy": e, "reference": float(g["energy"]), "abs_err": err}, f)
    assert err <= 1e-6, err
