"""Host logic of the device SCF driver (scf.SCFJob), on the CPU: the driver runs on torch CPU
tensors with a stand-in J/K engine whose builds come from the oracle (the C restatement of the
reference's J/K build) and whose one-electron matrices are the reference's own (golden S, T, V).
Its converged energies must match the reference's uhf() energies, in the same number of SCF
iterations.  The GPU runs of the same
driver with the CUDA engine are in test_scf_gpu.py."""
import numpy as np
import pytest

from conftest import golden, golden_basis, load_oracle, load_sqb200


class OracleJK:
    """Stand-in engine for host-logic tests only: J/K from the oracle, S/T/V from a fixture."""

    def __init__(self, g):
        self.port = load_oracle()
        self.g = g
        self.basis = golden_basis(g)
        self.nbf = self.basis.nbf
        self.sch = g["schwarz"]
        self.builds = []

    def oneint(self, Z, XYZ):
        return self.g["S"], self.g["T"], self.g["V"]

    def mem_cutoff(self, cutoff, max_mem_mb):
        return self.port.mem_cutoff(self.basis, self.sch, cutoff, max_mem_mb)

    def set_precision(self, tau):
        pass

    def build_tensors(self, PA, PB, JT, KA, KB=None, restricted=True, scf_cutoff=1e-10,
                      fixed_cutoff=None, dscreen_rmax=float("inf"), stream=None):
        import torch
        J, K, KBv, st = self.port.jk_build(self.basis, self.sch, PA.numpy(),
                                           None if restricted else PB.numpy(), restricted,
                                           scf_cutoff, fixed_cutoff, dscreen_rmax)
        self.builds.append((scf_cutoff, dscreen_rmax, int(st[0])))
        JT.copy_(torch.from_numpy(J))
        KA.copy_(torch.from_numpy(K))
        if KB is not None:
            KB.copy_(torch.from_numpy(KBv))

    def close(self):
        pass


@pytest.mark.parametrize("case", ["water_321g", "oh_321g_uhf"])
def test_scf_driver_reaches_reference_energy(case):
    import torch
    sqb = load_sqb200()
    g = golden(case)
    eng = OracleJK(g)
    job = sqb.scf.SCFJob([tuple(a) for a in g["atoms"]], str(g["basis"]), device=torch.device("cpu"),
                         restricted=bool(g["restricted"]), engine=eng)
    e = job.run()
    assert job.converged, (job.iters, job.dE, job.avgdP)
    # the reference's own loop (density DIIS, its convergence test): same energy, same steps
    assert abs(e - float(g["energy"])) < 1e-9, e - float(g["energy"])
    assert job.iters == int(g["scf_iters"])
    # first build: reference first visit (memory cutoff); later builds: full density screen
    assert eng.builds[0][1] == job.rmax_first and all(b[1] == float("inf") for b in eng.builds[1:])
    assert all(b[0] == job.cutoff for b in eng.builds)
    PA, PB, S = job.PA.numpy(), job.PB.numpy(), g["S"]
    if job.restricted:
        # the converged density matches the reference's converged density
        assert np.abs(PA - g["PA"]).max() < 1e-5
    else:
        # the doublet's occupied pi orbital is one of a degenerate pair: compare invariants
        assert abs(np.sum(PA * S) - job.nea) < 1e-10 and abs(np.sum(PB * S) - job.neb) < 1e-10
        assert abs(np.sum(PA * S) - np.sum(g["PA"] * S)) < 1e-10


def test_1step_cutoff_rule():
    import torch
    sqb = load_sqb200()
    g = golden("water_321g")
    job = sqb.scf.SCFJob([tuple(a) for a in g["atoms"]], str(g["basis"]), device=torch.device("cpu"),
                         engine=OracleJK(g))
    assert job.cutoff == pytest.approx(1e-8 / (25 + 25 + 25) / 50, rel=1e-15)
    assert float(torch.trace(job.PA)) == pytest.approx(5.0)
