"""Scheduler of the served stream (serve.Server) on the CPU: jobs run with a stand-in J/K engine
(oracle J/K, reference S/T/V fixtures), so admission (slots, memory budget, arrival order) and
the interleaved stepping can be checked without a GPU.  Every served result must equal the
job's result alone."""
import numpy as np
import pytest

from conftest import golden, load_sqb200
from test_scf_host import OracleJK

CASES = ["water_321g", "oh_321g_uhf"]


def _requests():
    reqs = []
    for i, c in enumerate(CASES * 2):
        g = golden(c)
        reqs.append({"id": i, "case": c, "atoms": [tuple(a) for a in g["atoms"]], "basis": str(g["basis"]),
                     "arrival": 0.0, "charge": 0, "mult": 1 if g["restricted"] else 2})
    return reqs


def _factory(sqb, torch):
    def make(r):
        g = golden(r["case"])
        return sqb.scf.SCFJob(r["atoms"], r["basis"], device=torch.device("cpu"),
                              restricted=bool(g["restricted"]), engine=OracleJK(g))
    return make


@pytest.mark.parametrize("max_active,budget", [(4, 10 ** 12), (2, 10 ** 12), (4, 150)])
def test_served_results_equal_alone(max_active, budget):
    import torch
    sqb = load_sqb200()
    reqs = _requests()
    srv = sqb.serve.Server(max_active=max_active, hbm_budget=budget, job_factory=_factory(sqb, torch),
                           footprint=lambda atoms, basis: 100)
    res = srv.run(reqs, realtime=False)
    cap = min(max_active, budget // 100) if budget >= 100 else 1
    assert srv.stats["peak_active"] <= max(1, cap)
    for r, out in zip(reqs, res):
        g = golden(r["case"])
        assert out["converged"]
        assert abs(out["energy"] - float(g["energy"])) < 1e-9
        assert out["iters"] == int(g["scf_iters"])
    # admission in arrival order: finish order never precedes the admission order of a slot
    assert all(o["admitted"] <= o["finished"] for o in res)


def test_fifo_latencies():
    sqb = load_sqb200()
    lat = sqb.serve.fifo_latencies([0.0, 0.5, 0.6], [1.0, 1.0, 1.0])
    assert np.allclose(lat, [1.0, 1.5, 2.4])


def test_poisson_requests_are_seeded():
    sqb = load_sqb200()
    a = sqb.serve.poisson_requests(7, 6, rate=2.0, heavy=(2, 4))
    b = sqb.serve.poisson_requests(7, 6, rate=2.0, heavy=(2, 4))
    assert [r["arrival"] for r in a] == [r["arrival"] for r in b]
    assert all(x["arrival"] < y["arrival"] for x, y in zip(a, a[1:]))
    for r in a:
        ne = sum(z for z, *_ in r["atoms"])
        assert (ne % 2 == 1) == (r["mult"] == 2)
