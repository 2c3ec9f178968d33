"""Served stream on the GPU: energy and energy+gradient jobs of different sizes and spins (RHF
and UHF doublets) run concurrently with continuous batching; each job's served result (energy,
and the gradient where asked) must be the result it gets
alone (same SCF algorithm; only the order of FP64 atomics in the J/K builds differs), also when
the HBM budget holds only a few jobs at a time.  Tolerance: 1e-9 Eh and the same number of SCF
iterations (+-1)."""
import json

import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden, load_sqb200, results_path

TOL = 1e-9


def _requests(sqb):
    reqs = []
    for c in GOLDEN_CASES:
        g = golden(c)
        reqs.append({"atoms": [tuple(a) for a in g["atoms"]], "basis": str(g["basis"]), "charge": 0,
                     "mult": 1 if g["restricted"] else 2})
    rng = np.random.default_rng(11)
    for k in (3, 4):
        m = sqb.molecules.random_organic(rng, k)
        reqs.append({"atoms": m, "basis": "631g_star", "charge": 0, "mult": 1, "gradient": True})
        reqs.append({"atoms": sqb.molecules.remove_one_h(m, rng), "basis": "631g_star", "charge": 0, "mult": 2,
                     "gradient": True})
    for i, r in enumerate(reqs):
        r["id"] = i
        r["arrival"] = 0.05 * i
    return reqs


@pytest.mark.gpu
@pytest.mark.parametrize("batched", [True, False])
@pytest.mark.parametrize("two_slots_by_memory", [False, True])
def test_served_results_equal_alone(two_slots_by_memory, batched):
    """batched: the active jobs' J/K in one batched build per round (re-formed as jobs come and
    go); otherwise one build per job on its own stream."""
    sqb = load_sqb200()
    reqs = _requests(sqb)
    fps = [sqb.serve.footprint_bytes(r["atoms"], r["basis"]) for r in reqs]
    budget = max(fps) + min(fps) if two_slots_by_memory else None
    srv = sqb.serve.Server(max_active=8, hbm_budget=budget, batched=batched)
    res = srv.run(reqs, realtime=True)
    alone = [sqb.serve.solve_alone(r) for r in reqs]
    if two_slots_by_memory:
        # admitted footprints never exceed the budget (a job alone is always admitted)
        assert srv.stats["peak_bytes"] <= budget or srv.stats["peak_active"] == 1
        assert srv.stats["peak_active"] < len(reqs)
    else:
        assert srv.stats["peak_active"] >= 3          # jobs did overlap
    out = []
    for r, o, a in zip(reqs, res, alone):
        out.append({"mult": r["mult"], "nbf": o["nbf"], "served": o["energy"], "alone": a[0],
                    "iters": [o["iters"], a[1]], "latency": o["latency"]})
        assert o["converged"]
        assert abs(o["energy"] - a[0]) <= TOL, (r["id"], o["energy"], a[0])
        assert abs(o["iters"] - a[1]) <= 1
        if r.get("gradient"):
            assert np.abs(o["gradient"] - a[4]).max() <= 1e-8
    with open(results_path("serve_vs_alone_%d_%d.json" % (two_slots_by_memory, batched)), "w") as f:
        json.dump({"jobs": out, "stats": srv.stats}, f)
    # the golden molecules also reach the reference's energies
    for c, o in zip(GOLDEN_CASES, res):
        assert abs(o["energy"] - float(golden(c)["energy"])) <= 1e-8


@pytest.mark.gpu
def test_served_gradients_under_load():
    """Gradient jobs that finish while many other jobs keep the GPU busy get their alone
    gradient: every host read of a job's device state is ordered after the job's own stream."""
    sqb = load_sqb200()
    rng = np.random.default_rng(29)
    reqs = []
    for i in range(10):
        m = sqb.molecules.random_organic(rng, int(rng.integers(5, 10)))
        uhf = i % 2 == 1
        if uhf:
            m = sqb.molecules.remove_one_h(m, rng)
        reqs.append({"id": i, "atoms": m, "basis": "631g_star", "charge": 0, "mult": 2 if uhf else 1,
                     "gradient": True, "arrival": 0.0})
    srv = sqb.serve.Server(max_active=10)
    res = srv.run(reqs, realtime=False)
    assert srv.stats["peak_active"] >= 5
    checked = 0
    for r, o in zip(reqs, res):
        a = sqb.serve.solve_alone(r)
        if o["converged"] and a[4] is not None:
            assert abs(o["energy"] - a[0]) <= TOL
            assert np.abs(o["gradient"] - a[4]).max() <= 1e-8, r["id"]
            checked += 1
    assert checked >= 5
