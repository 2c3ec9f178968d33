"""Batched Fock builds (sqb200_batch_*): several molecules of different size and spin in one
launch per class kernel must give each molecule exactly its single-molecule build (which is
parity-tested against the reference), also when replayed from a captured CUDA graph and after
the tile autotuner; the batched SCF must reach every molecule's reference energy."""
import json

import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden, golden_basis, load_sqb200, results_path

TOL_SAME = 1e-12     # batch vs single build of the same molecule (atomic summation order only)
TOL_REF = 1e-10      # vs the reference's J/K (fixtures)


def _setup(cases):
    import torch
    sqb = load_sqb200()
    gs = [golden(c) for c in cases]
    engs = [sqb.JKEngine(golden_basis(g), schwarz=g["schwarz"]) for g in gs]
    batch = sqb.JKBatch(engs)
    dev = torch.device("cuda:0")
    T = batch.total
    PA = np.zeros(T)
    PB = np.zeros(T)
    for m, g in enumerate(gs):
        o, n = batch.offsets[m], engs[m].nbf
        PA[o:o + n * n] = g["PA"].reshape(-1)
        PB[o:o + n * n] = (g["PA"] if g["restricted"] else g["PB"]).reshape(-1)
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
    return sqb, gs, engs, batch, t(PA), t(PB)


def _outs(batch):
    import torch
    return [torch.full((batch.total,), float("nan"), dtype=torch.float64, device="cuda:0") for _ in range(3)]


def _block(x, batch, m, n):
    o = batch.offsets[m]
    return x[o:o + n * n].reshape(n, n)


@pytest.mark.gpu
def test_batch_matches_single_builds_and_reference():
    import torch
    sqb, gs, engs, batch, PA, PB = _setup(GOLDEN_CASES)
    restricted = [bool(g["restricted"]) for g in gs]
    batch.set_step(restricted, 1e-10, 1e-10, float("inf"))
    JT, KA, KB = _outs(batch)
    st = torch.cuda.Stream()
    batch.build_device(PA.data_ptr(), PB.data_ptr(), JT.data_ptr(), KA.data_ptr(), KB.data_ptr(), stream=st.cuda_stream)
    st.synchronize()
    bst = batch.stats()
    JT, KA, KB = (x.cpu().numpy() for x in (JT, KA, KB))
    q = 0
    for m, (g, e) in enumerate(zip(gs, engs)):
        n = e.nbf
        r = restricted[m]
        J1, K1, KB1 = e.build(g["PA"], None if r else g["PB"], restricted=r, scf_cutoff=1e-10)
        q += e.stats()["quartets"]
        for x, y in ((JT, J1), (KA, K1), (KB, KB1)):
            assert np.abs(_block(x, batch, m, n) - y).max() <= TOL_SAME
        assert np.abs(_block(JT, batch, m, n) - g["JT_dir"]).max() <= TOL_REF
        assert np.abs(_block(KA, batch, m, n) - g["KA_dir"]).max() <= TOL_REF
        assert np.abs(_block(KB, batch, m, n) - g["KB_dir"]).max() <= TOL_REF
    assert bst["quartets"] == q
    batch.close()


@pytest.mark.gpu
def test_batch_graph_replay_and_autotune():
    import torch
    sqb, gs, engs, batch, PA, PB = _setup(["benzene_631gs", "h2co_631gs", "water_321g"])
    batch.set_step([True] * 3, 1e-10, 1e-10, 0.0)      # no density screen: J, K linear in P
    st = torch.cuda.Stream()
    JT, KA, KB = _outs(batch)
    args = lambda: (PA.data_ptr(), PB.data_ptr(), JT.data_ptr(), KA.data_ptr(), KB.data_ptr())
    with torch.cuda.stream(st):
        batch.build_device(*args(), stream=st.cuda_stream)
        st.synchronize()
        ref = [x.clone() for x in (JT, KA)]
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=st):
            batch.build_device(*args(), stream=st.cuda_stream)
        for x in (JT, KA):
            x.fill_(float("nan"))
        g.replay()
        st.synchronize()
        for x, y in zip((JT, KA), ref):
            assert torch.abs(x - y).max().item() <= TOL_SAME
        # a new density through the same graph
        PA.mul_(0.5)
        PB.mul_(0.5)
        g.replay()
        st.synchronize()
        for x, y in zip((JT, KA), ref):      # J and K are linear in the density
            assert torch.abs(2 * x - y).max().item() <= 4 * TOL_SAME
        PA.mul_(2.0)
        PB.mul_(2.0)
        del g
        batch.autotune(PA.data_ptr(), PB.data_ptr(), stream=st.cuda_stream)
        batch.build_device(*args(), stream=st.cuda_stream)
        st.synchronize()
        for x, y in zip((JT, KA), ref):
            assert torch.abs(x - y).max().item() <= TOL_SAME
    batch.close()


@pytest.mark.gpu
def test_single_context_autotune_keeps_results():
    import torch
    sqb = load_sqb200()
    g = golden("benzene_631gs")
    eng = sqb.JKEngine(golden_basis(g), schwarz=g["schwarz"])
    dev = torch.device("cuda:0")
    PA = torch.tensor(g["PA"], dtype=torch.float64, device=dev)
    t0 = eng.tiles()
    assert (t0 != 1).all()                      # narrow tiles until tuned
    eng.autotune(PA.data_ptr(), restricted=True, scf_cutoff=1e-10)
    t1 = eng.tiles()
    assert ((t1 >= -1) & (t1 <= 2)).all() and (t1 >= 0).sum() > 0
    J, K, _ = eng.build(g["PA"], scf_cutoff=1e-10)
    q = eng.stats()["quartets"]
    assert np.abs(J - g["JT_dir"]).max() <= TOL_REF
    assert np.abs(K - g["KA_dir"]).max() <= TOL_REF
    # every class in its wide form, then in its swapped form, gives the same J/K
    for form in (1, 2):
        eng.set_tiles(np.full(len(t1), form, np.int32))
        J2, K2, _ = eng.build(g["PA"], scf_cutoff=1e-10)
        assert np.abs(J2 - J).max() <= TOL_SAME and np.abs(K2 - K).max() <= TOL_SAME
        assert eng.stats()["quartets"] == q
    eng.close()


@pytest.mark.gpu
def test_batched_scf_reaches_reference_energies():
    sqb = load_sqb200()
    gs = [golden(c) for c in GOLDEN_CASES]
    jobs = [{"atoms": [tuple(a) for a in g["atoms"]], "basis": str(g["basis"]),
             "restricted": bool(g["restricted"])} for g in gs]
    bs = sqb.batch_scf.BatchSCF(jobs)
    E = bs.run()
    conv = bs.converged.copy()
    iters, secs = bs.iter_count.copy(), bs.seconds
    bs.close()
    err = np.abs(E - np.array([float(g["energy"]) for g in gs]))
    with open(results_path("batched_scf.json"), "w") as f:
        json.dump({"energies": E.tolist(), "abs_err": err.tolist(), "iters": iters.tolist(), "seconds": secs}, f)
    assert conv.all()
    assert (err <= 1e-8).all(), err
    # the reference's loop: each molecule takes the reference's number of iterations
    assert (np.abs(iters - np.array([int(g["scf_iters"]) for g in gs])) <= 1).all(), iters
