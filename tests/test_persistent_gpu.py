"""Persistent work-queue launches (sqb200_jk_set_persistent / sqb200_batch_set_persistent): the
class kernels run as a grid of one CTA per resident slot taking (work item, pass) units from a
device counter.  The J/K must equal the one-CTA-per-unit launch's (1e-10, the plain-FP64 bar)
and the reference's, for single builds in every tile form and for batched builds."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden, golden_basis, load_sqb200

TOL = 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["benzene_631gs", "oh_321g_uhf"])
def test_persistent_single_build_matches(case):
    sqb = load_sqb200()
    g = golden(case)
    restricted = bool(g["restricted"])
    PB = None if restricted else g["PB"]
    eng = sqb.JKEngine(golden_basis(g), schwarz=g["schwarz"])
    for form in (0, 1, 2):
        eng.set_tiles(np.full(256, form, np.int32))
        eng.set_persistent(False)
        ref = eng.build(g["PA"], PB, restricted=restricted, scf_cutoff=1e-10)
        eng.set_persistent(True)
        got = eng.build(g["PA"], PB, restricted=restricted, scf_cutoff=1e-10)
        for a, b in zip(ref, got):
            assert np.abs(a - b).max() <= TOL, (case, form, np.abs(a - b).max())
        assert np.abs(got[0] - g["JT_dir"]).max() <= TOL
        assert np.abs(got[1] - g["KA_dir"]).max() <= TOL
    eng.close()


@pytest.mark.gpu
def test_persistent_batched_build_matches():
    import torch
    sqb = load_sqb200()
    dev = torch.device("cuda", 0)
    gs = [golden(c) for c in GOLDEN_CASES]
    engs = [sqb.JKEngine(golden_basis(g), schwarz=g["schwarz"]) for g in gs]
    batch = sqb.engine.JKBatch(engs)
    T = batch.total
    PA = np.zeros(T); PB = np.zeros(T)
    for m, g in enumerate(gs):
        o, n = batch.offsets[m], len(g["nprim"])
        PA[o:o + n * n] = g["PA"].reshape(-1)
        PB[o:o + n * n] = (g["PA"] if g["restricted"] else g["PB"]).reshape(-1)
    dPA = torch.tensor(PA, device=dev)
    dPB = torch.tensor(PB, device=dev)
    batch.set_step([bool(g["restricted"]) for g in gs], 1e-10)
    outs = []
    for persistent in (False, True):
        batch.set_persistent(persistent)
        JT, KA, KB = (torch.zeros(T, dtype=torch.float64, device=dev) for _ in range(3))
        batch.build_device(dPA.data_ptr(), dPB.data_ptr(), JT.data_ptr(), KA.data_ptr(), KB.data_ptr())
        torch.cuda.synchronize()
        outs.append([x.cpu().numpy() for x in (JT, KA, KB)])
    for a, b in zip(*outs):
        assert np.abs(a - b).max() <= TOL
    for m, g in enumerate(gs):
        o, n = batch.offsets[m], len(g["nprim"])
        assert np.abs(outs[1][0][o:o + n * n] - g["JT_dir"].reshape(-1)).max() <= TOL
        assert np.abs(outs[1][1][o:o + n * n] - g["KA_dir"].reshape(-1)).max() <= TOL
    batch.close()
    for e in engs:
        e.close()
