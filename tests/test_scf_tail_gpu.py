"""The SCF tail's segmented dot products (sqb200_segdots_*, engine.SegmentDots) against plain
FP64 sums in numpy: several segments per slot, empty segments, a slot without segments,
products and plain sums; repeated runs agree bit for bit.  Tolerance 1e-12 relative (the sums
are taken in a different order)."""
import numpy as np
import pytest

from conftest import load_sqb200


@pytest.mark.gpu
def test_segment_dots_match_numpy_and_repeat_exactly():
    import torch
    sqb = load_sqb200()
    rng = np.random.default_rng(3)
    total = 300_000
    vecs = [rng.normal(size=total) for _ in range(4)]
    dv = [torch.tensor(v, device="cuda:0") for v in vecs]
    starts, lens, slots = [], [], []
    nslot = 7
    for k in range(40):
        L = int(rng.choice([0, 1, 17, 16384, 16385, 40000]))
        s0 = int(rng.integers(0, total - L + 1))
        starts.append(s0)
        lens.append(L)
        slots.append(int(rng.integers(0, nslot - 1)))      # the last slot gets no segment
    plan = sqb.engine.SegmentDots(starts, lens, slots, nslot, 0)
    pairs = [(0, 0), (0, 1), (1, 3), (2, 2), (3, -1), (2, 0)]
    out = plan(dv, pairs).cpu().numpy()
    ref = np.zeros((nslot, len(pairs)))
    for s0, L, sl in zip(starts, lens, slots):
        for p, (i, j) in enumerate(pairs):
            x = vecs[i][s0:s0 + L]
            ref[sl, p] += (x * vecs[j][s0:s0 + L]).sum() if j >= 0 else x.sum()
    scale = np.maximum(1.0, np.abs(ref))
    assert (np.abs(out - ref) / scale).max() <= 1e-12
    assert (out[nslot - 1] == 0.0).all()
    again = plan(dv, pairs).cpu().numpy()
    assert np.array_equal(out, again)
    # all ten DIIS products of four residual vectors in one run
    ten = sqb.scf.DensityDIIS4.PAIRS
    out10 = plan(dv, ten).cpu().numpy()
    for p, (i, j) in enumerate(ten):
        k = pairs.index((i, j)) if (i, j) in pairs else None
        if k is not None:
            assert np.array_equal(out10[:, p], out[:, k])
    with pytest.raises(ValueError):
        plan([dv[0][:10]], [(0, 0)])                         # shorter than the segments
    plan.close()
