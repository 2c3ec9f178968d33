"""The batched FP64 eigensolver of the SCF tail (sqb200_syev_batched, cusolverDnXsyevBatched)
against torch.linalg.eigh on seeded symmetric stacks."""
import numpy as np
import pytest

from conftest import load_sqb200


@pytest.mark.gpu
@pytest.mark.parametrize("n,batch", [(32, 5), (96, 3), (224, 2)])
def test_syev_batched_matches_eigh(n, batch):
    import torch
    sqb = load_sqb200()
    rng = np.random.default_rng(n)
    A = rng.normal(size=(batch, n, n))
    A = torch.tensor(A + A.transpose(0, 2, 1), dtype=torch.float64, device="cuda:0")
    W, V = sqb.engine.syev_batched(A)
    torch.cuda.synchronize()
    W0, _ = torch.linalg.eigh(A)
    scale = W0.abs().max().item()
    assert (W - W0).abs().max().item() <= 1e-12 * scale
    # A V = V diag(W) and V orthonormal
    assert (A @ V - V * W[:, None, :]).abs().max().item() <= 1e-11 * scale
    eye = torch.eye(n, dtype=torch.float64, device="cuda:0")
    assert (V.transpose(1, 2) @ V - eye).abs().max().item() <= 1e-12 * n
