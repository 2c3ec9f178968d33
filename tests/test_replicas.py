"""bench.py on N GPUs runs N independent replicas (one build runs on one GPU; the path is not
sharded): the job time is the maximum of the ranks' times and the value counts every
rank's work.  Checked here with two gloo ranks on the CPU."""
import os
import socket

import pytest

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import sys
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench
    t = bench.max_over_ranks(dist, 1.0 + rank, torch.device("cpu"))
    out[rank] = t
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    ps = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    assert dict(out) == {0: 2.0, 1: 2.0}
    # value = world * steps / t_max: two replicas of 10 steps in max 2 s -> 10 steps/s
    steps, world = 10, 2
    assert world * steps / out[0] == pytest.approx(10.0)


def test_single_process_passthrough():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 3.5, None) == 3.5
