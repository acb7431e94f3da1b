"""bench.py --gpus N runs N independent replicas of the estimation (the north
star fixes one GPU; samples are independent, so replicas are the multi-GPU
form).  Its only cross-rank step combines the ranks' numbers: total samples,
slowest rank's time.  Checked here with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import sys
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        res = bench.combine_replicas(dist, 1000.0 * (rank + 1), 0.5 + rank, 10.0 * (rank + 1),
                                     2.0 - rank)
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_two_replicas_combine():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        got = dict(out)
    for r in (0, 1):
        samples, t, e2e_s, e2e_t = got[r]
        assert samples == 3000.0      # 1000 + 2000
        assert t == 1.5               # slowest rank
        assert e2e_s == 30.0
        assert e2e_t == 2.0


def test_one_rank_is_identity():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.combine_replicas(None, 5, 1.0, 6, 2.0) == (5, 1.0, 6, 2.0)
