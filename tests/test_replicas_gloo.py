"""The N > 1 bench path runs independent replicas; its only collective is the
max over ranks of the device time.  Check that reduction with two gloo ranks
on the CPU (world size 2, 127.0.0.1 rendezvous)."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        out[rank] = bench.max_over_ranks(10.0 * (rank + 1), world, "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        assert dict(out) == {0: 20.0, 1: 20.0}


def test_max_over_ranks_single_process():
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
