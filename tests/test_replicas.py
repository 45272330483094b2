"""Multi-GPU is replicas only: each rank runs its own reconstruction and the bench reports
the slowest rank.  The host-side plumbing (rendezvous, the max-over-ranks reduction every
rank takes part in) runs here as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        # rank r took 10 + r ms: every rank must see the slowest, 10 + world - 1
        out[rank] = bench.replica_max(10.0 + rank, world, "cpu")
        out[world + rank] = bench.replica_max(3.5, world, "cpu")      # equal ranks
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_replica_max_over_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        assert out[r] == 10.0 + world - 1
        assert out[world + r] == 3.5


def test_replica_max_single_rank_is_identity():
    import bench
    assert bench.replica_max(7.25, 1) == 7.25
