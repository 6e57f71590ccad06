"""The multi-GPU path is replicas (and ensemble shards) with no collective on the data path:
the only cross-rank step is the max-over-ranks of the timed region.  Checked with two gloo
ranks on the CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    ms = bench.max_over_ranks(10.0 * (rank + 1), world, "cpu")
    out[rank] = ms
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
        assert dict(out) == {0: 20.0, 1: 20.0}


def test_ensemble_shards_partition_the_members():
    from sailfish_b200 import ensemble
    world = 3
    allm = ensemble.ensemble_members(seed=4, n=2 * world)
    shards = [allm[r::world] for r in range(world)]
    assert sum(len(sh) for sh in shards) == len(allm)
    ids = sorted(id(x) for sh in shards for x in sh)
    assert ids == sorted(id(x) for x in allm)
