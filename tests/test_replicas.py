"""Multi-rank host logic of the replica runs, on CPU with the gloo backend."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from contactmechanics_b200.replicas import assign, max_over_ranks


def test_assign_partitions_work():
    parts = [assign(10, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == list(range(10))
    assert parts[0] == [0, 3, 6, 9]
    with pytest.raises(ValueError):
        assign(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        m = max_over_ranks(1.5 + rank, dist=dist)
        out[rank] = (m, assign(7, rank, world))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert out[0][0] == out[1][0] == 2.5
        assert sorted(out[0][1] + out[1][1]) == list(range(7))
