"""The multi-GPU path of bench.py is N independent replicas: the process
group carries only the barrier and the max/sum over ranks.  Two gloo ranks on
the CPU check that reduction (no device needed)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    r, w, _ = bench.dist_setup(world)
    assert (r, w) == (rank, world) and dist.get_backend() == "gloo"
    # Rank r processed (r + 1) * 1000 units in (r + 1) * 0.5 seconds.
    value, secs, units = bench.replica_value((rank + 1) * 1000, (rank + 1) * 0.5)
    dist.barrier()
    out[rank] = (value, secs, units)
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_replica_throughput_is_sum_over_max():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(90)
            assert p.exitcode == 0
        for r in range(world):
            value, secs, units = out[r]
            assert secs == 1.0 and units == 3000.0 and value == 3000.0
