"""The multi-GPU form of bench.py (one process per GPU, independent replicas,
no collective on the data path) exercised on CPU with world size 2 over
gloo: each rank builds its own replica inputs, the timings are reduced as the
maximum over ranks, and the aggregate counts every rank's queries."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        grid, vps = bench.make_inputs(rank)
        # a rank's own timings: rank 1 is the slower one
        mine = [1.0 + rank, 2.0 + 3 * rank, 0.5 + rank]
        red = bench.max_over_ranks(mine, world, "cpu")
        out[rank] = (grid.shape, vps.tolist(), red, bench.aggregate_entries_per_s(world, len(vps), red[0]))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_replicas_reduce_to_the_slowest_rank():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    shape0, vps0, red0, agg0 = res[0]
    shape1, vps1, red1, agg1 = res[1]
    assert shape0 == shape1 == (512, 512)          # the same workload on every rank
    assert vps0 != vps1                             # independent replicas: own viewpoints
    assert red0 == red1 == [2.0, 5.0, 1.5]          # each timing is the max over ranks
    k = len(vps0)
    assert agg0 == pytest.approx(world * k * k / 2.0e-3)   # both ranks' queries over the slowest time
