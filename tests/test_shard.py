"""Sharding of independent traversals across ranks (host logic), on CPU with
gloo and world size 2, as bench.py uses it under torchrun."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from indigo2suite_b200.shard import gather_results, max_over_ranks, run_shard, shard_range


@pytest.mark.parametrize("n,world", [(0, 1), (1, 2), (64, 2), (64, 3), (513, 8), (7, 8)])
def test_shard_range_covers_units_once_and_balanced(n, world):
    seen = []
    sizes = []
    for r in range(world):
        lo, hi = shard_range(n, r, world)
        seen.extend(range(lo, hi))
        sizes.append(hi - lo)
    assert seen == list(range(n))
    assert max(sizes) - min(sizes) <= 1


def test_shard_range_rejects_bad_arguments():
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)
    with pytest.raises(ValueError):
        shard_range(10, 0, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        units = list(range(64))
        # each unit's "traversal": a deterministic result and a rank-dependent time
        secs, res = run_shard(units, rank, world, lambda u: (0.001 * (rank + 1), u * u))
        job = max_over_ranks(secs, world)
        allres = gather_results(res, world)
        out[rank] = (secs, job, allres)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_gloo_sharding():
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        r0, r1 = out[0], out[1]
    assert r0[2] == r1[2] == [u * u for u in range(64)]
    assert r0[1] == r1[1] == pytest.approx(max(r0[0], r1[0]))
    assert r1[0] == pytest.approx(2 * r0[0])
