"""Multi-rank host logic of the batched reanalysis, on CPU with the gloo
backend (world size 2): every rank derives the same partition of the
variants, solves only its own (here: a stand-in computation on the CPU),
and the ranks exchange only the final statistics and the max timing."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from openfea_b200.multirank import gather_by_variant, max_over_ranks, partition_variants


def test_partition_is_a_balanced_cover():
    costs = [3 * 441 * n * 16 for n in np.random.default_rng(4).integers(20, 61, size=64)]
    for world in (1, 2, 3, 4, 8):
        parts = partition_variants(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)  # greedy longest-first bound
    assert partition_variants(costs, 2) == partition_variants(list(costs), 2)  # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, costs, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = partition_variants(costs, world)[rank]
        local = {i: {"iterations": int(costs[i] % 97), "rank": rank} for i in mine}
        merged = gather_by_variant(local, dist)
        t = max_over_ranks(0.25 + rank, dist)
        q.put((rank, sorted(merged), {k: v["rank"] for k, v in merged.items()}, t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_partition_and_gather():
    costs = [float(3 * 441 * n) for n in np.random.default_rng(7).integers(20, 61, size=20)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = partition_variants(costs, 2)
    for rank, keys, owner, t in res:
        assert keys == list(range(20))           # every rank sees all variants' stats
        for r in range(2):
            assert all(owner[i] == r for i in parts[r])
        assert t == pytest.approx(1.25)          # max over ranks
