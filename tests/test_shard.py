"""CPU tests of the batch partition over ranks, including a world-size-2
gloo run in which each rank computes its share independently."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from bksp_b200 import problems as P
from bksp_b200 import shard


def test_partition_covers_and_balances():
    w = [float(L) ** 3 * 7 for L in P.kappa_batch_edges()]
    for parts in (1, 2, 3, 4, 8):
        shares = shard.partition(w, parts)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(w)))
        loads = [sum(w[i] for i in s) for s in shares]
        # LPT: the heaviest share exceeds the lightest by at most one system
        assert max(loads) - min(loads) <= max(w) + 1e-9
    assert shard.partition([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        shard.partition(w, 0)


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    w = [float(L) ** 3 * 7 for L in P.kappa_batch_edges()]
    mine = shard.my_share(w, world, rank)
    got = [None] * world
    dist.all_gather_object(got, mine)
    if rank == 0:
        out.put(got)
    dist.destroy_process_group()


def test_ranks_agree_on_disjoint_shares():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    a, b = map(set, got)
    assert not (a & b) and (a | b) == set(range(64))
    w = [float(L) ** 3 * 7 for L in P.kappa_batch_edges()]
    assert got == shard.partition(w, 2)


def test_batch_subset_matches_full_batch():
    full = P.kappa_batch(count=4, lo=4, hi=6)
    sub = P.kappa_batch(count=4, lo=4, hi=6, indices=[1, 3])
    for (a, b) in zip([full[1], full[3]], sub):
        for x, y in zip(a, b):
            assert np.array_equal(np.asarray(x), np.asarray(y))
