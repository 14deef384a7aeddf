"""The N > 1 host logic on CPU: two gloo ranks on 127.0.0.1 take disjoint,
covering shares of a list (the path shards with no exchange step) and agree on
the max-over-ranks time that bench.py reports."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, n, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    lo, hi = bench.shard(n, rank, world)
    t = bench.max_over_ranks(1.0 + rank * 2.5, dist, "cpu")
    dist.barrier()
    out[rank] = (lo, hi, t)
    dist.destroy_process_group()


@pytest.mark.parametrize("n", [4096, 7, 1])
def test_two_gloo_ranks_shard_and_reduce(n):
    world = 2
    # A spawned manager: forking this (possibly multi-threaded) test process
    # could deadlock the child.
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), n, out), nprocs=world, join=True)
        res = dict(out)
    shares = sorted((res[r][0], res[r][1]) for r in range(world))
    assert shares[0][0] == 0 and shares[-1][1] == n
    assert all(shares[i][1] == shares[i + 1][0] for i in range(world - 1))
    assert all(res[r][2] == 3.5 for r in range(world))


def test_shard_is_balanced():
    for n in (10, 4096, 3):
        sizes = [bench.shard(n, r, 8)[1] - bench.shard(n, r, 8)[0] for r in range(8)]
        assert sum(sizes) == n and max(sizes) - min(sizes) <= 1


def test_balance_is_longest_first_and_respects_devices(tp):
    """The assignment behind contract_batched_sharded: items in decreasing
    cost go to the least-loaded part of their output's device."""
    # Six items on any device over three parts: LPT gives loads 9, 9, 9.
    part = tp.balance([5, 4, 3, 3, 2, 2][::-1], [0, 0, 0])
    costs = [5, 4, 3, 3, 2, 2][::-1]
    loads = [sum(c for c, q in zip(costs, part) if q == k) for k in range(3)]
    assert sorted(loads) == [6, 6, 7]
    # Homes: items on device 1 go only to parts on device 1.
    part = tp.balance([10, 1, 1, 10], [0, 1, 1], homes=[1, 0, None, 1])
    assert part[0] in (1, 2) and part[3] in (1, 2) and part[0] != part[3] and part[1] == 0
    with pytest.raises(tp.TprimsError) as ei:
        tp.balance([1, 1], [0, 0], homes=[0, 3])
    assert ei.value.status == tp.ERR_DEVICE
    assert tp.balance([], [0]) == []
