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


def _contract_share(tp, items, share):
    """Each item of `share` through the three binary steps of the C4 update,
    planned by the library (Problem::from_labels, Plan::new on the CPU) and
    executed on the host through the plan's own scatter vectors, the way the
    kernels address memory (A' = A[h_a + a_m + a_k], B' = B[h_b + b_k + b_n],
    D[h_d + d_m + d_n] = A' B')."""
    import numpy as np

    results = {}
    for q in share:
        it = items[q]
        ext = bench.c4_extents(it)
        bufs = {k: it[k].astype(np.complex128) for k in ("E", "Ma", "W", "Mb")}
        code = tp.C64 if it["E"].dtype == np.complex128 else tp.F64
        for xa, la, xb, lb, xd, ld, cj in bench.C4_STEPS:
            ea, eb, ed = ([ext[x] for x in ls] for ls in (la, lb, ld))
            plan = tp.Plan(tp.Problem.from_labels(code, tp.OperandSpec(tp.LayoutSpec.col_major(ea)),
                                                  tp.OperandSpec(tp.LayoutSpec.col_major(eb), cj),
                                                  tp.OperandSpec(tp.LayoutSpec.col_major(ed)), la, lb, ld))
            sc = {n: np.array(tp.product_scatter(plan.product, n), dtype=np.int64) for n in tp.SCATTER_NAMES}
            one = np.zeros(1, np.int64)
            h_a, h_b, h_d = (sc[n] if len(sc[n]) else one for n in ("h_a", "h_b", "h_d"))
            out = np.zeros(int(np.prod(ed)), dtype=np.complex128)
            A, B = bufs[xa], (np.conj(bufs[xb]) if cj else bufs[xb])
            for h in range(max(len(sc["h_d"]), 1)):
                Am = A[h_a[h] + sc["a_m"][:, None] + sc["a_k"][None, :]]
                Bn = B[h_b[h] + sc["b_k"][:, None] + sc["b_n"][None, :]]
                out[h_d[h] + sc["d_m"][:, None] + sc["d_n"][None, :]] = Am @ Bn
            bufs[xd] = out
        results[q] = bufs["Ep"]
    return results


def _rank_contracts(rank, world, port, dt, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import tprims_b200 as tp

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    items = bench.c4_items(12, dt, seed=4321)
    costs = [it["a"] * it["s"] * it["b"] * it["p"] * it["a"] for it in items]
    part = tp.balance(costs, [0] * world)  # the same longest-first assignment on every rank
    mine = [q for q in range(len(items)) if part[q] == rank]
    res = _contract_share(tp, items, mine)
    gathered = [None] * world
    dist.all_gather_object(gathered, sorted(res))
    dist.barrier()
    out[rank] = (gathered, {q: v.tolist() for q, v in res.items()})
    dist.destroy_process_group()


@pytest.mark.parametrize("dt", ["float64", "complex128"])
def test_two_gloo_ranks_contract_disjoint_shares_of_a_list(tp, dt):
    """Two gloo ranks each plan and contract their own share of an uneven list
    of environment updates (no exchange step on the data path); the shares are
    disjoint, cover the list, and every result equals the four-tensor
    contraction in complex128."""
    import numpy as np

    world = 2
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_contracts, args=(world, _free_port(), dt, out), nprocs=world, join=True)
        res = dict(out)
    items = bench.c4_items(12, dt, seed=4321)
    shares = [set(res[r][1]) for r in range(world)]
    assert shares[0].isdisjoint(shares[1]) and shares[0] | shares[1] == set(range(len(items)))
    assert all(s for s in shares), "a rank received no items"
    assert res[0][0] == res[1][0] == [sorted(s) for s in shares]
    for r in range(world):
        for q, v in res[r][1].items():
            it = items[q]
            got = np.array(v).reshape((it["a"], it["s"], it["b"]), order="F")
            want = bench.c4_reference(it)
            assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-12, (r, q)


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
