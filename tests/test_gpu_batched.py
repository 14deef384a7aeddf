"""contract_batched on the GPU: the config-4 list of environment updates (three
binary steps per item over uneven extents), run as grouped persistent launches
replayed from cached CUDA graphs (a replay bitwise equal to the captured run),
against the same list run one launch per item (each item on the single-launch
family the model picks for it, a packed 3m or DMMA tile where the grouped list
runs a direct one: equal within the plain bound 1e-13) and against the
four-tensor contraction in complex128."""
import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


@pytest.mark.parametrize("dt", ["float64", "complex128"])
def test_grouped_list_matches_per_item_and_the_full_contraction(tp, torch_cuda, dt):
    torch = torch_cuda
    ex = tp.Executor()
    tdt = tp.C64 if dt == "complex128" else tp.F64
    items = bench.c4_items(40, dt, seed=777)
    dev, lists = [], [[], [], []]
    for it in items:
        ext = bench.c4_extents(it)
        t = {k: torch.from_numpy(it[k]).cuda() for k in ("E", "Ma", "W", "Mb")}
        for name, labs in (("T1", bench.C4_STEPS[0][5]), ("T2", bench.C4_STEPS[1][5]), ("Ep", bench.C4_STEPS[2][5])):
            t[name] = torch.zeros(int(np.prod([ext[l] for l in labs])), dtype=t["E"].dtype, device="cuda")
        dev.append(t)
        for si, (xa, la, xb, lb, xd, ld, cj) in enumerate(bench.C4_STEPS):
            prob = tp.Problem.from_labels(
                tdt, tp.OperandSpec(tp.LayoutSpec.col_major([ext[l] for l in la])),
                tp.OperandSpec(tp.LayoutSpec.col_major([ext[l] for l in lb]), cj),
                tp.OperandSpec(tp.LayoutSpec.col_major([ext[l] for l in ld])), la, lb, ld)
            lists[si].append(tp.Item(tp.Plan(prob), 1.0, t[xa].data_ptr(), t[xb].data_ptr(), t[xd].data_ptr()))
    prepared = [tp.PreparedBatch(l) for l in lists]
    torch.cuda.synchronize()  # the inputs are written on torch's stream

    def run(grouping):
        ex.set_grouping(grouping)
        for pb in prepared:
            pb.run(ex)
        ex.synchronize()
        return [d["Ep"].cpu().numpy().copy() for d in dev]

    single = run(False)
    grouped = run(True)   # captures the graphs
    replay = run(True)    # replays them
    for s, g, r in zip(single, grouped, replay):
        assert np.array_equal(g, r)
        assert np.linalg.norm(s - g) <= 1e-13 * np.linalg.norm(g)
    # New input values behind the same pointers: the replayed graph reads them.
    for d in dev:
        d["W"].mul_(2.0)
    torch.cuda.synchronize()
    doubled = run(True)
    for g, d2 in zip(grouped, doubled):
        assert np.allclose(d2, 2 * g, rtol=1e-13, atol=1e-15)
    for d in dev:
        d["W"].mul_(0.5)
    torch.cuda.synchronize()
    for i in np.random.default_rng(5).choice(len(items), size=10, replace=False):
        it = items[i]
        want = bench.c4_reference(it)
        got = grouped[i].reshape((it["a"], it["s"], it["b"]), order="F")
        assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-12, i
    ex.close()
