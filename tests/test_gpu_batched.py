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


def test_short_k_f64_list_on_the_skinny_tiles(tp, torch_cuda, orc):
    """A grouped f64 list of short-K items (K <= 64, N <= 64, M >= 128: the
    skinny FMA tiles of grouped lists), in both operand orders (k-fast and
    rows-fast A), with alpha, beta and C, against the oracle at the plain
    bound and against the same list run one launch per item."""
    torch = torch_cuda
    rng = np.random.default_rng(2026)
    shapes = [(130, 8, 8, True), (257, 16, 33, False), (512, 32, 64, True), (128, 64, 17, False), (300, 40, 64, True),
              (999, 1, 5, False), (200, 33, 1, True), (260, 24, 30, False)]
    ex = tp.Executor()
    items, hosts, devs = [], [], []
    for (m, n, k, kfast) in shapes:
        a = rng.uniform(-1, 1, m * k)
        b = rng.uniform(-1, 1, k * n)
        c = rng.uniform(-1, 1, m * n)
        sa = [k, 1] if kfast else [1, m]
        la, lb, lc = [0, 2], [2, 1], [0, 1]
        prob = tp.Problem.from_labels(tp.F64, tp.OperandSpec(tp.LayoutSpec([m, k], sa)),
                                      tp.OperandSpec(tp.LayoutSpec([k, n], [1, k])),
                                      tp.OperandSpec(tp.LayoutSpec([m, n], [1, m])), la, lb, lc,
                                      c=tp.OperandSpec(tp.LayoutSpec([m, n], [1, m])), lc=lc)
        t = {"a": torch.from_numpy(a).cuda(), "b": torch.from_numpy(b).cuda(), "c": torch.from_numpy(c).cuda(),
             "d": torch.zeros(m * n, dtype=torch.float64, device="cuda")}
        devs.append(t)
        hosts.append((a, b, c, sa))
        items.append(tp.Item(tp.Plan(prob), 0.75, t["a"].data_ptr(), t["b"].data_ptr(), t["d"].data_ptr(),
                             beta=-1.5, c=t["c"].data_ptr()))
    pb = tp.PreparedBatch(items)
    torch.cuda.synchronize()

    def run(grouping):
        ex.set_grouping(grouping)
        pb.run(ex)
        ex.synchronize()
        return [t["d"].cpu().numpy().copy() for t in devs]

    grouped = run(True)
    single = run(False)
    for (m, n, k, kfast), (a, b, c, sa), g, s in zip(shapes, hosts, grouped, single):
        want = np.zeros(m * n)
        orc.packed_contract(0.75, orc.View(a, [m, k], sa, [0, 2]), orc.View(b, [k, n], [1, k], [2, 1]), -1.5,
                            orc.View(c, [m, n], [1, m], [0, 1]), orc.View(want, [m, n], [1, m], [0, 1]))
        assert orc.rel_frobenius(g, want) <= 1e-13, (m, n, k, kfast)
        assert np.linalg.norm(s - g) <= 1e-13 * np.linalg.norm(g), (m, n, k, kfast)
    ex.close()
