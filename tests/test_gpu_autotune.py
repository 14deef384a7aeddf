"""The autotuner on a B200: tile family and split-K measured on the first
execution of a Problem signature, cached in the executor, persisted as a
versioned file; grouped lists get their tile policy measured the same way.

Every result is checked against float64 / complex128 sums on the host
(relative Frobenius <= 1e-13 for f64 / c64, the plain path's stated bound),
including in-place accumulation (beta = 1, C = D), where the timed candidate
runs must leave D as one execution leaves it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "the -m gpu tests need a CUDA device"
    torch.cuda.init()
    return torch


def rel(got, want):
    return float(np.linalg.norm(got - want) / np.linalg.norm(want))


def gemm_problem(tp, dtype, m, n, k):
    """D[m,n] = sum_k A[m,k] B[k,n], all column-major."""
    return tp.Problem.from_labels(dtype, tp.OperandSpec(tp.LayoutSpec.col_major([m, k])),
                                  tp.OperandSpec(tp.LayoutSpec.col_major([k, n])),
                                  tp.OperandSpec(tp.LayoutSpec.col_major([m, n])), [0, 2], [2, 1], [0, 1])


def operands(torch, dtype, m, n, k, seed):
    g = np.random.default_rng(seed)
    cplx = dtype == 3

    def draw(shape):
        x = g.uniform(-1, 1, shape)
        return x + 1j * g.uniform(-1, 1, shape) if cplx else x

    A, B, D0 = draw((m, k)), draw((k, n)), draw((m, n))
    dev = lambda x: torch.from_numpy(np.asfortranarray(x).ravel(order="F").copy()).cuda()
    return A, B, D0, dev(A), dev(B), dev(D0)


def host(t, m, n):
    return t.cpu().numpy().reshape((m, n), order="F")


@pytest.mark.parametrize("dtype,m,n,k", [(1, 576, 576, 576), (1, 256, 256, 8192), (3, 200, 136, 1000)])
def test_autotuned_choice_is_measured_cached_and_exact(tp, torch_cuda, dtype, m, n, k):
    torch = torch_cuda
    ex = tp.Executor()
    A, B, _, a, b, _ = operands(torch, dtype, m, n, k, 20261203 + m + k)
    d = torch.zeros(m * n, dtype=a.dtype, device="cuda")
    plan = tp.Plan(gemm_problem(tp, dtype, m, n, k), tp.PlanConfig(autotune=True))
    plan.execute_into(ex, 1.0, a.data_ptr(), b.data_ptr(), d.data_ptr())
    rep = plan.report()
    assert rep["choice"] == "autotuned"
    assert rel(host(d, m, n), A @ B) <= 1e-13
    cache = ex.tuning()["single"]
    entry = cache[rep["signature"] + ";plain;c=0"]
    assert entry["tuned"] and entry["tried"] >= 2 and entry["ms"] > 0
    # A second plan of the same signature reuses the measurement.
    again = tp.Plan(gemm_problem(tp, dtype, m, n, k), tp.PlanConfig(autotune=True))
    d2 = torch.full_like(d, 7.0)
    again.execute_into(ex, 1.0, a.data_ptr(), b.data_ptr(), d2.data_ptr())
    assert again.report()["choice"] == "tuning-cache"
    assert again.report()["family"] == rep["family"] and again.report()["split_k"] == rep["split_k"]
    assert rel(host(d2, m, n), A @ B) <= 1e-13
    assert len(ex.tuning()["single"]) == 1
    ex.close()


@pytest.mark.parametrize("m,n,k", [(256, 256, 8192), (96, 96, 64)])
def test_tuning_an_in_place_accumulation_adds_once(tp, torch_cuda, m, n, k):
    """beta = 1 with C = D: every candidate run reads D, so the tuner restores
    D between runs; the caller sees D0 + A B exactly once."""
    torch = torch_cuda
    ex = tp.Executor()
    A, B, D0, a, b, d = operands(torch, 1, m, n, k, 99 + k)
    plan = tp.Plan(gemm_problem(tp, 1, m, n, k), tp.PlanConfig(autotune=True))
    plan.execute_into_accum(ex, 1.0, a.data_ptr(), b.data_ptr(), 1.0, d.data_ptr())
    assert plan.report()["choice"] == "autotuned"
    assert rel(host(d, m, n), D0 + A @ B) <= 1e-13
    assert ex.tuning()["single"][plan.report()["signature"] + ";plain;c=1"]["tried"] >= 2
    ex.close()


def test_tuning_file_round_trip(tp, torch_cuda, tmp_path):
    torch = torch_cuda
    m = n = 320
    k = 640
    ex = tp.Executor()
    A, B, _, a, b, d = operands(torch, 1, m, n, k, 5)
    plan = tp.Plan(gemm_problem(tp, 1, m, n, k), tp.PlanConfig(autotune=True))
    plan.execute_into(ex, 1.0, a.data_ptr(), b.data_ptr(), d.data_ptr())
    path = tmp_path / "tune.txt"
    ex.save_tuning(str(path))
    text = path.read_text()
    assert text.startswith("tprims-b200-tune 1 ")
    assert text.count("\nsingle ") == 1
    # A new executor created with the file uses the entry without measuring.
    ex2 = tp.Executor(tuning=str(path))
    assert ex2.tuning()["single"] == ex.tuning()["single"]
    other = tp.Plan(gemm_problem(tp, 1, m, n, k), tp.PlanConfig(autotune=True))
    d2 = torch.zeros_like(d)
    other.execute_into(ex2, 1.0, a.data_ptr(), b.data_ptr(), d2.data_ptr())
    assert other.report()["choice"] == "tuning-cache"
    assert rel(host(d2, m, n), A @ B) <= 1e-13
    # Entries measured on another kind of device are skipped.
    head, rest = text.split("\n", 1)
    fields = head.split(" ")
    fields[2] = "7"
    foreign = tmp_path / "foreign.txt"
    foreign.write_text(" ".join(fields) + "\n" + rest)
    ex3 = tp.Executor(tuning=str(foreign))
    assert ex3.tuning()["single"] == {}
    # A malformed file is refused and adds nothing.
    bad = tmp_path / "bad.txt"
    bad.write_text(head + "\nsingle only-a-key 3\n")
    with pytest.raises(tp.TprimsError) as ei:
        ex3.load_tuning(str(bad))
    assert ei.value.status == 1
    assert ex3.tuning()["single"] == {}
    with pytest.raises(tp.TprimsError):
        ex3.load_tuning(str(tmp_path / "missing.txt"))
    ex2.clear_tuning()
    assert ex2.tuning()["single"] == {}
    for e in (ex, ex2, ex3):
        e.close()


def test_grouped_list_tile_policy_is_measured(tp, torch_cuda):
    """A list of uneven f64 products whose plans all autotune: the grouped
    launch's tile policy is timed once per list signature, and every item is
    exact."""
    torch = torch_cuda
    ex = tp.Executor()
    g = np.random.default_rng(11)
    items, want, outs = [], [], []
    for i in range(24):
        m, n, k = (int(x) for x in g.integers(16, 200, size=3))
        if i % 3 == 0:
            n = int(g.integers(4, 32))  # narrow outputs: the tall tile is a candidate
        A, B, _, a, b, _ = operands(torch, 1, m, n, k, 1000 + i)
        d = torch.zeros(m * n, dtype=torch.float64, device="cuda")
        plan = tp.Plan(gemm_problem(tp, 1, m, n, k), tp.PlanConfig(autotune=True))
        items.append(tp.Item(plan, 1.0, a.data_ptr(), b.data_ptr(), d.data_ptr()))
        want.append((A @ B, m, n))
        outs.append((a, b, d))
    tp.contract_batched(items, ex)
    for (w, m, n), (_, _, d) in zip(want, outs):
        assert rel(host(d, m, n), w) <= 1e-13
    lists = ex.tuning()["list"]
    assert len(lists) == 1
    entry = next(iter(lists.values()))
    assert entry["tuned"] and entry["tried"] >= 2 and 0 <= entry["policy"] < 4
    for _, _, d in outs:
        d.zero_()
    tp.contract_batched(items, ex)  # replays the captured graph
    for (w, m, n), (_, _, d) in zip(want, outs):
        assert rel(host(d, m, n), w) <= 1e-13
    assert len(ex.tuning()["list"]) == 1
    ex.close()


def test_split_k_pin_runs_exactly(tp, torch_cuda):
    torch = torch_cuda
    ex = tp.Executor()
    m, n, k = 128, 96, 4096
    A, B, D0, a, b, d = operands(torch, 1, m, n, k, 3)
    for s in (1, 2, 5, 64):
        plan = tp.Plan(gemm_problem(tp, 1, m, n, k), tp.PlanConfig(split_k=s))
        dd = d.clone()
        plan.execute_into_accum(ex, 0.5, a.data_ptr(), b.data_ptr(), -1.0, dd.data_ptr())
        rep = plan.report()
        assert rep["choice"] == "pinned" and rep["split_k"] == s
        assert rel(host(dd, m, n), 0.5 * (A @ B) - D0) <= 1e-13
    ex.close()
