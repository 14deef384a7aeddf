"""The reference harness's TCCG corpus (benchmarks/benchmarks/tcbench/
corpus.rs:262, 49 contractions of CCSD, AO2MO, InTensLi, CCSD(T) and a
transposed C; tests/golden/tccg.json) on a B200 through Problem::from_labels
and execute_into, plain precision:
  * every case and dtype at the small sizing against the packed oracle run in
    float64 / complex128 on every output (plain bounds f32 / c32 1e-6,
    f64 / c64 1e-13);
  * the published sizing (64 MiB nominal tensors) for one case of each group
    and dtype at 32 sampled outputs against float64 sums."""
import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu

CASES = bench.tccg_cases()
TOL = {"f32": 1e-6, "c32": 1e-6, "f64": 1e-13, "c64": 1e-13}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "the -m gpu tests need a CUDA device"
    return torch


@pytest.fixture(scope="module")
def ex(tp, torch_cuda):
    e = tp.Executor()
    yield e
    e.close()


@pytest.mark.parametrize("dt", ["f32", "f64", "c32", "c64"])
def test_tccg_every_case_small_against_the_packed_oracle(tp, ex, torch_cuda, orc, dt):
    torch = torch_cuda
    wide = np.complex128 if dt[0] == "c" else np.float64
    for i, case in enumerate(CASES):
        plan, t, _ = bench.tccg_case(tp, torch, case, dt, "small", 20261203 + 9100 + i)
        plan.execute_into(ex, 1.0, t["a"].data_ptr(), t["b"].data_ptr(), t["c"].data_ptr())
        torch.cuda.synchronize()
        ext = case["extents"]["small"]
        views = {}
        for k in ("a", "b"):
            dims, st, _ = bench.tccg_layout(case[k], ext)
            views[k] = orc.View(t[k].cpu().numpy().astype(wide), dims, st, [ord(ch) for ch in case[k]])
        dims, st, n = bench.tccg_layout(case["c"], ext)
        want = np.zeros(n, dtype=wide)
        orc.packed_contract(1.0, views["a"], views["b"], 0.0, None,
                            orc.View(want, dims, st, [ord(ch) for ch in case["c"]]))
        err = orc.rel_frobenius(t["c"].cpu().numpy(), want)
        assert err <= TOL[dt], (case["name"], dt, err, plan.report()["family"])


@pytest.mark.parametrize("dt", ["f32", "f64", "c32", "c64"])
def test_tccg_published_sizing_sampled(tp, ex, torch_cuda, dt):
    torch = torch_cuda
    seen = set()
    for i, case in enumerate(CASES):
        if case["group"] in seen:
            continue
        seen.add(case["group"])
        plan, t, _ = bench.tccg_case(tp, torch, case, dt, "tccg64", 20261203 + 9200 + i)
        plan.execute_into(ex, 1.0, t["a"].data_ptr(), t["b"].data_ptr(), t["c"].data_ptr())
        torch.cuda.synchronize()
        err = bench.tccg_sampled_error(torch, case, dt, t, "tccg64", seed=i)
        assert err <= TOL[dt], (case["name"], dt, err, plan.report()["family"])
        del t
