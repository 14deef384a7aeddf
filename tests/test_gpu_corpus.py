"""The reference's dot_general benchmark corpus (169 entries: tensor-network
shapes from tenferro, batched GEMMs, elementwise-like batches) executed on the
GPU through Problem::from_dot_general / execute_into with seeded inputs, each
checked at 64 sampled outputs against float64 (complex128) sums over the full
contracted index set. Tolerances: the plain path's stated bounds (f32/c32
1e-6 relative Frobenius, widened to 5e-6 for sampled sets; f64/c64 1e-13)."""
import pytest

import bench

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ex(tp):
    import torch

    assert torch.cuda.is_available()
    e = tp.Executor()
    yield e
    e.close()


@pytest.mark.parametrize("i", range(len(bench.corpus_entries())))
def test_corpus_entry_matches_float64(tp, ex, i):
    import torch

    e = bench.corpus_entries()[i]
    plan, bufs, ptrs = bench.corpus_case(tp, torch, e, 20261203 + 7000 + i)
    plan.execute_into(ex, 1.0, ptrs["a"], ptrs["b"], ptrs["c"])
    ex.synchronize()
    err = bench.corpus_sampled_error(torch, e, bufs, seed=i)
    tol = 5e-6 if e["dtype"] in ("f32", "c32") else 1e-13
    assert err <= tol, (e["name"], err, plan.report()["family"])
