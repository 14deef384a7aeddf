"""Failure detection without a GPU fault: a kernel's bounded wait that runs out
is reported as an error status and leaves the context usable; a workspace cap
refuses a call before anything is written (allocation-failure injection); an
injected launch failure (simulated stream error) is reported and later calls
run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_timeout_is_reported_and_the_context_survives(tp):
    import torch

    ex = tp.Executor()
    st = ex.selftest_wait(1_000_000)  # 1 ms on a flag nothing sets
    assert st == tp.ERR_INTERNAL
    assert "bounded wait" in tp.last_error()
    # The same executor keeps working: a contraction right after succeeds.
    A = torch.randn(5, 3, dtype=torch.float64, device="cuda")
    B = torch.randn(3, 4, dtype=torch.float64, device="cuda")
    D = torch.zeros(5, 4, dtype=torch.float64, device="cuda")
    rep = tp.contract([0, 2], A, [2, 1], B, [0, 1], D, exec_=ex)
    torch.cuda.synchronize()
    assert torch.allclose(D, A @ B, rtol=1e-13, atol=1e-13), rep
    assert ex.selftest_wait(1_000_000) == tp.ERR_INTERNAL  # and the status word was cleared in between
    ex.close()


def test_workspace_cap_refuses_before_writing(tp):
    ex = tp.Executor()
    ex.set_workspace_limit(1024)
    a = np.ones((64, 64))
    b = np.ones((64, 64))
    d = np.full((64, 64), 7.0)
    with pytest.raises(tp.TprimsError) as e:
        tp.contract([0, 2], a, [2, 1], b, [0, 1], d, exec_=ex)  # host operands need staging space
    assert e.value.status == tp.ERR_INTERNAL and "limit" in e.value.message
    assert np.all(d == 7.0)
    ex.set_workspace_limit(0)
    tp.contract([0, 2], a, [2, 1], b, [0, 1], d, exec_=ex)
    assert np.all(d == 64.0)
    ex.close()


def test_injected_launch_failure_is_reported_and_later_calls_run(tp):
    """Simulated stream errors: the chosen launch is refused on the host with an
    error status before it reaches the GPU, the output keeps its old value, and
    the same executor then runs the next calls normally (single items and a
    grouped list)."""
    import torch

    ex = tp.Executor()
    A = torch.randn(96, 64, dtype=torch.float64, device="cuda")
    B = torch.randn(64, 80, dtype=torch.float64, device="cuda")
    D = torch.full((96, 80), 7.0, dtype=torch.float64, device="cuda")
    ex.inject_launch_failure(1)  # the second launch from now
    tp.contract([0, 2], A, [2, 1], B, [0, 1], D, exec_=ex)  # first launch runs
    torch.cuda.synchronize()
    assert torch.allclose(D, A @ B, rtol=1e-13, atol=1e-13)
    D.fill_(7.0)
    with pytest.raises(tp.TprimsError) as e:
        tp.contract([0, 2], A, [2, 1], B, [0, 1], D, exec_=ex)
    assert e.value.status == tp.ERR_INTERNAL and "injected" in e.value.message
    torch.cuda.synchronize()
    assert bool(torch.all(D == 7.0))
    tp.contract([0, 2], A, [2, 1], B, [0, 1], D, exec_=ex)  # the hook fired once
    torch.cuda.synchronize()
    assert torch.allclose(D, A @ B, rtol=1e-13, atol=1e-13)
    # A grouped list whose graph launch is refused, then replayed.
    outs = [torch.full((96, 80), 7.0, dtype=torch.float64, device="cuda") for _ in range(3)]
    items = []
    for o in outs:  # torch's row-major storage: strides (64, 1), (80, 1), (80, 1)
        prob = tp.Problem.from_labels(1, tp.OperandSpec(tp.LayoutSpec([96, 64], [64, 1])),
                                      tp.OperandSpec(tp.LayoutSpec([64, 80], [80, 1])),
                                      tp.OperandSpec(tp.LayoutSpec([96, 80], [80, 1])), [0, 2], [2, 1], [0, 1])
        items.append(tp.Item(tp.Plan(prob), 1.0, A.data_ptr(), B.data_ptr(), o.data_ptr()))
    ex.inject_launch_failure(0)
    with pytest.raises(tp.TprimsError) as e:
        tp.contract_batched(items, ex)
    assert "injected" in e.value.message
    torch.cuda.synchronize()
    assert all(bool(torch.all(o == 7.0)) for o in outs)
    tp.contract_batched(items, ex)
    torch.cuda.synchronize()
    assert all(torch.allclose(o, A @ B, rtol=1e-13, atol=1e-13) for o in outs)
    ex.close()
