"""Failure detection without a GPU fault: a kernel's bounded wait that runs out
is reported as an error status and leaves the context usable; a workspace cap
refuses a call before anything is written (allocation-failure injection)."""
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
