"""Concurrent host threads on a B200: calls on one executor are serialized
(the reference's SPMD mutex, crates/tprims-capi/src/exec.rs:243-250; here the
executor's lock around its stream and workspace), calls on two executors run
side by side, and every result is exact to the plain path's bound. ctypes
releases the GIL for the duration of each C call, so the threads really are
inside the library at the same time."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "the -m gpu tests need a CUDA device"
    torch.cuda.init()
    return torch


def test_threads_share_one_executor_and_use_a_second(tp, torch_cuda):
    torch = torch_cuda
    ex1, ex2 = tp.Executor(), tp.Executor()
    errors = []

    def worker(seed):
        try:
            g = np.random.default_rng(seed)
            m, n, k = 120 + 7 * seed, 90 + 5 * seed, 70 + 3 * seed
            A, B = g.uniform(-1, 1, (m, k)), g.uniform(-1, 1, (k, n))
            a = torch.from_numpy(A.ravel(order="F").copy()).cuda()
            b = torch.from_numpy(B.ravel(order="F").copy()).cuda()
            d = torch.zeros(m * n, dtype=torch.float64, device="cuda")
            plan = tp.Plan(tp.Problem.from_labels(1, tp.OperandSpec(tp.LayoutSpec.col_major([m, k])),
                                                  tp.OperandSpec(tp.LayoutSpec.col_major([k, n])),
                                                  tp.OperandSpec(tp.LayoutSpec.col_major([m, n])), [0, 2], [2, 1],
                                                  [0, 1]))
            want = A @ B
            for r in range(12):
                ex = ex1 if (seed + r) % 3 else ex2
                plan.execute_into(ex, 1.0 + r, a.data_ptr(), b.data_ptr(), d.data_ptr())
                got = d.cpu().numpy().reshape((m, n), order="F")
                err = float(np.linalg.norm(got - (1.0 + r) * want) / np.linalg.norm((1.0 + r) * want))
                assert err <= 1e-13, (seed, r, err)
                # Host operands too: staged through the executor's shared workspace.
                hd = np.zeros(m * n)
                plan.execute_into(ex, 1.0, A.ravel(order="F").copy(), B.ravel(order="F").copy(), hd)
                assert float(np.linalg.norm(hd.reshape((m, n), order="F") - want) / np.linalg.norm(want)) <= 1e-13
        except Exception as e:  # collected and re-raised on the main thread
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(s,)) for s in range(6)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=120)
    assert not any(t.is_alive() for t in threads), "a worker did not finish"
    assert not errors, errors[0]
    ex1.close()
    ex2.close()


def test_sharded_list_over_two_executors(tp, torch_cuda):
    """contract_batched_sharded: a list balanced over two executors (both on
    this GPU, as two GPUs would each hold one), every item exact, host-staged
    outputs included."""
    torch = torch_cuda
    g = np.random.default_rng(31)
    execs = [tp.Executor(), tp.Executor()]
    items, wants, outs = [], [], []
    for q in range(10):
        m, n, k = (int(x) for x in g.integers(20, 160, size=3))
        A, B = g.uniform(-1, 1, (m, k)), g.uniform(-1, 1, (k, n))
        a = torch.from_numpy(A.ravel(order="F").copy()).cuda()
        b = torch.from_numpy(B.ravel(order="F").copy()).cuda()
        d = torch.zeros(m * n, dtype=torch.float64, device="cuda") if q % 3 else np.zeros(m * n)
        plan = tp.Plan(tp.Problem.from_labels(1, tp.OperandSpec(tp.LayoutSpec.col_major([m, k])),
                                              tp.OperandSpec(tp.LayoutSpec.col_major([k, n])),
                                              tp.OperandSpec(tp.LayoutSpec.col_major([m, n])), [0, 2], [2, 1], [0, 1]))
        items.append(tp.Item(plan, 1.0, a, b, d, _keep=[a, b]))
        wants.append((A @ B, m, n))
        outs.append(d)
    part = tp.balance([it.plan.report()["macs"] for it in items], [0, 0])
    assert set(part) == {0, 1}  # both executors get work
    tp.contract_batched_sharded(items, execs)
    for (w, m, n), d in zip(wants, outs):
        got = (d.cpu().numpy() if hasattr(d, "cpu") else d).reshape((m, n), order="F")
        assert float(np.linalg.norm(got - w) / np.linalg.norm(w)) <= 1e-13
    for e in execs:
        e.close()
