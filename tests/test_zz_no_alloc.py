"""The split-precision entry point that allocates no device memory
(tprims_b200_execute_product_noalloc), through the C ABI on a B200.

It exists for callers that cannot call cudaMalloc: code running inside a memory
pool that another component owns, or code that must not let an allocation
synchronise the device. Its scratch is the library's fixed device array, shared
by every call, so the tests run two different contractions in a row and check
each against TAPP_execute_product on the same plan (same kernels, so the
results agree to well within the bf16x6 / bf16x3 bounds used elsewhere:
relative Frobenius 1e-6 / 2e-5). This file is collected last on purpose."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F32 = 0


def col_major(ext):
    st, s = [], 1
    for e in ext:
        st.append(s)
        s *= e
    return st


def product(tp, specs, precision):
    """specs: (extents, strides, labels) of A, B, C, D."""
    h = tp.Handle()
    infos = [tp.TensorInfo(F32, e, s) for e, s, _ in specs]
    p = tp.TensorProduct.create(h, *[(0, i, l) for i, (_, _, l) in zip(infos, specs)])
    p._keep = (h, infos)
    if precision:
        p.set_precision(precision)
    return p


def rel(got, want):
    return float(np.linalg.norm((got - want).astype(np.float64)) / np.linalg.norm(want.astype(np.float64)))


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "the -m gpu tests need a CUDA device"
    return torch


def test_two_calls_in_a_row_match_the_allocating_entry_point(tp, torch_cuda):
    torch = torch_cuda
    ex = tp.Executor()
    stream = torch.cuda.current_stream().cuda_stream
    g = torch.Generator(device="cuda").manual_seed(20261203)
    cases = [
        # (1) bf16x6, a permuted 4-mode contraction, beta = 0.
        dict(prec=tp.PREC_BF16X6, tol=1e-6, alpha=1.0, beta=0.0,
             a=([40, 24, 36, 20], [0, 4, 1, 5]), b=([20, 48, 24, 28], [5, 2, 4, 3]), d=([40, 36, 48, 28], [0, 1, 2, 3])),
        # (2) bf16x3, a batched contraction with beta != 0 reading C (a
        # different plan and sizes: the shared scratch holds call 1's data).
        dict(prec=tp.PREC_BF16X3, tol=2e-5, alpha=0.75, beta=-0.5,
             a=([6, 130, 200], [0, 1, 2]), b=([6, 200, 90], [0, 2, 3]), d=([6, 130, 90], [0, 1, 3])),
    ]
    for case in cases:
        (ea, la), (eb, lb), (ed, ld) = case["a"], case["b"], case["d"]
        specs = [(ea, col_major(ea), la), (eb, col_major(eb), lb), (ed, col_major(ed), ld), (ed, col_major(ed), ld)]
        p = product(tp, specs, case["prec"])
        A = torch.randn(int(np.prod(ea)), dtype=torch.float32, device="cuda", generator=g)
        B = torch.randn(int(np.prod(eb)), dtype=torch.float32, device="cuda", generator=g)
        Cm = torch.randn(int(np.prod(ed)), dtype=torch.float32, device="cuda", generator=g)
        D_ref = torch.full_like(Cm, 123.0)
        D_new = torch.full_like(Cm, -77.0)
        c_ptr = Cm.data_ptr() if case["beta"] != 0 else None
        torch.cuda.synchronize()
        assert p.execute(ex, case["alpha"], A.data_ptr(), B.data_ptr(), case["beta"], c_ptr, D_ref.data_ptr()) == 0, \
            tp.last_error()
        st = p.execute_noalloc(stream, case["alpha"], A.data_ptr(), B.data_ptr(), case["beta"], c_ptr,
                               D_new.data_ptr())
        assert st == 0, tp.last_error()
        torch.cuda.synchronize()
        ref, new = D_ref.cpu().numpy(), D_new.cpu().numpy()
        assert np.all(np.isfinite(new))
        assert rel(new, ref) <= case["tol"], (case["prec"], rel(new, ref))
    ex.close()


def test_refusals_leave_the_output_untouched(tp, torch_cuda):
    torch = torch_cuda
    stream = torch.cuda.current_stream().cuda_stream
    n = 4096  # bf16x6 planes of two 4096 x 4096 operands: 192 MiB > the fixed 64 MiB
    e2 = [n, n]
    big = product(tp, [(e2, col_major(e2), [0, 2]), (e2, col_major(e2), [2, 1]), (e2, col_major(e2), [0, 1]),
                       (e2, col_major(e2), [0, 1])], tp.PREC_BF16X6)
    A = torch.ones(n * n, dtype=torch.float32, device="cuda")
    D = torch.full((n * n,), 5.0, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    assert big.execute_noalloc(stream, 1.0, A.data_ptr(), A.data_ptr(), 0.0, None, D.data_ptr()) == tp.ERR_SHAPE
    assert "64 MiB" in tp.last_error()
    e1 = [64, 64]
    plain = product(tp, [(e1, col_major(e1), [0, 2]), (e1, col_major(e1), [2, 1]), (e1, col_major(e1), [0, 1]),
                         (e1, col_major(e1), [0, 1])], tp.PREC_PLAIN)
    assert plain.execute_noalloc(stream, 1.0, A.data_ptr(), A.data_ptr(), 0.0, None, D.data_ptr()) == \
        tp.ERR_UNSUPPORTED
    torch.cuda.synchronize()
    assert bool(torch.all(D == 5.0))
