"""The split-precision entry point that allocates no device memory
(tprims_b200_execute_product_noalloc), through the C ABI on a B200.

It exists for callers that cannot call cudaMalloc: code running inside a memory
pool that another component owns, or code that must not let an allocation
synchronise the device. Its scratch is the library's fixed device array, shared
by every call, so the tests run several different contractions in a row and
check each (1) against TAPP_execute_product on the same plan and (2) against
the extended-precision label oracle, at the split schemes' stated bounds
(relative Frobenius bf16x6 <= 1e-6, bf16x3 <= 2e-5). They also check that a
call makes no device allocation: neither the library's own allocation counter
nor torch's allocator moves across it. This file is collected last on purpose."""
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


def oracle_want(orc, specs, a, b, c, d0, alpha, beta):
    """D = alpha * A B + beta * C by the label oracle, in float64."""
    (ea, sa, la), (eb, sb, lb), (ec, sc, lc), (ed, sd, ld) = specs
    out = d0.astype(np.float64)
    orc.label_contract(alpha, orc.View(a, ea, sa, la), orc.View(b, eb, sb, lb), beta,
                       None if c is None else orc.View(c, ec, sc, lc), orc.View(out, ed, sd, ld), out_f64=True)
    return out


CASES = [
    # (1) bf16x6, a permuted 4-mode contraction, beta = 0.
    dict(prec="BF16X6", tol=1e-6, alpha=1.0, beta=0.0, inplace=False,
         a=([40, 24, 36, 20], [0, 4, 1, 5]), b=([20, 48, 24, 28], [5, 2, 4, 3]), d=([40, 36, 48, 28], [0, 1, 2, 3])),
    # (2) bf16x3, a batched contraction with beta != 0 reading C (a different
    # plan and sizes: the shared scratch still holds call 1's data).
    dict(prec="BF16X3", tol=2e-5, alpha=0.75, beta=-0.5, inplace=False,
         a=([6, 130, 200], [0, 1, 2]), b=([6, 200, 90], [0, 2, 3]), d=([6, 130, 90], [0, 1, 3])),
    # (3) alpha = 0 with beta != 0: the output-only pass (A and B unread).
    dict(prec="BF16X6", tol=1e-6, alpha=0.0, beta=1.5, inplace=False,
         a=([70, 33], [0, 2]), b=([33, 50], [2, 1]), d=([70, 50], [0, 1])),
    # (4) in place: C is D (beta * D + alpha * A B written over D).
    dict(prec="BF16X6", tol=1e-6, alpha=-1.25, beta=0.5, inplace=True,
         a=([96, 300], [0, 2]), b=([300, 80], [2, 1]), d=([96, 80], [0, 1])),
]


def run_cases(tp, torch, orc, ex, stream, g):
    for case in CASES:
        (ea, la), (eb, lb), (ed, ld) = case["a"], case["b"], case["d"]
        specs = [(ea, col_major(ea), la), (eb, col_major(eb), lb), (ed, col_major(ed), ld), (ed, col_major(ed), ld)]
        p = product(tp, specs, getattr(tp, "PREC_" + case["prec"]))
        A = torch.randn(int(np.prod(ea)), dtype=torch.float32, device="cuda", generator=g)
        B = torch.randn(int(np.prod(eb)), dtype=torch.float32, device="cuda", generator=g)
        Cm = torch.randn(int(np.prod(ed)), dtype=torch.float32, device="cuda", generator=g)
        if case["inplace"]:
            D_ref, D_new = Cm.clone(), Cm.clone()
            c_ref, c_new = D_ref.data_ptr(), D_new.data_ptr()
        else:
            D_ref = torch.full_like(Cm, 123.0)
            D_new = torch.full_like(Cm, -77.0)
            c_ref = c_new = Cm.data_ptr() if case["beta"] != 0 else None
        torch.cuda.synchronize()
        assert p.execute(ex, case["alpha"], A.data_ptr(), B.data_ptr(), case["beta"], c_ref, D_ref.data_ptr()) == 0, \
            tp.last_error()
        before_lib = tp.device_allocations()
        before_torch = torch.cuda.memory_allocated()
        st = p.execute_noalloc(stream, case["alpha"], A.data_ptr(), B.data_ptr(), case["beta"], c_new,
                               D_new.data_ptr())
        assert st == 0, tp.last_error()
        torch.cuda.synchronize()
        assert tp.device_allocations() == before_lib, "the no-allocation entry point allocated device memory"
        assert torch.cuda.memory_allocated() == before_torch
        ref, new = D_ref.cpu().numpy(), D_new.cpu().numpy()
        assert np.all(np.isfinite(new))
        assert rel(new, ref) <= case["tol"], (case["prec"], rel(new, ref))
        cm = Cm.cpu().numpy()
        want = oracle_want(orc, specs, A.cpu().numpy(), B.cpu().numpy(), cm if case["beta"] != 0 else None,
                           cm if case["inplace"] else np.zeros_like(cm), case["alpha"], case["beta"])
        assert rel(new, want) <= case["tol"], (case["prec"], "vs oracle", rel(new, want))


def test_calls_in_a_row_match_the_allocating_entry_point_and_the_oracle(tp, torch_cuda, orc):
    torch = torch_cuda
    ex = tp.Executor()
    stream = torch.cuda.current_stream().cuda_stream
    g = torch.Generator(device="cuda").manual_seed(20261203)
    run_cases(tp, torch, orc, ex, stream, g)
    # Again, in the same order: every call starts from what the previous one left.
    run_cases(tp, torch, orc, ex, stream, g)
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
