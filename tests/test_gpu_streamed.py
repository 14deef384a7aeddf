"""Streamed execution of host operands on a B200, through TAPP_execute_product:
a large contraction of host A, B and D runs in chunks along the outermost
column axis of its output, the copies in and out overlapping the kernels.
The result must equal the oracle's at the bound of the scheme (bf16x6 1e-6,
plain f64 1e-13) and agree with the same call run unstreamed; the chunked
launches show in the executor's per-kernel launch counts."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "the -m gpu tests need a CUDA device"
    return torch


def col_major(ext):
    st, acc = [], 1
    for e in ext:
        st.append(acc)
        acc *= e
    return st


def product(tp, dtype, specs, precision=0):
    h = tp.Handle()
    infos = [tp.TensorInfo(dtype, e, s) for e, s, _ in specs]
    p = tp.TensorProduct.create(h, *[(0, i, l) for i, (_, _, l) in zip(infos, specs)])
    p._keep = (h, infos)
    if precision:
        p.set_precision(precision)
    return p


def launches(kt, fragment):
    return sum(v["launches"] for k, v in kt.items() if fragment in k)


@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
def test_c2_layout_streamed_bf16x6(tp, torch_cuda, orc, pinned):
    """f32 D[m1,n1,m2,n2] = sum A[k1,m1,k2,m2] B[n1,k2,n2,k1], extents 48,
    A with leading stride 2: A spans twice B's bytes, so B is copied whole and
    A goes in contiguous chunks of its outermost axis m2, D out in pitched
    copies (m2 is not D's outermost axis)."""
    torch = torch_cuda
    e = 48
    sa = [2, 2 * e, 2 * e * e, 2 * e ** 3]
    cm = col_major([e] * 4)
    g = np.random.default_rng(20261203 + 77)
    a = g.standard_normal(2 * e ** 4, dtype=np.float32)
    b = g.standard_normal(e ** 4, dtype=np.float32)
    specs = [([e] * 4, sa, [10, 0, 11, 1]), ([e] * 4, cm, [2, 11, 3, 10]), ([e] * 4, cm, [0, 2, 1, 3]),
             ([e] * 4, cm, [0, 2, 1, 3])]
    p = product(tp, tp.F32, specs, tp.PREC_BF16X6)
    if pinned:
        ah, bh = torch.from_numpy(a).pin_memory(), torch.from_numpy(b).pin_memory()
        dh = torch.full((e ** 4,), np.nan, dtype=torch.float32).pin_memory()
        pa, pb, pd = ah.data_ptr(), bh.data_ptr(), dh.data_ptr()
        dview = dh.numpy()
    else:
        dview = np.full(e ** 4, np.nan, dtype=np.float32)
        pa, pb, pd = a.ctypes.data, b.ctypes.data, dview.ctypes.data
    ex = tp.Executor()
    ex.set_profiling(True)
    tp.check(p.execute(ex, 1.0, pa, pb, 0.0, None, pd))
    kt = ex.kernel_times(reset=True)
    assert launches(kt, "tc_bf16x6_gemm") >= 2, kt  # chunks of m2 (24, 12, 6, 6)
    streamed = dview.copy()
    ex.set_streaming(False)
    tp.check(p.execute(ex, 1.0, pa, pb, 0.0, None, pd))
    kt = ex.kernel_times(reset=True)
    assert launches(kt, "tc_bf16x6_gemm") == 1, kt
    whole = dview.copy()
    ex.close()
    want = np.zeros(e ** 4)
    orc.packed_contract(1.0, orc.View(a.astype(np.float64), [e] * 4, sa, [10, 0, 11, 1]),
                        orc.View(b.astype(np.float64), [e] * 4, cm, [2, 11, 3, 10]), 0.0, None,
                        orc.View(want, [e] * 4, cm, [0, 2, 1, 3]))
    assert np.all(np.isfinite(streamed))
    assert orc.rel_frobenius(streamed, want) <= 1e-6
    assert orc.rel_frobenius(whole, want) <= 1e-6
    assert orc.rel_frobenius(streamed, whole) <= 1e-6


def test_plain_f64_streamed_and_a_layout_that_does_not_stream(tp, torch_cuda, orc):
    """A plain f64 product of host operands (2048 x 1536 x 1024, 40 MiB in
    all) runs streamed: row chunks of A, the larger operand, would be too
    small for a wave of tiles without split-K, so it runs in column chunks of
    B; the same product with D's columns reversed (a negative stride) cannot
    be chunked into pitched copies on either side and runs unstreamed. Both
    agree with the oracle at 1e-13."""
    m, n, k = 2048, 1536, 1024
    g = np.random.default_rng(20261203 + 78)
    a = g.uniform(-1, 1, m * k)
    b = g.uniform(-1, 1, k * n)
    ex = tp.Executor()
    ex.set_profiling(True)
    specs = [([m, k], [1, m], [0, 2]), ([k, n], [1, k], [2, 1]), ([m, n], [1, m], [0, 1]), ([m, n], [1, m], [0, 1])]
    p = product(tp, tp.F64, specs)
    d = np.full(m * n, np.nan)
    tp.check(p.execute(ex, 1.0, a.ctypes.data, b.ctypes.data, 0.0, None, d.ctypes.data))
    kt = ex.kernel_times(reset=True)
    fam = p.report()["family"]
    assert launches(kt, fam) >= 2, (fam, kt)  # column chunks (768, 384, 384)
    want = np.zeros(m * n)
    orc.packed_contract(1.0, orc.View(a, [m, k], [1, m], [0, 2]), orc.View(b, [k, n], [1, k], [2, 1]), 0.0, None,
                        orc.View(want, [m, n], [1, m], [0, 1]))
    assert orc.rel_frobenius(d, want) <= 1e-13
    # D with its columns reversed: origin at the last column, stride -m.
    rev = [([m, k], [1, m], [0, 2]), ([k, n], [1, k], [2, 1]), ([m, n], [1, -m], [0, 1]), ([m, n], [1, -m], [0, 1])]
    q = product(tp, tp.F64, rev)
    d2 = np.full(m * n, np.nan)
    origin = d2.ctypes.data + (n - 1) * m * 8
    tp.check(q.execute(ex, 1.0, a.ctypes.data, b.ctypes.data, 0.0, None, origin))
    kt = ex.kernel_times(reset=True)
    assert launches(kt, q.report()["family"]) == 1, kt
    got = d2.reshape(n, m)[::-1].ravel()  # column j of D sits at column n - 1 - j of the buffer
    assert orc.rel_frobenius(got, want) <= 1e-13
    ex.close()
