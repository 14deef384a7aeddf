"""The Ozaki INT8 slice scheme (f64 / c64 on tcgen05 kind::i8) against the
extended-precision label oracle, through the C ABI. Stated bound: relative
Frobenius error <= 1e-12 with the default 6 slices."""
import numpy as np
import pytest

from test_gpu_parity import Op, make_product, oracle_ref, rnd, run

pytestmark = pytest.mark.gpu

OZ = 3  # TPRIMS_PREC_OZAKI_INT8


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def ex(tp, torch_cuda):
    e = tp.Executor()
    yield e
    e.close()


def _run_prepared(tp, ex, torch, p, A, B, C, D, alpha, beta):
    tens = {}

    def dptr(o, b, key):
        t = torch.from_numpy(b.copy()).cuda()
        tens[key] = t
        return t.data_ptr() + o.offset * b.itemsize

    pa, pb, pd = dptr(A, A.buf, "a"), dptr(B, B.buf, "b"), dptr(D, D.buf, "d")
    pc = None if C is None else (pd if C.buf is D.buf else dptr(C, C.buf, "c"))
    st = p.execute(ex, alpha, pa, pb, beta, pc, pd)
    torch.cuda.synchronize()
    assert st == 0, tp.last_error()
    return tens["d"].cpu().numpy()


def oz(tp, ex, torch, dt, A, B, C, D, alpha, beta, slices=0):
    p = make_product(tp, dt, A, B, C, D)
    p.set_precision(OZ, slices)
    return _run_prepared(tp, ex, torch, p, A, B, C, D, alpha, beta), p


@pytest.mark.parametrize("dt", ["float64", "complex128"])
def test_ozaki_ragged_batched_general_strides(tp, ex, torch_cuda, orc, dt):
    rng = np.random.default_rng(41)
    # h = 40: batch index innermost with at least 32 entries (the batch-innermost
    # packing), not a multiple of 32.
    for (m, n, k, h) in [(1, 1, 1, 1), (7, 13, 5, 1), (130, 257, 70, 1), (65, 33, 129, 3), (70, 45, 100, 40)]:
        A = Op(rnd(rng, dt, h * m * k), [h, k, m], [1, h, h * k], [9, 2, 0])  # k before m
        B = Op(rnd(rng, dt, h * k * n), [h, n, k], [1, h * k, h], [9, 1, 2])
        C = Op(rnd(rng, dt, h * m * n), [h, m, n], [1, h, h * m], [9, 0, 1])
        d0 = np.zeros(h * m * n, dtype=dt)
        D = Op(d0, [h, m, n], [1, h, h * m], [9, 0, 1])
        al, be = (complex(0.5, -0.25), complex(-1.5, 0.5)) if dt == "complex128" else (0.75, -1.5)
        want = oracle_ref(orc, dt, A, B, C, D, al, be, d0)
        got, p = oz(tp, ex, torch_cuda, dt, A, B, C, D, al, be)
        err = orc.rel_frobenius(got, want)
        assert err <= 1e-12, (m, n, k, h, err, p.report()["family"])


@pytest.mark.parametrize("mask", range(16))
def test_ozaki_complex_every_conjugation(tp, ex, torch_cuda, orc, mask):
    rng = np.random.default_rng(500 + mask)
    dt = "complex128"
    A = Op(rnd(rng, dt, 20 * 9), [20, 9], [1, 20], [0, 2], conj=bool(mask & 1))
    B = Op(rnd(rng, dt, 9 * 11), [9, 11], [11, 1], [2, 1], conj=bool(mask & 2))
    C = Op(rnd(rng, dt, 20 * 11), [20, 11], [1, 20], [0, 1], conj=bool(mask & 4))
    d0 = np.zeros(220, dtype=dt)
    D = Op(d0, [20, 11], [1, 20], [0, 1], conj=bool(mask & 8))
    al, be = complex(1.25, -0.5), complex(0.75, 0.5)
    want = oracle_ref(orc, dt, A, B, C, D, al, be, d0)
    got, _ = oz(tp, ex, torch_cuda, dt, A, B, C, D, al, be)
    assert orc.rel_frobenius(got, want) <= 1e-12


def test_ozaki_c1_full_size(tp, ex, torch_cuda, orc):
    rng = np.random.default_rng(20261203 + 1000 + 10)
    e = 24
    cm = [1, e, e * e, e ** 3]
    A = Op(rng.uniform(-1, 1, e ** 4), [e] * 4, cm, [0, 4, 1, 5])
    B = Op(rng.uniform(-1, 1, e ** 4), [e] * 4, cm, [5, 2, 4, 3])
    C = Op(rng.uniform(-1, 1, e ** 4), [e] * 4, cm, [0, 1, 2, 3])
    d0 = np.zeros(e ** 4)
    D = Op(d0, [e] * 4, cm, [0, 1, 2, 3])
    want = oracle_ref(orc, "float64", A, B, C, D, 1.0, 0.5, d0)
    got, _ = oz(tp, ex, torch_cuda, "float64", A, B, C, D, 1.0, 0.5)
    assert orc.rel_frobenius(got, want) <= 1e-12


@pytest.mark.parametrize("dt", ["float64", "complex128"])
def test_ozaki_deep_k_is_split_into_exact_chunks(tp, ex, torch_cuda, orc, dt):
    # K = 40000 exceeds one INT32-exact chunk (about 21800 at 6 slices); later
    # chunks accumulate into D with beta = 1 and op_C = op_D.
    rng = np.random.default_rng(43)
    m, n, k = 5, 6, 40000
    A = Op(rnd(rng, dt, m * k), [m, k], [1, m], [0, 2])
    B = Op(rnd(rng, dt, k * n), [k, n], [1, k], [2, 1])
    C = Op(rnd(rng, dt, m * n), [m, n], [1, m], [0, 1])
    d0 = np.zeros(m * n, dtype=dt)
    D = Op(d0, [m, n], [1, m], [0, 1], conj=dt == "complex128")
    want = oracle_ref(orc, dt, A, B, C, D, 1.0, 0.5, d0)
    got, _ = oz(tp, ex, torch_cuda, dt, A, B, C, D, 1.0, 0.5)
    assert orc.rel_frobenius(got, want) <= 1e-12


def test_ozaki_error_falls_with_slices(tp, ex, torch_cuda, orc):
    rng = np.random.default_rng(44)
    m, n, k = 96, 80, 200
    A = Op(rnd(rng, "float64", m * k), [m, k], [1, m], [0, 2])
    B = Op(rnd(rng, "float64", k * n), [k, n], [1, k], [2, 1])
    d0 = np.zeros(m * n)
    D = Op(d0, [m, n], [1, m], [0, 1])
    want = oracle_ref(orc, "float64", A, B, None, D, 1.0, 0.0, d0)
    errs = []
    for s in (4, 5, 6, 7, 8):
        got, _ = oz(tp, ex, torch_cuda, "float64", A, B, None, D, 1.0, 0.0, slices=s)
        errs.append(orc.rel_frobenius(got, want))
    assert all(errs[i + 1] < errs[i] for i in range(3)), errs
    assert errs[3] <= 1e-12 and errs[4] <= 1e-13, errs


def test_ozaki_non_finite_rows_give_nan(tp, ex, torch_cuda, orc):
    rng = np.random.default_rng(45)
    a = rng.standard_normal(8 * 6)
    a[3 + 8 * 2] = np.inf  # row 3 of A
    A = Op(a, [8, 6], [1, 8], [0, 2])
    B = Op(rng.standard_normal(6 * 5), [6, 5], [1, 6], [2, 1])
    D = Op(np.zeros(40), [8, 5], [1, 8], [0, 1])
    got, _ = oz(tp, ex, torch_cuda, "float64", A, B, None, D, 1.0, 0.0)
    G = got.reshape(5, 8).T
    assert np.all(np.isnan(G[3])) and np.all(np.isfinite(np.delete(G, 3, axis=0)))


def test_ozaki_batch_innermost_conjugated_c3_layout(tp, ex, torch_cuda, orc):
    """Config-3 layout at reduced size: D[b,i,j] = sum_k conj(A[b,k,i]) B[b,k,j],
    c64, column-major in the listed order (batch stride 1 in every operand)."""
    rng = np.random.default_rng(43)
    dt, b, n = "complex128", 48, 96
    ext = [b, n, n]
    st = [1, b, b * n]
    A = Op(rnd(rng, dt, b * n * n), ext, st, [0, 3, 1], conj=True)
    B = Op(rnd(rng, dt, b * n * n), ext, st, [0, 3, 2])
    d0 = np.zeros(b * n * n, dtype=dt)
    D = Op(d0, ext, st, [0, 1, 2])
    want = oracle_ref(orc, dt, A, B, None, D, 1.0, 0.0, d0)
    got, p = oz(tp, ex, torch_cuda, dt, A, B, None, D, 1.0, 0.0)
    assert orc.rel_frobenius(got, want) <= 1e-12, p.report()


@pytest.mark.parametrize("dt,k", [("float64", 37), ("complex128", 37), ("float64", 900), ("complex128", 450)],
                         ids=["f64-k37", "c64-k37", "f64-k900-two-pass", "c64-k450-two-pass"])
def test_ozaki_batch_innermost_depths(tp, ex, torch_cuda, orc, dt, k):
    """Batch-innermost operands (h = 35 entries, stride 1) at a depth that is
    not a multiple of four (one pass over the operand: the whole depth of 16
    batch entries in shared memory) and at depths past that kernel's shared
    memory bound (the exponent scan and the slicing as two passes)."""
    rng = np.random.default_rng(47 + k)
    h, m, n = 35, 23, 19
    A = Op(rnd(rng, dt, h * k * m), [h, k, m], [1, h, h * k], [9, 2, 0], conj=dt == "complex128")
    B = Op(rnd(rng, dt, h * k * n), [h, k, n], [1, h, h * k], [9, 2, 1])
    d0 = np.zeros(h * m * n, dtype=dt)
    D = Op(d0, [h, m, n], [1, h, h * m], [9, 0, 1])
    want = oracle_ref(orc, dt, A, B, None, D, 1.0, 0.0, d0)
    got, p = oz(tp, ex, torch_cuda, dt, A, B, None, D, 1.0, 0.0)
    assert orc.rel_frobenius(got, want) <= 1e-12, p.report()


@pytest.mark.parametrize("dt", ["float64", "complex128"])
def test_ozaki_batch_innermost_non_finite(tp, ex, torch_cuda, orc, dt):
    """A NaN in one batch entry of one row of a batch-innermost A gives NaN in
    that entry's output row only."""
    rng = np.random.default_rng(49)
    h, m, n, k = 40, 9, 7, 30
    a = rnd(rng, dt, h * k * m)
    a[5 + h * 11 + h * k * 4] = np.nan  # batch 5, k 11, row 4
    A = Op(a, [h, k, m], [1, h, h * k], [9, 2, 0])
    B = Op(rnd(rng, dt, h * k * n), [h, k, n], [1, h, h * k], [9, 2, 1])
    D = Op(np.zeros(h * m * n, dtype=dt), [h, m, n], [1, h, h * m], [9, 0, 1])
    got, _ = oz(tp, ex, torch_cuda, dt, A, B, None, D, 1.0, 0.0)
    G = got.reshape(n, m, h)  # [j, i, b]
    bad = np.isnan(G.real) | np.isnan(G.imag) if dt == "complex128" else np.isnan(G)
    assert np.all(bad[:, 4, 5])
    bad[:, 4, 5] = False
    assert not np.any(bad)


@pytest.mark.parametrize("dt", ["float64", "complex128"])
def test_ozaki_extreme_digits(tp, ex, torch_cuda, orc, dt):
    # Entries at the top of their row's range, (1 - 2^-53) 2^p, round to
    # T = 2^(8S-2): the top digit at its bound (64) over all-zero low digits.
    # Exact powers of two, their negations and values one unit of the last
    # slice apart exercise the digit -128 and its negation in the complex
    # embedding (-Im A).
    rng = np.random.default_rng(46)
    m, n, k = 40, 24, 64
    top = 1.0 - 2.0 ** -53
    a = rng.choice([top, -top, 0.5, -0.5, 0.5 + 2.0 ** -47, -(0.5 + 2.0 ** -46), 2.0 ** -30], size=m * k)
    a = a * np.repeat(2.0 ** rng.integers(-20, 20, size=m), k).reshape(m, k).T.reshape(-1)
    b = rng.choice([top, -top, 0.25, -0.75, 2.0 ** -40], size=k * n)
    if dt == "complex128":
        a = a + 1j * np.roll(a, 3)
        b = b - 1j * np.roll(b, 5)
    A = Op(a.astype(dt), [m, k], [1, m], [0, 2], conj=dt == "complex128")
    B = Op(b.astype(dt), [k, n], [1, k], [2, 1])
    d0 = np.zeros(m * n, dtype=dt)
    D = Op(d0, [m, n], [1, m], [0, 1])
    want = oracle_ref(orc, dt, A, B, None, D, 1.0, 0.0, d0)
    got, p = oz(tp, ex, torch_cuda, dt, A, B, None, D, 1.0, 0.0)
    assert ".s6." in p.report()["family"], p.report()["family"]
    assert orc.rel_frobenius(got, want) <= 1e-12
