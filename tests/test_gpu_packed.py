"""The packed plain families on a B200, through the C ABI: the pack pass
(operands gathered through their scatter vectors into dense panels) and the
TMA-fed tiles over the panels: FP32 FFMA (f32; c32 as the 1m real embedding)
and FP64 DMMA (f64; c64 as 3m, three real products per complex MAC).

Against the extended-precision label oracle at the plain bounds (relative
Frobenius f32 / c32 <= 1e-6, f64 / c64 <= 1e-13), on ragged shapes, both
operand orders (k or the free index unit-stride), batches, every conjugation
mask, alpha / beta with C, split-K, and shapes where the model picks them."""
import numpy as np
import pytest

from test_gpu_parity import Op, make_product, oracle_ref, plain_tol, rnd, run

pytestmark = pytest.mark.gpu

PACKED = {"float32": 10, "complex64": 11, "float64": 12, "complex128": 13}
HALF = {"float32": 14, "complex64": 15}  # the half-width FFMA tiles
DTYPES = list(PACKED)


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


@pytest.mark.parametrize("dt", DTYPES)
def test_packed_family_on_ragged_shapes(tp, ex, torch_cuda, orc, dt):
    rng = np.random.default_rng(61)
    for (m, n, k, kfast) in [(1, 1, 1, True), (7, 13, 5, False), (65, 33, 17, True), (130, 257, 70, False),
                             (200, 129, 300, True), (129, 200, 33, False)]:
        if kfast:
            A = Op(rnd(rng, dt, m * k), [m, k], [k, 1], [0, 2])
            B = Op(rnd(rng, dt, k * n), [k, n], [1, k], [2, 1])
        else:
            A = Op(rnd(rng, dt, m * k), [m, k], [1, m], [0, 2])
            B = Op(rnd(rng, dt, k * n), [k, n], [n, 1], [2, 1])
        d0 = np.zeros(m * n, dtype=dt)
        D = Op(d0, [m, n], [1, m], [0, 1])
        want = oracle_ref(orc, dt, A, B, None, D, 1.0, 0.0, d0)
        st, got, p = run(tp, ex, torch_cuda, dt, A, B, None, D, 1.0, 0.0, kernel=PACKED[dt])
        assert st == 0, tp.last_error()
        assert p.report()["family"].startswith("sm100") and "tma" in p.report()["family"]
        assert orc.rel_frobenius(got, want) <= plain_tol(dt), (m, n, k, kfast)


@pytest.mark.parametrize("dt", list(HALF))
def test_half_width_ffma_tiles(tp, ex, torch_cuda, orc, dt):
    """The 128 x 64 FFMA tiles (f32; c32 as 1m): ragged shapes of both operand
    orders, conjugated A for c32, alpha / beta with C, and a split K."""
    rng = np.random.default_rng(65)
    for (m, n, k, kfast) in [(1, 1, 1, True), (65, 33, 17, False), (200, 129, 300, True), (129, 200, 33, False)]:
        if kfast:
            A = Op(rnd(rng, dt, m * k), [m, k], [k, 1], [0, 2], conj=dt == "complex64")
            B = Op(rnd(rng, dt, k * n), [k, n], [1, k], [2, 1])
        else:
            A = Op(rnd(rng, dt, m * k), [m, k], [1, m], [0, 2])
            B = Op(rnd(rng, dt, k * n), [k, n], [n, 1], [2, 1], conj=dt == "complex64")
        C = Op(rnd(rng, dt, m * n), [m, n], [1, m], [0, 1])
        d0 = np.zeros(m * n, dtype=dt)
        D = Op(d0, [m, n], [1, m], [0, 1])
        al, be = (complex(0.5, -0.25), complex(-1.5, 0.5)) if dt.startswith("complex") else (0.75, -1.5)
        want = oracle_ref(orc, dt, A, B, C, D, al, be, d0)
        st, got, p = run(tp, ex, torch_cuda, dt, A, B, C, D, al, be, kernel=HALF[dt])
        assert st == 0, tp.last_error()
        assert "x64x32" in p.report()["family"], p.report()["family"]
        assert orc.rel_frobenius(got, want) <= plain_tol(dt), (m, n, k, kfast)
    m, n, k = 96, 80, 1500
    A = Op(rnd(rng, dt, m * k), [m, k], [1, m], [0, 2])
    B = Op(rnd(rng, dt, k * n), [k, n], [1, k], [2, 1])
    d0 = np.zeros(m * n, dtype=dt)
    D = Op(d0, [m, n], [1, m], [0, 1])
    want = oracle_ref(orc, dt, A, B, None, D, 1.0, 0.0, d0)
    p = make_product(tp, dt, A, B, None, D)
    p.set_kernel(HALF[dt])
    p.set_split_k(3)
    torch = torch_cuda
    ta, tb = (torch.from_numpy(x.buf.copy()).cuda() for x in (A, B))
    td = torch.from_numpy(d0.copy()).cuda()
    assert p.execute(ex, 1.0, ta.data_ptr(), tb.data_ptr(), 0.0, None, td.data_ptr()) == 0, tp.last_error()
    torch.cuda.synchronize()
    assert p.report().get("split_k", 1) == 3
    assert orc.rel_frobenius(td.cpu().numpy(), want) <= plain_tol(dt)


@pytest.mark.parametrize("dt", DTYPES)
def test_packed_batched_general_strides_alpha_beta(tp, ex, torch_cuda, orc, dt):
    """A batch index, permuted modes on every operand, alpha and beta with a C
    of its own layout, and D with a leading dimension larger than M."""
    rng = np.random.default_rng(62)
    h, m, n, k = 3, 70, 45, 100
    A = Op(rnd(rng, dt, h * m * k), [h, k, m], [1, h, h * k], [9, 2, 0])
    B = Op(rnd(rng, dt, h * k * n), [h, n, k], [1, h * k, h], [9, 1, 2])
    C = Op(rnd(rng, dt, h * m * n), [h, m, n], [m * n, 1, m], [9, 0, 1])
    ld = m + 3
    d0 = np.zeros(h * ld * n, dtype=dt)
    D = Op(d0, [h, m, n], [ld * n, 1, ld], [9, 0, 1])
    al, be = (complex(0.5, -0.25), complex(-1.5, 0.5)) if dt.startswith("complex") else (0.75, -1.5)
    want = oracle_ref(orc, dt, A, B, C, D, al, be, d0)
    st, got, _ = run(tp, ex, torch_cuda, dt, A, B, C, D, al, be, kernel=PACKED[dt])
    assert st == 0, tp.last_error()
    assert orc.rel_frobenius(got, want) <= plain_tol(dt)
    gap = got.reshape(h, n, ld)[:, :, m:]
    assert np.all(gap == 0), "a write landed between the columns of D"


@pytest.mark.parametrize("dt", ["complex64", "complex128"])
@pytest.mark.parametrize("mask", range(16))
def test_packed_complex_every_conjugation(tp, ex, torch_cuda, orc, dt, mask):
    """1m (c32) and 3m (c64) with each of A, B, C, D conjugated or not: the
    conjugation of A and B is folded into the packed planes' signs."""
    rng = np.random.default_rng(900 + mask)
    A = Op(rnd(rng, dt, 40 * 19), [40, 19], [1, 40], [0, 2], conj=bool(mask & 1))
    B = Op(rnd(rng, dt, 19 * 23), [19, 23], [23, 1], [2, 1], conj=bool(mask & 2))
    C = Op(rnd(rng, dt, 40 * 23), [40, 23], [1, 40], [0, 1], conj=bool(mask & 4))
    d0 = np.zeros(40 * 23, dtype=dt)
    D = Op(d0, [40, 23], [1, 40], [0, 1], conj=bool(mask & 8))
    al, be = complex(1.25, -0.5), complex(0.75, 0.5)
    want = oracle_ref(orc, dt, A, B, C, D, al, be, d0)
    st, got, _ = run(tp, ex, torch_cuda, dt, A, B, C, D, al, be, kernel=PACKED[dt])
    assert st == 0, tp.last_error()
    assert orc.rel_frobenius(got, want) <= plain_tol(dt)


@pytest.mark.parametrize("dt", DTYPES)
def test_packed_split_k(tp, ex, torch_cuda, orc, dt):
    """A deep contraction with few output tiles, split along K into 3 chunks
    whose partials the reduce kernel adds in order."""
    rng = np.random.default_rng(63)
    m, n, k = 96, 80, 1500
    A = Op(rnd(rng, dt, m * k), [m, k], [1, m], [0, 2])
    B = Op(rnd(rng, dt, k * n), [k, n], [1, k], [2, 1])
    C = Op(rnd(rng, dt, m * n), [m, n], [1, m], [0, 1])
    d0 = np.zeros(m * n, dtype=dt)
    D = Op(d0, [m, n], [1, m], [0, 1])
    want = oracle_ref(orc, dt, A, B, C, D, 1.0, 0.5, d0)
    p = make_product(tp, dt, A, B, C, D)
    p.set_kernel(PACKED[dt])
    p.set_split_k(3)
    torch = torch_cuda
    ta, tb, tc = (torch.from_numpy(x.buf.copy()).cuda() for x in (A, B, C))
    td = torch.from_numpy(d0.copy()).cuda()
    assert p.execute(ex, 1.0, ta.data_ptr(), tb.data_ptr(), 0.5, tc.data_ptr(), td.data_ptr()) == 0, tp.last_error()
    torch.cuda.synchronize()
    rep = p.report()
    assert rep.get("split_k", 1) == 3, rep
    assert orc.rel_frobenius(td.cpu().numpy(), want) <= plain_tol(dt)


@pytest.mark.parametrize("dt", DTYPES)
def test_model_picks_the_packed_family_for_large_shapes(tp, ex, torch_cuda, orc, dt):
    """A contraction with more than a wave of packed tiles: the model's choice
    is the packed family, checked against float64 products at 256 sampled
    outputs (the full oracle would take long on the CPU)."""
    torch = torch_cuda
    n = 2048 if dt in ("float32", "complex64") else 1024
    code = {"float32": tp.F32, "float64": tp.F64, "complex64": tp.C32, "complex128": tp.C64}[dt]
    tdt = getattr(torch, dt)
    g = torch.Generator(device="cuda").manual_seed(64)
    A = torch.randn(n * n, dtype=tdt, device="cuda", generator=g)
    B = torch.randn(n * n, dtype=tdt, device="cuda", generator=g)
    D = torch.zeros(n * n, dtype=tdt, device="cuda")
    lay = tp.LayoutSpec([n, n], [1, n])
    plan = tp.Plan(tp.Problem.from_labels(code, tp.OperandSpec(lay, dt.startswith("complex")), tp.OperandSpec(lay),
                                          tp.OperandSpec(lay), [2, 0], [2, 1], [0, 1]))
    plan.execute_into(ex, 1.0, A.data_ptr(), B.data_ptr(), D.data_ptr())
    torch.cuda.synchronize()
    assert ".tma." in plan.report()["family"], plan.report()
    wide = torch.complex128 if dt.startswith("complex") else torch.float64
    Am = A.view(n, n).to(wide)  # Am[m, k] = A[k + n m] : A[k, m] column-major
    Bm = B.view(n, n).to(wide)  # Bm[n', k] = B[k, n']
    if dt.startswith("complex"):
        Am = Am.conj()
    rs = torch.from_numpy(np.random.default_rng(1).integers(0, n, size=(256, 2))).cuda()
    ref = (Am[rs[:, 0]] * Bm[rs[:, 1]]).sum(dim=1)
    got = D.view(n, n).T.to(wide)[rs[:, 0], rs[:, 1]]  # D[m, n'] column-major
    err = float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref))
    assert err <= plain_tol(dt), err
