"""Parity of the CUDA path with the oracle, through the C ABI (TAPP_execute_product
and the B200 extensions), on a B200.

Tolerances (relative Frobenius against the extended-precision label oracle):
plain f32 / c32 <= 1e-6 and plain f64 / c64 <= 1e-13 (the stated targets of the
plain path); bf16x6 <= 1e-6, bf16x3 <= 2e-5 (their stated bounds). Cases mirror
the reference's C-ABI conformance suite (crates/tprims-capi/tests/
tapp_conformance.rs) and its driver sweep (driver/tests/correctness.rs)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))
DTYPES = ["float32", "float64", "complex64", "complex128"]
TAPP_DT = {"float32": 0, "float64": 1, "complex64": 2, "complex128": 3}


def plain_tol(dt):
    return 1e-6 if dt in ("float32", "complex64") else 1e-13


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "the -m gpu tests need a CUDA device"
    torch.cuda.init()
    return torch


@pytest.fixture(scope="module")
def ex(tp, torch_cuda):
    e = tp.Executor()
    yield e
    e.close()


class Op:
    """An operand: backing array + layout + labels (origin at element `offset`)."""

    def __init__(self, buf, ext, st, lab, offset=0, conj=False):
        self.buf, self.ext, self.st, self.lab, self.offset, self.conj = buf, list(ext), list(st), list(lab), offset, conj

    def view(self, orc, buf=None):
        return orc.View(self.buf if buf is None else buf, self.ext, self.st, self.lab, self.offset, self.conj)


def make_product(tp, dt, A, B, C, D):
    h = tp.Handle()
    ops = [A, B, C if C is not None else D, D]
    infos = [tp.TensorInfo(TAPP_DT[dt], o.ext, o.st) for o in ops]
    p = tp.TensorProduct.create(h, *[(1 if o.conj else 0, i, o.lab) for o, i in zip(ops, infos)])
    p._keep = (h, infos)
    return p


def run(tp, ex, torch, dt, A, B, C, D, alpha, beta, device=True, precision=0, kernel=0, d_init=None):
    """Execute through TAPP_execute_product; returns (status, D buffer after)."""
    p = make_product(tp, dt, A, B, C, D)
    if precision:
        p.set_precision(precision)
    if kernel:
        p.set_kernel(kernel)
    dbuf = (D.buf if d_init is None else d_init).copy()
    if not device:
        ptr = lambda o, b: b.ctypes.data + o.offset * b.itemsize
        st = p.execute(ex, alpha, ptr(A, A.buf), ptr(B, B.buf), beta,
                       None if C is None else ptr(C, C.buf), ptr(D, dbuf))
        return st, dbuf, p
    tens = {}

    def dptr(o, b, key):
        t = torch.from_numpy(b.copy()).cuda()
        tens[key] = t
        return t.data_ptr() + o.offset * b.itemsize

    pa, pb = dptr(A, A.buf, "a"), dptr(B, B.buf, "b")
    pd = dptr(D, dbuf, "d")
    pc = None if C is None else (pd if C.buf is D.buf else dptr(C, C.buf, "c"))
    st = p.execute(ex, alpha, pa, pb, beta, pc, pd)
    torch.cuda.synchronize()
    return st, tens["d"].cpu().numpy(), p


def rnd(rng, dt, n):
    x = rng.uniform(-1, 1, n)
    if dt.startswith("complex"):
        x = x + 1j * rng.uniform(-1, 1, n)
    return x.astype(dt)


def layout(ext, rng, permute=True):
    order = rng.permutation(len(ext)) if permute else np.arange(len(ext))
    st = [0] * len(ext)
    acc = 1
    for p in order:
        st[p] = acc
        acc *= max(ext[p], 1)
    return list(ext), st, max(acc, 1)


def oracle_ref(orc, dt, A, B, C, D, alpha, beta, d_init):
    """The label oracle's result in float64 / complex128 (extended accumulation)."""
    wide = "complex128" if dt.startswith("complex") else "float64"
    out = d_init.astype(wide)
    orc.label_contract(alpha, A.view(orc), B.view(orc), beta, None if C is None else C.view(orc),
                       D.view(orc, out), out_f64=True)
    return out


# ----------------------------------------------------------------- known answers
@pytest.mark.parametrize("name", sorted(GOLD["cases"]))
@pytest.mark.parametrize("device", [True, False], ids=["device", "host"])
def test_known_answers_exact(tp, ex, torch_cuda, name, device):
    case = GOLD["cases"][name]
    for dt in case["dtypes"]:
        cplx = dt.startswith("complex")
        vals = lambda v: np.array([complex(*x) if isinstance(x, list) else x for x in v]).astype(
            dt if cplx else "complex128").real.astype(dt) if not cplx else np.array(
            [complex(*x) if isinstance(x, list) else x for x in v]).astype(dt)
        a = vals(case["a"].get("data", case["a"].get("data_c")))
        b = vals(case["b"].get("data", case["b"].get("data_c")))
        d = np.full(int(np.prod(case["d"]["ext"])), -1, dtype=dt)
        A = Op(a, case["a"]["ext"], case["a"]["str"], case["a"]["lab"])
        B = Op(b, case["b"]["ext"], case["b"]["str"], case["b"]["lab"])
        D = Op(d, case["d"]["ext"], case["d"]["str"], case["d"]["lab"])
        st, got, _ = run(tp, ex, torch_cuda, dt, A, B, None, D, complex(*case["alpha"]), complex(*case["beta"]),
                         device=device)
        assert st == 0, tp.last_error()
        want = case.get("want") or (case["want_complex"] if cplx else case["want_real"])
        want = np.array([complex(*w) if cplx else w[0] for w in want]).astype(dt)
        assert np.array_equal(got, want), (name, dt, got, want)


# ---------------------------------------------------------------- semantic sweep
SWEEP = [
    ([0, 2], [2, 1], [0, 1], {0: 5, 1: 4, 2: 3}),
    ([7, 0, 2], [2, 1], [0, 1, 7], {0: 4, 1: 5, 2: 3, 7: 2}),
    ([3, 0, 2], [3, 2, 1], [3, 0, 1], {0: 4, 1: 5, 2: 3, 3: 2}),
    ([0, 0], [0, 1], [1], {0: 4, 1: 5}),
    ([0, 0, 0], [0, 1], [1], {0: 4, 1: 5}),
    ([0, 2], [2], [0, 0], {0: 4, 2: 3}),
    ([0, 2, 9], [2, 1], [0, 1], {0: 4, 1: 5, 2: 3, 9: 2}),
    ([0, 2], [2, 1, 9], [0, 1], {0: 4, 1: 5, 2: 3, 9: 2}),
    ([0, 1], [0, 1], [], {0: 4, 1: 3}),
    ([0, 2], [2, 1], [0, 1], {0: 3, 1: 2, 2: 600}),
    ([0, 5, 2], [5, 2, 1], [1, 0], {0: 37, 1: 29, 2: 11, 5: 7}),
]


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("ci", range(len(SWEEP)))
def test_semantic_sweep_every_conjugation_mask(tp, ex, torch_cuda, orc, dt, ci):
    rng = np.random.default_rng(2000 + ci)
    la, lb, ld, E = SWEEP[ci]
    for mask in range(16):
        ea, sa, na = layout([E[l] for l in la], rng)
        eb, sb, nb = layout([E[l] for l in lb], rng)
        ed, sd, nd = layout([E[l] for l in ld], rng)
        A = Op(rnd(rng, dt, na), ea, sa, la, conj=bool(mask & 1))
        B = Op(rnd(rng, dt, nb), eb, sb, lb, conj=bool(mask & 2))
        C = Op(rnd(rng, dt, nd), ed, sd, ld, conj=bool(mask & 4))
        d0 = rnd(rng, dt, nd)
        D = Op(d0, ed, sd, ld, conj=bool(mask & 8))
        al, be = complex(0.5, -0.25), complex(-2, 0.75)
        st, got, _ = run(tp, ex, torch_cuda, dt, A, B, C, D, al, be, device=(mask % 2 == 0))
        assert st == 0, tp.last_error()
        want = oracle_ref(orc, dt, A, B, C, D, al, be, d0)
        err = orc.rel_frobenius(got, want)
        assert err <= plain_tol(dt), (mask, err)


@pytest.mark.parametrize("dt", DTYPES)
def test_beta_zero_never_reads_c_alpha_zero_never_reads_ab(tp, ex, torch_cuda, dt):
    rng = np.random.default_rng(5)
    A = Op(rnd(rng, dt, 12), [4, 3], [1, 4], [0, 2])
    B = Op(rnd(rng, dt, 15), [3, 5], [1, 3], [2, 1])
    D = Op(np.zeros(20, dtype=dt), [4, 5], [1, 4], [0, 1])
    poison = Op(np.full(20, np.nan, dtype=dt), [4, 5], [1, 4], [0, 1])
    st, got, _ = run(tp, ex, torch_cuda, dt, A, B, poison, D, 1.0, 0.0)
    assert st == 0 and np.all(np.isfinite(got))
    c = Op(rnd(rng, dt, 20), [4, 5], [1, 4], [0, 1])
    nanA = Op(np.full(12, np.nan, dtype=dt), [4, 3], [1, 4], [0, 2])
    st, got, _ = run(tp, ex, torch_cuda, dt, nanA, B, c, D, 0.0, 1.0)
    assert st == 0 and np.array_equal(got, c.buf)


@pytest.mark.parametrize("dt", DTYPES)
def test_null_c_with_nonzero_beta_leaves_d_alone(tp, ex, torch_cuda, dt):
    rng = np.random.default_rng(6)
    A = Op(rnd(rng, dt, 12), [4, 3], [1, 4], [0, 2])
    B = Op(rnd(rng, dt, 15), [3, 5], [1, 3], [2, 1])
    before = rnd(rng, dt, 20)
    D = Op(before, [4, 5], [1, 4], [0, 1])
    st, got, _ = run(tp, ex, torch_cuda, dt, A, B, None, D, 1.0, 1.0)
    assert st == tp.ERR_UNSUPPORTED and np.array_equal(got, before)


@pytest.mark.parametrize("dt", DTYPES)
def test_accumulate_in_place_across_kc_depths(tp, ex, torch_cuda, orc, dt):
    rng = np.random.default_rng(7)
    for kk in (3, 600):
        A = Op(rnd(rng, dt, 3 * kk), [3, kk], [1, 3], [0, 2])
        B = Op(rnd(rng, dt, kk * 2), [kk, 2], [1, kk], [2, 1])
        d0 = rnd(rng, dt, 6)
        D = Op(d0, [3, 2], [1, 3], [0, 1])
        st, got, _ = run(tp, ex, torch_cuda, dt, A, B, D, D, 1.25, complex(3, -1))
        assert st == 0, tp.last_error()
        want = oracle_ref(orc, dt, A, B, Op(d0, [3, 2], [1, 3], [0, 1]), D, 1.25, complex(3, -1), d0)
        assert orc.rel_frobenius(got, want) <= plain_tol(dt)


@pytest.mark.parametrize("dt", DTYPES)
def test_c_with_a_different_layout(tp, ex, torch_cuda, orc, dt):
    rng = np.random.default_rng(8)
    A = Op(rnd(rng, dt, 12), [4, 3], [1, 4], [0, 2])
    B = Op(rnd(rng, dt, 15), [3, 5], [1, 3], [2, 1])
    C = Op(rnd(rng, dt, 20), [4, 5], [5, 1], [0, 1])
    d0 = np.zeros(20, dtype=dt)
    D = Op(d0, [4, 5], [1, 4], [0, 1])
    st, got, _ = run(tp, ex, torch_cuda, dt, A, B, C, D, 1.0, complex(1.5, -0.5))
    assert st == 0
    want = oracle_ref(orc, dt, A, B, C, D, 1.0, complex(1.5, -0.5), d0)
    assert orc.rel_frobenius(got, want) <= plain_tol(dt)


def test_negative_strides(tp, ex, torch_cuda):
    rng = np.random.default_rng(9)
    a = rng.uniform(-1, 1, 15)
    M = a.reshape(3, 5).T  # A[i, k] = a[i + 5k]
    rev = M[::-1, :].ravel(order="F").copy()
    B = Op(rng.uniform(-1, 1, 12), [3, 4], [4, 1], [2, 1])
    D = Op(np.zeros(20), [5, 4], [1, 5], [0, 1])
    st1, d1, _ = run(tp, ex, torch_cuda, "float64", Op(a, [5, 3], [1, 5], [0, 2]), B, None, D, 1.0, 0.0)
    st2, d2, _ = run(tp, ex, torch_cuda, "float64", Op(rev, [5, 3], [-1, 5], [0, 2], offset=4), B, None, D, 1.0, 0.0)
    assert st1 == 0 and st2 == 0
    assert np.allclose(d1, d2, rtol=0, atol=1e-14)


def test_batched_product_matches_single_products(tp, ex, torch_cuda):
    rng = np.random.default_rng(10)
    A = Op(np.zeros(12), [4, 3], [1, 4], [0, 2])
    B = Op(np.zeros(15), [3, 5], [1, 3], [2, 1])
    D = Op(np.zeros(20), [4, 5], [1, 4], [0, 1])
    p = make_product(tp, "float64", A, B, None, D)
    As = [rng.uniform(-1, 1, 12) for _ in range(3)]
    Bs = [rng.uniform(-1, 1, 15) for _ in range(3)]
    Ds = [np.zeros(20) for _ in range(3)]
    assert p.execute_batched(ex, 1.0, As, Bs, 0.0, None, Ds) == 0
    for i in range(3):
        d = np.zeros(20)
        assert p.execute(ex, 1.0, As[i], Bs[i], 0.0, None, d) == 0
        assert np.array_equal(d, Ds[i])


# ----------------------------------------------------------- tiles and families
FAMILIES = {"float32": [1, 2], "float64": [3, 4, 8], "complex64": [5], "complex128": [6, 7, 9]}


@pytest.mark.parametrize("dt", DTYPES)
def test_every_family_on_ragged_shapes_and_bitwise_across_tiles(tp, ex, torch_cuda, orc, dt):
    rng = np.random.default_rng(11)
    for (m, n, k) in [(1, 1, 1), (7, 13, 5), (65, 33, 17), (130, 257, 70)]:
        A = Op(rnd(rng, dt, m * k), [m, k], [k, 1], [0, 2])  # k fastest in A
        B = Op(rnd(rng, dt, k * n), [k, n], [1, k], [2, 1])
        d0 = np.zeros(m * n, dtype=dt)
        D = Op(d0, [m, n], [1, m], [0, 1])
        want = oracle_ref(orc, dt, A, B, None, D, 1.0, 0.0, d0)
        outs = []
        for fam in FAMILIES[dt]:
            st, got, _ = run(tp, ex, torch_cuda, dt, A, B, None, D, 1.0, 0.0, kernel=fam)
            assert st == 0, tp.last_error()
            assert orc.rel_frobenius(got, want) <= plain_tol(dt), (m, n, k, fam)
            outs.append(got)
        for o in outs[1:]:
            assert np.array_equal(o, outs[0]), "results differ bitwise across tile sizes"


def test_c1_full_size_f64(tp, ex, torch_cuda, orc):
    """Config 1 at its full size: D[a,b,c,d] = sum_{e,f} A[a,e,b,f] B[f,c,e,d] + 0.5 C."""
    rng = np.random.default_rng(20261203 + 1000 * 1)
    e = 24
    cm = [1, e, e * e, e ** 3]
    A = Op(rng.uniform(-1, 1, e ** 4), [e] * 4, cm, [0, 4, 1, 5])
    B = Op(rng.uniform(-1, 1, e ** 4), [e] * 4, cm, [5, 2, 4, 3])
    C = Op(rng.uniform(-1, 1, e ** 4), [e] * 4, cm, [0, 1, 2, 3])
    d0 = np.zeros(e ** 4)
    D = Op(d0, [e] * 4, cm, [0, 1, 2, 3])
    st, got, _ = run(tp, ex, torch_cuda, "float64", A, B, C, D, 1.0, 0.5)
    assert st == 0
    want = d0.copy()
    orc.packed_contract(1.0, A.view(orc), B.view(orc), 0.5, C.view(orc), D.view(orc, want))
    assert orc.rel_frobenius(got, want) <= 1e-13


# ----------------------------------------------------------------- tiny batches
@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("shape", [(1, 1, 1, (12, 11)), (2, 3, 5, (10, 9)), (4, 1, 16, (70,))],
                         ids=["hadamard", "small", "vecmat"])
def test_tiny_batched_products(tp, ex, torch_cuda, orc, dt, shape):
    """Batches of tiny products (M N K <= 256) take the one-thread-per-output
    kernel: batch axes folded or not (B's two batch axes are transposed, so
    its batch scatter is not a sequence), conjugation, alpha, beta and C."""
    m, n, k, hb = shape
    rng = np.random.default_rng(55)
    cplx = dt.startswith("complex")
    h = int(np.prod(hb))
    hl = list(range(10, 10 + len(hb)))
    # A[batch..., m, k] batch-first; B[k, n, batch reversed]; C, D [m, n, batch...]
    ea = list(hb) + [m, k]
    A = Op(rnd(rng, dt, h * m * k), ea, layout(ea, rng, permute=False)[1], hl + [0, 2], conj=cplx)
    eb = [k, n] + list(reversed(hb))
    B = Op(rnd(rng, dt, h * k * n), eb, layout(eb, rng, permute=False)[1], [2, 1] + list(reversed(hl)))
    ed = [m, n] + list(hb)
    C = Op(rnd(rng, dt, h * m * n), ed, layout(ed, rng, permute=True)[1], [0, 1] + hl)
    d0 = rnd(rng, dt, h * m * n)
    D = Op(d0, ed, layout(ed, rng, permute=False)[1], [0, 1] + hl)
    al, be = (complex(0.5, 0.25), complex(-1.0, 0.5)) if cplx else (1.5, -0.75)
    want = oracle_ref(orc, dt, A, B, C, D, al, be, d0)
    st, got, p = run(tp, ex, torch_cuda, dt, A, B, C, D, al, be)
    assert st == 0, tp.last_error()
    assert "tiny-batched" in p.report()["family"], p.report()
    assert orc.rel_frobenius(got, want) <= plain_tol(dt)


# ----------------------------------------------------------------- split-K
@pytest.mark.parametrize("dt", DTYPES)
def test_split_k_on_deep_contractions_with_few_tiles(tp, ex, torch_cuda, orc, dt):
    """Few output tiles and a deep K: the launch splits K across CTAs, writes
    partial tiles and reduces them in a fixed order before the epilogue (the
    KC-slab accumulation of the reference's driver, spread over SMs). Batch,
    conjugation, beta and a permuted C layout all pass through the reduce."""
    rng = np.random.default_rng(77)
    m, n, k, h = {"float32": (100, 90, 4096, 1), "float64": (70, 65, 3000, 1),
                  "complex64": (50, 60, 2500, 2), "complex128": (40, 33, 2100, 2)}[dt]
    cplx = dt.startswith("complex")
    A = Op(rnd(rng, dt, h * m * k), [k, m, h], [1, k, k * m], [2, 0, 9], conj=cplx)
    B = Op(rnd(rng, dt, h * k * n), [h, n, k], [1, h, h * n], [9, 1, 2])
    C = Op(rnd(rng, dt, h * m * n), [n, h, m], [1, n, n * h], [1, 9, 0])
    d0 = rnd(rng, dt, h * m * n)
    D = Op(d0, [m, n, h], [1, m, m * n], [0, 1, 9])
    al, be = (complex(0.5, -1.0), complex(0.25, 0.75)) if cplx else (1.25, -0.5)
    want = oracle_ref(orc, dt, A, B, C, D, al, be, d0)
    st, got, p = run(tp, ex, torch_cuda, dt, A, B, C, D, al, be)
    assert st == 0, tp.last_error()
    assert p.report()["split_k"] > 1, p.report()
    assert orc.rel_frobenius(got, want) <= plain_tol(dt), (dt, orc.rel_frobenius(got, want))


# ----------------------------------------------------------------- split paths
def _c2_layout(e):
    """Config 2 layout at extent e per mode: A[k1,m1,k2,m2] with a non-unit
    leading stride (2) in a 2x allocation, B[n1,k2,n2,k1] and D[m1,n1,m2,n2]
    column-major."""
    sa = [2, 2 * e, 2 * e * e, 2 * e ** 3]
    cm = [1, e, e * e, e ** 3]
    return sa, cm


@pytest.mark.parametrize("scheme,bound", [(1, 2e-5), (2, 1e-6)], ids=["bf16x3", "bf16x6"])
@pytest.mark.parametrize("e", [6, 16])
def test_split_precision_c2_layout(tp, ex, torch_cuda, orc, scheme, bound, e):
    rng = np.random.default_rng(20261203 + 1000 * 2 + e)
    sa, cm = _c2_layout(e)
    A = Op(rng.standard_normal(2 * e ** 4).astype("float32"), [e] * 4, sa, [10, 0, 11, 1])
    B = Op(rng.standard_normal(e ** 4).astype("float32"), [e] * 4, cm, [2, 11, 3, 10])
    d0 = np.zeros(e ** 4, dtype="float32")
    D = Op(d0, [e] * 4, cm, [0, 2, 1, 3])
    want = oracle_ref(orc, "float32", A, B, None, D, 1.0, 0.0, d0)
    st, got, p = run(tp, ex, torch_cuda, "float32", A, B, None, D, 1.0, 0.0, precision=scheme)
    assert st == 0, tp.last_error()
    assert p.report()["scheme"] in ("bf16x3", "bf16x6")
    err = orc.rel_frobenius(got, want)
    assert err <= bound, err
    st, plain, _ = run(tp, ex, torch_cuda, "float32", A, B, None, D, 1.0, 0.0)
    assert orc.rel_frobenius(plain, want) <= 1e-6


@pytest.mark.parametrize("scheme", [1, 2], ids=["bf16x3", "bf16x6"])
def test_split_precision_ragged_with_beta_and_batch(tp, ex, torch_cuda, orc, scheme):
    rng = np.random.default_rng(31)
    for (m, n, k, h) in [(1, 1, 1, 1), (200, 300, 100, 1), (129, 257, 65, 3)]:
        A = Op(rng.standard_normal(h * m * k).astype("float32"), [h, m, k], [1, h, h * m], [9, 0, 2])
        B = Op(rng.standard_normal(h * k * n).astype("float32"), [h, n, k], [1, h * k, h], [9, 1, 2])
        C = Op(rng.standard_normal(h * m * n).astype("float32"), [h, m, n], [1, h, h * m], [9, 0, 1])
        d0 = np.zeros(h * m * n, dtype="float32")
        D = Op(d0, [h, m, n], [1, h, h * m], [9, 0, 1])
        want = oracle_ref(orc, "float32", A, B, C, D, 0.75, -1.5, d0)
        st, got, _ = run(tp, ex, torch_cuda, "float32", A, B, C, D, 0.75, -1.5, precision=scheme)
        assert st == 0, tp.last_error()
        assert orc.rel_frobenius(got, want) <= (2e-5 if scheme == 1 else 1e-6), (m, n, k, h)


def test_split_precision_full_c2_sampled(tp, ex, torch_cuda):
    """Config 2 at its full size (M = N = K = 4096): bf16x6 and plain FP32 against
    exact float64 dot products at 512 sampled output elements."""
    torch = torch_cuda
    e = 64
    sa, cm = _c2_layout(e)
    g = np.random.default_rng(20261203 + 1000 * 2)
    a = g.standard_normal(2 * e ** 4, dtype=np.float32)
    b = g.standard_normal(e ** 4, dtype=np.float32)
    A = Op(a, [e] * 4, sa, [10, 0, 11, 1])
    B = Op(b, [e] * 4, cm, [2, 11, 3, 10])
    D = Op(np.zeros(e ** 4, dtype="float32"), [e] * 4, cm, [0, 2, 1, 3])
    idx = g.integers(0, e, size=(512, 4))  # m1, m2, n1, n2
    A4 = np.lib.stride_tricks.as_strided(a, (e, e, e, e), [s * 4 for s in sa])  # [k1,m1,k2,m2]
    B4 = b.reshape(e, e, e, e, order="F")  # [n1,k2,n2,k1]
    for scheme, bound in ((2, 1e-6), (0, 1e-6)):
        st, got, _ = run(tp, ex, torch, "float32", A, B, None, D, 1.0, 0.0, precision=scheme)
        assert st == 0, tp.last_error()
        num = den = 0.0
        for m1, m2, n1, n2 in idx:
            ref = np.dot(A4[:, m1, :, m2].astype(np.float64).ravel(), B4[n1, :, n2, :].T.astype(np.float64).ravel())
            val = got[m1 + e * n1 + e * e * m2 + e ** 3 * n2]
            num += (val - ref) ** 2
            den += ref ** 2
        assert (num / den) ** 0.5 <= bound, (scheme, (num / den) ** 0.5)


@pytest.mark.parametrize("scheme,bound", [(1, 2e-5), (2, 1e-6)], ids=["bf16x3", "bf16x6"])
def test_split_precision_tail_split_against_float64(tp, ex, torch_cuda, scheme, bound):
    """160 output tiles on 148 SMs: the 12 tiles of the partial last wave run
    as K halves whose FP32 sums are added by a reduce kernel before the
    epilogue (alpha, beta, a transposed C). Checked at every element against
    float64 products."""
    torch = torch_cuda
    rng = np.random.default_rng(91)
    m, n, k = 2560, 2048, 1024
    a = rng.standard_normal(m * k).astype(np.float32)  # A[k, m], k fastest
    b = rng.standard_normal(k * n).astype(np.float32)  # B[k, n]
    c = rng.standard_normal(m * n).astype(np.float32)  # C[n, m] (transposed)
    A = Op(a, [k, m], [1, k], [2, 0])
    B = Op(b, [k, n], [1, k], [2, 1])
    C = Op(c, [n, m], [1, n], [1, 0])
    D = Op(np.zeros(m * n, dtype=np.float32), [m, n], [1, m], [0, 1])
    st, got, _ = run(tp, ex, torch, "float32", A, B, C, D, 0.75, -0.5, precision=scheme)
    assert st == 0, tp.last_error()
    a2 = a.reshape(m, k).astype(np.float64)  # [m, k]
    b2 = b.reshape(n, k).astype(np.float64)  # [n, k]
    want = 0.75 * a2 @ b2.T - 0.5 * c.reshape(m, n).astype(np.float64)  # C[n, m] stored n fastest
    gotm = got.reshape(n, m).T  # D[m, n], m fastest
    err = np.linalg.norm(gotm - want) / np.linalg.norm(want)
    assert err <= bound, err


# ------------------------------------------------------------ front ends, DLPack
def test_dot_general_execute_into_and_accum(tp, ex, torch_cuda, orc):
    torch = torch_cuda
    a = tp.OperandSpec(tp.LayoutSpec.col_major([3, 5, 4]))
    b = tp.OperandSpec(tp.LayoutSpec.col_major([3, 4, 2]))
    d = tp.OperandSpec(tp.LayoutSpec.col_major([5, 2, 3]))
    plan = tp.Plan(tp.Problem.from_dot_general(tp.F64, a, b, d, tp.DotGeneral([2], [1], [0], [0])))
    g = torch.Generator().manual_seed(0)
    A = torch.rand(3 * 5 * 4, generator=g, dtype=torch.float64).cuda()
    B = torch.rand(3 * 4 * 2, generator=g, dtype=torch.float64).cuda()
    D = torch.zeros(5 * 2 * 3, dtype=torch.float64).cuda()
    plan.execute_into(ex, 1.0, A.data_ptr(), B.data_ptr(), D.data_ptr())
    torch.cuda.synchronize()
    Ah = A.cpu().numpy().reshape(4, 5, 3).transpose(2, 1, 0)  # [b, i, k] col-major
    Bh = B.cpu().numpy().reshape(2, 4, 3).transpose(2, 1, 0)  # [b, k, j]
    want = np.einsum("bik,bkj->ijb", Ah, Bh)
    got = D.cpu().numpy().reshape(3, 2, 5).transpose(2, 1, 0)
    assert np.allclose(got, want, rtol=1e-13, atol=1e-13)
    plan.execute_into_accum(ex, 1.0, A.data_ptr(), B.data_ptr(), 2.0, D.data_ptr())
    torch.cuda.synchronize()
    got2 = D.cpu().numpy().reshape(3, 2, 5).transpose(2, 1, 0)
    assert np.allclose(got2, 3 * want, rtol=1e-13, atol=1e-13)


def test_contract_batched_uneven_items(tp, ex, torch_cuda, orc):
    torch = torch_cuda
    rng = np.random.default_rng(12)
    items, refs = [], []
    for (m, n, k, dt) in [(16, 40, 8, tp.F64), (100, 3, 50, tp.F64), (33, 65, 17, tp.C64)]:
        npdt = "complex128" if dt == tp.C64 else "float64"
        a = rnd(rng, npdt, m * k)
        b = rnd(rng, npdt, k * n)
        ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        td = torch.zeros(m * n, dtype=ta.dtype).cuda()
        A = tp.OperandSpec(tp.LayoutSpec.col_major([m, k]))
        B = tp.OperandSpec(tp.LayoutSpec.col_major([k, n]))
        D = tp.OperandSpec(tp.LayoutSpec.col_major([m, n]))
        plan = tp.Plan(tp.Problem.from_labels(dt, A, B, D, [0, 2], [2, 1], [0, 1]))
        items.append(tp.Item(plan, 1.0, ta.data_ptr(), tb.data_ptr(), td.data_ptr()))
        refs.append((a.reshape(k, m).T @ b.reshape(n, k).T, td, (ta, tb)))
    tp.contract_batched(items, ex)
    torch.cuda.synchronize()
    for want, td, _ in refs:
        got = td.cpu().numpy().reshape(want.shape[1], want.shape[0]).T
        assert np.allclose(got, want, rtol=1e-12, atol=1e-12)


def test_dlpack_execute_with_cuda_tensors(tp, ex, torch_cuda):
    import ctypes as C

    torch = torch_cuda

    class DLDevice(C.Structure):
        _fields_ = [("device_type", C.c_int), ("device_id", C.c_int32)]

    class DLDataType(C.Structure):
        _fields_ = [("code", C.c_uint8), ("bits", C.c_uint8), ("lanes", C.c_uint16)]

    class DLTensor(C.Structure):
        _fields_ = [("data", C.c_void_p), ("device", DLDevice), ("ndim", C.c_int32), ("dtype", DLDataType),
                    ("shape", C.POINTER(C.c_int64)), ("strides", C.POINTER(C.c_int64)), ("byte_offset", C.c_uint64)]

    class Tns(C.Structure):
        _fields_ = [("view", C.POINTER(DLTensor)), ("flags", C.c_uint64)]

    keep = []

    def dl(t):
        sh = (C.c_int64 * t.dim())(*t.shape)
        st = (C.c_int64 * t.dim())(*t.stride())
        x = DLTensor(t.data_ptr(), DLDevice(2, t.device.index or 0), t.dim(), DLDataType(2, 64, 1), sh, st, 0)
        keep.extend([sh, st, x])
        return Tns(C.pointer(x), 0)

    A = torch.randn(6, 4, dtype=torch.float64, device="cuda")
    B = torch.randn(4, 5, dtype=torch.float64, device="cuda")
    D = torch.zeros(6, 5, dtype=torch.float64, device="cuda")
    h = tp.Handle()
    ia = tp.TensorInfo(tp.F64, [6, 4], list(A.stride()))
    ib = tp.TensorInfo(tp.F64, [4, 5], list(B.stride()))
    idd = tp.TensorInfo(tp.F64, [6, 5], list(D.stride()))
    p = tp.TensorProduct.create(h, (0, ia, [0, 2]), (0, ib, [2, 1]), (0, idd, [0, 1]), (0, idd, [0, 1]))
    f = tp.lib.tprims_b200_execute_product_dlpack
    f.argtypes = [C.c_ssize_t, C.c_ssize_t, C.c_void_p, C.c_void_p, Tns, Tns, C.c_void_p, Tns, Tns]
    al, be = tp.scalar_bytes(tp.F64, 1.0), tp.scalar_bytes(tp.F64, 0.0)
    st = f(p.h, ex.h, None, C.cast(al, C.c_void_p), dl(A), dl(B), C.cast(be, C.c_void_p), Tns(None, 0), dl(D))
    assert st == 0, tp.last_error()
    torch.cuda.synchronize()
    assert torch.allclose(D, A @ B, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("prog", ["standard_consumer", "abi_test", "c_consumer"])
def test_reference_c_consumers_run_against_this_library(prog):
    """The reference's own C programs (crates/tprims-capi/tests/c/standard_consumer.c,
    abi_test.c, examples/c-consumer/main.c), built from their sources against the
    reference's headers and linked to libtprims_b200 (oracle/Makefile ref_consumers)."""
    import subprocess

    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", prog)
    if not os.path.exists(exe):
        pytest.skip("reference consumers not built (the reference tree was absent at build time)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.parametrize("dt", ["float32", "complex64"])
def test_contract_batched_single_precision_lists(tp, ex, torch_cuda, dt):
    """Grouped lists of f32 items (SIMT tiles) and c32 items (SIMT tiles fed by
    the cp.async ring, the conjugation variant chosen per tile) of uneven
    extents, against float64 / complex128 sums (plain bound 1e-6)."""
    torch = torch_cuda
    rng = np.random.default_rng(13)
    code = tp.F32 if dt == "float32" else tp.C32
    items, refs = [], []
    for q, (m, n, k) in enumerate([(16, 40, 8), (100, 3, 50), (33, 65, 17), (130, 70, 90), (64, 64, 64),
                                   (7, 200, 33), (257, 129, 40)]):
        conj_a = dt == "complex64" and q % 2 == 1
        a, b = rnd(rng, dt, m * k), rnd(rng, dt, k * n)
        ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        td = torch.zeros(m * n, dtype=ta.dtype, device="cuda")
        plan = tp.Plan(tp.Problem.from_labels(code, tp.OperandSpec(tp.LayoutSpec.col_major([m, k]), conj_a),
                                              tp.OperandSpec(tp.LayoutSpec.col_major([k, n])),
                                              tp.OperandSpec(tp.LayoutSpec.col_major([m, n])), [0, 2], [2, 1], [0, 1]))
        items.append(tp.Item(plan, 1.0, ta.data_ptr(), tb.data_ptr(), td.data_ptr()))
        A = a.astype(np.complex128 if dt == "complex64" else np.float64).reshape(k, m).T
        B = b.astype(A.dtype).reshape(n, k).T
        refs.append(((np.conj(A) if conj_a else A) @ B, td, (ta, tb)))
    tp.contract_batched(items, ex)
    torch.cuda.synchronize()
    for want, td, _ in refs:
        got = td.cpu().numpy().astype(want.dtype).reshape(want.shape[1], want.shape[0]).T
        assert float(np.linalg.norm(got - want) / np.linalg.norm(want)) <= 1e-6
