"""The CPU oracle pinned against the reference's known answers, and its two
implementations (brute-force label oracle, restated packed driver) checked
against each other on the reference's semantic cases: every conjugation mask,
diagonals on inputs and on the output, reductions, batch indices, a rank-0
output, several KC slabs, negative strides, alpha == 0 and beta == 0 with a
poisoned C."""
import json
import os

import numpy as np
import pytest

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))
DTYPES = ["float32", "float64", "complex64", "complex128"]


def tol(dt):
    # crates/tprims-capi/tests/common/mod.rs:57-63
    return 2e-4 if dt in ("float32", "complex64") else 1e-11


def _mk(dt, vals):
    vals = [complex(*v) if isinstance(v, list) else v for v in vals]
    if not dt.startswith("complex"):
        vals = [complex(v).real for v in vals]
    return np.array(vals).astype(dt)


@pytest.mark.parametrize("name", sorted(GOLD["cases"]))
@pytest.mark.parametrize("impl", ["label", "packed"])
def test_known_answers(orc, name, impl):
    case = GOLD["cases"][name]
    for dt in case["dtypes"]:
        cplx = dt.startswith("complex")
        a = _mk(dt, case["a"].get("data", case["a"].get("data_c")))
        b = _mk(dt, case["b"].get("data", case["b"].get("data_c")))
        n = int(np.prod(case["d"]["ext"]))
        d = np.full(n, -1, dtype=dt)
        A = orc.View(a, case["a"]["ext"], case["a"]["str"], case["a"]["lab"])
        B = orc.View(b, case["b"]["ext"], case["b"]["str"], case["b"]["lab"])
        D = orc.View(d, case["d"]["ext"], case["d"]["str"], case["d"]["lab"])
        fn = orc.label_contract if impl == "label" else orc.packed_contract
        fn(complex(*case["alpha"]), A, B, complex(*case["beta"]), None, D)
        want = case.get("want") or (case["want_complex"] if cplx else case["want_real"])
        want = np.array([complex(*w) if cplx else w[0] for w in want]).astype(dt)
        assert np.array_equal(d, want), (name, dt, d, want)


def test_seq_generator_is_the_reference_sequence():
    # Values are multiples of 1/2048 in [-1, 1) (common/mod.rs:65-71).
    for re, im in GOLD["seq"]["seed_1_real_8"]:
        assert -1 <= re < 1 and (re * 2048) == int(re * 2048) and im == 0


def _layout(ext, rng, permute=True):
    order = rng.permutation(len(ext)) if permute else np.arange(len(ext))
    st = [0] * len(ext)
    acc = 1
    for p in order:
        st[p] = acc
        acc *= max(ext[p], 1)
    return list(ext), st, max(acc, 1)


CASES = [
    # (labels A, labels B, labels D, extents)
    ([0, 2], [2, 1], [0, 1], {0: 5, 1: 4, 2: 3}),  # case 1
    ([7, 0, 2], [2, 1], [0, 1, 7], {0: 4, 1: 5, 2: 3, 7: 2}),  # general strides
    ([3, 0, 2], [3, 2, 1], [3, 0, 1], {0: 4, 1: 5, 2: 3, 3: 2}),  # case 2: batch
    ([0, 0], [0, 1], [1], {0: 4, 1: 5}),  # case 3: diagonal in A
    ([0, 0, 0], [0, 1], [1], {0: 4, 1: 5}),  # label repeated three times
    ([0, 2], [2], [0, 0], {0: 4, 2: 3}),  # diagonal in the output
    ([0, 2, 9], [2, 1], [0, 1], {0: 4, 1: 5, 2: 3, 9: 2}),  # case 4: reduction in A
    ([0, 2], [2, 1, 9], [0, 1], {0: 4, 1: 5, 2: 3, 9: 2}),  # reduction in B
    ([0, 1], [0, 1], [], {0: 4, 1: 3}),  # full reduction, rank-0 D
    ([0, 2], [2, 1], [0, 1], {0: 3, 1: 2, 2: 600}),  # several KC slabs
]


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_label_and_packed_oracles_agree(orc, dt, ci):
    rng = np.random.default_rng(1000 + ci)
    la, lb, ld, E = CASES[ci]
    cplx = dt.startswith("complex")

    def rnd(n):
        x = rng.uniform(-1, 1, n)
        if cplx:
            x = x + 1j * rng.uniform(-1, 1, n)
        return x.astype(dt)

    for mask in range(16):
        ea, sa, na = _layout([E[l] for l in la], rng)
        eb, sb, nb = _layout([E[l] for l in lb], rng)
        ed, sd, nd = _layout([E[l] for l in ld], rng)
        a, b, c = rnd(na), rnd(nb), rnd(nd)
        d1 = rnd(nd)
        d2 = d1.copy()
        al, be = complex(0.5, -0.25), complex(-2, 0.75)
        A = orc.View(a, ea, sa, la, conj=bool(mask & 1))
        B = orc.View(b, eb, sb, lb, conj=bool(mask & 2))
        Cv = orc.View(c, ed, sd, ld, conj=bool(mask & 4))
        orc.label_contract(al, A, B, be, Cv, orc.View(d1, ed, sd, ld, conj=bool(mask & 8)))
        orc.packed_contract(al, A, B, be, Cv, orc.View(d2, ed, sd, ld, conj=bool(mask & 8)))
        assert orc.rel_frobenius(d2, d1) <= tol(dt), (mask,)


@pytest.mark.parametrize("dt", DTYPES)
def test_beta_zero_never_reads_c_and_alpha_zero_never_reads_ab(orc, dt):
    # tapp_conformance.rs:491-537 and c_modes.rs:340-383
    rng = np.random.default_rng(7)
    a = rng.uniform(-1, 1, 12).astype(dt)
    b = rng.uniform(-1, 1, 15).astype(dt)
    poison_c = np.full(20, np.nan, dtype=dt)
    for impl in (orc.label_contract, orc.packed_contract):
        d = np.zeros(20, dtype=dt)
        impl(1.0, orc.View(a, [4, 3], [1, 4], [0, 2]), orc.View(b, [3, 5], [1, 3], [2, 1]), 0.0,
             orc.View(poison_c, [4, 5], [1, 4], [0, 1]), orc.View(d, [4, 5], [1, 4], [0, 1]))
        assert np.all(np.isfinite(d))
        if impl is orc.label_contract:
            continue  # the brute-force oracle (like oracle.rs:178) always forms alpha * acc
        c = rng.uniform(-1, 1, 20).astype(dt)
        nan_a = np.full(12, np.nan, dtype=dt)
        impl(0.0, orc.View(nan_a, [4, 3], [1, 4], [0, 2]), orc.View(b, [3, 5], [1, 3], [2, 1]), 1.0,
             orc.View(c, [4, 5], [1, 4], [0, 1]), orc.View(d, [4, 5], [1, 4], [0, 1]))
        assert np.array_equal(d, c)


def test_negative_strides(orc):
    # tapp_conformance.rs:319-390: reversing A's rows and negating the row stride is the identity.
    rng = np.random.default_rng(3)
    a = rng.uniform(-1, 1, (3, 5)).T.copy(order="F")  # 5x3 column-major
    b = rng.uniform(-1, 1, 12)
    rev = a[::-1, :].copy(order="F")
    d1 = np.zeros(20)
    d2 = np.zeros(20)
    buf = rev.ravel(order="F")
    orc.packed_contract(1.0, orc.View(a.ravel(order="F"), [5, 3], [1, 5], [0, 2]), orc.View(b, [3, 4], [4, 1], [2, 1]),
                        0.0, None, orc.View(d1, [5, 4], [1, 5], [0, 1]))
    orc.packed_contract(1.0, orc.View(buf, [5, 3], [-1, 5], [0, 2], offset=4), orc.View(b, [3, 4], [4, 1], [2, 1]),
                        0.0, None, orc.View(d2, [5, 4], [1, 5], [0, 1]))
    assert np.allclose(d1, d2, rtol=0, atol=1e-14)
