"""The C ABI without a GPU: the library loads, exports every declared symbol,
and plans (lowering, folding, scatter vectors, orientation) and refuses what
the reference refuses, with the reference's status codes. Nothing here
launches a kernel."""
import json
import os
import re

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = json.load(open(os.path.join(REPO, "tests", "golden", "known_answers.json")))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(REPO, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(REPO, "include", fn)).read()
            names |= set(re.findall(r"(?m)^TPRIMS_B200_EXPORT[^;(]*?\b(\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol(tp):
    decl = declared_symbols()
    assert len(decl) >= 40
    for name in sorted(decl):
        assert hasattr(tp.lib, name), name
    assert set(tp.ABI_SYMBOLS) == decl


def test_header_matches_the_reference_headers_as_the_compiler_sees_them():
    """Every prototype (types after typedefs, parameter names dropped), enum
    value, status code and DLPack struct size of the reference's pinned
    headers (crates/tprims-capi/include/tapp.h, tprims/tprims.h; fixture
    tests/golden/tapp_abi.json by tests/golden/make_abi_golden.py) is the same
    in include/tprims_b200.h, compiled by gcc."""
    import sys

    sys.path.insert(0, os.path.join(REPO, "tests", "golden"))
    from abi_extract import extract

    ref = json.load(open(os.path.join(REPO, "tests", "golden", "tapp_abi.json")))
    hdr = os.path.join(REPO, "include", "tprims_b200.h")
    ours = extract([os.path.join(REPO, "include")], ["tprims_b200.h"], [hdr])
    assert len(ref["prototypes"]) >= 30 and len(ref["values"]) >= 30
    for name, proto in ref["prototypes"].items():
        assert ours["prototypes"].get(name) == proto, (name, proto, ours["prototypes"].get(name))
    for name, value in ref["values"].items():
        assert ours["values"].get(name) == value, (name, value, ours["values"].get(name))


def test_identity_queries(tp):
    assert tp.lib.tprims_abi_version() == 100
    assert tp.lib.tprims_has_part(b"core") == 1 and tp.lib.tprims_has_part(b"tapp") == 1
    assert tp.lib.tprims_has_part(b"blas") == 0 and tp.lib.tprims_has_part(None) == 0
    assert tp.lib.TAPP_implementation_version().decode() == "0.1.0"
    assert tp.lib.TAPP_check_success(0) and not tp.lib.TAPP_check_success(14)
    assert tp.explain(14) == "invalid index labels"


def test_explain_error_truncates_like_snprintf(tp):
    import ctypes as C

    full = tp.lib.TAPP_explain_error(2, 0, None)
    buf = C.create_string_buffer(5)
    assert tp.lib.TAPP_explain_error(2, 5, buf) == full
    assert buf.value == b"inco"


def test_attributes_refuse_every_key(tp):
    import ctypes as C

    v = C.c_void_p(1234)
    assert tp.lib.TAPP_attr_get(1, 0, C.byref(v)) == tp.ERR_UNSUPPORTED and v.value is None
    assert tp.lib.TAPP_attr_set(1, 0, None) == tp.ERR_UNSUPPORTED
    assert tp.lib.TAPP_attr_clear(1, 0) == tp.ERR_UNSUPPORTED


def _product(tp, a, b, d, c=None, prec=-1, dtype=None, ops=(0, 0, 0, 0)):
    dtype = tp.F64 if dtype is None else dtype
    h = tp.Handle()
    infos = [tp.TensorInfo(dtype, x["ext"], x["str"]) for x in (a, b, c or d, d)]
    labs = [a["lab"], b["lab"], (c or d)["lab"], d["lab"]]
    p = tp.TensorProduct.create(h, *[(ops[i], infos[i], labs[i]) for i in range(4)], prec=prec)
    p._keep = (h, infos)
    return p


@pytest.mark.parametrize("name", sorted(GOLD["plans"]))
def test_planner_matches_the_reference_analysis_tests(tp, name):
    case = GOLD["plans"][name]
    p = _product(tp, case["a"], case["b"], case["d"])
    rep = p.report()
    if "mnkb" in case:
        assert [rep["m"], rep["n"], rep["k"], rep["batch"]] == case["mnkb"]
        assert rep["is_pure_gemm"] == case["pure_gemm"]
    if "m_axes" in case:
        assert len(rep["m_axes"]) == case["m_axes"]
    if "vector" in case:
        v = tp.product_scatter(p, case["vector"])
        if "want" in case:
            assert v == case["want"]
        if "want_prefix" in case:
            assert v[: len(case["want_prefix"])] == case["want_prefix"]
        assert rep["k"] == case["k"]


@pytest.mark.parametrize("name", sorted(GOLD["scatters"]))
def test_scatter_vectors(tp, name):
    case = GOLD["scatters"][name]
    # A one-role plan whose M scatter is the vector under test: D[m...] = A[m...,k] B[k].
    ext, st = case["extents"], case["strides"]
    n = len(ext)
    span = 1 + sum((e - 1) * abs(s) for e, s in zip(ext, st))
    a = {"ext": ext + [1], "str": st + [span], "lab": list(range(n)) + [99]}
    b = {"ext": [1], "str": [1], "lab": [99]}
    # D is column-major, so sorting the M axes by |stride in D| keeps the
    # example's fastest-first order and A's strides generate the vector.
    d = {"ext": ext, "str": [int(np.prod(ext[:i])) for i in range(n)], "lab": list(range(n))}
    p = _product(tp, a, b, d)
    assert tp.product_scatter(p, "a_m") == case["want"]


def test_c1_plan_shape(tp):
    # D[a,b,c,d] = sum_{e,f} A[a,e,b,f] B[f,c,e,d], extents 24, column-major.
    cm = lambda n: [24 ** i for i in range(n)]
    A = {"ext": [24] * 4, "str": cm(4), "lab": [0, 4, 1, 5]}
    B = {"ext": [24] * 4, "str": cm(4), "lab": [5, 2, 4, 3]}
    D = {"ext": [24] * 4, "str": cm(4), "lab": [0, 1, 2, 3]}
    rep = _product(tp, A, B, D).report()
    assert (rep["m"], rep["n"], rep["k"], rep["batch"]) == (576, 576, 576, 1)
    assert len(rep["m_axes"]) == 2 and len(rep["k_axes"]) == 2
    assert rep["swapped"] is False and rep["d_mfast"] is True


def test_c2_plan_shape(tp):
    # A[k1,m1,k2,m2] with strides (2,128,8192,524288), B[n1,k2,n2,k1], D[m1,n1,m2,n2] column-major.
    cm = lambda n: [64 ** i for i in range(n)]
    A = {"ext": [64] * 4, "str": [2, 128, 8192, 524288], "lab": [10, 0, 11, 1]}
    B = {"ext": [64] * 4, "str": cm(4), "lab": [2, 11, 3, 10]}
    D = {"ext": [64] * 4, "str": cm(4), "lab": [0, 2, 1, 3]}
    rep = _product(tp, A, B, D, dtype=tp.F32).report()
    assert (rep["m"], rep["n"], rep["k"]) == (4096, 4096, 4096)
    assert rep["a_kfast"] is True and rep["b_kfast"] is False


REJECT = [
    # (description, A, B, D, expected status)
    ("extent mismatch", {"ext": [2, 3], "str": [1, 2], "lab": [0, 2]},
     {"ext": [4, 2], "str": [1, 4], "lab": [2, 1]}, None, 2),
    ("output-only label", None, None, {"ext": [2, 2, 3], "str": [1, 2, 4], "lab": [0, 1, 9]}, 15),
    ("non-injective D", None, None, {"ext": [2, 2], "str": [1, 1], "lab": [0, 1]}, 6),
    ("negative extent", {"ext": [2, -2], "str": [1, 2], "lab": [0, 2]}, None, None, 2),
]


@pytest.mark.parametrize("desc,A,B,D,status", REJECT, ids=[r[0] for r in REJECT])
def test_rejections(tp, desc, A, B, D, status):
    A = A or {"ext": [2, 2], "str": [1, 2], "lab": [0, 2]}
    B = B or {"ext": [2, 2], "str": [1, 2], "lab": [2, 1]}
    D = D or {"ext": [2, 2], "str": [1, 2], "lab": [0, 1]}
    with pytest.raises(tp.TprimsError) as e:
        _product(tp, A, B, D)
    assert e.value.status == status, e.value.message


def test_c_and_d_must_carry_the_same_labels(tp):
    # validate.rs:236-238: OutputLabelMismatch maps to LABELS (abi.rs:100-102).
    with pytest.raises(tp.TprimsError) as e:
        _product(tp, {"ext": [2, 2], "str": [1, 2], "lab": [0, 2]}, {"ext": [2, 2], "str": [1, 2], "lab": [2, 1]},
                 {"ext": [2, 2], "str": [1, 2], "lab": [0, 1]}, c={"ext": [2, 2], "str": [1, 2], "lab": [0, 2]})
    assert e.value.status == tp.ERR_LABELS


def test_mixed_dtypes_and_precisions(tp):
    h = tp.Handle()
    i64 = tp.TensorInfo(tp.F64, [2, 2], [1, 2])
    i32 = tp.TensorInfo(tp.F32, [2, 2], [1, 2])
    L = ([0, 2], [2, 1], [0, 1], [0, 1])
    with pytest.raises(tp.TprimsError) as e:
        tp.TensorProduct.create(h, (0, i64, L[0]), (0, i32, L[1]), (0, i64, L[2]), (0, i64, L[3]))
    assert e.value.status == tp.ERR_DTYPE
    for prec, ok in ((-1, True), (1, True), (0, False), (6, False), (42, False)):
        if ok:
            tp.TensorProduct.create(h, (0, i64, L[0]), (0, i64, L[1]), (0, i64, L[2]), (0, i64, L[3]), prec=prec)
        else:
            with pytest.raises(tp.TprimsError) as e:
                tp.TensorProduct.create(h, (0, i64, L[0]), (0, i64, L[1]), (0, i64, L[2]), (0, i64, L[3]), prec=prec)
            assert e.value.status == tp.ERR_UNSUPPORTED
    with pytest.raises(tp.TprimsError) as e:
        tp.TensorProduct.create(h, (2, i64, L[0]), (0, i64, L[1]), (0, i64, L[2]), (0, i64, L[3]))
    assert e.value.status == tp.ERR_UNSUPPORTED


def test_tensor_info_setters_and_f16_refusal(tp):
    import ctypes as C

    t = tp.TensorInfo(tp.F64, [5, 3], [1, 5])
    assert t.extents() == [5, 3] and t.strides() == [1, 5]
    assert tp.lib.TAPP_set_nmodes(t.h, 3) == 0
    assert t.extents() == [5, 3, 1] and t.strides() == [1, 5, 0]
    ext = (C.c_int64 * 3)(2, 2, 2)
    assert tp.lib.TAPP_set_extents(t.h, ext) == 0 and t.extents() == [2, 2, 2]
    out = C.c_ssize_t(0)
    assert tp.lib.TAPP_create_tensor_info(C.byref(out), tp.F16, 0, None, None) == tp.ERR_DTYPE
    assert tp.lib.TAPP_get_nmodes(0) == -1
    assert tp.lib.TAPP_destroy_tensor_info(0) == tp.ERR_INVALID_ARGUMENT


def test_null_c_with_nonzero_beta_is_rejected_before_any_device_work(tp):
    # execute.rs:34-39: refused during validation, which precedes any CUDA call.
    p = _product(tp, {"ext": [2, 2], "str": [1, 2], "lab": [0, 2]}, {"ext": [2, 2], "str": [1, 2], "lab": [2, 1]},
                 {"ext": [2, 2], "str": [1, 2], "lab": [0, 1]})
    a, b, d = np.ones(4), np.ones(4), np.zeros(4)
    assert p.execute(None, 1.0, a, b, 1.0, None, d) == tp.ERR_UNSUPPORTED
    assert np.all(d == 0)
    # D overlapping A is ALIASED, also before any device work.
    assert p.execute(None, 1.0, a, b, 0.0, None, a) == tp.ERR_ALIASED


def test_dot_general_front_end(tp):
    # DotGeneral::new(&[2], &[1], &[0], &[0]) on [3,5,4] x [3,4,2] -> [5,2,3] (dot_general.rs:14-18)
    a = tp.OperandSpec(tp.LayoutSpec.col_major([3, 5, 4]))
    b = tp.OperandSpec(tp.LayoutSpec.col_major([3, 4, 2]))
    d = tp.OperandSpec(tp.LayoutSpec.col_major([5, 2, 3]))
    plan = tp.Plan(tp.Problem.from_dot_general(tp.F64, a, b, d, tp.DotGeneral([2], [1], [0], [0])))
    rep = plan.report()
    assert (rep["m"], rep["n"], rep["k"], rep["batch"]) == (5, 2, 4, 3)
    bad = tp.OperandSpec(tp.LayoutSpec.col_major([5, 3, 2]))
    with pytest.raises(tp.TprimsError) as e:
        tp.Plan(tp.Problem.from_dot_general(tp.F64, a, b, bad, tp.DotGeneral([2], [1], [0], [0])))
    assert e.value.status == tp.ERR_SHAPE
    with pytest.raises(tp.TprimsError) as e:
        tp.Plan(tp.Problem.from_dot_general(tp.F64, a, b, d, tp.DotGeneral([2, 1], [1], [0], [0])))
    assert e.value.status == tp.ERR_INVALID_ARGUMENT


def test_split_precision_applies_to_f32_only(tp):
    p = _product(tp, {"ext": [2, 2], "str": [1, 2], "lab": [0, 2]}, {"ext": [2, 2], "str": [1, 2], "lab": [2, 1]},
                 {"ext": [2, 2], "str": [1, 2], "lab": [0, 1]})
    with pytest.raises(tp.TprimsError) as e:
        p.set_precision(tp.PREC_BF16X3)
    assert e.value.status == tp.ERR_UNSUPPORTED
    q = _product(tp, {"ext": [2, 2], "str": [1, 2], "lab": [0, 2]}, {"ext": [2, 2], "str": [1, 2], "lab": [2, 1]},
                 {"ext": [2, 2], "str": [1, 2], "lab": [0, 1]}, dtype=tp.F32)
    q.set_precision(tp.PREC_BF16X6)
    assert q.report()["scheme"] == "bf16x6"


def test_ozaki_slice_count_default_and_range(tp):
    """The Ozaki scheme takes 4 to 8 INT8 slices, six by default (21 slice
    products), and applies to f64 / c64 only."""
    specs = ({"ext": [2, 2], "str": [1, 2], "lab": [0, 2]}, {"ext": [2, 2], "str": [1, 2], "lab": [2, 1]},
             {"ext": [2, 2], "str": [1, 2], "lab": [0, 1]})
    for dt in (tp.F64, tp.C64):
        p = _product(tp, *specs, dtype=dt)
        p.set_precision(tp.PREC_OZAKI_INT8)
        assert ".ozaki-int8.s6." in p.report()["family"], p.report()
        p.set_precision(tp.PREC_OZAKI_INT8, 8)
        assert ".ozaki-int8.s8." in p.report()["family"]
        for bad in (3, 9):
            with pytest.raises(tp.TprimsError) as e:
                p.set_precision(tp.PREC_OZAKI_INT8, bad)
            assert e.value.status == tp.ERR_INVALID_ARGUMENT
    q = _product(tp, *specs, dtype=tp.F32)
    with pytest.raises(tp.TprimsError) as e:
        q.set_precision(tp.PREC_OZAKI_INT8)
    assert e.value.status == tp.ERR_UNSUPPORTED


def test_ozaki_workspace_follows_the_slice_count(tp):
    """The Ozaki workspace of the C3 shape (c64, batch 64 innermost, 384^3,
    conj A): S INT8 planes of the embedded A' (2M rows, padded to 128; depth
    2K, each half padded to 64) and of B' (N rows, padded to 64), plus the
    per-row and per-column exponents."""
    b, e = 64, 384
    h = tp.Handle()
    info = tp.TensorInfo(tp.C64, [b, e, e], [1, b, b * e])
    p = tp.TensorProduct.create(h, (1, info, [9, 2, 0]), (0, info, [9, 2, 1]), (0, info, [9, 0, 1]),
                                (0, info, [9, 0, 1]))
    p._keep = (h, info)

    def expected(s):
        k_emb = 2 * ((e + 63) // 64 * 64)
        m_pad, n_pad = (2 * e + 127) // 128 * 128, (e + 63) // 64 * 64
        exps = (b * ((e + 31) // 32 * 32 + 32) + b * n_pad) * 4
        return s * b * m_pad * k_emb + s * b * n_pad * k_emb + exps + 1024

    for s in (6, 7, 4, 8):
        p.set_precision(tp.PREC_OZAKI_INT8, s)
        assert p.report()["scratch_bytes"] == expected(s), (s, p.report()["scratch_bytes"], expected(s))
    p.set_precision(tp.PREC_OZAKI_INT8)
    assert p.report()["scratch_bytes"] == expected(6)


def test_executor_handles_without_a_gpu(tp):
    import ctypes as C

    h = C.c_ssize_t(0)
    assert tp.lib.tprims_tapp_executor_create_rayon(C.byref(h), 0, None) == tp.ERR_INVALID_ARGUMENT
    assert tp.lib.tprims_tapp_executor_create_rayon(C.byref(h), 4, None) == 0
    ps, bd = C.c_size_t(), C.c_size_t()
    assert tp.lib.tprims_tapp_executor_set_budget(h.value, 2) == 0
    assert tp.lib.tprims_tapp_executor_get_threads(h.value, C.byref(ps), C.byref(bd)) == 0
    assert (ps.value, bd.value) == (4, 2)
    assert tp.lib.TAPP_destroy_executor(h.value) == 0
    assert tp.lib.TAPP_destroy_executor(0) == 0


def test_planner_splits_k_only_for_deep_contractions_with_few_tiles(tp):
    """The launch choice (reported per plan, for 148 SMs): split-K when the
    large-tile grid has fewer tiles than SMs and K is deep (packed tiles: at
    least two chunks of 128); never otherwise."""
    def report(m, n, k, dt=1):
        h = tp.Handle()
        infos = [tp.TensorInfo(dt, [m, k], [1, m]), tp.TensorInfo(dt, [k, n], [1, k]),
                 tp.TensorInfo(dt, [m, n], [1, m]), tp.TensorInfo(dt, [m, n], [1, m])]
        p = tp.TensorProduct.create(h, (0, infos[0], [0, 2]), (0, infos[1], [2, 1]), (0, infos[2], [0, 1]),
                                    (0, infos[3], [0, 1]))
        return p.report()

    deep = report(512, 512, 32768)
    assert deep["split_k"] > 1 and "64x64" in deep["family"]
    assert report(4096, 4096, 4096, dt=0)["split_k"] == 1  # enough tiles
    assert report(64, 64, 192)["split_k"] == 1  # shallow
    c1_like = report(576, 576, 576)  # 81 packed tiles, K = 576: three chunks of 192
    assert c1_like["split_k"] == 3 and ".tma." in c1_like["family"], c1_like


def test_launch_choices_reported_per_plan(tp):
    """The plan report names the launch shape the executor will use (for 148
    SMs): the tcgen05 split GEMM cuts the partial last wave of C2 (512 tiles)
    into K halves, and batches of tiny products take the one-thread-per-output
    kernel."""
    def product(dt, ext_a, st_a, la, ext_b, st_b, lb, ext_d, st_d, ld, prec=0):
        h = tp.Handle()
        infos = [tp.TensorInfo(dt, ext_a, st_a), tp.TensorInfo(dt, ext_b, st_b), tp.TensorInfo(dt, ext_d, st_d),
                 tp.TensorInfo(dt, ext_d, st_d)]
        p = tp.TensorProduct.create(h, (0, infos[0], la), (0, infos[1], lb), (0, infos[2], ld), (0, infos[3], ld))
        p._keep = (h, infos)
        if prec:
            p.set_precision(prec)
        return p

    n = 4096
    c2 = product(0, [n, n], [1, n], [2, 0], [n, n], [1, n], [2, 1], [n, n], [1, n], [0, 1], prec=tp.PREC_BF16X6)
    assert c2.report()["tail_parts"] == 2
    m = 2048
    sq = product(0, [m, m], [1, m], [2, 0], [m, m], [1, m], [2, 1], [m, m], [1, m], [0, 1], prec=tp.PREC_BF16X6)
    assert sq.report()["tail_parts"] == 1  # 128 tiles: one partial wave of whole tiles
    hb = 1 << 20
    had = product(1, [hb], [1], [9], [hb], [1], [9], [hb], [1], [9])
    assert "tiny-batched" in had.report()["family"]


def _gemm_product(tp, m, n, k, dt=1, lda=None):
    """D[m,n] = sum_k A[m,k] B[k,n], column-major; `lda` widens A's column stride."""
    lda = lda or m
    h = tp.Handle()
    infos = [tp.TensorInfo(dt, [m, k], [1, lda]), tp.TensorInfo(dt, [k, n], [1, k]),
             tp.TensorInfo(dt, [m, n], [1, m]), tp.TensorInfo(dt, [m, n], [1, m])]
    p = tp.TensorProduct.create(h, (0, infos[0], [0, 2]), (0, infos[1], [2, 1]), (0, infos[2], [0, 1]),
                                (0, infos[3], [0, 1]))
    p._keep = (h, infos)
    return p


def test_problem_signature_keys_the_folded_layout(tp):
    """The autotuner's cache key: equal for two plans of the same folded
    layout, different when a stride, an extent or the dtype differs."""
    a = _gemm_product(tp, 300, 200, 100).report()
    b = _gemm_product(tp, 300, 200, 100).report()
    assert a["signature"] == b["signature"] and " " not in a["signature"]
    assert a["signature"].startswith("f64;")
    assert _gemm_product(tp, 300, 200, 100, lda=320).report()["signature"] != a["signature"]
    assert _gemm_product(tp, 300, 200, 101).report()["signature"] != a["signature"]
    assert _gemm_product(tp, 300, 200, 100, dt=0).report()["signature"] != a["signature"]


def test_split_k_and_autotune_switches(tp):
    """PlanConfig's pins and autotune switch: the split-K pin is reported
    before any execution as the pinned choice (chunks of whole 64-deep blocks),
    out-of-range factors are refused, and an autotuning plan reports the model's
    choice until it has run."""
    p = _gemm_product(tp, 512, 512, 4096)
    assert p.report()["choice"] == "model" and p.report()["autotune"] is False
    p.set_split_k(4)
    rep = p.report()
    assert rep["choice"] == "pinned" and rep["split_k"] == 4
    p.set_split_k(1)
    assert p.report()["split_k"] == 1
    p.set_split_k(3)
    assert p.report()["split_k"] == 3  # chunks of 1408 = 22 blocks of 64
    for bad in (-1, 65):
        with pytest.raises(tp.TprimsError) as ei:
            p.set_split_k(bad)
        assert ei.value.status == 1  # INVALID_ARGUMENT
    q = _gemm_product(tp, 512, 512, 4096)
    q.set_autotune(True)
    assert q.report()["autotune"] is True and q.report()["choice"] == "model"
    plan = tp.Plan(tp.Problem.from_labels(1, tp.OperandSpec(tp.LayoutSpec([8, 8], [1, 8])),
                                          tp.OperandSpec(tp.LayoutSpec([8, 8], [1, 8])),
                                          tp.OperandSpec(tp.LayoutSpec([8, 8], [1, 8])), [0, 2], [2, 1], [0, 1]),
                   tp.PlanConfig(autotune=True, split_k=1))
    assert plan.report()["autotune"] is True and plan.report()["choice"] == "pinned"


def test_autotune_candidates(tp):
    """What the autotuner times (for 148 SMs): the model's choice first, every
    tile family of the dtype, split-K only while tiles x splits <= 4 x SMs and
    the chunks stay at least 128 deep."""
    c1 = _gemm_product(tp, 576, 576, 576).report()["autotune_candidates"]
    assert c1[0].startswith(_gemm_product(tp, 576, 576, 576).report()["family"])  # the model's choice first
    assert {"sm100.f64.dmma884.64x64x16", "sm100.f64.dmma884.32x32x16", "sm100.f64.dmma884.128x32x16"} <= set(c1)
    assert any("+splitk" in c for c in c1) and len(c1) == len(set(c1))
    big = _gemm_product(tp, 4096, 4096, 4096, dt=0).report()["autotune_candidates"]
    assert big[0] == "sm100.f32.simt.tma.packed.128x128x32"  # the model: packed, a full wave of tiles
    assert sorted(big) == ["sm100.f32.simt.128x128x16", "sm100.f32.simt.64x64x16",
                           "sm100.f32.simt.tma.packed.128x128x32",
                           "sm100.f32.simt.tma.packed.128x64x32"]  # enough tiles: no split
    shallow = _gemm_product(tp, 64, 64, 128).report()["autotune_candidates"]
    assert not any("+splitk" in c for c in shallow)  # halves of K = 128 would be 64 deep
    c32 = _gemm_product(tp, 300, 300, 300, dt=2).report()["autotune_candidates"]
    assert c32[0].startswith("sm100.c32.simt.tma.1m")  # packed 1m, K split in two (15 tiles)
    assert any(c.startswith("sm100.c32.simt.ring") for c in c32)


def test_plain_c_consumer_compiles_links_and_runs(tmp_path):
    """tests/c/abi_consumer.c: the header as strict C99 (-Wall -Wextra -Werror
    -pedantic), linked against the built library, run without a GPU (handles,
    infos, products, report, refusals, network planning)."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    libdir = os.path.join(REPO, "tensoralgebra-rs_b200", "tprims_b200")
    exe = str(tmp_path / "abi_consumer")
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "c", "abi_consumer.c"), "-L", libdir, "-ltprims_b200",
                    "-Wl,-rpath," + libdir, "-o", exe], check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"


def test_report_tile_ctas_and_scratch(tp):
    """The report's launch geometry for 148 SMs: CTA tile, CTAs of the main
    launch (tiles x K chunks) and the workspace the scheme needs."""
    r = _gemm_product(tp, 576, 576, 576).report()
    bm, bn = r["tile"]
    assert r["ctas"] == -(-576 // bm) * -(-576 // bn) * r["split_k"]
    # The packed family's panels (576 x 576 of A and B, f64) plus the split-K partials.
    assert r["scratch_bytes"] >= 2 * 576 * 576 * 8 + r["split_k"] * 576 * 576 * 8
    small = _gemm_product(tp, 96, 96, 96).report()  # direct tiles, no split: no scratch
    assert small["split_k"] == 1 and small["scratch_bytes"] == 0 and ".tma." not in small["family"]
    deep = _gemm_product(tp, 512, 512, 32768).report()
    assert deep["split_k"] > 1 and deep["ctas"] == 64 * deep["split_k"]
    assert deep["scratch_bytes"] >= deep["split_k"] * 512 * 512 * 8  # the split-K partials


def test_check_raw_decides_aliasing_from_addresses(tp):
    """Plan::check_raw (plan/mod.rs:384-428) from the origins alone: nothing is
    dereferenced, so plain integers serve as addresses here."""
    m, n, k = 6, 5, 4
    plan = tp.Plan(tp.Problem.from_labels(1, tp.OperandSpec(tp.LayoutSpec.col_major([m, k])),
                                          tp.OperandSpec(tp.LayoutSpec.col_major([k, n])),
                                          tp.OperandSpec(tp.LayoutSpec.col_major([m, n])), [0, 2], [2, 1], [0, 1]),
                   tp.PlanConfig.packed())
    A, B, D = 0x100000, 0x200000, 0x300000
    plan.check_raw(A, B, None, D)
    plan.check_raw(A, B, D, D)  # C = D, the same mapping: an in-place update
    plan.check_raw(None, None, None, D)  # absent operands are not checked
    plan.check_raw(A, B, None, None)
    for a, b, c, d in [(A, B, None, A + 8 * (m * k - 1)),  # D's first element is A's last
                       (A, B, None, B - 8 * (m * n - 1)),  # D's last element is B's first
                       (A, B, D + 8, D)]:  # C shifted by one element over D
        with pytest.raises(tp.TprimsError) as ei:
            plan.check_raw(a, b, c, d)
        assert ei.value.status == tp.ERR_ALIASED
    plan.check_raw(A, B, None, A + 8 * m * k)  # just past A's range


def _random_problem(g):
    """Random labels over roles batch / M / N / K (with a diagonal or a
    reduction now and then), random extents, permuted and sometimes negative
    or padded strides; returns (a, b, d) dicts for _product and the base
    offsets that keep every addressed element inside its buffer."""
    roles = {"h": g.integers(0, 2), "m": g.integers(1, 3), "n": g.integers(1, 3), "k": g.integers(1, 3)}
    labels, nxt = {}, 0
    for r, cnt in roles.items():
        labels[r] = list(range(nxt, nxt + int(cnt)))
        nxt += int(cnt)
    ext = {l: int(g.integers(1, 5)) for ls in labels.values() for l in ls}
    la = labels["h"] + labels["m"] + labels["k"]
    lb = labels["h"] + labels["k"] + labels["n"]
    ld = labels["h"] + labels["m"] + labels["n"]
    if g.random() < 0.3:  # a reduction label only in A
        r = nxt
        ext[r] = int(g.integers(2, 4))
        la = la + [r]
    if g.random() < 0.3 and labels["k"]:  # a diagonal: one K label twice in A
        la = la + [labels["k"][0]]

    def layout(ls):
        ls = [ls[i] for i in g.permutation(len(ls))]
        st, acc = [], 1
        for l in ls:
            st.append(acc * (-1 if g.random() < 0.2 else 1))
            acc *= ext[l] + (1 if g.random() < 0.3 else 0)
        lo = sum((ext[l] - 1) * s for l, s in zip(ls, st) if s < 0)
        return {"ext": [ext[l] for l in ls], "str": st, "lab": ls}, -lo, acc

    return layout(la), layout(lb), layout(ld), ext


@pytest.mark.parametrize("seed", range(40))
def test_scatter_vectors_reproduce_the_contraction(tp, orc, seed):
    """The plan's 12 scatter vectors (as the kernels address memory: h + m + k
    for A, h + k + n for B, h + m + n for D) contract random data exactly as
    the brute-force oracle does, in whichever orientation the planner picked."""
    g = np.random.default_rng(1000 + seed)
    (a, oa, na), (b, ob, nb), (d, od, nd), ext = _random_problem(g)
    p = _product(tp, a, b, d)
    sc = {name: np.array(tp.product_scatter(p, name), dtype=np.int64) for name in tp.SCATTER_NAMES}
    A = g.uniform(-1, 1, na + 8)
    B = g.uniform(-1, 1, nb + 8)
    D = np.zeros(nd + 8)
    h_n = max(len(sc["h_d"]), 1)
    h_a = sc["h_a"] if len(sc["h_a"]) else np.zeros(1, np.int64)
    h_b = sc["h_b"] if len(sc["h_b"]) else np.zeros(1, np.int64)
    h_d = sc["h_d"] if len(sc["h_d"]) else np.zeros(1, np.int64)
    for h in range(h_n):
        Am = A[oa + h_a[h] + sc["a_m"][:, None] + sc["a_k"][None, :]]
        Bn = B[ob + h_b[h] + sc["b_k"][:, None] + sc["b_n"][None, :]]
        D[od + h_d[h] + sc["d_m"][:, None] + sc["d_n"][None, :]] = Am @ Bn
    want = np.zeros(nd + 8)
    orc.label_contract(1.0, orc.View(A, a["ext"], a["str"], a["lab"], oa), orc.View(B, b["ext"], b["str"], b["lab"], ob),
                       0.0, None, orc.View(want, d["ext"], d["str"], d["lab"], od))
    np.testing.assert_allclose(D, want, rtol=1e-12, atol=1e-12)


def test_tuning_file_format_is_checked_without_a_gpu(tp, tmp_path):
    """The autotuner cache file (versioned text): header, single-contraction and
    list entries; malformed lines and other versions are refused."""
    sig = _gemm_product(tp, 64, 64, 64).report()["signature"] + ";plain;c=0"
    good = tmp_path / "tune.txt"
    good.write_text("tprims-b200-tune 1 148 NVIDIA_B200\n"
                    f"single {sig} 3 1 0 0 1 0.0123 4\n"
                    f"single {sig}-split 3 4 1024 0 1 0.5 7\n"
                    "single tiny-signature 0 1 0 1 0 0 0\n"
                    "\n"
                    "list list-0123456789abcdef-n3 2 1 1.5 3\n")
    assert tp.tuning_file_info(str(good)) == {"sms": 148, "device": "NVIDIA_B200", "single": 3, "list": 1}
    bad_lines = [
        "single sig 16 1 0 0 1 0.1 1",    # no kernel family 16
        "single sig 3 2 0 0 1 0.1 1",     # split without a chunk
        "single sig 3 65 64 0 1 0.1 1",   # more than 64 chunks
        "single sig 3 1 0 0 1 0.1",       # a field short
        "single sig 3 1 0 0 1 0.1 1 9",   # a field too many
        "list sig 4 1 0.1 1",             # no list policy 4
        "pair sig 1 1 0.1 1",             # unknown kind
    ]
    for i, line in enumerate(bad_lines):
        p = tmp_path / f"bad{i}.txt"
        p.write_text("tprims-b200-tune 1 148 NVIDIA_B200\n" + line + "\n")
        with pytest.raises(tp.TprimsError) as ei:
            tp.tuning_file_info(str(p))
        assert ei.value.status == tp.ERR_INVALID_ARGUMENT and "line 2" in ei.value.message, line
    other = tmp_path / "v2.txt"
    other.write_text("tprims-b200-tune 2 148 NVIDIA_B200\n")
    with pytest.raises(tp.TprimsError) as ei:
        tp.tuning_file_info(str(other))
    assert ei.value.status == tp.ERR_UNSUPPORTED
    for text in ["", "something else 1 148 x\n"]:
        p = tmp_path / "junk.txt"
        p.write_text(text)
        with pytest.raises(tp.TprimsError):
            tp.tuning_file_info(str(p))
    with pytest.raises(tp.TprimsError):
        tp.tuning_file_info(str(tmp_path / "missing.txt"))
