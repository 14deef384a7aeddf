"""The benchmark configurations at their full sizes, every output checked, on a
B200, through the C ABI (TAPP_execute_product, the plan VJP, contract_batched).

The reference checks every size class it times with its randomized driver
sweep (crates/tprims-contract/src/driver/tests/correctness.rs:77-89). Here the
checker for whole outputs is the oracle's restated packed CPU driver
(oracle_packed_contract, OpenMP on the host cores), run in float64 /
complex128 on the same inputs; it is itself pinned to the reference's
known answers and to the brute-force label oracle (tests/test_oracle.py).

Bounds (relative Frobenius): plain f64 / c64 <= 1e-13, plain f32 <= 1e-6,
bf16x6 <= 1e-6, bf16x3 <= 2e-5, Ozaki INT8 (6 slices) <= 1e-12."""
import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu


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


def col_major(ext):
    st, acc = [], 1
    for e in ext:
        st.append(acc)
        acc *= e
    return st


def product(tp, dtype, specs, ops=(0, 0, 0, 0)):
    """specs: (extents, strides, labels) of A, B, C, D."""
    h = tp.Handle()
    infos = [tp.TensorInfo(dtype, e, s) for e, s, _ in specs]
    p = tp.TensorProduct.create(h, *[(ops[i], infos[i], specs[i][2]) for i in range(4)])
    p._keep = (h, infos)
    return p


# --------------------------------------------------------------------- config 2
@pytest.mark.parametrize("scheme,bound", [(0, 1e-6), (1, 2e-5), (2, 1e-6)], ids=["plain", "bf16x3", "bf16x6"])
def test_c2_every_output_against_the_packed_oracle(tp, ex, torch_cuda, orc, scheme, bound):
    """f32 D[m1,n1,m2,n2] = sum_{k1,k2} A[k1,m1,k2,m2] B[n1,k2,n2,k1], extents
    64 (M = N = K = 4096), A strides (2, 128, 8192, 524288): all 16.8 M outputs
    against the packed oracle in float64."""
    torch = torch_cuda
    a, b = bench.host_inputs()
    A, B = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    D = torch.full((bench.E ** 4,), np.nan, dtype=torch.float32, device="cuda")
    p = product(tp, tp.F32, [([bench.E] * 4, bench.SA, bench.LAB_A), ([bench.E] * 4, bench.CM, bench.LAB_B),
                             ([bench.E] * 4, bench.CM, bench.LAB_D), ([bench.E] * 4, bench.CM, bench.LAB_D)])
    if scheme:
        p.set_precision(scheme)
    tp.check(p.execute(ex, 1.0, A.data_ptr(), B.data_ptr(), 0.0, None, D.data_ptr()))
    torch.cuda.synchronize()
    got = D.cpu().numpy()
    want = np.zeros(bench.E ** 4)
    e4 = [bench.E] * 4
    orc.packed_contract(1.0, orc.View(a.astype(np.float64), e4, bench.SA, bench.LAB_A),
                        orc.View(b.astype(np.float64), e4, bench.CM, bench.LAB_B), 0.0, None,
                        orc.View(want, e4, bench.CM, bench.LAB_D))
    assert np.all(np.isfinite(got))
    err = orc.rel_frobenius(got, want)
    assert err <= bound, (scheme, err)


# --------------------------------------------------------------------- config 3
C3_NB, C3_N = 64, 384


def c3_inputs():
    nb, n = C3_NB, C3_N
    g = lambda i: (np.random.default_rng(20261203 + 3000 + 30 + i).uniform(-1, 1, nb * n * n)
                   + 1j * np.random.default_rng(20261203 + 3000 + 30 + i + 100).uniform(-1, 1, nb * n * n))
    return g(0), g(1)


@pytest.mark.parametrize("scheme,bound", [(0, 1e-13), (3, 1e-12)], ids=["plain", "ozaki"])
def test_c3_every_output_against_the_packed_oracle(tp, ex, torch_cuda, orc, scheme, bound):
    """c64 D[b,i,j] = sum_k conj(A[b,k,i]) B[b,k,j], b = 64, i = j = k = 384,
    every operand column-major in the listed order (the batch index has stride
    1): all 9.4 M outputs against the packed oracle in complex128."""
    torch = torch_cuda
    nb, n = C3_NB, C3_N
    ext = [nb, n, n]
    cm = col_major(ext)
    a, b = c3_inputs()
    specs = [(ext, cm, [9, 2, 0]), (ext, cm, [9, 2, 1]), (ext, cm, [9, 0, 1]), (ext, cm, [9, 0, 1])]
    p = product(tp, tp.C64, specs, ops=(1, 0, 0, 0))
    if scheme:
        p.set_precision(scheme)
    A, B = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    D = torch.full_like(A, complex(np.nan, np.nan))
    tp.check(p.execute(ex, 1.0, A.data_ptr(), B.data_ptr(), 0.0, None, D.data_ptr()))
    torch.cuda.synchronize()
    got = D.cpu().numpy()
    want = np.zeros(nb * n * n, dtype=np.complex128)
    orc.packed_contract(1.0, orc.View(a, ext, cm, [9, 2, 0], conj=True), orc.View(b, ext, cm, [9, 2, 1]), 0.0, None,
                        orc.View(want, ext, cm, [9, 0, 1]))
    assert np.all(np.isfinite(got))
    err = orc.rel_frobenius(got, want)
    assert err <= bound, (scheme, p.report()["family"], err)


# --------------------------------------------------------------------- config 5
@pytest.mark.parametrize("dt", ["float64", "float32"])
def test_c5_forward_and_vjp_full_size(tp, ex, torch_cuda, orc, dt):
    """D[i,j] = sum_{k,l} A[i,k,k,l] B[l,j,k] with i = j = 512, k = 128,
    l = 256 (A a full [512,128,128,256] allocation: 2^31 elements, of which
    only the diagonal k1 = k2 is read), its forward and Plan::vjp:
      * D, dB and the diagonal of dA at every element against the packed
        oracle (float64) on the diagonal's dense copy Ad[i,k,l] = A[i,k,k,l]
        (the adjoint-label contractions dA_d[i,k,l] = sum_j dD[i,j] B[l,j,k],
        dB[l,j,k] = sum_i Ad[i,k,l] dD[i,j]);
      * dA is zero off the diagonal: its nonzero count equals the diagonal's."""
    torch = torch_cuda
    i, k, l = 512, 128, 256
    tdt = torch.float64 if dt == "float64" else torch.float32
    code = tp.F64 if dt == "float64" else tp.F32
    bound = 1e-13 if dt == "float64" else 1e-6
    ea, eb, ed = [i, k, k, l], [l, i, k], [i, i]
    gen = torch.Generator(device="cuda").manual_seed(20261203 + 5000 + (10 if dt == "float64" else 0))
    A = torch.randn(i * k * k * l, dtype=tdt, device="cuda", generator=gen)
    B = torch.randn(l * i * k, dtype=tdt, device="cuda", generator=gen)
    dD = torch.randn(i * i, dtype=tdt, device="cuda", generator=gen)
    D = torch.full((i * i,), np.nan, dtype=tdt, device="cuda")
    dA = torch.full_like(A, 7.0)  # poison: every element must be written or zeroed
    dB = torch.full_like(B, 7.0)
    p = product(tp, code, [(ea, col_major(ea), [0, 2, 2, 3]), (eb, col_major(eb), [3, 1, 2]),
                           (ed, col_major(ed), [0, 1]), (ed, col_major(ed), [0, 1])])
    tp.check(p.execute(ex, 1.0, A.data_ptr(), B.data_ptr(), 0.0, None, D.data_ptr()))
    tp.check(p.vjp(ex, 1.0, A.data_ptr(), B.data_ptr(), dD.data_ptr(), dA.data_ptr(), dB.data_ptr()))
    torch.cuda.synchronize()
    diag = (1, i + i * k, i * k * k)  # element strides of A[i,k,k,l] along i, k (both k modes), l
    Ad = torch.as_strided(A, (i, k, l), diag).double().cpu().numpy().ravel(order="F")
    dAd = torch.as_strided(dA, (i, k, l), diag).double().cpu().numpy().ravel(order="F")
    nz_all = int(torch.count_nonzero(dA).item())
    nz_diag = int(torch.count_nonzero(torch.as_strided(dA, (i, k, l), diag)).item())
    assert nz_all == nz_diag, "dA is not zero off the diagonal"
    del A, dA
    torch.cuda.empty_cache()
    b64, dd64 = B.double().cpu().numpy(), dD.double().cpu().numpy()
    eadd = [i, k, l]
    V = orc.View
    # Forward.
    want = np.zeros(i * i)
    orc.packed_contract(1.0, V(Ad, eadd, col_major(eadd), [0, 2, 3]), V(b64, eb, col_major(eb), [3, 1, 2]), 0.0, None,
                        V(want, ed, col_major(ed), [0, 1]))
    assert orc.rel_frobenius(D.cpu().numpy(), want) <= bound
    # dA on the diagonal.
    want = np.zeros(i * k * l)
    orc.packed_contract(1.0, V(dd64, ed, col_major(ed), [0, 1]), V(b64, eb, col_major(eb), [3, 1, 2]), 0.0, None,
                        V(want, eadd, col_major(eadd), [0, 2, 3]))
    assert orc.rel_frobenius(dAd, want) <= bound
    # dB.
    want = np.zeros(l * i * k)
    orc.packed_contract(1.0, V(Ad, eadd, col_major(eadd), [0, 2, 3]), V(dd64, ed, col_major(ed), [0, 1]), 0.0, None,
                        V(want, eb, col_major(eb), [3, 1, 2]))
    assert orc.rel_frobenius(dB.cpu().numpy(), want) <= bound


# --------------------------------------------------------------------- config 4
@pytest.mark.parametrize("dt", ["float64", "complex128"])
def test_c4_all_4096_updates(tp, torch_cuda, dt):
    """The uneven list of 4096 environment updates, three binary steps each,
    as grouped persistent launches from cached CUDA graphs (a replay bitwise
    equal to the captured run), within the plain bound 1e-13 of the same list
    run one launch per item (on the single-launch families), and 64 sampled
    items against the four-tensor contraction in complex128 (1e-13)."""
    torch = torch_cuda
    ex = tp.Executor()
    tdt = tp.C64 if dt == "complex128" else tp.F64
    items = bench.c4_items(4096, dt)
    plans, dev, lists = {}, [], [[], [], []]
    for it in items:
        ext = bench.c4_extents(it)
        t = {k: torch.from_numpy(it[k]).cuda() for k in ("E", "Ma", "W", "Mb")}
        for name, labs in (("T1", bench.C4_STEPS[0][5]), ("T2", bench.C4_STEPS[1][5]), ("Ep", bench.C4_STEPS[2][5])):
            t[name] = torch.zeros(int(np.prod([ext[l] for l in labs])), dtype=t["E"].dtype, device="cuda")
        dev.append(t)
        for si, (xa, la, xb, lb, xd, ld, cj) in enumerate(bench.C4_STEPS):
            key = (si, tuple(ext[x] for x in la), tuple(ext[x] for x in lb))
            if key not in plans:
                plans[key] = tp.Plan(tp.Problem.from_labels(
                    tdt, tp.OperandSpec(tp.LayoutSpec.col_major([ext[x] for x in la])),
                    tp.OperandSpec(tp.LayoutSpec.col_major([ext[x] for x in lb]), cj),
                    tp.OperandSpec(tp.LayoutSpec.col_major([ext[x] for x in ld])), la, lb, ld))
            lists[si].append(tp.Item(plans[key], 1.0, t[xa].data_ptr(), t[xb].data_ptr(), t[xd].data_ptr()))
    prepared = [tp.PreparedBatch(x) for x in lists]
    torch.cuda.synchronize()

    def run(grouping):
        ex.set_grouping(grouping)
        for pb in prepared:
            pb.run(ex)
        ex.synchronize()
        return torch.cat([d["Ep"] for d in dev]).cpu().numpy()

    single = run(False)
    grouped = run(True)
    replay = run(True)
    assert np.array_equal(grouped, replay)
    assert np.linalg.norm(single - grouped) <= 1e-13 * np.linalg.norm(grouped)
    for q in np.random.default_rng(11).choice(len(items), size=64, replace=False):
        it = items[q]
        want = bench.c4_reference(it)
        got = dev[q]["Ep"].cpu().numpy().reshape((it["a"], it["s"], it["b"]), order="F")
        assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-13, q
    ex.close()
