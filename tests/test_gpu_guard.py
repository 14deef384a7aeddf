"""Guard checks on a B200, the counterparts of the reference's memory-safety
harnesses (panels ending flush against a PROT_NONE page; allocation counters,
crates/tprims-kernel/tests/cplx_tile.rs:1-5, packed_workspace_alloc.rs):

* writes stay inside D: sentinel elements before and after D and in the gaps
  between its columns (a leading dimension larger than M) are untouched by
  every plain tile family, split-K, the bf16x6 and Ozaki paths, the tiny
  batched kernel and a grouped list, and D itself matches float64 sums;
* a steady-state execution allocates nothing: once a call has run, repeating
  it leaves the library's device-allocation count unchanged."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SENTINEL = 1234.5
PAD = 1000
TORCH_DT = {0: "float32", 1: "float64", 2: "complex64", 3: "complex128"}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "the -m gpu tests need a CUDA device"
    torch.cuda.init()
    return torch


def draw(g, shape, cplx):
    x = g.uniform(-1, 1, shape)
    return x + 1j * g.uniform(-1, 1, shape) if cplx else x


class GappedOut:
    """D[m,n] column-major with leading dimension m + gap, PAD sentinel
    elements on each side, in one device buffer."""

    def __init__(self, torch, dt, m, n, gap):
        self.m, self.n, self.ld = m, n, m + gap
        self.total = PAD + self.ld * n + PAD
        self.buf = torch.full((self.total,), SENTINEL, dtype=getattr(torch, TORCH_DT[dt]), device="cuda")
        self.layout = None

    def spec(self, tp):
        return tp.OperandSpec(tp.LayoutSpec([self.m, self.n], [1, self.ld]))

    def ptr(self):
        return self.buf.data_ptr() + PAD * self.buf.element_size()

    def check(self, want, tol):
        h = self.buf.cpu().numpy()
        inside = np.zeros(self.total, dtype=bool)
        idx = PAD + np.arange(self.m)[:, None] + self.ld * np.arange(self.n)[None, :]
        inside[idx.ravel()] = True
        assert np.all(h[~inside] == SENTINEL), "a kernel wrote outside D"
        got = h[idx]
        assert float(np.linalg.norm(got - want) / np.linalg.norm(want)) <= tol


CASES = [
    # (dtype, m, n, k, precision, tile family, split-K, tolerance)
    (1, 131, 70, 90, 0, 3, 0, 1e-13),
    (1, 131, 70, 90, 0, 4, 0, 1e-13),
    (1, 131, 20, 90, 0, 8, 0, 1e-13),
    (3, 75, 41, 66, 0, 6, 0, 1e-13),
    (3, 75, 41, 66, 0, 7, 0, 1e-13),
    (3, 150, 20, 66, 0, 9, 0, 1e-13),
    (0, 200, 150, 70, 0, 1, 0, 1e-6),
    (0, 200, 150, 70, 0, 2, 0, 1e-6),
    (2, 99, 77, 55, 0, 5, 0, 1e-6),
    (1, 64, 48, 2048, 0, 0, 5, 1e-13),
    (2, 64, 48, 1024, 0, 0, 3, 1e-6),
    (0, 260, 140, 300, 2, 0, 0, 1e-6),
    (1, 140, 90, 200, 3, 0, 0, 1e-12),
    (3, 140, 90, 200, 3, 0, 0, 1e-12),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"dt{c[0]}-{c[1]}x{c[2]}x{c[3]}-p{c[4]}-f{c[5]}-s{c[6]}")
def test_writes_stay_inside_d(tp, torch_cuda, case):
    torch = torch_cuda
    dt, m, n, k, prec, fam, split, tol = case
    cplx = dt in (2, 3)
    g = np.random.default_rng(m * 7 + n + k)
    A, B = draw(g, (m, k), cplx), draw(g, (k, n), cplx)
    d = GappedOut(torch, dt, m, n, gap=3)
    prob = tp.Problem.from_labels(dt, tp.OperandSpec(tp.LayoutSpec.col_major([m, k])),
                                  tp.OperandSpec(tp.LayoutSpec.col_major([k, n])), d.spec(tp), [0, 2], [2, 1], [0, 1])
    plan = tp.Plan(prob, tp.PlanConfig(precision=prec, kernel=fam, split_k=split))
    tdt = getattr(torch, TORCH_DT[dt])
    a = torch.from_numpy(A.ravel(order="F").copy()).to(tdt).cuda()
    b = torch.from_numpy(B.ravel(order="F").copy()).to(tdt).cuda()
    ex = tp.Executor()
    plan.execute_into(ex, 1.0, a.data_ptr(), b.data_ptr(), d.ptr())
    d.check(A @ B, tol)
    # Accumulating in place (beta = 1, C = D) touches the same elements only.
    plan.execute_into_accum(ex, 1.0, a.data_ptr(), b.data_ptr(), 1.0, d.ptr())
    d.check(2 * (A @ B), tol)
    ex.close()


def test_tiny_batched_and_grouped_list_stay_inside_d(tp, torch_cuda):
    torch = torch_cuda
    g = np.random.default_rng(17)
    ex = tp.Executor()
    # Batches of tiny products: D[i,j,h] with strides (1, 5, 23), i = j = k = 4, h = 100.
    i = j = kk = 4
    h = 100
    A, B = draw(g, (i, kk, h), False), draw(g, (kk, j, h), False)
    total = PAD + 23 * h + PAD
    buf = torch.full((total,), SENTINEL, dtype=torch.float64, device="cuda")
    prob = tp.Problem.from_labels(1, tp.OperandSpec(tp.LayoutSpec.col_major([i, kk, h])),
                                  tp.OperandSpec(tp.LayoutSpec.col_major([kk, j, h])),
                                  tp.OperandSpec(tp.LayoutSpec([i, j, h], [1, 5, 23])), [0, 2, 9], [2, 1, 9], [0, 1, 9])
    plan = tp.Plan(prob)
    assert "tiny-batched" in plan.report()["family"]
    a = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    b = torch.from_numpy(B.ravel(order="F").copy()).cuda()
    plan.execute_into(ex, 1.0, a.data_ptr(), b.data_ptr(), buf.data_ptr() + PAD * 8)
    hb = buf.cpu().numpy()
    idx = PAD + np.arange(i)[:, None, None] + 5 * np.arange(j)[None, :, None] + 23 * np.arange(h)[None, None, :]
    inside = np.zeros(total, dtype=bool)
    inside[idx.ravel()] = True
    assert np.all(hb[~inside] == SENTINEL)
    want = np.einsum("ikh,kjh->ijh", A, B)
    assert float(np.linalg.norm(hb[idx] - want) / np.linalg.norm(want)) <= 1e-13
    # A grouped list: three items, each into its own gapped D.
    items, checks = [], []
    for q, (m, n, k) in enumerate([(70, 33, 40), (129, 65, 17), (40, 9, 300)]):
        A, B = draw(g, (m, k), False), draw(g, (k, n), False)
        d = GappedOut(torch, 1, m, n, gap=2 + q)
        prob = tp.Problem.from_labels(1, tp.OperandSpec(tp.LayoutSpec.col_major([m, k])),
                                      tp.OperandSpec(tp.LayoutSpec.col_major([k, n])), d.spec(tp), [0, 2], [2, 1],
                                      [0, 1])
        a = torch.from_numpy(A.ravel(order="F").copy()).cuda()
        b = torch.from_numpy(B.ravel(order="F").copy()).cuda()
        items.append(tp.Item(tp.Plan(prob), 1.0, a.data_ptr(), b.data_ptr(), d.ptr(), _keep=[a, b]))
        checks.append((d, A @ B))
    tp.contract_batched(items, ex)
    for d, want in checks:
        d.check(want, 1e-13)
    ex.close()


def test_steady_state_executions_allocate_nothing(tp, torch_cuda):
    torch = torch_cuda
    g = np.random.default_rng(23)
    ex = tp.Executor()

    def gemm(dt, m, n, k, prec=0, split=0):
        cplx = dt in (2, 3)
        tdt = getattr(torch, TORCH_DT[dt])
        a = torch.from_numpy(draw(g, m * k, cplx)).to(tdt).cuda()
        b = torch.from_numpy(draw(g, k * n, cplx)).to(tdt).cuda()
        d = torch.zeros(m * n, dtype=tdt, device="cuda")
        prob = tp.Problem.from_labels(dt, tp.OperandSpec(tp.LayoutSpec.col_major([m, k])),
                                      tp.OperandSpec(tp.LayoutSpec.col_major([k, n])),
                                      tp.OperandSpec(tp.LayoutSpec.col_major([m, n])), [0, 2], [2, 1], [0, 1])
        plan = tp.Plan(prob, tp.PlanConfig(precision=prec, split_k=split))
        return lambda: plan.execute_into(ex, 1.0, a.data_ptr(), b.data_ptr(), d.data_ptr())

    host_a = draw(g, 96 * 80, False)
    host_b = draw(g, 80 * 64, False)
    host_d = np.zeros(96 * 64)
    host_plan = tp.Plan(tp.Problem.from_labels(1, tp.OperandSpec(tp.LayoutSpec.col_major([96, 80])),
                                               tp.OperandSpec(tp.LayoutSpec.col_major([80, 64])),
                                               tp.OperandSpec(tp.LayoutSpec.col_major([96, 64])), [0, 2], [2, 1],
                                               [0, 1]))
    ts = [torch.from_numpy(draw(g, 64 * 64, False)).cuda() for _ in range(6)]
    list_items = [tp.Item(tp.Plan(tp.Problem.from_labels(
        1, tp.OperandSpec(tp.LayoutSpec.col_major([64, 64])), tp.OperandSpec(tp.LayoutSpec.col_major([64, 64])),
        tp.OperandSpec(tp.LayoutSpec.col_major([64, 64])), [0, 2], [2, 1], [0, 1])), 1.0, ts[2 * q].data_ptr(),
        ts[2 * q + 1].data_ptr(), torch.zeros(64 * 64, dtype=torch.float64, device="cuda")) for q in range(3)]
    calls = {
        "plain f64": gemm(1, 300, 200, 150),
        "split-K f64": gemm(1, 64, 64, 4096, split=4),
        "bf16x6 f32": gemm(0, 512, 384, 256, prec=2),
        "ozaki c64": gemm(3, 200, 100, 150, prec=3),
        "host operands": lambda: host_plan.execute_into(ex, 1.0, host_a, host_b, host_d),
        "grouped list": lambda: tp.contract_batched(list_items, ex),
    }
    for name, fn in calls.items():
        fn()
        fn()
        ex.synchronize()
        before = tp.device_allocations()
        for _ in range(5):
            fn()
        ex.synchronize()
        assert tp.device_allocations() == before, name
    ex.close()
