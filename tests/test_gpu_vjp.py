"""Plan::vjp on the GPU: D[i,j] = alpha * sum_{k,l} op_A(A[i,k,k,l]) op_B(B[l,j,k])
(a repeated index k on A) and its cotangents dA (written onto A's diagonal,
zero elsewhere) and dB.

Checks: (1) against the oracle's contraction of the adjoint labels (the
brute-force label oracle with a repeated *output* label, the construction of
crates/tprims-capi/tests/tapp_conformance.rs:217-232); (2) directional central
finite differences in f64 of L(A, B) = Re <dD, D(A, B)> with step 1e-6 along
seeded random directions; (3) every conjugation of A, B and D for c64."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TAPP = {"float32": 0, "float64": 1, "complex64": 2, "complex128": 3}


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


def col_major(ext):
    s, acc = [], 1
    for e in ext:
        s.append(acc)
        acc *= e
    return s


def rnd(rng, dt, n):
    x = rng.standard_normal(n)
    if dt.startswith("complex"):
        x = x + 1j * rng.standard_normal(n)
    return x.astype(dt)


class C5:
    """The config-5 contraction at extents (i, k, l) with i = j."""

    def __init__(self, tp, dt, i, k, l, conj=(False, False, False)):
        self.dt, self.i, self.k, self.l = dt, i, k, l
        self.ea, self.eb, self.ed = [i, k, k, l], [l, i, k], [i, i]
        self.la, self.lb, self.ld = [0, 2, 2, 3], [3, 1, 2], [0, 1]
        self.conj = conj
        h = tp.Handle()
        infos = [tp.TensorInfo(TAPP[dt], e, col_major(e)) for e in (self.ea, self.eb, self.ed, self.ed)]
        ops = [1 if conj[0] else 0, 1 if conj[1] else 0, 0, 1 if conj[2] else 0]
        self.p = tp.TensorProduct.create(h, (ops[0], infos[0], self.la), (ops[1], infos[1], self.lb),
                                         (ops[2], infos[2], self.ld), (ops[3], infos[3], self.ld))
        self._keep = (h, infos)

    def forward(self, tp, ex, torch, alpha, A, B):
        D = torch.zeros(self.i * self.i, dtype=A.dtype, device="cuda")
        tp.check(self.p.execute(ex, alpha, A.data_ptr(), B.data_ptr(), 0.0, None, D.data_ptr()))
        torch.cuda.synchronize()
        return D

    def vjp(self, tp, ex, torch, alpha, A, B, dD):
        dA = torch.full_like(A, 7.0)  # poison: every element must be written or zeroed
        dB = torch.full_like(B, 7.0)
        tp.check(self.p.vjp(ex, alpha, A.data_ptr(), B.data_ptr(), dD.data_ptr(), dA.data_ptr(), dB.data_ptr()))
        torch.cuda.synchronize()
        return dA, dB


def test_vjp_matches_adjoint_label_contraction_f64(tp, ex, torch_cuda, orc):
    torch = torch_cuda
    rng = np.random.default_rng(20261203 + 5000 + 10)
    c = C5(tp, "float64", 6, 5, 4)
    a = rnd(rng, "float64", 6 * 5 * 5 * 4)
    b = rnd(rng, "float64", 4 * 6 * 5)
    dd = rnd(rng, "float64", 36)
    A, B, dD = (torch.from_numpy(x).cuda() for x in (a, b, dd))
    dA, dB = c.vjp(tp, ex, torch, 1.5, A, B, dD)
    # dA[i,k,k,l] = 1.5 * sum_j dD[i,j] B[l,j,k]  (oracle, repeated output label), 0 elsewhere
    want_a = np.zeros_like(a)
    orc.label_contract(1.5, orc.View(dd, c.ed, col_major(c.ed), c.ld), orc.View(b, c.eb, col_major(c.eb), c.lb), 0.0,
                       None, orc.View(want_a, c.ea, col_major(c.ea), c.la))
    want_b = np.zeros_like(b)
    orc.label_contract(1.5, orc.View(a, c.ea, col_major(c.ea), c.la), orc.View(dd, c.ed, col_major(c.ed), c.ld), 0.0,
                       None, orc.View(want_b, c.eb, col_major(c.eb), c.lb))
    got_a, got_b = dA.cpu().numpy(), dB.cpu().numpy()
    assert orc.rel_frobenius(got_a, want_a) <= 1e-13
    assert orc.rel_frobenius(got_b, want_b) <= 1e-13
    A4 = got_a.reshape(4, 5, 5, 6)  # [l, k2, k1, i]
    off = A4.copy()
    for kk in range(5):
        off[:, kk, kk, :] = 0
    assert np.all(off == 0), "dA is not zero off the diagonal"


@pytest.mark.parametrize("dt", ["float64", "float32"])
def test_vjp_central_finite_differences(tp, ex, torch_cuda, dt):
    torch = torch_cuda
    rng = np.random.default_rng(20261203 + 5000 + (10 if dt == "float64" else 0))
    i, k, l = 8, 6, 5
    c = C5(tp, dt, i, k, l)
    a = rnd(rng, dt, i * k * k * l)
    b = rnd(rng, dt, l * i * k)
    dd = rnd(rng, dt, i * i)
    A, B, dD = (torch.from_numpy(x).cuda() for x in (a, b, dd))
    dA, dB = c.vjp(tp, ex, torch, 1.0, A, B, dD)
    # Central differences are taken on an f64 copy of the problem (step 1e-6).
    c64 = C5(tp, "float64", i, k, l)
    A64, B64, dD64 = A.double(), B.double(), dD.double()
    tol = 1e-6 if dt == "float64" else 2e-4
    h = 1e-6
    for trial in range(4):
        for which in ("A", "B"):
            V = torch.from_numpy(rng.standard_normal(A64.numel() if which == "A" else B64.numel())).cuda()
            if which == "A":
                fp = c64.forward(tp, ex, torch, 1.0, A64 + h * V, B64)
                fm = c64.forward(tp, ex, torch, 1.0, A64 - h * V, B64)
                grad = dA.double()
            else:
                fp = c64.forward(tp, ex, torch, 1.0, A64, B64 + h * V)
                fm = c64.forward(tp, ex, torch, 1.0, A64, B64 - h * V)
                grad = dB.double()
            fd = float(torch.dot(dD64, (fp - fm) / (2 * h)))
            an = float(torch.dot(grad, V))
            assert abs(fd - an) <= tol * max(1.0, abs(an)), (which, trial, fd, an)


@pytest.mark.parametrize("mask", range(8))
def test_vjp_complex_conjugations(tp, ex, torch_cuda, mask):
    """c64 with op_A, op_B, op_D each identity or conjugate: the cotangents match
    central differences of L = Re <dD, D> (conjugate-Wirtinger convention)."""
    torch = torch_cuda
    rng = np.random.default_rng(700 + mask)
    conj = (bool(mask & 1), bool(mask & 2), bool(mask & 4))
    i, k, l = 5, 4, 3
    c = C5(tp, "complex128", i, k, l, conj)
    a = rnd(rng, "complex128", i * k * k * l)
    b = rnd(rng, "complex128", l * i * k)
    dd = rnd(rng, "complex128", i * i)
    alpha = complex(0.75, -0.5)
    A, B, dD = (torch.from_numpy(x).cuda() for x in (a, b, dd))
    dA, dB = c.vjp(tp, ex, torch, alpha, A, B, dD)
    h = 1e-6
    for which in ("A", "B"):
        n = A.numel() if which == "A" else B.numel()
        V = torch.from_numpy(rnd(rng, "complex128", n)).cuda()
        if which == "A":
            fp, fm, grad = c.forward(tp, ex, torch, alpha, A + h * V, B), c.forward(tp, ex, torch, alpha, A - h * V, B), dA
        else:
            fp, fm, grad = c.forward(tp, ex, torch, alpha, A, B + h * V), c.forward(tp, ex, torch, alpha, A, B - h * V), dB
        fd = float(torch.real(torch.sum(torch.conj(dD) * (fp - fm) / (2 * h))))
        an = float(torch.real(torch.sum(torch.conj(grad) * V)))
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (mask, which, fd, an)


def test_vjp_host_operands(tp, ex, orc):
    """Host (numpy) operands go through the executor's staging; dA's off-diagonal
    zeros are written on the host before its staged copy."""
    rng = np.random.default_rng(3)
    c = C5(tp, "float64", 4, 3, 2)
    a = rnd(rng, "float64", 4 * 3 * 3 * 2)
    b = rnd(rng, "float64", 2 * 4 * 3)
    dd = rnd(rng, "float64", 16)
    da = np.full_like(a, 7.0)
    db = np.full_like(b, 7.0)
    tp.check(c.p.vjp(ex, 1.0, a, b, dd, da, db))
    want_a = np.zeros_like(a)
    orc.label_contract(1.0, orc.View(dd, c.ed, col_major(c.ed), c.ld), orc.View(b, c.eb, col_major(c.eb), c.lb), 0.0,
                       None, orc.View(want_a, c.ea, col_major(c.ea), c.la))
    assert orc.rel_frobenius(da, want_a) <= 1e-13
