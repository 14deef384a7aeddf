"""N-ary contraction networks on a B200: every result against numpy
tensordot steps in float64 / complex128 on the host (relative Frobenius <= 1e-13, the plain
path's bound; <= 1e-12 for the Ozaki scheme), with explicit and greedy paths,
device and host operands, alpha / beta on the output, caller workspaces, and a
list of networks of different extents run step by step as grouped
submissions."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F64, C64 = 1, 3


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


def rel(got, want):
    return float(np.linalg.norm(got - want) / np.linalg.norm(want))


def draw(g, dims, cplx):
    x = g.uniform(-1, 1, dims)
    return x + 1j * g.uniform(-1, 1, dims) if cplx else x


def env_update(tp, g, a, b, s, p, dtype, path=((0, 1), (2, 0), (1, 0))):
    """E'[a',s',b'] = sum E[a,s,b] M[a,p,a'] W[s,p,s',q] conj(M'[b,q,b'])."""
    cplx = dtype == C64
    A, S, B, P, A2, S2, Q, B2 = range(8)
    dims = [[a, s, b], [a, p, a], [s, p, s, p], [b, p, b]]
    labels = [[A, S, B], [A, P, A2], [S, P, S2, Q], [B, Q, B2]]
    conj = [False, False, False, cplx]
    arrays = [draw(g, d, cplx) for d in dims]
    inputs = [(tp.OperandSpec(tp.LayoutSpec.col_major(d), c), l) for d, l, c in zip(dims, labels, conj)]
    net = tp.Network(dtype, inputs, (tp.LayoutSpec.col_major([a, s, b]), [A2, S2, B2]),
                     None if path is None else list(path))
    x3 = np.conj(arrays[3]) if cplx else arrays[3]
    # The reference by three BLAS contractions: T1[s,b,p,a'], T2[b,a',s',q], E'[a',s',b'].
    t1 = np.tensordot(arrays[0], arrays[1], axes=([0], [0]))
    t2 = np.tensordot(t1, arrays[2], axes=([0, 2], [0, 1]))
    want = np.tensordot(t2, x3, axes=([0, 3], [0, 1]))
    return net, arrays, want


def flat(x):
    return np.ascontiguousarray(x.ravel(order="F"))


@pytest.mark.parametrize("dtype", [F64, C64])
@pytest.mark.parametrize("path", ["given", "greedy"])
def test_network_matches_einsum(tp, torch_cuda, ex, dtype, path):
    torch = torch_cuda
    g = np.random.default_rng(7 + dtype)
    a, b, s, p = 40, 56, 8, 4
    net, arrays, want = env_update(tp, g, a, b, s, p, dtype, path=None if path == "greedy" else ((0, 1), (2, 0), (1, 0)))
    dev = [torch.from_numpy(flat(x)).cuda() for x in arrays]
    d0 = draw(g, [a, s, b], dtype == C64)
    out = torch.from_numpy(flat(d0)).cuda()
    net.execute(ex, 0.5, dev, out, beta=-1.0)
    got = out.cpu().numpy().reshape((a, s, b), order="F")
    assert rel(got, 0.5 * want - d0) <= 1e-13
    # Host operands and output (staged by the executor), beta = 0.
    host_out = np.zeros(a * s * b, dtype=arrays[0].dtype)
    net.execute(ex, 1.0, [flat(x) for x in arrays], host_out)
    assert rel(host_out.reshape((a, s, b), order="F"), want) <= 1e-13
    net.close()


def test_network_list_in_grouped_steps(tp, torch_cuda, ex):
    torch = torch_cuda
    g = np.random.default_rng(11)
    nets, ins, outs, wants, shapes, wss = [], [], [], [], [], []
    for i in range(12):
        a, b = (int(x) for x in g.integers(16, 96, size=2))
        s, p = int(g.choice([4, 8, 16])), int(g.choice([2, 4]))
        net, arrays, want = env_update(tp, g, a, b, s, p, F64)
        nets.append(net)
        ins.append([torch.from_numpy(flat(x)).cuda() for x in arrays])
        outs.append(torch.zeros(a * s * b, dtype=torch.float64, device="cuda"))
        wants.append(want)
        shapes.append((a, s, b))
        # Half of the networks run in a caller workspace.
        wss.append(torch.empty(net.workspace_size(), dtype=torch.uint8, device="cuda") if i % 2 else None)
    for rep in range(2):  # the second pass replays the cached step graphs
        for o in outs:
            o.zero_()
        tp.execute_networks(ex, nets, ins, outs, workspaces=wss)
        for o, w, sh in zip(outs, wants, shapes):
            assert rel(o.cpu().numpy().reshape(sh, order="F"), w) <= 1e-13
    for n in nets:
        n.close()


def test_network_in_ozaki_precision(tp, torch_cuda, ex):
    torch = torch_cuda
    g = np.random.default_rng(3)
    net, arrays, want = env_update(tp, g, 48, 40, 8, 2, C64)
    net.set_precision(tp.PREC_OZAKI_INT8)
    assert all(st["plan"]["scheme"] == "ozaki-int8" for st in net.report()["steps"])
    dev = [torch.from_numpy(flat(x)).cuda() for x in arrays]
    out = torch.zeros(48 * 8 * 40, dtype=torch.complex128, device="cuda")
    net.execute(ex, 1.0, dev, out)
    assert rel(out.cpu().numpy().reshape((48, 8, 40), order="F"), want) <= 1e-12
    net.close()


@pytest.mark.parametrize("dtype", ["float64", "complex128"])
def test_einsum_front_end(tp, torch_cuda, ex, dtype):
    """tp.einsum over torch tensors (row-major, device), a given output layout,
    conjugation, and host numpy operands, against torch.einsum."""
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(3)
    cplx = dtype == "complex128"

    def rnd(*shape):
        x = torch.randn(*shape, dtype=torch.float64, device="cuda", generator=g)
        return torch.complex(x, torch.randn(*shape, dtype=torch.float64, device="cuda", generator=g)) if cplx else x

    def rel(got, want):
        return float(torch.linalg.norm(got - want) / torch.linalg.norm(want))

    x, y, z = rnd(30, 40), rnd(40, 25), rnd(25, 12)
    got = tp.einsum("ij,jk,kl->il", x, y, z, exec_=ex)
    assert got.shape == (30, 12) and rel(got, x @ y @ z) <= 1e-13
    a, b = rnd(8, 20, 30), rnd(8, 30, 10)
    out = torch.zeros(10, 8, 20, dtype=a.dtype, device="cuda")
    assert tp.einsum("bij,bjk->kbi", a, b, exec_=ex, out=out, conj=[True, False]) is out
    assert rel(out, torch.einsum("bij,bjk->kbi", a.conj().resolve_conj(), b)) <= 1e-13
    xn, yn = x.cpu().numpy(), y.cpu().numpy()
    res = tp.einsum("ij,jk->ik", xn, yn, exec_=ex)
    assert float(np.linalg.norm(res - xn @ yn) / np.linalg.norm(xn @ yn)) <= 1e-13
