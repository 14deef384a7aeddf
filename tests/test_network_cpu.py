"""N-ary contraction networks without a GPU: path walking, the labels and
extents of every intermediate, the arena layout, the greedy path and the
refusals (TAPP status codes). Execution is covered by test_gpu_network.py."""
import numpy as np
import pytest

F64, C64 = 1, 3


def spec(tp, dims, conj=False):
    return tp.OperandSpec(tp.LayoutSpec.col_major(dims), conj)


def env_update(tp, a=20, b=24, s=4, p=2, dtype=C64, path=((0, 1), (2, 0), (1, 0))):
    """The environment update of the list benchmark as one network:
    E'[a',s',b'] = sum E[a,s,b] M[a,p,a'] W[s,p,s',q] conj(M[b,q,b'])."""
    A, S, B, P, A2, S2, Q, B2 = range(8)
    inputs = [(spec(tp, [a, s, b]), [A, S, B]), (spec(tp, [a, p, a]), [A, P, A2]),
              (spec(tp, [s, p, s, p]), [S, P, S2, Q]), (spec(tp, [b, p, b], conj=True), [B, Q, B2])]
    out = (tp.LayoutSpec.col_major([a, s, b]), [A2, S2, B2])
    return tp.Network(dtype, inputs, out, path)


def test_environment_update_steps_match_the_hand_built_lists(tp):
    rep = env_update(tp).report()
    st = rep["steps"]
    assert [s["last"] for s in st] == [False, False, True]
    # T1[s,b,p,a'], T2[b,a',s',q], then the output E'[a',s',b'].
    assert st[0]["labels"] == [1, 2, 3, 4] and st[0]["dims"] == [4, 24, 2, 20]
    assert st[1]["labels"] == [2, 4, 5, 6] and st[1]["dims"] == [24, 20, 4, 2]
    assert st[2]["labels"] == [4, 5, 7]
    assert (st[0]["a"], st[0]["b"]) == (0, 1) and (st[1]["a"], st[1]["b"]) == (4, 2) and (st[2]["a"], st[2]["b"]) == (5, 3)
    # Dense intermediates in one arena, 256-byte aligned, complex128 elements.
    t1 = 4 * 24 * 2 * 20 * 16
    assert st[0]["offset"] == 0 and st[1]["offset"] == (t1 + 255) // 256 * 256
    assert rep["arena_bytes"] == st[1]["offset"] + (24 * 20 * 4 * 2 * 16 + 255) // 256 * 256
    # MACs: a s b p a' + b a' s p s' q + a' s' b q b'.
    assert rep["macs"] == 20 * 4 * 24 * 2 * 20 + 24 * 20 * 4 * 2 * 4 * 2 + 20 * 4 * 24 * 2 * 24
    # The conjugation of the last input reaches its step's plan.
    assert st[2]["plan"]["dtype"] == "c64" and rep["greedy_path"] is False


def test_greedy_path_is_complete_and_avoids_outer_products(tp):
    net = env_update(tp, path=None)
    rep = net.report()
    assert rep["greedy_path"] is True and len(rep["path"]) == 3
    for s in rep["steps"]:
        assert set(s["labels_a"]) & set(s["labels_b"]), s  # every step contracts or batches a shared label
    assert net.workspace_size() == rep["arena_bytes"]


def test_reductions_and_batch_labels(tp):
    # D[i] = sum_{j,k} X[i,j] Y[j,k] Z[i,k]: the last step batches i and contracts k.
    I, J, K = 0, 1, 2
    inputs = [(spec(tp, [5, 6]), [I, J]), (spec(tp, [6, 7]), [J, K]), (spec(tp, [5, 7]), [I, K])]
    rep = tp.Network(F64, inputs, (tp.LayoutSpec.col_major([5]), [I]), [(0, 1), (1, 0)]).report()
    assert rep["steps"][0]["labels"] == [I, K]
    assert rep["steps"][1]["plan"]["batch"] == 5 and rep["steps"][1]["plan"]["k"] == 7
    # A label of one input needed nowhere else is summed in its first step.
    inputs = [(spec(tp, [5, 6, 3]), [I, J, 9]), (spec(tp, [6, 7]), [J, K])]
    rep = tp.Network(F64, inputs, (tp.LayoutSpec.col_major([5, 7]), [I, K]), None).report()
    assert rep["steps"][0]["plan"]["k"] == 18


@pytest.mark.parametrize("case,status", [
    ("extent", 2), ("broadcast", 15), ("short_path", 1), ("bad_position", 1), ("one_input", 15), ("labels", 14),
])
def test_refusals(tp, case, status):
    I, J, K = 0, 1, 2
    inputs = [(spec(tp, [5, 6]), [I, J]), (spec(tp, [6, 7]), [J, K])]
    out = (tp.LayoutSpec.col_major([5, 7]), [I, K])
    path = [(0, 1)]
    if case == "extent":
        inputs[1] = (spec(tp, [8, 7]), [J, K])
    elif case == "broadcast":
        out = (tp.LayoutSpec.col_major([5, 7, 2]), [I, K, 3])
    elif case == "short_path":
        path = [(0, 1), (0, 1)]
    elif case == "bad_position":
        path = [(0, 2)]
    elif case == "one_input":
        inputs = inputs[:1]
        out = (tp.LayoutSpec.col_major([5]), [I])
        path = None
    elif case == "labels":
        inputs[0] = (spec(tp, [5, 6]), [I])
    with pytest.raises(tp.TprimsError) as ei:
        tp.Network(F64, inputs, out, path)
    assert ei.value.status == status


def test_prepared_networks_marshal_every_pointer(tp, monkeypatch):
    """The argument arrays handed to tprims_b200_networks_execute (the C call
    is replaced by a recorder: nothing runs without a GPU)."""
    import ctypes as C

    import numpy as np

    nets = [env_update(tp, a=10 + i, b=12, dtype=F64) for i in range(3)]
    inputs = [[np.zeros(4, dtype=np.float64) for _ in range(4)] for _ in nets]
    outs = [np.zeros(4, dtype=np.float64) for _ in nets]
    wss = [None, np.zeros(8, dtype=np.uint8), None]
    seen = {}

    def recorder(exec_h, n, hs, al, ins, be, ou, ws):
        seen["n"] = n
        seen["hs"] = [hs[i] for i in range(n)]
        seen["ins"] = [[ins[i][j] for j in range(4)] for i in range(n)]
        seen["outs"] = [ou[i] for i in range(n)]
        seen["ws"] = [ws[i] for i in range(n)]
        seen["alpha"] = [C.cast(al[i], C.POINTER(C.c_double))[0] for i in range(n)]
        seen["beta"] = [C.cast(be[i], C.POINTER(C.c_double))[0] for i in range(n)]
        return 0

    monkeypatch.setattr(tp.lib, "tprims_b200_networks_execute", recorder)
    prep = tp.PreparedNetworks(nets, inputs, outs, alphas=[1.0, 0.5, -2.0], betas=[0.0, 1.0, 0.25], workspaces=wss)
    prep.run(None)
    prep.run(None)  # the arrays stay valid across runs
    assert seen["n"] == 3 and seen["hs"] == [n.h for n in nets]
    assert seen["ins"] == [[x.ctypes.data for x in row] for row in inputs]
    assert seen["outs"] == [o.ctypes.data for o in outs]
    assert seen["ws"] == [None, wss[1].ctypes.data, None]
    assert seen["alpha"] == [1.0, 0.5, -2.0] and seen["beta"] == [0.0, 1.0, 0.25]
    with pytest.raises(tp.TprimsError):
        tp.PreparedNetworks(nets, inputs[:2], outs)
    for n in nets:
        n.close()


def _chain_through_oracle(orc, rep, arrays, conj):
    """Runs a network's reported steps with the CPU oracle's brute-force binary
    contraction: every intermediate dense column-major with the step's labels
    and extents, exactly as the GPU arena holds them."""
    import numpy as np

    n = len(arrays)
    cm = lambda dims: [int(np.prod(dims[:i])) for i in range(len(dims))]
    ops = {i: (np.ascontiguousarray(a.ravel(order="F")), list(a.shape), conj[i]) for i, a in enumerate(arrays)}
    out = None
    for s, st in enumerate(rep["steps"]):
        (ba, ea, ca), (bb, eb, cb) = ops[st["a"]], ops[st["b"]]
        dims = st["dims"]
        buf = np.zeros(int(np.prod(dims)), dtype=arrays[0].dtype)
        orc.label_contract(1.0, orc.View(ba, ea, cm(ea), st["labels_a"], conj=ca),
                           orc.View(bb, eb, cm(eb), st["labels_b"], conj=cb), 0.0, None,
                           orc.View(buf, dims, cm(dims), st["labels"]))
        ops[n + s] = (buf, dims, False)
        out = buf.reshape(dims, order="F")
    return out


@pytest.mark.parametrize("greedy", [False, True])
def test_network_steps_compose_to_the_whole_contraction(tp, orc, greedy):
    """The planner's step labels, extents and intermediate layouts, chained
    through the oracle, give the full network contraction (numpy einsum)."""
    import numpy as np

    g = np.random.default_rng(5)
    a, b, s, p = 5, 4, 3, 2
    dims = [[a, s, b], [a, p, a], [s, p, s, p], [b, p, b]]
    arrays = [g.uniform(-1, 1, d) + 1j * g.uniform(-1, 1, d) for d in dims]
    net = env_update(tp, a=a, b=b, s=s, p=p, dtype=C64, path=None if greedy else ((0, 1), (2, 0), (1, 0)))
    got = _chain_through_oracle(orc, net.report(), arrays, [False, False, False, True])
    want = np.einsum("asb,apc,spdq,bqe->cde", arrays[0], arrays[1], arrays[2], np.conj(arrays[3]))
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    net.close()


def test_five_tensor_network_with_batch_and_reduction(tp, orc):
    """A ring of five tensors with a batch label kept to the output and a
    label summed inside one input, on the greedy path."""
    import numpy as np

    g = np.random.default_rng(6)
    ext = {0: 3, 1: 4, 2: 2, 3: 5, 4: 3, 5: 2, 6: 3}  # 6: batch (kept), 5: summed in input 0 only
    labels = [[0, 1, 5, 6], [1, 2, 6], [2, 3], [3, 4, 6], [4, 0]]
    arrays = [g.uniform(-1, 1, [ext[l] for l in ls]) for ls in labels]
    inputs = [(spec(tp, [ext[l] for l in ls]), ls) for ls in labels]
    net = tp.Network(F64, inputs, (tp.LayoutSpec.col_major([ext[6]]), [6]), None)
    rep = net.report()
    assert rep["greedy_path"] and len(rep["steps"]) == 4
    got = _chain_through_oracle(orc, rep, arrays, [False] * 5)
    want = np.einsum("abfg,bcg,cd,deg,ea->g", *arrays)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    net.close()


def test_greedy_path_orders_a_matrix_chain_by_cost(tp):
    # A(10x100) B(100x5) C(5x50): (AB) first costs 5000 MACs, (BC) first 25000.
    inputs = [(spec(tp, [10, 100]), [0, 1]), (spec(tp, [100, 5]), [1, 2]), (spec(tp, [5, 50]), [2, 3])]
    rep = tp.Network(F64, inputs, (tp.LayoutSpec.col_major([10, 50]), [0, 3]), None).report()
    assert rep["path"][0] == [0, 1] and rep["macs"] == 10 * 100 * 5 + 10 * 5 * 50


def test_einsum_parsing_and_refusals(tp):
    import numpy as np

    a, b = np.zeros((3, 4)), np.zeros((4, 5))
    net, shape = tp.einsum_network("ab,bc->ac", a, b)
    assert shape == [3, 5] and net.report()["steps"][0]["labels"] == [ord("a"), ord("c")]
    assert tp.einsum_network("ab,bc", a, b)[1] == [3, 5]  # implicit output: letters seen once, sorted
    assert tp.einsum_network("ba,cb", a.T, b.T)[1] == [5, 3][::-1]
    for args, status in [(("ab,bc,cd->ad", a, b), 14), (("a1,bc->ac", a, b), 14), (("ab,bc->az", a, b), 15),
                         (("abc,bc->a", a, b), 14), (("ab,bc->ac", a, b.astype(np.float32)), 3)]:
        with pytest.raises(tp.TprimsError) as ei:
            tp.einsum_network(*args)
        assert ei.value.status == status, args


@pytest.mark.parametrize("expr,shapes,want", [
    ("ii->", [(4, 4)], lambda x: np.trace(x)),
    ("abc->cab", [(2, 3, 4)], lambda x: np.transpose(x, (2, 0, 1))),
    ("ij->j", [(5, 3)], lambda x: x.sum(axis=0)),
    ("ij,jk,kl->il", [(3, 4), (4, 5), (5, 2)], lambda x, y, z: x @ y @ z),
])
def test_einsum_plans_compose_through_the_oracle(tp, orc, expr, shapes, want):
    """The einsum front end's networks (a single operand paired with a rank-0
    one) chained through the CPU oracle equal numpy's result."""
    g = np.random.default_rng(4)
    arrays = [g.uniform(-1, 1, s) for s in shapes]
    net, shape = tp.einsum_network(expr, *arrays)
    ins = list(arrays) + ([np.ones(())] if len(arrays) == 1 else [])
    got = _chain_through_oracle(orc, net.report(), ins, [False] * len(ins))
    assert list(np.shape(got)) == shape
    np.testing.assert_allclose(got, want(*arrays), rtol=1e-12, atol=1e-12)
    net.close()


def test_einsum_glue_hands_the_right_pointers(tp, monkeypatch):
    """einsum's allocation and argument passing, with the C execute replaced
    by a recorder (no GPU): numpy operands give a column-major numpy result,
    torch operands a column-major tensor, and a single operand gets a
    one-element partner holding 1."""
    import ctypes as C

    import torch

    seen = {}

    def recorder(net_h, exec_h, alpha, ins, beta, out, ws):
        seen["ins"] = [ins[i] for i in range(len(ins))]
        seen["second"] = C.cast(ins[1], C.POINTER(C.c_double))[0]  # read while the call's buffers live
        seen["out"] = out
        seen["alpha"] = C.cast(alpha, C.POINTER(C.c_double))[0]
        return 0

    monkeypatch.setattr(tp.lib, "tprims_b200_network_execute", recorder)
    a, b = np.ones((3, 4)), np.ones((4, 5))
    out = tp.einsum("ab,bc->ac", a, b, alpha=2.0)
    assert out.shape == (3, 5) and out.flags["F_CONTIGUOUS"]
    assert seen["ins"][:2] == [a.ctypes.data, b.ctypes.data] and seen["out"] == out.ctypes.data
    assert seen["alpha"] == 2.0
    t = torch.ones(6, 2, dtype=torch.float64)
    res = tp.einsum("ij->ji", t)
    assert tuple(res.shape) == (2, 6) and res.stride() == (1, 2)
    assert seen["ins"][0] == t.data_ptr() and seen["second"] == 1.0
    given = np.zeros((5, 3))  # C order: the result is written through its strides
    assert tp.einsum("ab,bc->ca", a, b, out=given) is given and seen["out"] == given.ctypes.data
    with pytest.raises(tp.TprimsError):
        tp.einsum("ab,bc->ca", a, b, out=np.zeros((3, 5)))


@pytest.mark.parametrize("seed", range(30))
def test_random_networks_compose_through_the_oracle(tp, orc, seed):
    """Random networks of 3 to 5 tensors (labels shared by one to three
    tensors, some kept in the output, some summed inside one tensor), planned
    on the greedy path or a random valid path, chained through the oracle,
    equal numpy's einsum."""
    g = np.random.default_rng(500 + seed)
    n_t = int(g.integers(3, 6))
    n_l = int(g.integers(3, 8))
    ext = [int(g.integers(1, 4)) for _ in range(n_l)]
    labels = [[] for _ in range(n_t)]
    for l in range(n_l):
        for t in g.choice(n_t, size=int(g.integers(1, 4)), replace=False):
            labels[t].append(l)
    for t in range(n_t):  # no empty tensor
        if not labels[t]:
            labels[t].append(int(g.integers(0, n_l)))
    present = sorted({l for ls in labels for l in ls})
    out = [l for l in present if g.random() < 0.35]
    arrays = [g.uniform(-1, 1, [ext[l] for l in ls]) for ls in labels]
    inputs = [(spec(tp, [ext[l] for l in ls]), ls) for ls in labels]
    if seed % 2:
        path, m = [], n_t
        while m > 1:
            i, j = (int(x) for x in g.choice(m, size=2, replace=False))
            path.append((i, j))
            m -= 1
    else:
        path = None
    net = tp.Network(F64, inputs, (tp.LayoutSpec.col_major([ext[l] for l in out]), out), path)
    got = _chain_through_oracle(orc, net.report(), arrays, [False] * n_t)
    letters = "abcdefgh"
    expr = ",".join("".join(letters[l] for l in ls) for ls in labels) + "->" + "".join(letters[l] for l in out)
    want = np.einsum(expr, *arrays)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)
    net.close()


def test_c_entry_refusals_need_no_gpu(tp):
    """Argument checks of the network and sharded-list entry points run before
    any executor is touched, so they answer without a GPU."""
    import ctypes as C

    lib = tp.lib
    assert lib.tprims_b200_network_destroy(0) == tp.ERR_INVALID_ARGUMENT
    assert lib.tprims_b200_network_report(0, None, 0) == 0
    size = C.c_size_t(0)
    assert lib.tprims_b200_network_workspace_size(0, C.byref(size)) == tp.ERR_INVALID_ARGUMENT
    h = tp._ip(0)
    # Null descriptions, a negative count, too few inputs.
    assert lib.tprims_b200_network_create(C.byref(h), 1, 2, None, None, None, None, None, 0, None, None, None, 0,
                                          None) == tp.ERR_INVALID_ARGUMENT
    assert lib.tprims_b200_network_create(C.byref(h), 1, -1, None, None, None, None, None, 0, None, None, None, 0,
                                          None) == tp.ERR_SHAPE
    assert lib.tprims_b200_network_create(None, 1, 2, None, None, None, None, None, 0, None, None, None, 0,
                                          None) == tp.ERR_INVALID_ARGUMENT
    nets = (tp._ip * 1)(0)
    ptrs = (tp._vp * 1)()
    ins = (C.POINTER(tp._vp) * 1)()
    assert lib.tprims_b200_networks_execute(0, 1, nets, ptrs, ins, ptrs, ptrs, ptrs) == tp.ERR_INVALID_ARGUMENT
    assert lib.tprims_b200_networks_execute(0, 0, None, None, None, None, None, None) == tp.OK
    # The sharded list: no executors, a null item array, a null plan.
    execs = (tp._ip * 1)(0)
    assert lib.tprims_b200_contract_batched_sharded(None, 0, 0, None) == tp.ERR_INVALID_ARGUMENT
    assert lib.tprims_b200_contract_batched_sharded(execs, 1, 2, None) == tp.ERR_INVALID_ARGUMENT
    items = (tp.BatchItem * 1)()
    assert lib.tprims_b200_contract_batched_sharded(execs, 1, 1, items) == tp.ERR_INVALID_ARGUMENT
    assert lib.tprims_b200_balance(2, None, None, 1, None, None) == tp.ERR_INVALID_ARGUMENT
