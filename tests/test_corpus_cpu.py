"""The reference's dot_general benchmark corpus (tests/golden/corpus.json,
written by tests/golden/make_corpus.py) planned on the CPU: every entry lowers
through Problem::from_dot_general, and the plan's batch and contracted sizes
and its free sizes match the entry's axis lists."""
import pytest

import bench


@pytest.mark.parametrize("i", range(len(bench.corpus_entries())))
def test_corpus_entry_plans(tp, i):
    e = bench.corpus_entries()[i]
    code, _ = bench.CORPUS_DT[e["dtype"]]
    spec = lambda side, conj: tp.OperandSpec(tp.LayoutSpec(list(e[side]["dims"]), list(e[side]["strides"])), conj)
    prob = tp.Problem.from_dot_general(code, spec("a", bool(e["conj"][0])), spec("b", bool(e["conj"][1])),
                                       spec("c", False), tp.DotGeneral(e["lc"], e["rc"], e["lb"], e["rb"]))
    rep = tp.Plan(prob).report()
    H, M, N, K, _ = bench.corpus_dims(e)
    assert rep["batch"] == H and rep["k"] == K, (e["name"], rep)
    assert sorted([rep["m"], rep["n"]]) == sorted([M, N]), (e["name"], rep)
