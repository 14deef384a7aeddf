"""Writes tests/golden/corpus.json: the dot_general shape corpus of the
reference's contraction benchmark (benchmarks/benchmarks/tprims/corpus/*.json,
replayed there by `contract --corpus`, benchmarks/benchmarks/tprims/contract/
README.md:37), reduced to what a replay needs: per entry the dtype, the
operand and output dims and strides, the contracted and batch axes of each
side, the conjugation flags and the recorded call count. No values: the
replay draws seeded inputs of these shapes.

The reference tree is read in place here; the fixture is what travels to the
machines that run the GPU tests and bench.py (--config corpus).

Run: python tests/golden/make_corpus.py <reference-root>/benchmarks/benchmarks/tprims/corpus
"""
import glob
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_corpus.py <reference-root>/benchmarks/benchmarks/tprims/corpus")
    src = sys.argv[1]
    out = {"source": "benchmarks/benchmarks/tprims/corpus/*.json of the reference", "files": [], "entries": []}
    for path in sorted(glob.glob(os.path.join(src, "*.json"))):
        with open(path) as f:
            doc = json.load(f)
        fname = os.path.basename(path)
        out["files"].append(fname)
        for e in doc.get("entries", []):
            if e.get("op") != "dot_general":
                continue
            out["entries"].append({
                "file": fname,
                "name": e["name"],
                "dtype": e["dtype"],
                "a": {"dims": e["a"]["dims"], "strides": e["a"]["strides"]},
                "b": {"dims": e["b"]["dims"], "strides": e["b"]["strides"]},
                "c": {"dims": e["c"]["dims"], "strides": e["c"]["strides"]},
                "lc": e["lc"], "rc": e["rc"], "lb": e["lb"], "rb": e["rb"],
                "conj": e.get("conj", [False, False]),
                "calls": e.get("calls", 1),
            })
    with open(os.path.join(HERE, "corpus.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(f"{len(out['entries'])} entries from {len(out['files'])} files")


if __name__ == "__main__":
    main()
