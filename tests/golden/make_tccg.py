"""Writes tests/golden/tccg.json: the TCCG contraction corpus as the
reference's benchmark harness defines it (benchmarks/benchmarks/tcbench/
corpus.rs:262 `corpus()`: the CCSD, AO2MO, InTensLi, CCSD(T) and transpose-C
groups, de-duplicated after the label normalisation of `normalize`,
corpus.rs:305-347), read from that file in place, with each case's extents
under the harness's sizing rule (corpus.rs:27-45, `size_case_stressed`
:407-441) at the nominal tensor sizes the reference publishes numbers for
(64 MiB: docs/archive/tensorprimitives/results.md:80-93) and a small size for
the parity tests.

The sizing rule, restated: avg = (bytes / 8) ** (1 / max_ndim) (8 bytes per
element for every dtype); an index that is the first (stride-1, column-major)
label of any of C, A, B is rounded up to a multiple of 24; every other index
to the nearest multiple of 4 (at least 4; ties go down).

Run: python tests/golden/make_tccg.py <reference-root>
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
GROUPS = [("ccsd", "CCSD"), ("ao2mo", "AO2MO"), ("intensli", "INTENSLI"), ("ccsd_t", "CCSD_T"),
          ("transC", "TRANS_C")]
SIZES_MIB = {"tccg64": 64, "small": 1.0 / 16}


def read_groups(text):
    out = []
    for group, const in GROUPS:
        m = re.search(r"const\s+" + const + r"\s*:\s*&\[&str\]\s*=\s*&\[(.*?)\];", text, re.S)
        if not m:
            sys.exit(f"make_tccg: {const} not found in corpus.rs")
        out.append((group, re.findall(r'"([a-z-]+)"', m.group(1))))
    return out


def normalize(spec):
    """corpus.rs:305-347: rename C's labels A, B, ... in order, then A's labels
    not in C, lower-case the result."""
    c, a, b = (list(x) for x in spec.split("-"))
    nxt = ord("A")

    def rename(frm, to):
        for v in (a, b, c):
            for i, x in enumerate(v):
                if x == frm:
                    v[i] = to

    for ch in list(c):
        rename(ch, chr(nxt))
        nxt += 1
    for ch in list(a):
        if ch not in c and ch.islower():
            rename(ch, chr(nxt))
            nxt += 1
    return ("".join(c) + "-" + "".join(a) + "-" + "".join(b)).lower()


def size_case(c, a, b, tensor_bytes):
    """corpus.rs:407-441 (Stress::None)."""
    max_ndim = max(len(a), len(b), len(c))
    avg = (tensor_bytes / 8.0) ** (1.0 / max_ndim)
    labels = []
    for s in (c, a, b):
        for ch in s:
            if ch not in labels:
                labels.append(ch)
    stride1 = [s[0] for s in (c, a, b) if s]
    ext = {}
    for ch in labels:
        if ch in stride1:
            ext[ch] = int((avg + 23.0) / 24.0) * 24
        else:
            up = int((avg + 3.0) / 4.0) * 4
            down = max(int(avg / 4.0) * 4, 4)
            ext[ch] = up if abs(avg - up) < abs(avg - down) else down
    return ext


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_tccg.py <reference-root>")
    path = os.path.join(sys.argv[1], "benchmarks", "benchmarks", "tcbench", "corpus.rs")
    with open(path) as f:
        text = f.read()
    seen, cases = set(), []
    for group, specs in read_groups(text):
        for spec in specs:
            norm = normalize(spec)
            if norm in seen:
                continue
            seen.add(norm)
            c, a, b = spec.split("-")
            case = {"name": spec, "group": group, "c": c, "a": a, "b": b, "extents": {}}
            for key, mib in SIZES_MIB.items():
                case["extents"][key] = size_case(c, a, b, mib * 1024 * 1024)
            cases.append(case)
    doc = {"source": "benchmarks/benchmarks/tcbench/corpus.rs of the reference (corpus(), size_case_stressed)",
           "sizes_mib": SIZES_MIB, "layout": "column-major, first label stride 1", "cases": cases}
    with open(os.path.join(HERE, "tccg.json"), "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")
    print(f"{len(cases)} cases")


if __name__ == "__main__":
    main()
