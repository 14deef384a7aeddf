"""Writes tests/golden/known_answers.json: the hand-checkable answers the
reference's own tests pin, transcribed with their file:line, plus the
deterministic value sequence its C-ABI conformance suite uses.

The reference (Rust) cannot be built or run in this environment, so these are
the reference's known-answer tests read as text; the oracle and the GPU path
are both checked against them (tests/test_oracle.py, tests/test_gpu_parity.py).

Run: python tests/golden/make_golden.py
"""
import json
import os


def seq(n, seed, complex_):
    """The conformance suite's value sequence (crates/tprims-capi/tests/common/
    mod.rs:72-92): xorshift64 (13, 7, 17), multiples of 1/2048 in [-1, 1)."""
    mask = (1 << 64) - 1
    s = ((seed * 0x9E3779B97F4A7C15) & mask) | 1
    out = []

    def nxt():
        nonlocal s
        s ^= (s << 13) & mask
        s ^= s >> 7
        s ^= (s << 17) & mask
        return (s >> 52) / 2048.0 - 1.0

    for _ in range(n):
        re = nxt()
        im = nxt() if complex_ else 0.0
        out.append([re, im])
    return out


CASES = {
    # crates/tprims-capi/tests/tapp_conformance.rs:111-135
    "small_real_2x2": {
        "cite": "crates/tprims-capi/tests/tapp_conformance.rs:111-135",
        "a": {"ext": [2, 2], "str": [1, 2], "lab": [0, 2], "data": [1, 3, 2, 4]},
        "b": {"ext": [2, 2], "str": [1, 2], "lab": [2, 1], "data": [5, 7, 6, 8]},
        "d": {"ext": [2, 2], "str": [1, 2], "lab": [0, 1]},
        "alpha": [1, 0], "beta": [0, 0],
        "want": [[19, 0], [43, 0], [22, 0], [50, 0]],
        "dtypes": ["float32", "float64", "complex64", "complex128"],
    },
    # tapp_conformance.rs:88-108 (complex); real types keep only the real parts: 1*3 = 3
    "single_complex_product": {
        "cite": "crates/tprims-capi/tests/tapp_conformance.rs:88-108",
        "a": {"ext": [1, 1], "str": [1, 1], "lab": [0, 2], "data_c": [[1, 2]]},
        "b": {"ext": [1, 1], "str": [1, 1], "lab": [2, 1], "data_c": [[3, 4]]},
        "d": {"ext": [1, 1], "str": [1, 1], "lab": [0, 1]},
        "alpha": [1, 0], "beta": [0, 0],
        "want_complex": [[-5, 10]], "want_real": [[3, 0]],
        "dtypes": ["float32", "float64", "complex64", "complex128"],
    },
    # crates/tprims-capi/tests/c/standard_consumer.c:15-39
    "standard_consumer": {
        "cite": "crates/tprims-capi/tests/c/standard_consumer.c:15-39",
        "a": {"ext": [2, 3], "str": [1, 2], "lab": [105, 107], "data": [1, 2, 3, 4, 5, 6]},
        "b": {"ext": [3, 2], "str": [1, 3], "lab": [107, 106], "data": [1, 2, 3, 4, 5, 6]},
        "d": {"ext": [2, 2], "str": [1, 2], "lab": [105, 106]},
        "alpha": [1, 0], "beta": [0, 0],
        "want": [[22, 0], [28, 0], [49, 0], [64, 0]],
        "dtypes": ["float64"],
    },
    # crates/tprims-capi/src/lib.rs:44-85 (D = A * identity)
    "identity_product": {
        "cite": "crates/tprims-capi/src/lib.rs:44-85",
        "a": {"ext": [2, 2], "str": [1, 2], "lab": [105, 107], "data": [1, 2, 3, 4]},
        "b": {"ext": [2, 2], "str": [1, 2], "lab": [107, 106], "data": [1, 0, 0, 1]},
        "d": {"ext": [2, 2], "str": [1, 2], "lab": [105, 106]},
        "alpha": [1, 0], "beta": [0, 0],
        "want": [[1, 0], [2, 0], [3, 0], [4, 0]],
        "dtypes": ["float64"],
    },
}

# Scatter / fold unit tests of the planner.
SCATTERS = {
    "scatter_two_modes": {"cite": "crates/tprims-kernel/src/pack/scatter.rs:61-64",
                          "extents": [2, 3], "strides": [1, 10], "want": [0, 1, 10, 11, 20, 21]},
    "scatter_col_major": {"cite": "crates/tprims-kernel/src/pack/scatter.rs:293-297",
                          "extents": [2, 3], "strides": [1, 2], "want": [0, 1, 2, 3, 4, 5]},
    "scatter_permuted": {"cite": "crates/tprims-kernel/src/pack/scatter.rs:305-306",
                         "extents": [2, 3], "strides": [3, 1], "want": [0, 3, 1, 4, 2, 5]},
}

# Plans whose packed scatter vectors the reference's analysis tests pin.
PLANS = {
    # plan/analysis.rs:368-386: D[j] = sum_i A[i,i] B[i,j]; a_k = [0, 5, 10, 15]
    "diagonal_a_k": {"cite": "crates/tprims-contract/src/plan/analysis.rs:374-386",
                     "a": {"ext": [4, 4], "str": [1, 4], "lab": [0, 0]},
                     "b": {"ext": [4, 6], "str": [1, 4], "lab": [0, 1]},
                     "d": {"ext": [6], "str": [1], "lab": [1]},
                     "vector": "a_k", "want": [0, 5, 10, 15], "k": 4},
    # plan/analysis.rs:355-366: D[i,j] = sum_{k,r} A[i,k,r] B[k,j]; b_k prefix [0,1,2,3,4,0]
    "reduction_b_k": {"cite": "crates/tprims-contract/src/plan/analysis.rs:355-366",
                      "a": {"ext": [4, 5, 3], "str": [1, 4, 20], "lab": [0, 2, 7]},
                      "b": {"ext": [5, 6], "str": [1, 5], "lab": [2, 1]},
                      "d": {"ext": [4, 6], "str": [1, 4], "lab": [0, 1]},
                      "vector": "b_k", "want_prefix": [0, 1, 2, 3, 4, 0], "k": 15},
    # plan/analysis.rs:329-340: plain matmul folds to one GEMM (4, 6, 5, batch 1)
    "plain_matmul": {"cite": "crates/tprims-contract/src/plan/analysis.rs:329-340",
                     "a": {"ext": [4, 5], "str": [1, 4], "lab": [0, 2]},
                     "b": {"ext": [5, 6], "str": [1, 5], "lab": [2, 1]},
                     "d": {"ext": [4, 6], "str": [1, 4], "lab": [0, 1]},
                     "mnkb": [4, 6, 5, 1], "pure_gemm": True},
    # plan/analysis.rs:342-353: a and b adjacent in A and D fold into one M axis of 12
    "adjacent_fold": {"cite": "crates/tprims-contract/src/plan/analysis.rs:342-353",
                      "a": {"ext": [4, 3, 5], "str": [1, 4, 12], "lab": [0, 1, 3]},
                      "b": {"ext": [5, 6], "str": [1, 5], "lab": [3, 2]},
                      "d": {"ext": [4, 3, 6], "str": [1, 4, 12], "lab": [0, 1, 2]},
                      "mnkb": [12, 6, 5, 1], "pure_gemm": True, "m_axes": 1},
    # plan/analysis.rs:355-366 (hadamard): D[b,i,j] = A[b,i,k] B[b,k,j]
    "hadamard": {"cite": "crates/tprims-contract/src/plan/analysis.rs:342-366",
                 "a": {"ext": [2, 4, 5], "str": [1, 2, 8], "lab": [9, 0, 3]},
                 "b": {"ext": [2, 5, 6], "str": [1, 2, 10], "lab": [9, 3, 1]},
                 "d": {"ext": [2, 4, 6], "str": [1, 2, 8], "lab": [9, 0, 1]},
                 "mnkb": [4, 6, 5, 2], "pure_gemm": False},
}


def main():
    out = {"cases": CASES, "scatters": SCATTERS, "plans": PLANS,
           "seq": {"cite": "crates/tprims-capi/tests/common/mod.rs:72-92",
                   "seed_1_real_8": seq(8, 1, False), "seed_2_complex_4": seq(4, 2, True)}}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_answers.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    main()
