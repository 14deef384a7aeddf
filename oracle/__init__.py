"""ctypes loader of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arms as the checker. The library under tensoralgebra-rs_b200/ never imports this.

``label_contract`` restates the reference's brute-force oracle
(crates/tprims-testkit/src/oracle.rs:92-204) with extended-precision
accumulation; ``packed_contract`` restates the reference's packed CPU driver
(see the header of oracle.c for the file:line list). Parity of the restatement
is pinned against the golden vectors of the reference's own tests
(tests/golden/, tests/test_oracle.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


def _cpu_flags() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            return f.read()
    except OSError:
        return ""


def _cpu_has_avx2() -> bool:
    txt = _cpu_flags()
    return " avx2" in txt and " fma" in txt


def _cpu_has_avx512() -> bool:
    txt = _cpu_flags()
    return all(f" {f}" in txt for f in ("avx512f", "avx512dq", "avx512bw", "avx512vl", "avx512cd"))


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    names = ((["liboracle_v4.so"] if _cpu_has_avx512() else []) + (["liboracle_v3.so"] if _cpu_has_avx2() else [])
             + ["liboracle_base.so"])
    for n in names:
        p = os.path.join(_HERE, n)
        if os.path.exists(p):
            return C.CDLL(p)
    build()
    return C.CDLL(os.path.join(_HERE, names[0]))


_lib = _load()


class _Operand(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("rank", C.c_int),
        ("ext", C.POINTER(C.c_int64)),
        ("str", C.POINTER(C.c_int64)),
        ("lab", C.POINTER(C.c_int64)),
        ("conj", C.c_int),
    ]


_lib.oracle_label_contract.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(_Operand),
                                       C.POINTER(_Operand), C.POINTER(C.c_double), C.POINTER(_Operand),
                                       C.POINTER(_Operand)]
_lib.oracle_packed_contract.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(_Operand), C.POINTER(_Operand),
                                        C.POINTER(C.c_double), C.POINTER(_Operand), C.POINTER(_Operand), C.c_int]
_lib.oracle_layout_sums.argtypes = [C.c_int, C.POINTER(_Operand), C.POINTER(C.c_double), C.POINTER(C.c_double)]

_DT = {"float32": 0, "float64": 1, "complex64": 2, "complex128": 3}


def dtype_code(x: np.ndarray) -> int:
    return _DT[str(x.dtype)]


class View:
    """An operand for the oracle: the backing array, the element offset of index
    (0,..,0), extents, element strides, labels and conjugation."""

    def __init__(self, buf: np.ndarray, extents, strides, labels, offset: int = 0, conj: bool = False):
        self.buf = buf
        self.extents = [int(e) for e in extents]
        self.strides = [int(s) for s in strides]
        self.labels = [int(l) for l in labels]
        self.offset = int(offset)
        self.conj = bool(conj)

    @staticmethod
    def of(arr: np.ndarray, labels, conj: bool = False) -> "View":
        it = arr.itemsize
        base = arr
        while base.base is not None and isinstance(base.base, np.ndarray):
            base = base.base
        return View(arr, arr.shape, [s // it for s in arr.strides], labels, 0, conj)

    def _struct(self, keep):
        n = len(self.extents)
        ext = (C.c_int64 * max(n, 1))(*self.extents)
        st = (C.c_int64 * max(n, 1))(*self.strides)
        lab = (C.c_int64 * max(n, 1))(*self.labels)
        keep += [ext, st, lab]
        ptr = self.buf.ctypes.data + self.offset * self.buf.itemsize
        return _Operand(ptr, n, ext, st, lab, 1 if self.conj else 0)


def _scalar(v, complex_: bool):
    v = complex(v)
    return (C.c_double * 2)(v.real, v.imag if complex_ else 0.0)


def label_contract(alpha, a: View, b: View, beta, c, d: View, out_f64: bool = False) -> None:
    """Brute-force oracle; writes into d.buf (as float64/complex128 when out_f64)."""
    keep = []
    dt = dtype_code(a.buf)
    cplx = dt >= 2
    r = _lib.oracle_label_contract(dt, 1 if out_f64 else 0, _scalar(alpha, cplx), C.byref(a._struct(keep)),
                                   C.byref(b._struct(keep)), _scalar(beta, cplx),
                                   C.byref(c._struct(keep)) if c is not None else None, C.byref(d._struct(keep)))
    if r != 0:
        raise ValueError(f"oracle refused the labels (code {r})")


def packed_contract(alpha, a: View, b: View, beta, c, d: View, nthreads: int = 0) -> None:
    """The restated packed CPU driver (OpenMP over the static output grid)."""
    keep = []
    dt = dtype_code(a.buf)
    cplx = dt >= 2
    r = _lib.oracle_packed_contract(dt, _scalar(alpha, cplx), C.byref(a._struct(keep)), C.byref(b._struct(keep)),
                                    _scalar(beta, cplx), C.byref(c._struct(keep)) if c is not None else None,
                                    C.byref(d._struct(keep)), int(nthreads))
    if r != 0:
        raise ValueError(f"packed oracle refused the problem (code {r})")


def layout_sums(x: View):
    keep = []
    s, q = C.c_double(), C.c_double()
    _lib.oracle_layout_sums(dtype_code(x.buf), C.byref(x._struct(keep)), C.byref(s), C.byref(q))
    return s.value, q.value


def rel_frobenius(got: np.ndarray, want: np.ndarray) -> float:
    """Relative Frobenius error ||got - want|| / ||want|| in float64 (complex128)."""
    g = got.astype(np.complex128).ravel()
    w = want.astype(np.complex128).ravel()
    num = np.linalg.norm(g - w)
    den = np.linalg.norm(w)
    return float(num / den) if den > 0 else float(num)
