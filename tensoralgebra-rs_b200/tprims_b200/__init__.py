"""Python host mirror of the tprims contraction interface over libtprims_b200.

The library is a C ABI (``include/tprims_b200.h``); this module binds it with
ctypes and mirrors the reference's two front ends so that tests and callers
read like the reference's own:

* the TAPP objects (``Handle``, ``Executor``, ``TensorInfo``, ``TensorProduct``)
  of ``crates/tprims-capi/src/{handle,executor,tensor_info,product,execute}.rs``;
* the Rust API of ``crates/tprims-contract``: ``Problem.from_labels``
  (``api/problem.rs:370``), ``Problem.from_dot_general`` (``api/problem.rs:396``),
  ``Plan`` with ``execute_into`` / ``execute_into_accum`` (``plan/mod.rs:271``,
  ``:309``), ``Plan.report`` (``plan/mod.rs:237``) and ``contract_batched``
  (``batch.rs:125``).

Operands are numpy arrays (host memory, staged by the library) or torch CUDA
tensors (device memory, used in place); strides are taken from the array. There
is no Python or CPU fallback: every contraction runs in the CUDA library, and
importing this module fails if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libtprims_b200.so")
if not os.path.exists(_LIB_PATH):
    raise ImportError(
        f"libtprims_b200.so is not built ({_LIB_PATH}); run `make -C tensoralgebra-rs_b200` "
        "(or __graft_entry__.build()) first"
    )
lib = C.CDLL(_LIB_PATH)

# --------------------------------------------------------------- constants
F32, F64, C32, C64, F16, BF16 = 0, 1, 2, 3, 4, 5
DEFAULT_PREC = -1
IDENTITY, CONJUGATE = 0, 1

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_SHAPE = 2
ERR_DTYPE = 3
ERR_DEVICE = 4
ERR_ALIASED = 6
BUSY = 9
ERR_PANIC = 12
ERR_INTERNAL = 13
ERR_LABELS = 14
ERR_UNSUPPORTED = 15

PREC_PLAIN, PREC_BF16X3, PREC_BF16X6, PREC_OZAKI_INT8 = 0, 1, 2, 3

ABI_SYMBOLS = [
    "TAPP_check_success", "TAPP_explain_error", "TAPP_attr_set", "TAPP_attr_get", "TAPP_attr_clear",
    "TAPP_create_handle", "TAPP_destroy_handle", "TAPP_create_executor", "TAPP_destroy_executor",
    "TAPP_destroy_status", "TAPP_create_tensor_info", "TAPP_destroy_tensor_info", "TAPP_get_nmodes",
    "TAPP_set_nmodes", "TAPP_get_extents", "TAPP_set_extents", "TAPP_get_strides", "TAPP_set_strides",
    "TAPP_create_tensor_product", "TAPP_destroy_tensor_product", "TAPP_execute_product",
    "TAPP_execute_batched_product", "tprims_tensor_borrow_versioned", "tprims_tensor_borrow_raw",
    "tprims_last_error", "tprims_abi_version", "tprims_has_part", "TAPP_implementation_name",
    "TAPP_implementation_version", "tprims_tapp_executor_create_rayon", "tprims_tapp_executor_set_budget",
    "tprims_tapp_executor_get_threads", "tprims_b200_executor_create", "tprims_b200_executor_stream",
    "tprims_b200_executor_set_sync", "tprims_b200_executor_synchronize", "tprims_b200_product_set_precision",
    "tprims_b200_product_set_tile", "tprims_b200_product_report", "tprims_b200_product_from_dot_general",
    "tprims_b200_execute_product_dlpack", "tprims_b200_contract_batched", "tprims_b200_product_vjp",
    "tprims_b200_product_scatter", "tprims_b200_executor_set_profiling", "tprims_b200_executor_kernel_times",
    "tprims_b200_executor_set_grouping", "tprims_b200_executor_set_streaming", "tprims_b200_executor_set_workspace_limit",
    "tprims_b200_executor_selftest_wait", "tprims_b200_executor_probe_peak",
    "tprims_b200_execute_product_noalloc", "tprims_b200_product_set_split_k", "tprims_b200_product_set_autotune",
    "tprims_b200_executor_save_tuning", "tprims_b200_executor_load_tuning", "tprims_b200_executor_clear_tuning",
    "tprims_b200_executor_tuning", "tprims_b200_network_create", "tprims_b200_network_destroy",
    "tprims_b200_network_set_precision", "tprims_b200_network_set_autotune", "tprims_b200_network_workspace_size",
    "tprims_b200_network_report", "tprims_b200_network_execute", "tprims_b200_networks_execute",
    "tprims_b200_device_allocations", "tprims_b200_executor_inject_launch_failure", "tprims_b200_product_check_raw",
    "tprims_b200_contract_batched_sharded", "tprims_b200_balance", "tprims_b200_tuning_file_info",
]

_i64p = C.POINTER(C.c_int64)
_vp = C.c_void_p
_ip = C.c_ssize_t  # intptr_t

lib.TAPP_check_success.restype = C.c_bool
lib.TAPP_check_success.argtypes = [C.c_int]
lib.TAPP_explain_error.restype = C.c_size_t
lib.TAPP_explain_error.argtypes = [C.c_int, C.c_size_t, C.c_char_p]
lib.tprims_last_error.restype = C.c_char_p
lib.tprims_abi_version.restype = C.c_uint32
lib.tprims_has_part.restype = C.c_int32
lib.tprims_has_part.argtypes = [C.c_char_p]
lib.TAPP_implementation_name.restype = C.c_char_p
lib.TAPP_implementation_version.restype = C.c_char_p
lib.TAPP_create_handle.argtypes = [C.POINTER(_ip)]
lib.TAPP_destroy_handle.argtypes = [_ip]
lib.TAPP_create_executor.argtypes = [C.POINTER(_ip)]
lib.TAPP_destroy_executor.argtypes = [_ip]
lib.TAPP_destroy_status.argtypes = [_ip]
lib.TAPP_attr_set.argtypes = [_ip, C.c_int, _vp]
lib.TAPP_attr_get.argtypes = [_ip, C.c_int, C.POINTER(_vp)]
lib.TAPP_attr_clear.argtypes = [_ip, C.c_int]
lib.tprims_b200_executor_create.argtypes = [C.POINTER(_ip), C.c_int, C.c_size_t]
lib.tprims_b200_executor_stream.argtypes = [_ip, C.POINTER(C.c_size_t)]
lib.tprims_b200_executor_set_sync.argtypes = [_ip, C.c_int]
lib.tprims_b200_executor_synchronize.argtypes = [_ip]
lib.tprims_b200_executor_set_profiling.argtypes = [_ip, C.c_int]
lib.tprims_b200_executor_set_grouping.argtypes = [_ip, C.c_int]
lib.tprims_b200_executor_set_streaming.argtypes = [_ip, C.c_int]
lib.tprims_b200_executor_set_workspace_limit.argtypes = [_ip, C.c_size_t]
lib.tprims_b200_executor_selftest_wait.argtypes = [_ip, C.c_uint64]
lib.tprims_b200_executor_probe_peak.argtypes = [_ip, C.c_int, C.POINTER(C.c_double)]
lib.tprims_b200_execute_product_noalloc.argtypes = [_ip, C.c_size_t, _vp, _vp, _vp, _vp, _vp, _vp]
lib.tprims_b200_executor_kernel_times.argtypes = [_ip, C.c_char_p, C.c_size_t, C.c_int]
lib.tprims_b200_executor_kernel_times.restype = C.c_size_t
lib.tprims_tapp_executor_create_rayon.argtypes = [C.POINTER(_ip), C.c_size_t, _vp]
lib.tprims_tapp_executor_set_budget.argtypes = [_ip, C.c_size_t]
lib.tprims_tapp_executor_get_threads.argtypes = [_ip, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
lib.TAPP_create_tensor_info.argtypes = [C.POINTER(_ip), C.c_int, C.c_int, _i64p, _i64p]
lib.TAPP_destroy_tensor_info.argtypes = [_ip]
lib.TAPP_get_nmodes.argtypes = [_ip]
lib.TAPP_get_nmodes.restype = C.c_int
lib.TAPP_set_nmodes.argtypes = [_ip, C.c_int]
lib.TAPP_get_extents.argtypes = [_ip, _i64p]
lib.TAPP_get_extents.restype = None
lib.TAPP_set_extents.argtypes = [_ip, _i64p]
lib.TAPP_get_strides.argtypes = [_ip, _i64p]
lib.TAPP_get_strides.restype = None
lib.TAPP_set_strides.argtypes = [_ip, _i64p]
lib.TAPP_create_tensor_product.argtypes = [
    C.POINTER(_ip), _ip, C.c_int, _ip, _i64p, C.c_int, _ip, _i64p, C.c_int, _ip, _i64p, C.c_int, _ip, _i64p, C.c_int
]
lib.TAPP_destroy_tensor_product.argtypes = [_ip]
lib.TAPP_execute_product.argtypes = [_ip, _ip, C.POINTER(_ip), _vp, _vp, _vp, _vp, _vp, _vp]
lib.TAPP_execute_batched_product.argtypes = [
    _ip, _ip, C.POINTER(_ip), C.c_int, _vp, C.POINTER(_vp), C.POINTER(_vp), _vp, C.POINTER(_vp), C.POINTER(_vp)
]
lib.tprims_b200_product_set_precision.argtypes = [_ip, C.c_int, C.c_int]
lib.tprims_b200_product_set_tile.argtypes = [_ip, C.c_int]
lib.tprims_b200_product_set_split_k.argtypes = [_ip, C.c_int]
lib.tprims_b200_product_check_raw.argtypes = [_ip, _vp, _vp, _vp, _vp]
lib.tprims_b200_product_set_autotune.argtypes = [_ip, C.c_int]
lib.tprims_b200_executor_save_tuning.argtypes = [_ip, C.c_char_p]
lib.tprims_b200_executor_load_tuning.argtypes = [_ip, C.c_char_p]
lib.tprims_b200_executor_clear_tuning.argtypes = [_ip]
lib.tprims_b200_tuning_file_info.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.c_char_p, C.c_size_t,
                                             C.POINTER(C.c_int), C.POINTER(C.c_int)]
lib.tprims_b200_executor_tuning.argtypes = [_ip, C.c_char_p, C.c_size_t]
lib.tprims_b200_executor_tuning.restype = C.c_size_t
lib.tprims_b200_executor_inject_launch_failure.argtypes = [_ip, C.c_int]
lib.tprims_b200_device_allocations.argtypes = []
lib.tprims_b200_device_allocations.restype = C.c_uint64
_i64pp = C.POINTER(_i64p)
lib.tprims_b200_network_create.argtypes = [C.POINTER(_ip), C.c_int, C.c_int, C.POINTER(C.c_int), _i64pp, _i64pp,
                                           _i64pp, C.POINTER(C.c_int), C.c_int, _i64p, _i64p, _i64p, C.c_int,
                                           C.POINTER(C.c_int)]
lib.tprims_b200_network_destroy.argtypes = [_ip]
lib.tprims_b200_network_set_precision.argtypes = [_ip, C.c_int, C.c_int]
lib.tprims_b200_network_set_autotune.argtypes = [_ip, C.c_int]
lib.tprims_b200_network_workspace_size.argtypes = [_ip, C.POINTER(C.c_size_t)]
lib.tprims_b200_network_report.argtypes = [_ip, C.c_char_p, C.c_size_t]
lib.tprims_b200_network_report.restype = C.c_size_t
lib.tprims_b200_network_execute.argtypes = [_ip, _ip, _vp, C.POINTER(_vp), _vp, _vp, _vp]
lib.tprims_b200_networks_execute.argtypes = [_ip, C.c_int, C.POINTER(_ip), C.POINTER(_vp), C.POINTER(C.POINTER(_vp)),
                                             C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)]
lib.tprims_b200_product_report.argtypes = [_ip, C.c_char_p, C.c_size_t]
lib.tprims_b200_product_report.restype = C.c_size_t
lib.tprims_b200_product_from_dot_general.argtypes = [
    C.POINTER(_ip), C.c_int, C.c_int, _i64p, _i64p, C.c_int, C.c_int, _i64p, _i64p, C.c_int, C.c_int, _i64p, _i64p,
    C.c_int, C.c_int, _i64p, _i64p, C.c_int, _i64p, _i64p,
]
lib.tprims_b200_product_vjp.argtypes = [_ip, _ip, _vp, _vp, _vp, _vp, _vp, _vp]


class BatchItem(C.Structure):
    """``tprims_b200_batch_item``: one entry of ``contract_batched``."""

    _fields_ = [("plan", _ip), ("alpha", _vp), ("A", _vp), ("B", _vp), ("beta", _vp), ("C", _vp), ("D", _vp)]


lib.tprims_b200_contract_batched.argtypes = [_ip, C.c_int, C.POINTER(BatchItem)]
lib.tprims_b200_contract_batched_sharded.argtypes = [C.POINTER(_ip), C.c_int, C.c_int, C.POINTER(BatchItem)]
lib.tprims_b200_balance.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int,
                                    C.POINTER(C.c_int), C.POINTER(C.c_int)]


class TprimsError(RuntimeError):
    """A non-zero ``tprims_status`` with the library's last-error message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"tprims status {status}: {message}")
        self.status = status
        self.message = message


def last_error() -> str:
    return (lib.tprims_last_error() or b"").decode()


def check(status: int) -> None:
    if status != OK:
        raise TprimsError(status, last_error())


def explain(status: int) -> str:
    n = lib.TAPP_explain_error(status, 0, None)
    buf = C.create_string_buffer(n + 1)
    lib.TAPP_explain_error(status, n + 1, buf)
    return buf.value.decode()


def _arr(vals: Sequence[int]):
    vals = list(vals)
    if not vals:
        return None
    return (C.c_int64 * len(vals))(*[int(v) for v in vals])


# ------------------------------------------------------------- dtype helpers
_NP_NAMES = {F32: "float32", F64: "float64", C32: "complex64", C64: "complex128"}
_REAL_NP = {F32: "float32", F64: "float64", C32: "float32", C64: "float64"}
DTYPE_NAMES = {F32: "f32", F64: "f64", C32: "c32", C64: "c64"}


def dtype_of(x) -> int:
    """TAPP datatype of a numpy array or torch tensor."""
    name = str(x.dtype).replace("torch.", "")
    for k, v in _NP_NAMES.items():
        if v == name:
            return k
    raise TprimsError(ERR_DTYPE, f"unsupported dtype {x.dtype}")


def scalar_bytes(dtype: int, value) -> C.Array:
    """The bytes of a scalar of the plan's element type (alpha, beta)."""
    import numpy as np

    if dtype in (F32, F64):
        value = complex(value).real  # the imaginary part of a real scalar is dropped
    v = np.array([value], dtype=_NP_NAMES[dtype])
    buf = (C.c_char * v.nbytes).from_buffer_copy(v.tobytes())
    return buf


def layout_of(x):
    """(origin pointer, extents, strides in elements) of a numpy array / torch tensor."""
    try:
        import torch

        if isinstance(x, torch.Tensor):
            return x.data_ptr(), list(x.shape), list(x.stride())
    except ImportError:  # pragma: no cover
        pass
    import numpy as np

    if isinstance(x, np.ndarray):
        it = x.itemsize
        return x.ctypes.data, list(x.shape), [s // it for s in x.strides]
    if isinstance(x, int):
        raise TprimsError(ERR_INVALID_ARGUMENT, "a raw pointer needs explicit extents and strides")
    raise TprimsError(ERR_INVALID_ARGUMENT, f"unsupported operand type {type(x)}")


def ptr_of(x) -> Optional[int]:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return layout_of(x)[0]


# ------------------------------------------------------------------ TAPP layer
class Handle:
    def __init__(self):
        h = _ip(0)
        check(lib.TAPP_create_handle(C.byref(h)))
        self.h = h.value

    def close(self):
        if self.h:
            check(lib.TAPP_destroy_handle(self.h))
            self.h = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Executor:
    """A CUDA executor: one stream on one device plus a reusable workspace.

    ``device=None`` uses the current device; ``stream`` is an integer
    ``cudaStream_t`` (0: the executor creates its own). ``sync=True`` is the
    TAPP contract (every execute returns after the work is done)."""

    def __init__(self, device: Optional[int] = None, stream: int = 0, sync: bool = True,
                 tuning: Optional[str] = None):
        h = _ip(0)
        check(lib.tprims_b200_executor_create(C.byref(h), -1 if device is None else int(device), int(stream)))
        self.h = h.value
        if not sync:
            check(lib.tprims_b200_executor_set_sync(self.h, 0))
        if tuning is not None:
            self.load_tuning(tuning)

    def save_tuning(self, path: str):
        """Write the autotuner cache to ``path`` (versioned text)."""
        check(lib.tprims_b200_executor_save_tuning(self.h, os.fsencode(path)))

    def load_tuning(self, path: str):
        """Add the entries of a cache file written on the same kind of device."""
        check(lib.tprims_b200_executor_load_tuning(self.h, os.fsencode(path)))

    def clear_tuning(self):
        check(lib.tprims_b200_executor_clear_tuning(self.h))

    def tuning(self) -> dict:
        """The autotuner cache: {"single": {signature: entry}, "list": {...}}."""
        n = lib.tprims_b200_executor_tuning(self.h, None, 0)
        buf = C.create_string_buffer(n + 64)
        lib.tprims_b200_executor_tuning(self.h, buf, n + 64)
        return json.loads(buf.value.decode())

    @property
    def stream(self) -> int:
        s = C.c_size_t(0)
        check(lib.tprims_b200_executor_stream(self.h, C.byref(s)))
        return s.value

    def set_sync(self, sync: bool):
        check(lib.tprims_b200_executor_set_sync(self.h, 1 if sync else 0))

    def synchronize(self):
        check(lib.tprims_b200_executor_synchronize(self.h))

    def set_grouping(self, on: bool):
        """Grouped persistent launches (cached in CUDA graphs) for lists; off = one launch per item."""
        check(lib.tprims_b200_executor_set_grouping(self.h, 1 if on else 0))

    def set_streaming(self, on: bool):
        """Streamed execution of large host-operand contractions (chunked copies
        overlapping the kernels); off = copy in, run, copy out."""
        check(lib.tprims_b200_executor_set_streaming(self.h, 1 if on else 0))

    def set_workspace_limit(self, nbytes: int):
        """Cap the workspace arena (0 = no cap); larger requests are refused."""
        check(lib.tprims_b200_executor_set_workspace_limit(self.h, int(nbytes)))

    def inject_launch_failure(self, after: int):
        """Refuse the launch `after` launches from now (host-side fault injection; -1: off)."""
        check(lib.tprims_b200_executor_inject_launch_failure(self.h, int(after)))

    def selftest_wait(self, limit_ns: int) -> int:
        """Run the bounded-wait self-test kernel; returns the status it produced."""
        return lib.tprims_b200_executor_selftest_wait(self.h, int(limit_ns))

    def probe_peak(self, which: int) -> float:
        """Measured TFLOP/s (TOP/s) of the FP64 DMMA (0), FP32 FFMA (1), INT8
        tcgen05 (2) or BF16 tcgen05 (3) pipe on this device."""
        v = C.c_double(0)
        check(lib.tprims_b200_executor_probe_peak(self.h, int(which), C.byref(v)))
        return v.value

    def set_profiling(self, on: bool):
        """Record CUDA events around every kernel launch on this executor."""
        check(lib.tprims_b200_executor_set_profiling(self.h, 1 if on else 0))

    def kernel_times(self, reset: bool = False) -> dict:
        """{kernel family: {"ms": total ms, "launches": n}} (drains the stream)."""
        n = lib.tprims_b200_executor_kernel_times(self.h, None, 0, 0)
        buf = C.create_string_buffer(n + 64)
        lib.tprims_b200_executor_kernel_times(self.h, buf, n + 64, 1 if reset else 0)
        return json.loads(buf.value.decode() or "{}")

    def close(self):
        if self.h:
            check(lib.TAPP_destroy_executor(self.h))
            self.h = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TensorInfo:
    def __init__(self, dtype: int, extents: Sequence[int], strides: Sequence[int]):
        h = _ip(0)
        check(lib.TAPP_create_tensor_info(C.byref(h), int(dtype), len(extents), _arr(extents), _arr(strides)))
        self.h = h.value
        self.dtype = dtype

    @property
    def nmodes(self) -> int:
        return lib.TAPP_get_nmodes(self.h)

    def extents(self):
        n = self.nmodes
        a = (C.c_int64 * max(n, 1))()
        lib.TAPP_get_extents(self.h, a)
        return list(a)[:n]

    def strides(self):
        n = self.nmodes
        a = (C.c_int64 * max(n, 1))()
        lib.TAPP_get_strides(self.h, a)
        return list(a)[:n]

    def close(self):
        if self.h:
            check(lib.TAPP_destroy_tensor_info(self.h))
            self.h = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TensorProduct:
    """A planned product (``TAPP_create_tensor_product``). Owns no data."""

    def __init__(self, h: int):
        self.h = h

    @classmethod
    def create(cls, handle: Handle, a, b, c, d, prec: int = DEFAULT_PREC) -> "TensorProduct":
        """a, b, c, d: (op, TensorInfo, labels) triples."""
        out = _ip(0)
        args = []
        for op, info, labels in (a, b, c, d):
            args += [int(op), info.h, _arr(labels)]
        check(lib.TAPP_create_tensor_product(C.byref(out), handle.h, *args, int(prec)))
        p = cls(out.value)
        p.dtype = a[1].dtype
        return p

    def set_precision(self, scheme: int, slices: int = 0):
        check(lib.tprims_b200_product_set_precision(self.h, int(scheme), int(slices)))

    def set_kernel(self, kernel_id: int):
        check(lib.tprims_b200_product_set_tile(self.h, int(kernel_id)))

    def set_split_k(self, splits: int):
        """0: chosen; 1: never split K; 2..64: that many K chunks."""
        check(lib.tprims_b200_product_set_split_k(self.h, int(splits)))

    def set_autotune(self, on: bool):
        check(lib.tprims_b200_product_set_autotune(self.h, 1 if on else 0))

    def report(self) -> dict:
        n = lib.tprims_b200_product_report(self.h, None, 0)
        buf = C.create_string_buffer(n + 1)
        lib.tprims_b200_product_report(self.h, buf, n + 1)
        return json.loads(buf.value.decode())

    def execute(self, exec_: Optional[Executor], alpha, a, b, beta, c, d, status: bool = False) -> int:
        """``TAPP_execute_product`` on raw pointers / arrays. Returns the status."""
        al = scalar_bytes(self.dtype, alpha)
        be = scalar_bytes(self.dtype, beta)
        st = _ip(-1)
        return lib.TAPP_execute_product(
            self.h, exec_.h if exec_ else 0, C.byref(st) if status else None, al, ptr_of(a), ptr_of(b), be,
            ptr_of(c), ptr_of(d),
        )

    def execute_noalloc(self, stream: int, alpha, a, b, beta, c, d) -> int:
        """``tprims_b200_execute_product_noalloc``: the split-precision path with
        its scratch in the library's fixed device array, for callers that cannot
        allocate device memory. Device operands only; returns after ``stream``
        has drained. Returns the status."""
        al = scalar_bytes(self.dtype, alpha)
        be = scalar_bytes(self.dtype, beta)
        return lib.tprims_b200_execute_product_noalloc(self.h, int(stream), al, ptr_of(a), ptr_of(b), be,
                                                       ptr_of(c), ptr_of(d))

    def execute_batched(self, exec_: Optional[Executor], alpha, As, Bs, beta, Cs, Ds) -> int:
        n = len(As)
        al = scalar_bytes(self.dtype, alpha)
        be = scalar_bytes(self.dtype, beta)
        arr = lambda xs: (_vp * max(n, 1))(*[ptr_of(x) for x in xs]) if xs is not None else None
        return lib.TAPP_execute_batched_product(
            self.h, exec_.h if exec_ else 0, None, n, al, arr(As), arr(Bs), be, arr(Cs), arr(Ds)
        )

    def vjp(self, exec_: Optional[Executor], alpha, a, b, dd, da, db) -> int:
        al = scalar_bytes(self.dtype, alpha)
        return lib.tprims_b200_product_vjp(
            self.h, exec_.h if exec_ else 0, al, ptr_of(a), ptr_of(b), ptr_of(dd), ptr_of(da), ptr_of(db)
        )

    def close(self):
        if self.h:
            check(lib.TAPP_destroy_tensor_product(self.h))
            self.h = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ Rust API mirror
@dataclass
class LayoutSpec:
    """Extents and signed element strides (``api/problem.rs`` LayoutSpec)."""

    dims: Sequence[int]
    strides: Sequence[int]

    @staticmethod
    def col_major(dims: Sequence[int]) -> "LayoutSpec":
        s, acc = [], 1
        for d in dims:
            s.append(acc)
            acc *= max(int(d), 1)
        return LayoutSpec(list(dims), s)

    @staticmethod
    def row_major(dims: Sequence[int]) -> "LayoutSpec":
        s, acc = [0] * len(dims), 1
        for k in reversed(range(len(dims))):
            s[k] = acc
            acc *= max(int(dims[k]), 1)
        return LayoutSpec(list(dims), s)


@dataclass
class OperandSpec:
    layout: LayoutSpec
    conj: bool = False


@dataclass
class DotGeneral:
    """Contracted and batch axis lists of A and B (``api/dot_general.rs``)."""

    lhs_contract: Sequence[int]
    rhs_contract: Sequence[int]
    lhs_batch: Sequence[int] = ()
    rhs_batch: Sequence[int] = ()


@dataclass
class PlanConfig:
    """``plan/config.rs`` PlanConfig, with the B200 knobs: the precision scheme
    (plain / bf16x3 / bf16x6 / ozaki-int8), optional tile and split-K pins, and
    the autotuner switch (tile family and split-K measured on first execution
    per executor and cached by Problem signature)."""

    precision: int = PREC_PLAIN
    ozaki_slices: int = 0
    kernel: int = 0
    split_k: int = 0
    autotune: bool = False

    @staticmethod
    def packed() -> "PlanConfig":
        """``PlanConfig::packed()`` (plan/config.rs:134): the packed strategy,
        which is the only strategy here, in drop-in precision."""
        return PlanConfig()


class Problem:
    """A validated problem: built through ``from_labels`` or ``from_dot_general``.

    On the C side a problem and its plan are one object (a TAPP product); this
    class keeps the description and creates that object in ``Plan``."""

    def __init__(self, kind, dtype, args):
        self.kind, self.dtype, self.args = kind, dtype, args

    @staticmethod
    def from_labels(dtype: int, a: OperandSpec, b: OperandSpec, d: OperandSpec, la, lb, ld,
                    c: Optional[OperandSpec] = None, lc=None) -> "Problem":
        return Problem("labels", dtype, (a, b, c, d, la, lb, lc, ld))

    @staticmethod
    def from_dot_general(dtype: int, a: OperandSpec, b: OperandSpec, d: OperandSpec, dot: DotGeneral) -> "Problem":
        return Problem("dot_general", dtype, (a, b, d, dot))


class Plan:
    """``Plan::new(&problem, &config)``: lowering, folding and scatter vectors
    happen here, once; device copies are made on first execution."""

    def __init__(self, problem: Problem, config: PlanConfig = PlanConfig()):
        self.problem = problem
        self.dtype = problem.dtype
        if problem.kind == "dot_general":
            a, b, d, dot = problem.args
            out = _ip(0)
            check(lib.tprims_b200_product_from_dot_general(
                C.byref(out), int(problem.dtype),
                len(a.layout.dims), _arr(a.layout.dims), _arr(a.layout.strides), CONJUGATE if a.conj else IDENTITY,
                len(b.layout.dims), _arr(b.layout.dims), _arr(b.layout.strides), CONJUGATE if b.conj else IDENTITY,
                len(d.layout.dims), _arr(d.layout.dims), _arr(d.layout.strides), CONJUGATE if d.conj else IDENTITY,
                len(dot.lhs_contract), _arr(dot.lhs_contract), _arr(dot.rhs_contract),
                len(dot.lhs_batch), _arr(dot.lhs_batch), _arr(dot.rhs_batch)))
            self.product = TensorProduct(out.value)
            self.product.dtype = problem.dtype
        else:
            a, b, c, d, la, lb, lc, ld = problem.args
            handle = Handle()
            infos = []
            for spec in (a, b, c if c is not None else d, d):
                infos.append(TensorInfo(problem.dtype, spec.layout.dims, spec.layout.strides))
            ops = [CONJUGATE if s.conj else IDENTITY for s in (a, b, c if c is not None else d, d)]
            self.product = TensorProduct.create(
                handle, (ops[0], infos[0], la), (ops[1], infos[1], lb),
                (ops[2], infos[2], lc if lc is not None else ld), (ops[3], infos[3], ld))
        if config.precision != PREC_PLAIN:
            self.product.set_precision(config.precision, config.ozaki_slices)
        if config.kernel:
            self.product.set_kernel(config.kernel)
        if config.split_k:
            self.product.set_split_k(config.split_k)
        if config.autotune:
            self.product.set_autotune(True)

    def report(self) -> dict:
        return self.product.report()

    def check_raw(self, a, b, c, d):
        """``Plan::check_raw``: the aliasing preflight from the origins alone
        (nothing is read; None is absent). Raises TprimsError(ERR_ALIASED)."""
        check(lib.tprims_b200_product_check_raw(self.product.h, ptr_of(a), ptr_of(b), ptr_of(c), ptr_of(d)))

    def execute_raw(self, exec_: Optional[Executor], alpha, a, b, beta, c, d):
        """``Plan::execute_raw``: check_raw, then D = op_D(alpha AB + beta op_C(C))
        on raw origins (C may be D itself for an in-place update)."""
        self.check_raw(a, b, c, d)
        check(self.product.execute(exec_, alpha, a, b, beta, c, d))

    def execute_into(self, exec_: Optional[Executor], alpha, a, b, d):
        """The overwrite form: D = op_D(alpha * op_A(A) op_B(B)); D's old value is not read."""
        check(self.product.execute(exec_, alpha, a, b, 0, None, d))

    def execute_into_accum(self, exec_: Optional[Executor], alpha, a, b, beta, d, c=None):
        """D = op_D(alpha * AB + beta * op_C(C)); without ``c`` the source is D itself."""
        check(self.product.execute(exec_, alpha, a, b, beta, d if c is None else c, d))

    def vjp(self, exec_: Optional[Executor], alpha, a, b, dd, da=None, db=None):
        check(self.product.vjp(exec_, alpha, a, b, dd, da, db))


@dataclass
class Item:
    """``BatchItem``: a plan and its operands for ``contract_batched``."""

    plan: Plan
    alpha: object
    a: object
    b: object
    d: object
    beta: object = 0
    c: object = None
    _keep: list = field(default_factory=list)


class PreparedBatch:
    """A list of (plan, operands) frozen into the C item array once, for
    repeated submission without rebuilding it (see ``contract_batched``)."""

    def __init__(self, items: Sequence[Item]):
        self.n = len(items)
        self.arr = (BatchItem * max(self.n, 1))()
        self._keep = []
        for i, it in enumerate(items):
            al = scalar_bytes(it.plan.dtype, it.alpha)
            be = scalar_bytes(it.plan.dtype, it.beta)
            self._keep += [al, be, it.plan]
            self.arr[i] = BatchItem(it.plan.product.h, C.cast(al, _vp), ptr_of(it.a), ptr_of(it.b), C.cast(be, _vp),
                                    ptr_of(it.c), ptr_of(it.d))

    def run(self, exec_: Optional[Executor] = None):
        check(lib.tprims_b200_contract_batched(exec_.h if exec_ else 0, self.n, self.arr))


class Network:
    """An N-ary contraction network executed as binary steps on the GPU (the
    einsum layer the reference leaves to its callers).

    ``inputs``: (OperandSpec, labels) per input tensor; ``output``:
    (LayoutSpec, labels); ``path``: pairs of positions in the current operand
    list (opt_einsum convention), or None for the greedy path."""

    def __init__(self, dtype: int, inputs, output, path=None):
        self.dtype = dtype
        n = len(inputs)
        # The C call reads one label per mode; a mismatch is refused here,
        # before any array is read past its end.
        for i, (sp, labels) in enumerate(list(inputs) + [(OperandSpec(output[0]), output[1])]):
            if len(labels) != len(sp.layout.dims) or len(sp.layout.strides) != len(sp.layout.dims):
                what = "output" if i == n else f"input {i}"
                raise TprimsError(ERR_LABELS, f"{what}: {len(labels)} labels for {len(sp.layout.dims)} modes")
        nm = (C.c_int * max(n, 1))(*[len(sp.layout.dims) for sp, _ in inputs])
        self._arrs = []

        def arr(v):
            a = _arr(v)
            self._arrs.append(a)
            return C.cast(a, _i64p)

        ext = (_i64p * max(n, 1))(*[arr(sp.layout.dims) for sp, _ in inputs])
        st = (_i64p * max(n, 1))(*[arr(sp.layout.strides) for sp, _ in inputs])
        lab = (_i64p * max(n, 1))(*[arr(l) for _, l in inputs])
        ops = (C.c_int * max(n, 1))(*[CONJUGATE if sp.conj else IDENTITY for sp, _ in inputs])
        olay, olab = output
        pth = [x for pair in (path or []) for x in pair]
        parr = (C.c_int * max(len(pth), 1))(*pth)
        h = _ip(0)
        check(lib.tprims_b200_network_create(C.byref(h), int(dtype), n, nm, ext, st, lab, ops, len(olay.dims),
                                             arr(olay.dims), arr(olay.strides), arr(olab), len(pth) // 2, parr))
        self.h = h.value
        self.n_inputs = n

    def set_precision(self, scheme: int, slices: int = 0):
        check(lib.tprims_b200_network_set_precision(self.h, int(scheme), int(slices)))

    def set_autotune(self, on: bool):
        check(lib.tprims_b200_network_set_autotune(self.h, 1 if on else 0))

    def workspace_size(self) -> int:
        v = C.c_size_t(0)
        check(lib.tprims_b200_network_workspace_size(self.h, C.byref(v)))
        return v.value

    def report(self) -> dict:
        n = lib.tprims_b200_network_report(self.h, None, 0)
        buf = C.create_string_buffer(n + 1)
        lib.tprims_b200_network_report(self.h, buf, n + 1)
        return json.loads(buf.value.decode())

    def execute(self, exec_: Optional[Executor], alpha, inputs, out, beta=0.0, workspace=None):
        ins = (_vp * max(self.n_inputs, 1))(*[ptr_of(x) for x in inputs])
        al, be = scalar_bytes(self.dtype, alpha), scalar_bytes(self.dtype, beta)
        check(lib.tprims_b200_network_execute(self.h, exec_.h if exec_ else 0, C.cast(al, _vp), ins, C.cast(be, _vp),
                                              ptr_of(out), ptr_of(workspace)))

    def close(self):
        if getattr(self, "h", 0):
            check(lib.tprims_b200_network_destroy(self.h))
            self.h = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_allocations() -> int:
    """Device allocations the library has made in this process (diagnostics)."""
    return int(lib.tprims_b200_device_allocations())


class PreparedNetworks:
    """A list of networks and their operands frozen into the C argument arrays
    once (the network counterpart of PreparedBatch): repeated runs pay no
    per-network marshaling."""

    def __init__(self, nets: Sequence[Network], inputs, outs, alphas=None, betas=None, workspaces=None):
        n = len(nets)
        alphas = alphas if alphas is not None else [1.0] * n
        betas = betas if betas is not None else [0.0] * n
        workspaces = workspaces if workspaces is not None else [None] * n
        if not (len(inputs) == len(outs) == len(alphas) == len(betas) == len(workspaces) == n):
            raise TprimsError(ERR_INVALID_ARGUMENT, "one inputs list, output, alpha, beta and workspace per network")
        self.n = n
        self._keep = [list(nets)]
        self.hs = (_ip * max(n, 1))(*[x.h for x in nets])
        self.al = (_vp * max(n, 1))()
        self.be = (_vp * max(n, 1))()
        self.ins = (C.POINTER(_vp) * max(n, 1))()
        self.outs = (_vp * max(n, 1))(*[ptr_of(o) for o in outs])
        self.ws = (_vp * max(n, 1))(*[ptr_of(w) for w in workspaces])
        for i, net in enumerate(nets):
            if len(inputs[i]) != net.n_inputs:
                raise TprimsError(ERR_INVALID_ARGUMENT, f"network {i} takes {net.n_inputs} inputs")
            a, b = scalar_bytes(net.dtype, alphas[i]), scalar_bytes(net.dtype, betas[i])
            arr = (_vp * max(net.n_inputs, 1))(*[ptr_of(x) for x in inputs[i]])
            self._keep += [a, b, arr]
            self.al[i], self.be[i] = C.cast(a, _vp), C.cast(b, _vp)
            self.ins[i] = C.cast(arr, C.POINTER(_vp))

    def run(self, exec_: Optional[Executor] = None):
        check(lib.tprims_b200_networks_execute(exec_.h if exec_ else 0, self.n, self.hs, self.al, self.ins, self.be,
                                               self.outs, self.ws))


def execute_networks(exec_: Optional[Executor], nets: Sequence[Network], inputs, outs, alphas=None, betas=None,
                     workspaces=None):
    """Run a list of networks: step s of every network in one grouped submission."""
    PreparedNetworks(nets, inputs, outs, alphas, betas, workspaces).run(exec_)


def _parse_einsum(subscripts: str, n: int):
    """Input and output label lists of an einsum string ("ab,bc->ac"; without
    "->" the output is the letters that appear once, in alphabetical order).
    Labels are the letters' code points."""
    s = subscripts.replace(" ", "")
    if "->" in s:
        lhs, rhs = s.split("->")
    else:
        lhs, rhs = s, None
    terms = lhs.split(",")
    if len(terms) != n:
        raise TprimsError(ERR_LABELS, f"{len(terms)} input terms for {n} operands")
    for t in terms + ([rhs] if rhs is not None else []):
        if not all(ch.isalpha() for ch in t):
            raise TprimsError(ERR_LABELS, f"einsum term {t!r}: only letters are supported")
    if rhs is None:
        counts = {}
        for t in terms:
            for ch in t:
                counts[ch] = counts.get(ch, 0) + 1
        rhs = "".join(sorted(ch for ch, c in counts.items() if c == 1))
    return [[ord(ch) for ch in t] for t in terms], [ord(ch) for ch in rhs]


def einsum_network(subscripts: str, *operands, conj=None, path=None, out_layout=None):
    """The Network (and output extents) of an einsum over the given arrays or
    tensors: one network input per operand with its own extents and strides;
    a single operand is paired with a rank-0 one (a 1-element array), so traces,
    sums and permutations run as one binary step. ``out_layout``: (extents,
    strides) of the output, column-major when None."""
    if not operands:
        raise TprimsError(ERR_INVALID_ARGUMENT, "einsum needs at least one operand")
    labels, out_labels = _parse_einsum(subscripts, len(operands))
    dt = dtype_of(operands[0])
    conj = list(conj) if conj is not None else [False] * len(operands)
    if len(conj) != len(operands):
        raise TprimsError(ERR_INVALID_ARGUMENT, "one conj flag per operand")
    inputs, ext = [], {}
    for x, l, c in zip(operands, labels, conj):
        if dtype_of(x) != dt:
            raise TprimsError(ERR_DTYPE, "einsum operands have different dtypes")
        _, shape, strides = layout_of(x)
        if len(shape) != len(l):
            raise TprimsError(ERR_LABELS, f"term of {len(l)} letters for an operand of rank {len(shape)}")
        for e, lab in zip(shape, l):
            ext.setdefault(lab, e)
        inputs.append((OperandSpec(LayoutSpec(list(shape), list(strides)), bool(c)), list(l)))
    for lab in out_labels:
        if lab not in ext:
            raise TprimsError(ERR_UNSUPPORTED, f"output letter {chr(lab)!r} appears in no input")
    out_shape = [int(ext[lab]) for lab in out_labels]
    if out_layout is None:
        st, acc = [], 1
        for e in out_shape:
            st.append(acc)
            acc *= max(e, 1)
    else:
        oshape, st = [int(e) for e in out_layout[0]], [int(v) for v in out_layout[1]]
        if oshape != out_shape:
            raise TprimsError(ERR_SHAPE, f"out has shape {oshape}, the result {out_shape}")
    if len(inputs) == 1:
        inputs.append((OperandSpec(LayoutSpec([], [])), []))
    net = Network(dt, inputs, (LayoutSpec(out_shape, st), out_labels), path)
    return net, out_shape


def einsum(subscripts: str, *operands, exec_: Optional[Executor] = None, out=None, conj=None, path=None,
           precision: int = PREC_PLAIN, alpha=1.0, beta=0.0):
    """``out = alpha * einsum(subscripts, *operands) + beta * out`` through the
    network driver (binary steps on the GPU, intermediates in device memory).

    Operands are torch tensors (device or host) or numpy arrays of one dtype,
    with any strides; ``conj`` conjugates chosen operands; ``path`` is a
    pairwise path (opt_einsum convention) or None for the greedy one. Without
    ``out`` the result is a new column-major tensor (torch operands: on the
    first operand's device) or numpy array; with ``out`` its layout is used."""
    import numpy as np

    out_layout = None
    if out is not None:
        _, oshape, ostrides = layout_of(out)
        out_layout = (oshape, ostrides)
    net, out_shape = einsum_network(subscripts, *operands, conj=conj, path=path, out_layout=out_layout)
    try:
        if precision != PREC_PLAIN:
            net.set_precision(precision)
        first = operands[0]
        torch = None
        try:
            import torch
        except ImportError:  # pragma: no cover
            pass
        on_torch = torch is not None and isinstance(first, torch.Tensor)
        if out is None:
            if on_torch:
                n = int(np.prod(out_shape)) if out_shape else 1
                flat = torch.zeros(n, dtype=first.dtype, device=first.device)
                # Column-major: the reversed shape in row-major order, permuted back.
                out = flat.reshape(list(reversed(out_shape))).permute(*reversed(range(len(out_shape)))) \
                    if out_shape else flat.reshape(())
            else:
                out = np.zeros(out_shape, dtype=first.dtype, order="F")
        ins = list(operands)
        if len(ins) == 1:  # the rank-0 partner of a single operand
            ins.append(torch.ones(1, dtype=first.dtype, device=first.device) if on_torch
                       else np.ones(1, dtype=first.dtype))
        net.execute(exec_, alpha, ins, out, beta=beta)
    finally:
        net.close()
    return out


def tuning_file_info(path: str) -> dict:
    """Header and entry counts of an autotuner cache file (no GPU needed)."""
    sms, singles, lists = C.c_int(0), C.c_int(0), C.c_int(0)
    dev = C.create_string_buffer(256)
    check(lib.tprims_b200_tuning_file_info(os.fsencode(path), C.byref(sms), dev, 256, C.byref(singles),
                                           C.byref(lists)))
    return {"sms": sms.value, "device": dev.value.decode(), "single": singles.value, "list": lists.value}


def balance(costs, part_devices, homes=None):
    """Longest-first assignment of items (costs, home devices; None: any) to
    parts living on ``part_devices``; returns the part of each item."""
    n, p = len(costs), len(part_devices)
    c = (C.c_double * max(n, 1))(*[float(x) for x in costs])
    h = (C.c_int * max(n, 1))(*[(-1 if x is None else int(x)) for x in (homes or [None] * n)])
    d = (C.c_int * max(p, 1))(*[int(x) for x in part_devices])
    out = (C.c_int * max(n, 1))()
    check(lib.tprims_b200_balance(n, c, h, p, d, out))
    return [out[i] for i in range(n)]


def _batch_items(items: Sequence[Item]):
    arr = (BatchItem * max(len(items), 1))()
    keep = []
    for i, it in enumerate(items):
        al = scalar_bytes(it.plan.dtype, it.alpha)
        be = scalar_bytes(it.plan.dtype, it.beta)
        keep += [al, be]
        arr[i] = BatchItem(it.plan.product.h, C.cast(al, _vp), ptr_of(it.a), ptr_of(it.b), C.cast(be, _vp),
                           ptr_of(it.c), ptr_of(it.d))
    return arr, keep


def contract_batched_sharded(items: Sequence[Item], execs: Sequence[Executor]):
    """contract_batched over several executors (one per GPU, or several per
    GPU): items balanced by cost over the executors of their output's device,
    each share one grouped submission on its executor's stream."""
    arr, keep = _batch_items(items)
    hs = (_ip * max(len(execs), 1))(*[e.h for e in execs])
    check(lib.tprims_b200_contract_batched_sharded(hs, len(execs), len(items), arr))


def contract_batched(items: Sequence[Item], exec_: Optional[Executor] = None):
    """Validate every item, then run them as one grouped submission."""
    arr = (BatchItem * max(len(items), 1))()
    keep = []
    for i, it in enumerate(items):
        al = scalar_bytes(it.plan.dtype, it.alpha)
        be = scalar_bytes(it.plan.dtype, it.beta)
        keep += [al, be]
        arr[i] = BatchItem(it.plan.product.h, C.cast(al, _vp), ptr_of(it.a), ptr_of(it.b), C.cast(be, _vp),
                           ptr_of(it.c), ptr_of(it.d))
    check(lib.tprims_b200_contract_batched(exec_.h if exec_ else 0, len(items), arr))


def contract(labels_a, a, labels_b, b, labels_d, d, alpha=1.0, beta=0.0, c=None, conj=(False, False, False, False),
             exec_: Optional[Executor] = None, precision: int = PREC_PLAIN) -> dict:
    """One-shot TAPP contraction of arrays/tensors by labels; returns the plan report."""
    dt = dtype_of(a)
    h = Handle()
    infos = []
    for x in (a, b, c if c is not None else d, d):
        _, ext, st = layout_of(x)
        infos.append(TensorInfo(dt, ext, st))
    ops = [CONJUGATE if f else IDENTITY for f in conj]
    p = TensorProduct.create(h, (ops[0], infos[0], labels_a), (ops[1], infos[1], labels_b),
                             (ops[2], infos[2], labels_d), (ops[3], infos[3], labels_d))
    if precision != PREC_PLAIN:
        p.set_precision(precision)
    check(p.execute(exec_, alpha, a, b, beta, c, d))
    return p.report()


lib.tprims_b200_product_scatter.argtypes = [_ip, C.c_int, _i64p, C.c_int64]
lib.tprims_b200_product_scatter.restype = C.c_int64
SCATTER_NAMES = ["a_m", "a_k", "b_k", "b_n", "c_m", "c_n", "d_m", "d_n", "h_a", "h_b", "h_c", "h_d"]


def product_scatter(product: TensorProduct, name: str):
    """A scatter vector of the packed plan (before orientation), for tests."""
    w = SCATTER_NAMES.index(name)
    n = lib.tprims_b200_product_scatter(product.h, w, None, 0)
    if n < 0:
        raise TprimsError(ERR_INVALID_ARGUMENT, last_error())
    buf = (C.c_int64 * max(n, 1))()
    lib.tprims_b200_product_scatter(product.h, w, buf, n)
    return list(buf)[:n]
