"""ctypes binding of libqsim.so (the C-ABI declared in include/qsim.h).

The library is loaded from the package directory.  There is no fallback: if
the shared object is missing or fails to load, every simulator entry point
raises ``NativeLibraryError``.
"""
from __future__ import annotations

import atexit
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# QSIM_LIB overrides the library path (e.g. an instrumented build)
LIB_PATH = os.environ.get("QSIM_LIB") or os.path.join(_HERE, "libqsim.so")

# ---- constants mirrored from include/qsim.h --------------------------------
QS_OK, QS_EINVAL, QS_ECUDA, QS_EWORKSPACE, QS_ENOTSUP, QS_ETIMEOUT = 0, -1, -2, -3, -4, -5
QS_C64, QS_C128 = 0, 1
QS_K_DENSE, QS_K_DIAG, QS_K_ANTIDIAG, QS_K_SWAP = 0, 1, 2, 3
QS_OP_MAT, QS_OP_DIAG, QS_OP_ANTI, QS_OP_SWAP = 1, 2, 3, 4
QS_OP_EXPECT = 5
QS_OPF_UNIT, QS_OPF_DIAG = 1, 2
QS_MAX_PASS_MATS = 2048
QS_SRC_SV, QS_SRC_DM = 0, 1
QS_SAMPLE_CDF, QS_SAMPLE_SEQ = 0, 1
QS_MAX_TILE_BITS = 14
QS_MAX_PASS_OPS = 160
QS_NOALLOC_SAMPLE_MAX_QUBITS = 26
QS_JIT_OFF, QS_JIT_ASYNC, QS_JIT_SYNC = 0, 1, 2
JIT_STAT_KEYS = ("compiled", "failed", "pending", "compiled_launches", "generic_launches_while_pending",
                 "compile_ms", "cache_hits")


class NativeLibraryError(RuntimeError):
    """libqsim.so is missing or could not be loaded."""


class QsimError(RuntimeError):
    """A libqsim call returned a negative status."""

    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed ({code}): {msg}")
        self.code = code


class qs_op(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("m", C.c_int32),
        ("tgt", C.c_int32 * 4),
        ("gbit", C.c_int32 * 4),
        ("lctrl", C.c_uint32),
        ("flags", C.c_uint32),
        ("gctrl", C.c_uint64),
        ("mat", C.c_int64),
        ("mat_stride", C.c_int64),
        ("slot", C.c_int32),
        ("pad1", C.c_int32),
    ]


class qs_pass(C.Structure):
    _fields_ = [
        ("k", C.c_int32),
        ("nlow", C.c_int32),
        ("hi", C.c_int32 * QS_MAX_TILE_BITS),
        ("op_begin", C.c_int32),
        ("op_count", C.c_int32),
        ("inst_shift", C.c_int32),
        ("pair", C.c_int32),
    ]


class qs_batch_inst(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("fwd_begin", C.c_int32),
        ("nfwd", C.c_int32),
        ("bwd_begin", C.c_int32),
        ("nbwd", C.c_int32),
        ("term_begin", C.c_int32),
        ("nterms", C.c_int32),
        ("nslots", C.c_int32),
        ("nparams", C.c_int32),
        ("pad", C.c_int32),
        ("w_begin", C.c_int64),
    ]


class qs_batch_sizes(C.Structure):
    _fields_ = [
        ("blob_bytes", C.c_int64),
        ("state_elems", C.c_int64),
        ("partial_doubles", C.c_int64),
        ("grad_doubles", C.c_int64),
        ("energy_doubles", C.c_int64),
        ("ctrl_bytes", C.c_int64),
        ("smem_bytes", C.c_int64),
        ("threads", C.c_int32),
        ("nitems", C.c_int32),
        ("nstages", C.c_int32),
        ("big", C.c_int32),
        ("dtype", C.c_int32),
        ("jit_fns", C.c_int32),
        ("jit_key", C.c_uint64),
    ]


assert C.sizeof(qs_op) == 80
assert C.sizeof(qs_batch_inst) == 48 and C.sizeof(qs_batch_sizes) == 88
assert C.sizeof(qs_pass) == 8 + 4 * QS_MAX_TILE_BITS + 16

_vp, _i, _i64, _u64, _d, _sz = C.c_void_p, C.c_int, C.c_int64, C.c_uint64, C.c_double, C.c_size_t
_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)

# name -> (restype, argtypes)
SIGNATURES = {
    "qs_version": (_i, []),
    "qs_last_error": (C.c_char_p, []),
    "qs_device_sm_count": (_i, []),
    "qs_init_zero": (_i, [_vp, _i, _i, _vp]),
    "qs_scale": (_i, [_vp, _i, _i, _d, _d, _vp]),
    "qs_apply_1q": (_i, [_vp, _i, _i, _i, _u64, _i, _dp, _vp]),
    "qs_apply_2q": (_i, [_vp, _i, _i, _i, _i, _u64, _i, _dp, _vp]),
    "qs_apply_kq": (_i, [_vp, _i, _i, _i, _i32p, _u64, _vp, _vp]),
    "qs_apply_fused": (_i, [_vp, _i, _i, C.POINTER(qs_pass), _i, C.POINTER(qs_op), _i64, _vp, _i64, _vp]),
    "qs_adjoint_fused": (_i, [_vp, _vp, _i, _i, C.POINTER(qs_pass), _i, C.POINTER(qs_op), _i64, _vp, _i64, _vp,
                              _i64, _vp]),
    "qs_adjoint_pair": (_i, [_vp, _i, _i, C.POINTER(qs_pass), _i, C.POINTER(qs_op), _i64, _vp, _i64, _vp, _i64, _vp]),
    "qs_apply_pauli_sum": (_i, [_vp, _vp, _i, _i, _vp, _vp, _vp, _i, _vp]),
    "qs_inner_batched": (_i, [_vp, _vp, _i, _i, _i, _vp, _vp, _sz, _vp]),
    "qs_segment_sum": (_i, [_vp, _i64, _i64, _vp, _vp]),
    "qs_reduce_ws_bytes": (_sz, [_i]),
    "qs_prob0": (_i, [_vp, _i, _i, _i, _i, _vp, _sz, _vp, _vp]),
    "qs_norm2": (_i, [_vp, _i, _i, _i, _vp, _sz, _vp, _vp]),
    "qs_collapse": (_i, [_vp, _i, _i, _i, _i, _d, _vp]),
    "qs_reset": (_i, [_vp, _i, _i, _i, _d, _vp]),
    "qs_sample_ws_bytes": (_sz, [_i]),
    "qs_sample_prepare": (_i, [_vp, _i, _i, _i, _vp, _sz, _vp]),
    "qs_sample": (_i, [_vp, _i, _i, _i, _vp, _sz, _vp, _i64, _i, _vp, _vp]),
    "qs_histogram": (_i, [_vp, _i64, _vp, _i64, _vp]),
    "qs_sample_noalloc": (_i, [_vp, _i, _i, _i, _vp, _i64, _i, _vp, _vp]),
    "qs_apply_fused_ex": (_i, [_vp, _i, _i, C.POINTER(qs_pass), _i, C.POINTER(qs_op), _i64, _vp, _vp, _i64, _vp]),
    "qs_adjoint_pair_ex": (_i, [_vp, _i, _i, C.POINTER(qs_pass), _i, C.POINTER(qs_op), _i64, _vp, _vp, _i64, _vp,
                                _i64, _vp]),
    "qs_batch_plan": (_i, [_i, C.POINTER(qs_batch_inst), _i, C.POINTER(qs_pass), _i, C.POINTER(qs_op), _i64, _i64,
                           _vp, _i, _vp, _vp, _vp, _i, _vp, _i64, _i64, _i64, _vp, _sz, C.POINTER(qs_batch_sizes),
                           C.POINTER(C.c_int64)]),
    "qs_batch_link_check": (_i, [C.POINTER(qs_batch_sizes), C.POINTER(C.c_int64)]),
    "qs_batch_launch": (_i, [C.POINTER(qs_batch_sizes), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _d, _vp]),
    "qs_jit_shutdown": (_i, []),
    "qs_jit_set_mode": (_i, [_i]),
    "qs_jit_wait": (_i, [_d]),
    "qs_jit_stats": (_i, [C.POINTER(C.c_int64), _i]),
    "qs_jit_last_log": (C.c_char_p, []),
    "qs_jit_compile_check": (_i, [C.c_char_p, C.POINTER(C.c_int64)]),
    "qs_jit_pass_source": (_i, [_i, _i, C.POINTER(qs_pass), C.POINTER(qs_op), _i64, _vp, _i64, _i, C.c_char_p, _sz,
                                C.POINTER(C.c_int64)]),
}

_lib = None


def load() -> C.CDLL:
    """Load libqsim.so once; raise NativeLibraryError when it is unavailable."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NativeLibraryError(
            f"{LIB_PATH} not found: build it with `python -m quict_b200.build` (no CPU fallback exists)"
        )
    try:
        lib = C.CDLL(LIB_PATH)
    except OSError as e:  # pragma: no cover - depends on the machine
        raise NativeLibraryError(f"cannot load {LIB_PATH}: {e}") from e
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    # no pass compilation may still run while the interpreter shuts down
    atexit.register(lib.qs_jit_shutdown)
    return lib


def call(name: str, *args) -> int:
    """Call a status-returning entry point and raise QsimError on failure."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc < 0:
        msg = lib.qs_last_error().decode(errors="replace")
        raise QsimError(name, rc, msg)
    return rc


def mat_ptr(m: np.ndarray):
    """Host complex128 matrix -> (keepalive array, double*)."""
    a = np.ascontiguousarray(m, dtype=np.complex128)
    return a, a.ctypes.data_as(_dp)


def stream_ptr(stream) -> int | None:
    """torch.cuda.Stream (or None) -> raw cudaStream_t value for ctypes."""
    if stream is None:
        return None
    return int(stream.cuda_stream) or None


def jit_set_mode(mode: int) -> int:
    """Set libqsim's run-time compilation mode (QS_JIT_OFF / ASYNC / SYNC);
    returns the previous mode."""
    return call("qs_jit_set_mode", int(mode))


def jit_wait(timeout_s: float = -1.0) -> None:
    """Block until every queued pass compilation has finished."""
    call("qs_jit_wait", float(timeout_s))


def jit_stats() -> dict:
    out = (C.c_int64 * len(JIT_STAT_KEYS))()
    call("qs_jit_stats", out, len(JIT_STAT_KEYS))
    return dict(zip(JIT_STAT_KEYS, (int(v) for v in out)))
