"""ctypes binding of libqtxrgf.so (the C ABI declared in include/qtx_rgf.h).

The shared library is built in-tree by ``python -m quatrex_b200.build``.  There
is no fallback: if the library (or a CUDA device) is missing, every solver call
raises.
"""

from __future__ import annotations

import ctypes
import os
import threading
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqtxrgf.so")

QTX_OK = 0
QTX_E_INVAL = 1
QTX_E_NOMEM = 2
QTX_E_SINGULAR = 3
QTX_E_NOT_CONVERGED = 4
QTX_E_TIMEOUT = 5
QTX_E_CUDA = 6
QTX_E_UNSUPPORTED = 7

QTX_PREC_FP64 = 0
QTX_PREC_MIXED = 1

QTX_FLAG_RETURN_RETARDED = 0x1
QTX_FLAG_RETURN_CURRENT = 0x2
QTX_FLAG_SYMMETRIC_OUT = 0x4
QTX_FLAG_HOST_BUFFERS = 0x8
QTX_FLAG_RETARDED_OFFDIAG = 0x10
QTX_FLAG_GRAPH = 0x20

c_void_p = ctypes.c_void_p
c_int32 = ctypes.c_int32
c_int64 = ctypes.c_int64
c_uint32 = ctypes.c_uint32
c_double = ctypes.c_double


class BtdDesc(ctypes.Structure):
    _fields_ = [
        ("num_blocks", c_int32),
        ("block_sizes", ctypes.POINTER(c_int32)),
        ("block_offset", ctypes.POINTER(c_int64)),
        ("block_nnz", ctypes.POINTER(c_int64)),
        ("block_index", ctypes.POINTER(c_void_p)),
        ("stack_size", c_int64),
        ("stack_stride", c_int64),
    ]


class SpectralParams(ctypes.Structure):
    _fields_ = [
        ("min_decay", c_double),
        ("max_decay", c_double),
        ("min_propagation", c_double),
        ("residual_tolerance", c_double),
        ("eta_decay", c_double),
        ("residual_normalization", c_int32),
        ("num_ref_iterations", c_int32),
    ]


class Obc(ctypes.Structure):
    _fields_ = [
        ("retarded", ctypes.POINTER(c_void_p)),
        ("lesser", ctypes.POINTER(c_void_p)),
        ("greater", ctypes.POINTER(c_void_p)),
    ]


class TransportProblem(ctypes.Structure):
    _fields_ = [
        ("num_blocks", c_int32),
        ("block_size", c_int32),
        ("num_energies", c_int64),
        ("h_diag", c_void_p),
        ("h_upper", c_void_p),
        ("energies", c_void_p),
        ("eta", c_double),
        ("mu_left", c_double),
        ("mu_right", c_double),
        ("kt", c_double),
        ("sr_tol", c_double),
        ("sr_max_iterations", c_int32),
        ("max_batch_size", c_int64),
    ]


class TransportOutputs(ctypes.Structure):
    _fields_ = [
        ("gr_diag", c_void_p),
        ("gr_upper", c_void_p),
        ("gr_lower", c_void_p),
        ("gl_diag", c_void_p),
        ("gl_upper", c_void_p),
        ("gg_diag", c_void_p),
        ("gg_upper", c_void_p),
        ("density", c_void_p),
        ("hole_density", c_void_p),
        ("transmission", c_void_p),
        ("current_left", c_void_p),
        ("current_right", c_void_p),
        ("sr_iterations", c_void_p),
        ("dos", c_void_p),
        ("layer_current", c_void_p),
    ]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", c_int32), ("slots", c_int32), ("memory_budget", ctypes.c_size_t),
                ("group_max_block_size", c_int32)]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", c_int64), ("completed", c_int64), ("failed", c_int64), ("queued", c_int64),
        ("running", c_int64), ("peak_running", c_int64), ("solves", c_int64), ("memory_in_use", ctypes.c_size_t),
        ("p50_latency_s", c_double), ("p99_latency_s", c_double), ("mean_latency_s", c_double),
        ("grouped_launches", c_int64), ("grouped_requests", c_int64),
    ]


# (name, restype, argtypes) of every exported symbol, mirroring include/qtx_rgf.h
SIGNATURES = {
    "qtx_version": (ctypes.c_char_p, []),
    "qtx_ctx_create": (c_int32, [ctypes.c_int, ctypes.POINTER(c_void_p)]),
    "qtx_ctx_destroy": (c_int32, [c_void_p]),
    "qtx_last_error": (ctypes.c_char_p, [c_void_p]),
    "qtx_ctx_set_memory_limit": (c_int32, [c_void_p, ctypes.c_size_t]),
    "qtx_ctx_trim": (c_int32, [c_void_p]),
    "qtx_launch_count": (c_int64, [c_void_p]),
    "qtx_graph_replays": (c_int64, [c_void_p]),
    "qtx_ctx_release_graphs": (c_int32, [c_void_p, c_void_p]),
    "qtx_ctx_set_timing": (c_int32, [c_void_p, ctypes.c_int]),
    "qtx_ctx_timing_report": (
        c_int32, [c_void_p, c_int32, ctypes.POINTER(c_double), ctypes.POINTER(c_double), ctypes.POINTER(c_int64)]),
    "qtx_inv": (c_int32, [c_void_p, c_int32, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p]),
    "qtx_zgemm": (
        c_int32,
        [c_void_p, c_int32, c_int32, c_int32, c_int64, c_double, c_double, c_void_p, c_int64, c_int64, c_int32,
         c_void_p, c_int64, c_int64, c_int32, c_double, c_double, c_void_p, c_int64, c_int64, c_void_p, c_int64,
         c_int64, c_int32, c_void_p],
    ),
    "qtx_selected_inv": (
        c_int32,
        [c_void_p, ctypes.POINTER(BtdDesc), c_void_p, ctypes.POINTER(c_void_p), ctypes.POINTER(BtdDesc), c_void_p,
         c_int64, c_int32, c_uint32, c_void_p],
    ),
    "qtx_selected_solve": (
        c_int32,
        [c_void_p, ctypes.POINTER(BtdDesc), c_void_p, ctypes.POINTER(BtdDesc), c_void_p, ctypes.POINTER(BtdDesc),
         c_void_p, ctypes.POINTER(Obc), ctypes.POINTER(BtdDesc), c_void_p, ctypes.POINTER(BtdDesc), c_void_p,
         ctypes.POINTER(BtdDesc), c_void_p, c_void_p, c_int64, c_int32, c_uint32, c_void_p],
    ),
    "qtx_sancho_rubio": (
        c_int32,
        [c_void_p, c_int32, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_double, c_int32,
         c_void_p, c_void_p, c_void_p],
    ),
    "qtx_sancho_rubio_noalloc": (
        c_int32,
        [c_int32, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_double, c_int32, c_void_p,
         c_void_p, c_void_p, ctypes.c_char_p, c_int32],
    ),
    "qtx_block_combine": (
        c_int32,
        [c_void_p, c_int32, c_int32, c_int64, c_double, c_double, c_void_p, c_int64, c_int64, c_int32, c_double,
         c_double, c_void_p, c_int64, c_int64, c_int32, c_void_p, c_int64, c_int64, c_void_p],
    ),
    "qtx_beyn_moments": (
        c_int32,
        [c_void_p, c_int32, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_double, c_double,
         c_int32, c_void_p, c_int32, c_void_p, c_void_p, c_void_p],
    ),
    "qtx_spectral_surface": (
        c_int32,
        [c_void_p, c_int32, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p,
         c_int32, c_void_p, c_void_p, c_void_p, c_void_p],
    ),
    "qtx_obc_fixed_point": (
        c_int32,
        [c_void_p, c_int32, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p,
         c_void_p, c_void_p, c_void_p],
    ),
    "qtx_obc_assemble": (
        c_int32,
        [c_void_p, c_int32, c_int64, c_void_p, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p, c_void_p,
         c_void_p, c_void_p],
    ),
    "qtx_transport_solve": (
        c_int32,
        [c_void_p, ctypes.POINTER(TransportProblem), ctypes.POINTER(TransportOutputs), c_int32, c_uint32, c_void_p],
    ),
    "qtx_transport_footprint": (ctypes.c_size_t, [c_int32, c_int32, c_int64, c_int32]),
    "qtx_transport_solve_grouped": (
        c_int32,
        [c_void_p, c_int32, ctypes.POINTER(TransportProblem), ctypes.POINTER(TransportOutputs), c_int32, c_uint32,
         ctypes.POINTER(c_int32), c_void_p],
    ),
    "qtx_transport_grouped_footprint": (
        ctypes.c_size_t, [c_int32, ctypes.POINTER(c_int32), ctypes.POINTER(c_int64), c_int32]),
    "qtx_assemble_system": (
        c_int32, [c_void_p, c_int64, c_int64, c_void_p, c_double, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                  c_void_p, c_int64, c_void_p, c_int64, c_void_p]),
    "qtx_block_sort_index": (
        c_int32, [c_void_p, c_int64, c_void_p, c_void_p, c_int32, ctypes.POINTER(c_int32), c_void_p,
                  ctypes.POINTER(c_int64), c_void_p]),
    "qtx_server_create": (c_int32, [ctypes.POINTER(ServerConfig), ctypes.POINTER(c_void_p)]),
    "qtx_server_destroy": (c_int32, [c_void_p]),
    "qtx_server_submit": (
        c_int32,
        [c_void_p, ctypes.POINTER(TransportProblem), ctypes.POINTER(TransportOutputs), c_int32, c_uint32,
         ctypes.POINTER(c_int64)],
    ),
    "qtx_server_wait": (
        c_int32,
        [c_void_p, c_int64, c_int64, ctypes.POINTER(c_int32), ctypes.POINTER(c_double), ctypes.c_char_p, c_int32],
    ),
    "qtx_server_wait_any": (
        c_int32,
        [c_void_p, c_int64, ctypes.POINTER(c_int64), ctypes.POINTER(c_int32), ctypes.POINTER(c_double),
         ctypes.c_char_p, c_int32],
    ),
    "qtx_server_get_stats": (c_int32, [c_void_p, ctypes.POINTER(ServerStats)]),
}

_lib = None
_lib_lock = threading.Lock()
_ctx: dict[int, int] = {}


class QtxError(RuntimeError):
    """A non-OK status returned by libqtxrgf."""

    def __init__(self, status: int, message: str):
        super().__init__(f"qtx status {status}: {message}")
        self.status = status


def load() -> ctypes.CDLL:
    """Load libqtxrgf.so (raises if it has not been built)."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m quatrex_b200.build` (CUDA 12.9, sm_100a)"
            )
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def exported_symbols() -> list[str]:
    return list(SIGNATURES)


def context(device: int) -> int:
    """Per-device qtx_ctx handle (created on first use)."""
    lib = load()
    with _lib_lock:
        h = _ctx.get(device)
        if h is None:
            p = c_void_p()
            st = lib.qtx_ctx_create(device, ctypes.byref(p))
            if st != QTX_OK:
                raise QtxError(st, f"qtx_ctx_create(device={device}) failed")
            h = p.value
            _ctx[device] = h
        return h


def new_context(device: int) -> int:
    """A fresh qtx_ctx handle (one per host thread that drives its own stream)."""
    lib = load()
    p = c_void_p()
    st = lib.qtx_ctx_create(device, ctypes.byref(p))
    if st != QTX_OK:
        raise QtxError(st, f"qtx_ctx_create(device={device}) failed")
    return p.value


def destroy_context(ctx: int) -> None:
    load().qtx_ctx_destroy(ctx)


def status_error(status: int, what: str, msg: str):
    """The exception (or None for OK / not converged) of a status code."""
    if status in (QTX_OK, QTX_E_NOT_CONVERGED):
        return None
    if status == QTX_E_INVAL:
        return ValueError(f"{what}: {msg}")
    if status == QTX_E_SINGULAR:
        return np.linalg.LinAlgError(f"{what}: {msg}")
    if status == QTX_E_NOMEM:
        return MemoryError(f"{what}: {msg}")
    if status == QTX_E_UNSUPPORTED:
        return NotImplementedError(f"{what}: {msg}")
    return QtxError(status, f"{what}: {msg}")


def check(status: int, ctx: int, what: str) -> None:
    if status == QTX_OK:
        return
    msg = load().qtx_last_error(ctx)
    msg = msg.decode() if msg else ""
    if status == QTX_E_NOT_CONVERGED:
        warnings.warn(msg or "Surface Green's function did not converge.", RuntimeWarning, stacklevel=3)
        return
    if status == QTX_E_INVAL:
        raise ValueError(f"{what}: {msg}")
    if status == QTX_E_SINGULAR:
        raise np.linalg.LinAlgError(f"{what}: {msg}")
    if status == QTX_E_NOMEM:
        raise MemoryError(f"{what}: {msg}")
    if status == QTX_E_UNSUPPORTED:
        raise NotImplementedError(f"{what}: {msg}")
    raise QtxError(status, f"{what}: {msg}")


def launch_count(device: int = 0) -> int:
    return int(load().qtx_launch_count(context(device)))


def set_timing(enable: bool, device: int = 0) -> None:
    ctx = context(device)
    check(load().qtx_ctx_set_timing(ctx, 1 if enable else 0), ctx, "qtx_ctx_set_timing")


def timing_report(kind: int, device: int = 0) -> dict:
    """Summed device time (ms), algorithmic flops and launches of one kernel class
    (0 = complex GEMM, 1 = block inverse) since timing was enabled."""
    ctx = context(device)
    ms, fl, n = c_double(), c_double(), c_int64()
    check(load().qtx_ctx_timing_report(ctx, kind, ctypes.byref(ms), ctypes.byref(fl), ctypes.byref(n)), ctx,
          "qtx_ctx_timing_report")
    return {"ms": ms.value, "flops": fl.value, "launches": n.value}
