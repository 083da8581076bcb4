"""Continuous-batching transport server on one GPU (Python face of the
library's native server, ``qtx_server_*`` in include/qtx_rgf.h).

Requests (one device, its own energy grid and contacts) arrive at any time.
``submit`` puts the request's H and energies on the device and hands it to the
native server, whose worker threads (one CUDA stream and library context per
slot) admit the oldest waiting request as soon as a slot is free and its
device footprint fits in the budget next to the running ones; admitted
requests overlap on the GPU while new ones keep arriving.  Waiting FP64
requests of one block size <= 64 are taken together and solved in one
persistent launch (every energy of every request one work item).  A request's state
(H, the energy-call work space, outputs) stays on the device until it
completes; only its observables come back.  Latency = completion time -
submission time, measured by the native server.
"""

from __future__ import annotations

import ctypes
import threading
import warnings
from concurrent.futures import Future

import numpy as np
import torch

from quatrex_b200 import _lib
from quatrex_b200.autotune import Autotuner
from quatrex_b200.batching import OBSERVABLE_KEYS
from quatrex_b200.transport import allocate_outputs
from quatrex_b200.workloads import TransportDevice

_PRECISIONS = {"fp64": _lib.QTX_PREC_FP64, "mixed": _lib.QTX_PREC_MIXED}


class TransportServer:
    """Admit, run and complete transport requests concurrently.

    Parameters
    ----------
    slots : number of concurrently running requests (CUDA streams).
    memory_budget : device bytes the running requests' work spaces may hold
        together (default: half of the free memory at start).
    precision : "fp64" or "mixed" (for "mixed" the autotuner may still pick
        the FP64 products for a block size where they are faster).
    group_small : waiting FP64 requests of one block size <= 64 are solved
        together in one persistent launch (qtx_transport_solve_grouped).
    """

    def __init__(self, slots: int = 4, memory_budget: int | None = None, precision: str = "fp64",
                 tuner: Autotuner | None = None, cuda_device: int | None = None, keys=OBSERVABLE_KEYS,
                 group_small: bool = True):
        if not torch.cuda.is_available():
            raise RuntimeError("quatrex_b200 needs a CUDA device (B200, sm_100a); there is no CPU path")
        self.cuda = torch.cuda.current_device() if cuda_device is None else cuda_device
        if memory_budget is None:
            free, _ = torch.cuda.mem_get_info(self.cuda)
            memory_budget = int(free * 0.5)
        self.budget = int(memory_budget)
        self.precision = precision
        self.tuner = tuner if tuner is not None else Autotuner()
        self.keys = tuple(keys)
        self._lib = _lib.load()
        cfg = _lib.ServerConfig(device=self.cuda, slots=max(1, int(slots)), memory_budget=self.budget,
                                group_max_block_size=64 if group_small else 0)
        h = ctypes.c_void_p()
        st = self._lib.qtx_server_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != _lib.QTX_OK:
            raise _lib.status_error(st, "qtx_server_create", "") or RuntimeError("qtx_server_create")
        self._srv = h.value
        self._copy_stream = torch.cuda.Stream(device=self.cuda)
        self._live: dict[int, tuple] = {}
        self._lock = threading.Lock()
        self._closing = False
        self._collector = threading.Thread(target=self._collect, daemon=True)
        self._collector.start()

    # -- client side ---------------------------------------------------------
    def submit(self, device: TransportDevice, energies) -> Future:
        """Queue one request; the future resolves to a dict of host arrays of
        the observables plus 'latency_s'."""
        fut: Future = Future()
        if self._closing:
            fut.set_exception(RuntimeError("server is closed"))
            return fut
        energies = np.asarray(energies, dtype=np.float64)
        choice = self.tuner.best(device.block_size, len(energies), self.precision)
        path = choice.get("gemm_path", self.precision)
        ne_call = call_size(self._lib, device.num_blocks, device.block_size, len(energies),
                            int(choice["energies_per_call"]), path, self.budget)
        dev = f"cuda:{self.cuda}"
        nb, b, ne = device.num_blocks, device.block_size, len(energies)
        with torch.cuda.stream(self._copy_stream):
            h_diag = torch.from_numpy(device.h_diag).to(dev, non_blocking=False)
            h_upper = torch.from_numpy(device.h_upper).to(dev, non_blocking=False)
            e = torch.from_numpy(energies).to(dev, non_blocking=False)
            out = allocate_outputs(nb, b, ne, self.keys, self.cuda)
        # the inputs are on the device before any worker can pick the request up
        self._copy_stream.synchronize()
        p = _lib.TransportProblem(
            num_blocks=nb, block_size=b, num_energies=ne, h_diag=h_diag.data_ptr(), h_upper=h_upper.data_ptr(),
            energies=e.data_ptr(), eta=device.eta, mu_left=device.mu_left, mu_right=device.mu_right, kt=device.kt,
            sr_tol=device.sr_tol, sr_max_iterations=device.sr_max_iter, max_batch_size=ne_call)
        o = _lib.TransportOutputs(**{name: (out[name].data_ptr() if name in out else None)
                                     for name, _ in _lib.TransportOutputs._fields_})
        rid = ctypes.c_int64()
        with self._lock:
            st = self._lib.qtx_server_submit(self._srv, ctypes.byref(p), ctypes.byref(o), _PRECISIONS[path], 0,
                                             ctypes.byref(rid))
            if st != _lib.QTX_OK:
                need = self._lib.qtx_transport_footprint(nb, b, ne_call, _PRECISIONS[path])
                fut.set_exception(_lib.status_error(
                    st, "qtx_server_submit",
                    f"request needs {need} device bytes; server budget {self.budget}"))
                return fut
            # keep the request's device arrays alive until it completes
            self._live[rid.value] = (fut, out, (h_diag, h_upper, e))
        return fut

    def close(self, wait: bool = True):
        """Finish every submitted request, then stop the server (``wait`` is
        kept for compatibility: closing always drains the queue)."""
        self._closing = True
        self._collector.join()
        if self._srv:
            self._lib.qtx_server_destroy(self._srv)
            self._srv = None

    def stats(self) -> dict:
        st = _lib.ServerStats()
        self._lib.qtx_server_get_stats(self._srv, ctypes.byref(st))
        return {"submitted": st.submitted, "completed": st.completed, "failed": st.failed, "queued": st.queued,
                "running": st.running, "solves": st.solves, "p50_s": st.p50_latency_s, "p99_s": st.p99_latency_s,
                "mean_s": st.mean_latency_s, "peak_concurrency": st.peak_running,
                "memory_in_use": st.memory_in_use, "grouped_launches": st.grouped_launches,
                "grouped_requests": st.grouped_requests}

    # -- completions -----------------------------------------------------------
    def _collect(self):
        rid, status, lat = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_double()
        err = ctypes.create_string_buffer(512)
        while True:
            st = self._lib.qtx_server_wait_any(self._srv, 50, ctypes.byref(rid), ctypes.byref(status),
                                               ctypes.byref(lat), err, len(err))
            if st != _lib.QTX_OK:
                with self._lock:
                    if self._closing and not self._live:
                        return
                continue
            with self._lock:
                fut, out, _inputs = self._live.pop(rid.value)
            exc = _lib.status_error(status.value, "transport request", err.value.decode(errors="replace"))
            if exc is not None:
                fut.set_exception(exc)
                continue
            if status.value == _lib.QTX_E_NOT_CONVERGED:
                warnings.warn(err.value.decode(errors="replace") or "Surface Green's function did not converge.",
                              RuntimeWarning, stacklevel=2)
            res = {k: v.cpu().numpy() for k, v in out.items()}
            res["latency_s"] = lat.value
            fut.set_result(res)


def call_size(lib, num_blocks: int, block_size: int, num_energies: int, tuned: int, path: str,
              budget: int) -> int:
    """Energies per device call of one request: the tuned size (chosen on a
    short probe device), at most the request's energies, halved until one
    call's work space (``qtx_transport_footprint``) fits the budget, never
    below one; a request that does not fit even then is refused at
    submission by the native server."""
    ne_call = max(1, min(int(tuned), int(num_energies)))
    while ne_call > 1 and lib.qtx_transport_footprint(num_blocks, block_size, ne_call, _PRECISIONS[path]) > budget:
        ne_call = max(1, ne_call // 2)
    return ne_call


def poisson_arrivals(count: int, rate_hz: float, seed: int = 0) -> np.ndarray:
    """Arrival offsets (seconds) of a seeded Poisson stream."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_hz, size=count))
