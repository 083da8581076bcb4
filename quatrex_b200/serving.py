"""Continuous-batching transport server on one GPU.

Requests (one device, its own energy grid and contacts) arrive at any time.
A scheduler admits the oldest waiting request as soon as a slot is free and
its device-memory footprint (H, work space of one energy call, outputs) fits
in the budget next to the requests already running; every slot is a CUDA
stream with its own library context, so admitted requests overlap on the
GPU while new ones keep arriving.  State of a running request (H, the
energy-call work space, outputs) stays on the device until it completes; only
its observables come back.  Latency = completion time - submission time; the
server keeps every latency for p50/p99.
"""

from __future__ import annotations

import threading
import time
from collections import deque
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np
import torch

from quatrex_b200.autotune import Autotuner
from quatrex_b200.batching import OBSERVABLE_KEYS, Worker
from quatrex_b200.transport import TransportSolver
from quatrex_b200.workloads import TransportDevice


@dataclass
class Request:
    rid: int
    device: TransportDevice
    energies: np.ndarray
    submitted: float
    footprint: int
    choice: dict
    future: Future = field(default_factory=Future)


class TransportServer:
    """Admit, run and complete transport requests concurrently.

    Parameters
    ----------
    slots : number of concurrently running requests (CUDA streams).
    memory_budget : device bytes the running requests may hold together
        (default: half of the free memory at start).
    precision : "fp64" or "mixed".
    """

    def __init__(self, slots: int = 4, memory_budget: int | None = None, precision: str = "fp64",
                 tuner: Autotuner | None = None, cuda_device: int | None = None, keys=OBSERVABLE_KEYS):
        self.cuda = torch.cuda.current_device() if cuda_device is None else cuda_device
        if memory_budget is None:
            free, _ = torch.cuda.mem_get_info(self.cuda)
            memory_budget = int(free * 0.5)
        self.budget = int(memory_budget)
        self.precision = precision
        self.tuner = tuner if tuner is not None else Autotuner()
        self.keys = keys
        self.workers = [Worker(self.cuda) for _ in range(max(1, slots))]
        self._free_workers = list(self.workers)
        self._queue: deque[Request] = deque()
        self._used = 0
        self._next_id = 0
        self._cv = threading.Condition()
        self._closing = False
        self.latencies: list[float] = []
        self.completed = 0
        self.solves = 0
        self.peak_concurrency = 0
        self._running = 0
        self._scheduler = threading.Thread(target=self._schedule, daemon=True)
        self._scheduler.start()

    # -- client side ---------------------------------------------------------
    def submit(self, device: TransportDevice, energies) -> Future:
        energies = np.asarray(energies, dtype=np.float64)
        choice = self.tuner.best(device.block_size, len(energies), self.precision)
        ne_call = min(int(choice["energies_per_call"]), len(energies))
        fp = TransportSolver.footprint_bytes(device.num_blocks, device.block_size, ne_call,
                                             ("density", "transmission"))
        with self._cv:
            req = Request(self._next_id, device, energies, time.perf_counter(), fp, choice)
            self._next_id += 1
            if fp > self.budget:
                req.future.set_exception(MemoryError(
                    f"request needs {fp} device bytes, above the server budget of {self.budget}"))
                return req.future
            self._queue.append(req)
            self._cv.notify_all()
        return req.future

    def close(self, wait: bool = True):
        with self._cv:
            self._closing = True
            self._cv.notify_all()
        if wait:
            self._scheduler.join()
        for w in self.workers:
            w.close()

    def stats(self) -> dict:
        lat = np.array(self.latencies) if self.latencies else np.array([np.nan])
        return {"completed": self.completed, "solves": self.solves, "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_s": float(np.mean(lat)),
                "peak_concurrency": self.peak_concurrency}

    # -- server side ---------------------------------------------------------
    def _schedule(self):
        while True:
            with self._cv:
                while True:
                    if self._closing and not self._queue and self._running == 0:
                        return
                    head = self._queue[0] if self._queue else None
                    if head is not None and self._free_workers and self._used + head.footprint <= self.budget:
                        break
                    self._cv.wait(timeout=0.05)
                req = self._queue.popleft()
                worker = self._free_workers.pop()
                self._used += req.footprint
                self._running += 1
                self.peak_concurrency = max(self.peak_concurrency, self._running)
            threading.Thread(target=self._run, args=(req, worker), daemon=True).start()

    def _run(self, req: Request, worker: Worker):
        try:
            res = worker.solve(req.device, req.energies, self.precision, req.choice, self.keys)
            latency = time.perf_counter() - req.submitted
            res["latency_s"] = latency
            with self._cv:
                self.latencies.append(latency)
                self.completed += 1
                self.solves += len(req.energies)
            req.future.set_result(res)
        except BaseException as exc:  # noqa: BLE001 -- delivered to the caller
            req.future.set_exception(exc)
        finally:
            with self._cv:
                self._used -= req.footprint
                self._running -= 1
                self._free_workers.append(worker)
                self._cv.notify_all()


def poisson_arrivals(count: int, rate_hz: float, seed: int = 0) -> np.ndarray:
    """Arrival offsets (seconds) of a seeded Poisson stream."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_hz, size=count))
