"""Autotuner of the transport solve, keyed on (block size, batch, precision).

For a key it times a short probe device (the seeded generator at the key's
block size, few blocks) over the candidate settings

* energies per device call (the batch the kernels see; powers of two and
  148, one per SM of a B200, which fills one wave of the block inverse;
  bounded by a memory budget),
* the GEMM path: FP64 DMMA or the INT8 split-product path (for a "mixed" key
  both paths satisfy the accuracy contract, so the faster one wins; a "fp64"
  key only uses DMMA),
* CUDA-graph replay of the sweep on or off,

and keeps the setting with the highest solves/s.  Results persist as JSON so
a production run tunes once per GPU model.
"""

from __future__ import annotations

import json
import os
import threading
import time

import torch

from quatrex_b200.transport import TransportSolver
from quatrex_b200.workloads import make_device

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "quatrex_b200", "autotune.json")


def _bucket(n: int) -> int:
    """Power-of-two bucket of an energy count."""
    b = 1
    while b < n:
        b *= 2
    return b


class Autotuner:
    def __init__(self, cache_path: str | None = None, memory_budget: int | None = None,
                 candidates_ne=(8, 16, 32, 64, 128, 148, 256), probe_blocks: int = 6, repeats: int = 2):
        self.cache_path = cache_path
        self.memory_budget = memory_budget
        self.candidates_ne = tuple(candidates_ne)
        self.probe_blocks = probe_blocks
        self.repeats = repeats
        self.table: dict[str, dict] = {}
        self._lock = threading.Lock()
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.table = json.load(f)

    @staticmethod
    def key(block_size: int, batch: int, precision: str) -> str:
        return f"b{int(block_size)}-n{_bucket(int(batch))}-{precision}"

    def lookup(self, block_size: int, batch: int, precision: str) -> dict | None:
        return self.table.get(self.key(block_size, batch, precision))

    def _budget(self) -> int:
        if self.memory_budget is not None:
            return int(self.memory_budget)
        free, _ = torch.cuda.mem_get_info()
        return int(free * 0.5)

    def _time(self, dev, ne: int, precision: str, graph: bool) -> float:
        energies = torch.linspace(-1.5, 1.5, ne, dtype=torch.float64)
        s = TransportSolver(dev, max_batch_size=ne, precision=precision, use_graph=graph)
        keys = ("density", "transmission")
        out = s.allocate_outputs(ne, keys)
        try:
            s.solve(energies, out)  # warm-up (and graph capture)
            torch.cuda.synchronize()
            best = float("inf")
            for _ in range(self.repeats):
                t0 = time.perf_counter()
                s.solve(energies, out)
                torch.cuda.synchronize()
                best = min(best, time.perf_counter() - t0)
        finally:
            if graph:
                # the probe's captured sweep (and its work space) is of no further use
                s.release_graphs()
                torch.cuda.synchronize()
        return ne / best

    def tune(self, block_size: int, batch: int, precision: str) -> dict:
        """Measure the candidates for this key and store the best."""
        b = int(block_size)
        dev = make_device(num_blocks=self.probe_blocks, block_size=b, num_energies=4, seed=2024)
        budget = self._budget()
        paths = ("fp64",) if precision == "fp64" else ("fp64", "mixed")
        cap = _bucket(int(batch))
        results = []
        for ne in self.candidates_ne:
            if ne > max(cap, self.candidates_ne[0]):
                break
            # footprint of a realistic (long) device at this batch, not of the probe
            if TransportSolver.footprint_bytes(64, b, ne, ("density", "transmission")) > budget:
                break
            for path in paths:
                for graph in (False, True):
                    try:
                        rate = self._time(dev, ne, path, graph)
                    except (MemoryError, RuntimeError):
                        continue
                    results.append({"energies_per_call": ne, "gemm_path": path, "graph": graph,
                                    "probe_solves_per_s": rate})
        if not results:
            choice = {"energies_per_call": self.candidates_ne[0], "gemm_path": "fp64", "graph": False,
                      "probe_solves_per_s": None}
        else:
            choice = max(results, key=lambda r: r["probe_solves_per_s"])
        choice = dict(choice, candidates=len(results))
        with self._lock:
            self.table[self.key(b, batch, precision)] = choice
            self.save()
        return choice

    def best(self, block_size: int, batch: int, precision: str) -> dict:
        got = self.lookup(block_size, batch, precision)
        return got if got is not None else self.tune(block_size, batch, precision)

    def save(self) -> None:
        if not self.cache_path:
            return
        os.makedirs(os.path.dirname(os.path.abspath(self.cache_path)), exist_ok=True)
        tmp = self.cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.table, f, indent=1, sort_keys=True)
        os.replace(tmp, self.cache_path)
