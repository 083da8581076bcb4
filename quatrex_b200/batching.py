"""Uneven batches of transport instances on one GPU.

Instances differ in block size, number of blocks and energy grid.  The
instances of each block size b <= 64 run together in ONE persistent launch
(qtx_transport_solve_grouped: every (instance, energy) pair of the group is a
work item of one kernel, a CTA solves a whole energy, pairs are handed out
longest instance first).  Larger instances are solved one by one: per
instance the energy grid is cut into device calls of the size the autotuner
picked for (block size, number of energies, precision), and the sweep of every
full-size call is a replayed CUDA graph when the tuner found that faster.
Each job (a group or a large instance) runs on a worker that owns a CUDA
stream and its own library context, so several jobs share the device; jobs
are handed out longest first.

Only observables travel back to the host (per-block density and hole
density, transmission, contact currents, Sancho-Rubio iteration counts); the
Green's-function blocks stay on the device inside each call.
"""

from __future__ import annotations

import math
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np
import torch

from quatrex_b200 import _lib
from quatrex_b200.autotune import Autotuner
from quatrex_b200.transport import (GROUPED_MAX_BLOCK_SIZE, TransportSolver, grouped_footprint_bytes,
                                    solve_grouped)
from quatrex_b200.workloads import TransportDevice

# largest block size whose sweeps are captured as CUDA graphs
GRAPH_MAX_BLOCK_SIZE = 128

OBSERVABLE_KEYS = ("density", "hole_density", "transmission", "current_left", "current_right", "sr_iterations", "dos",
                   "layer_current")


def instance_flops(dev: TransportDevice, num_energies: int) -> float:
    """Algorithmic flops of one instance with observables only (8 b^3 per
    block product; 17 per block step, the G^R off-diagonal outputs not being
    formed; Sancho-Rubio at ~22 iterations per contact)."""
    b, nb = dev.block_size, dev.num_blocks
    return 8.0 * b ** 3 * (17 * (nb - 1) + 11 + 2 * (7 * 22 + 1)) * num_energies


class Worker:
    """A CUDA stream plus its own library context, driven by one host thread."""

    def __init__(self, cuda_device: int):
        self.cuda = cuda_device
        self.stream = torch.cuda.Stream(device=cuda_device)
        self.ctx = _lib.new_context(cuda_device)
        self.busy_s = 0.0

    def close(self):
        if self.ctx:
            torch.cuda.synchronize(self.cuda)
            _lib.destroy_context(self.ctx)
            self.ctx = None

    def solve(self, dev: TransportDevice, energies: np.ndarray, precision: str, choice: dict,
              keys=OBSERVABLE_KEYS) -> dict:
        """Solve one instance on this worker's stream; returns host arrays."""
        t0 = time.perf_counter()
        ne_call = int(choice["energies_per_call"])
        path = choice.get("gemm_path", precision)
        # a captured sweep pays off only when it is replayed: use it when the
        # instance has at least three full-size calls (same buffers each time)
        # and its launches are short (b <= 128; a captured sweep also keeps
        # its work space for the life of the instance)
        graph = (bool(choice.get("graph", False)) and len(energies) // max(ne_call, 1) >= 3
                 and dev.block_size <= GRAPH_MAX_BLOCK_SIZE)
        energies = np.asarray(energies, dtype=np.float64)
        results = {k: [] for k in keys}
        with torch.cuda.stream(self.stream):
            h_diag = torch.from_numpy(dev.h_diag).to(f"cuda:{self.cuda}", non_blocking=False)
            h_upper = torch.from_numpy(dev.h_upper).to(f"cuda:{self.cuda}", non_blocking=False)
            solver = TransportSolver(dev, max_batch_size=ne_call, precision=path, cuda_device=self.cuda,
                                     h_diag=h_diag, h_upper=h_upper, ctx=self.ctx, stream=self.stream,
                                     use_graph=graph)
            outs = {}
            for c0 in range(0, len(energies), ne_call):
                chunk = energies[c0:c0 + ne_call]
                n = len(chunk)
                if n not in outs:
                    outs[n] = solver.allocate_outputs(n, keys)
                try:
                    out = solver.solve(chunk, outs[n])
                except MemoryError:
                    # memory torch's caching allocator keeps for freed tensors is
                    # out of reach of the library's stream-ordered pool: hand it
                    # back, drop this instance's captured sweep (its work space
                    # stays allocated while it exists) and retry eagerly
                    if solver.use_graph:
                        solver.release_graphs()
                        solver.use_graph = False
                    torch.cuda.synchronize(self.cuda)
                    torch.cuda.empty_cache()
                    out = solver.solve(chunk, outs[n])
                for k in keys:
                    results[k].append(out[k].cpu())
            if solver.use_graph:
                # the captured sweeps reference this instance's buffers: drop them
                solver.release_graphs()
            self.stream.synchronize()
        self.busy_s += time.perf_counter() - t0
        return {k: torch.cat(v).numpy() for k, v in results.items()}

    def solve_group(self, devs: list[TransportDevice], energies: list, keys=OBSERVABLE_KEYS) -> list[dict]:
        """Every energy of several instances of one block size in one
        persistent launch on this worker's stream; returns host arrays."""
        t0 = time.perf_counter()
        dev = f"cuda:{self.cuda}"
        with torch.cuda.stream(self.stream):
            hs = [(torch.from_numpy(d.h_diag).to(dev), torch.from_numpy(d.h_upper).to(dev)) for d in devs]
            outs = solve_grouped(devs, [np.asarray(e, dtype=np.float64) for e in energies], keys=keys,
                                 cuda_device=self.cuda, hamiltonians=hs, ctx=self.ctx, stream=self.stream)
            res = [{k: v.cpu().numpy() for k, v in out.items()} for out in outs]
        self.busy_s += time.perf_counter() - t0
        return res


@dataclass
class Instance:
    device: TransportDevice
    energies: np.ndarray


class BatchedTransport:
    """Solve a list of uneven instances with ``streams`` concurrent workers."""

    def __init__(self, precision: str = "fp64", streams: int = 4, tuner: Autotuner | None = None,
                 cuda_device: int | None = None, keys=OBSERVABLE_KEYS, memory_budget: int | None = None,
                 group_small: bool = True):
        self.precision = precision
        # instances with b <= 64 share one persistent launch per block size
        # (FP64 products: the INT8 split products only pay off at b >= 512)
        self.group_small = group_small
        self.cuda = torch.cuda.current_device() if cuda_device is None else cuda_device
        if memory_budget is None:
            free, _ = torch.cuda.mem_get_info(self.cuda)
            memory_budget = int(free * 0.6)
        self.budget = int(memory_budget)
        self._used = 0
        self.tuner = tuner if tuner is not None else Autotuner()
        self.keys = keys
        self.workers = [Worker(self.cuda) for _ in range(max(1, streams))]
        self._free = list(self.workers)
        self._cv = threading.Condition()

    def close(self):
        for w in self.workers:
            w.close()

    def _take(self) -> Worker:
        with self._cv:
            while not self._free:
                self._cv.wait()
            return self._free.pop()

    def _give(self, w: Worker):
        with self._cv:
            self._free.append(w)
            self._cv.notify()

    def choice_for(self, inst: Instance) -> dict:
        """Tuned setting, with the energies per call capped so that one call of
        this instance (its actual number of blocks) fits in the budget."""
        c = dict(self.tuner.best(inst.device.block_size, len(inst.energies), self.precision))
        ne = int(c["energies_per_call"])
        while ne > 1 and self.footprint(inst, ne) > self.budget:
            ne //= 2
        c["energies_per_call"] = max(1, ne)
        return c

    def footprint(self, inst: Instance, ne_call: int) -> int:
        return TransportSolver.footprint_bytes(inst.device.num_blocks, inst.device.block_size,
                                               min(ne_call, len(inst.energies)), ("density", "transmission"),
                                               precision=self.precision)

    def group_footprint(self, members: list[Instance]) -> int:
        """Device bytes of one grouped launch: its work space, H and the outputs."""
        b = members[0].device.block_size
        ws = grouped_footprint_bytes([m.device.num_blocks for m in members], [len(m.energies) for m in members], b)
        h = sum(16 * b * b * (3 * m.device.num_blocks) for m in members)
        out = sum(64 * len(m.energies) * (m.device.num_blocks + 2) for m in members)
        return int(ws + h + out)

    def jobs(self, instances: list[Instance]) -> list[tuple[str, list[int]]]:
        """("group", members) per block size <= 64 when grouping, else ("one", [i]);
        longest first."""
        groups: dict[int, list[int]] = {}
        singles = []
        for i, x in enumerate(instances):
            b = x.device.block_size
            if self.group_small and b <= GROUPED_MAX_BLOCK_SIZE and len(x.energies) > 0:
                groups.setdefault(b, []).append(i)
            else:
                singles.append(i)
        cost = lambda idx: sum(instance_flops(instances[i].device, len(instances[i].energies)) for i in idx)
        out = [("group", idx) for idx in groups.values()] + [("one", [i]) for i in singles]
        return sorted(out, key=lambda j: -cost(j[1]))

    def run(self, instances: list[Instance]) -> list[dict]:
        """Results in input order; each dict also holds 'seconds' (wall time of
        its job on its worker: the whole group's for grouped instances) and
        'grouped' (whether it ran in a grouped launch)."""
        jobs = self.jobs(instances)
        # tune every key up front (serially), so workers only read the table
        for kind, idx in jobs:
            if kind == "one":
                self.choice_for(instances[idx[0]])
        results: list[dict | None] = [None] * len(instances)

        def job(j):
            kind, idx = j
            if kind == "one":
                choice = self.choice_for(instances[idx[0]])
                fp = self.footprint(instances[idx[0]], int(choice["energies_per_call"]))
            else:
                fp = self.group_footprint([instances[i] for i in idx])
            with self._cv:
                # admission by device-memory footprint next to the jobs already running
                while self._used + fp > self.budget and self._used > 0:
                    self._cv.wait()
                self._used += fp
            w = self._take()
            try:
                t0 = time.perf_counter()
                if kind == "one":
                    r = w.solve(instances[idx[0]].device, instances[idx[0]].energies, self.precision, choice,
                                self.keys)
                    r["seconds"] = time.perf_counter() - t0
                    r["grouped"] = False
                    results[idx[0]] = r
                else:
                    rs = w.solve_group([instances[i].device for i in idx], [instances[i].energies for i in idx],
                                       self.keys)
                    dt = time.perf_counter() - t0
                    for i, r in zip(idx, rs):
                        r["seconds"] = dt
                        r["grouped"] = True
                        results[i] = r
            finally:
                self._give(w)
                with self._cv:
                    self._used -= fp
                    self._cv.notify_all()

        with ThreadPoolExecutor(max_workers=len(self.workers)) as ex:
            list(ex.map(job, jobs))
        return results


def total_solves(instances: list[Instance]) -> int:
    return int(sum(len(x.energies) for x in instances))


def total_flops(instances: list[Instance]) -> float:
    return float(sum(instance_flops(x.device, len(x.energies)) for x in instances))


def geometric_energies(n: int, e_min: float = -2.0, e_max: float = 2.0) -> np.ndarray:
    return np.linspace(e_min, e_max, int(n))


def ceil_div(a: int, b: int) -> int:
    return int(math.ceil(a / b))
