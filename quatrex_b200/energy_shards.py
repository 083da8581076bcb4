"""Energy sharding across GPUs: one process per GPU, each solving its own
energies (the upstream stack distribution, ``src/qttools/datastructures/dsdbsparse.py:163-212``
with ``get_section_sizes`` ``src/qttools/utils/mpi_utils.py:16-67``).

Energies are independent, so the solve itself exchanges nothing; the only
collectives are the gather of per-energy observables at the end and the
max-over-ranks of timings.  Both go through ``torch.distributed`` (NCCL between
GPUs, gloo on CPU).
"""

from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def section_sizes(num: int, sections: int) -> list[int]:
    """Balanced split: the first ``num % sections`` sections get one more element."""
    q, r = divmod(int(num), int(sections))
    return [q + 1 if k < r else q for k in range(sections)]


def shard_slice(num: int, world: int, rank: int) -> slice:
    """Contiguous slice of ``num`` energies owned by ``rank``."""
    sizes = section_sizes(num, world)
    start = int(np.sum(sizes[:rank]))
    return slice(start, start + sizes[rank])


def gather_energy_results(local: torch.Tensor, num: int, group=None) -> torch.Tensor:
    """All-gather per-energy results (leading axis = this rank's energies) into
    the full ``num``-energy array on every rank (uneven shards are padded)."""
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return local
    world = dist.get_world_size(group)
    sizes = section_sizes(num, world)
    pad = max(sizes)
    buf = torch.zeros((pad,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    buf[: local.shape[0]] = local
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([p[:s] for p, s in zip(parts, sizes)], dim=0)


def max_over_ranks(value: float, device=None, group=None) -> float:
    """Maximum of a per-rank scalar (e.g. an elapsed time) over all ranks."""
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
