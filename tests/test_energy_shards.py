"""Multi-rank host logic of the energy sharding, run as world_size-2 gloo
process groups on the CPU (the data path itself exchanges nothing)."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from quatrex_b200.energy_shards import gather_energy_results, max_over_ranks, section_sizes, shard_slice


def test_section_sizes_match_upstream_rule():
    assert section_sizes(10, 3) == [4, 3, 3]
    assert section_sizes(7, 2) == [4, 3]
    assert sum(section_sizes(1024, 8)) == 1024
    slices = [shard_slice(13, 4, r) for r in range(4)]
    assert slices[0].start == 0 and slices[-1].stop == 13
    assert all(a.stop == b.start for a, b in zip(slices, slices[1:]))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, num, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sl = shard_slice(num, world, rank)
        energies = torch.linspace(-2, 2, num, dtype=torch.float64)[sl]
        # a per-energy "observable" computed locally: density-like (E, nb) and transmission-like (E,)
        local_density = torch.stack([energies * (k + 1) for k in range(3)], dim=1)
        local_t = energies ** 2 + rank * 0.0
        full_d = gather_energy_results(local_density, num)
        full_t = gather_energy_results(local_t, num)
        tmax = max_over_ranks(1.0 + rank)
        np.save(os.path.join(out_dir, f"r{rank}.npy"),
                np.concatenate([full_d.numpy().ravel(), full_t.numpy(), [tmax]]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("num", [8, 11])
def test_gather_and_max_two_ranks(tmp_path, num):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), num, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    e = np.linspace(-2, 2, num)
    want_d = np.stack([e * (k + 1) for k in range(3)], axis=1).ravel()
    want = np.concatenate([want_d, e ** 2, [2.0]])
    for r in range(world):
        got = np.load(tmp_path / f"r{r}.npy")
        assert np.allclose(got, want)
