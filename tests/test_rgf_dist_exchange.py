"""The reduced-system exchange of the partitioned RGF (``RGFDist`` with a
process group), as world_size 2 and 3 gloo process groups on the CPU.

Every rank builds the boundary slots of its own partition (stand-in blocks:
seeded random tensors of the shapes the elimination produces), packs them,
all-gathers them with the library's exchange and assembles the reduced block
lists; every rank must end with exactly the lists that the single-process
path assembles from all partitions (upstream all-gathers two slots per rank,
``src/qttools/greens_function_solver/_serinv.py:258-330``).  Constant and mixed
block sizes (upstream switches to a pickled gather for the latter, ``:111-201``;
here both go through one zero-padded buffer)."""

import os
import socket
import zlib

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from quatrex_b200.rgf_dist import (_exchange_slots, _local_slots, _pack_slots, _reduced_from,
                                   _reduced_from_gathered, _reduced_order, _slot_shapes, partition_bounds)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _blk(tag, rows, cols, batch=3):
    g = torch.Generator().manual_seed(zlib.crc32(repr(tag).encode()))  # the same on every rank
    re = torch.randn(batch, rows, cols, generator=g, dtype=torch.float64)
    im = torch.randn(batch, rows, cols, generator=g, dtype=torch.float64)
    return torch.complex(re, im)


class _StandInPart:
    """The fields of an eliminated partition that the exchange reads, filled
    with seeded blocks of the elimination's shapes (global block sizes bs)."""

    def __init__(self, p, P, s, e, bs):
        self.idx, self.P, self.s, self.e, self.n = p, P, s, e, e - s
        n, f, l = self.n, bs[s], bs[e - 1]
        self.bs = bs
        self.xr = [None] * n
        self.bl, self.bu = [None] * n, [None] * n
        self.x = {c: [None] * n for c in "lg"}
        self.xb = {c: [None] * n for c in "lg"}
        self.xr[0], self.xr[n - 1] = _blk((p, "xr0"), f, f), _blk((p, "xrn"), l, l)
        self.bl[n - 2], self.bu[n - 2] = _blk((p, "bl"), f, l), _blk((p, "bu"), l, f)
        for c in "lg":
            self.x[c][0], self.x[c][n - 1] = _blk((p, c, "x0"), f, f), _blk((p, c, "xn"), l, l)
            self.xb[c][n - 2] = _blk((p, c, "xb"), l, f)

    def a(self, i, j):
        gi, gj = self.s + i, self.s + j
        return _blk(("a", gi, gj), self.bs[gi], self.bs[gj])

    def sigma(self, c, i, j):
        gi, gj = self.s + i, self.s + j
        return _blk(("s", c, gi, gj), self.bs[gi], self.bs[gj])


def _worker(rank, world, port, sizes, ss, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bounds = partition_bounds(len(sizes), world)
        shapes = _slot_shapes(np.asarray(sizes), bounds)
        parts = [_StandInPart(p, world, s, e, sizes) for p, (s, e) in enumerate(bounds)]
        mine = parts[rank]
        buf = _pack_slots(_local_slots(mine, ss), ss, 3, max(sizes), "cpu")
        gathered = _exchange_slots(buf, dist.group.WORLD)
        red, neg_h = _reduced_from_gathered(gathered, shapes, world, ss)
        # the single-process assembly from every partition's own slots
        slots = [_local_slots(p, ss) for p in parts]
        want, want_neg = _reduced_from(lambda p, slot, kind: slots[p][(slot, kind)], world, ss)
        assert neg_h == want_neg
        ok = all(len(red[k]) == len(want[k]) for k in want)
        ok = ok and all(torch.equal(a.contiguous(), b) for k in want for a, b in zip(red[k], want[k]))
        # sizes of the reduced system: 2 (P - 1) diagonal blocks, one coupling fewer
        ok = ok and len(red["xr"]) == 2 * (world - 1) and len(red["up"]) == 2 * world - 3
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array([ok, len(neg_h)]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("sizes", [[3] * 8, [3, 4, 2, 5, 3, 4, 2, 3]], ids=["constant", "mixed"])
@pytest.mark.parametrize("ss", [False, True], ids=["inv", "solve"])
def test_reduced_system_exchange(tmp_path, world, sizes, ss):
    mp.start_processes(_worker, args=(world, _free_port(), sizes, ss, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        ok, nneg = np.load(tmp_path / f"r{r}.npy")
        assert ok
        assert nneg == (2 * (world - 2) if ss else 0)


def test_reduced_order_matches_upstream_slots():
    """Entry order of the reduced lists: partition by partition, first block
    row before last block row, the outer slots of the first and last
    partitions dropped (upstream keeps slots [1:-1] of its 2P gathered slots)."""
    order = _reduced_order(3, False)
    xr = [(p, s) for p, s, k in order if k == "xr"]
    assert xr == [(0, 1), (1, 0), (1, 1), (2, 0)]
    up = [(p, s) for p, s, k in order if k == "up"]
    assert up == [(0, 1), (1, 0), (1, 1)]
