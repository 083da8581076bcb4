"""The partitioned RGF (RGFDist, nested dissection) on the GPU.

Against the oracle (the plain RGF restatement, pinned to upstream fixtures,
which the partitioned restatement equals to rounding: tests/test_oracle.py),
per returned block at 1e-10 relative Frobenius error, for 2, 3 and 4
partitions: selected inversion and selected solve with contact blocks and
interior self-energies, stack batching, host (NumPy) operands, mixed block
sizes and symmetric-storage outputs.  Every block operation of the
partitioned solver runs in libqtxrgf (GEMM, inverse, block combination).
The process-group mode (one partition per rank) runs as 2 and 3 processes
sharing this GPU with a gloo group (the exchange goes through host memory, so
no kernel of one rank waits on another) and must return, on every rank, the
blocks of its partition exactly as the single-process solver does.
"""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp
from scipy import sparse

from oracle import rgf_oracle as orc
from quatrex_b200.datastructures import DSDBCOO, DSDBCSR
from quatrex_b200.greens_function_solver import RGF, OBCBlocks
from quatrex_b200.rgf_dist import RGFDist
from quatrex_b200.workloads import make_device

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _system(nb=10, b=6, ne=4, seed=0, sizes=None):
    rng = np.random.default_rng(seed)
    sizes = [b] * nb if sizes is None else sizes
    nb = len(sizes)

    def rnd(*s):
        return rng.standard_normal(s) + 1j * rng.standard_normal(s)

    def skew(x):
        return x - x.conj().swapaxes(-1, -2)

    diag = [rnd(ne, s, s) + 6 * np.eye(s) for s in sizes]
    upper = [rnd(ne, sizes[i], sizes[i + 1]) for i in range(nb - 1)]
    lower = [rnd(ne, sizes[i + 1], sizes[i]) for i in range(nb - 1)]
    sl_d = [skew(rnd(ne, s, s)) for s in sizes]
    sg_d = [skew(rnd(ne, s, s)) for s in sizes]
    sl_u = [rnd(ne, sizes[i], sizes[i + 1]) for i in range(nb - 1)]
    sg_u = [rnd(ne, sizes[i], sizes[i + 1]) for i in range(nb - 1)]
    pad = [None] * (nb - 2)
    obc = OBCBlocks(nb)
    obc.retarded[0], obc.retarded[-1] = rnd(ne, sizes[0], sizes[0]), rnd(ne, sizes[-1], sizes[-1])
    obc.lesser[0], obc.lesser[-1] = skew(rnd(ne, sizes[0], sizes[0])), skew(rnd(ne, sizes[-1], sizes[-1]))
    obc.greater[0], obc.greater[-1] = skew(rnd(ne, sizes[0], sizes[0])), skew(rnd(ne, sizes[-1], sizes[-1]))
    lists = dict(diag=diag, upper=upper, lower=lower, sl_d=sl_d, sl_u=sl_u, sg_d=sg_d, sg_u=sg_u,
                 obc_r=[obc.retarded[0], *pad, obc.retarded[-1]], obc_l=[obc.lesser[0], *pad, obc.lesser[-1]],
                 obc_g=[obc.greater[0], *pad, obc.greater[-1]])
    return lists, obc


def _lower_of(upper):
    return [-u.conj().swapaxes(-1, -2) for u in upper]


@pytest.mark.parametrize("num_partitions", [2, 3, 4])
@pytest.mark.parametrize("max_batch_size", [4, 3])
def test_rgf_dist_selected_inv(num_partitions, max_batch_size):
    L, obc = _system(nb=11, seed=num_partitions)
    A = DSDBCOO.from_blocks(L["diag"], L["upper"], L["lower"], device="cuda")
    out = DSDBCOO.zeros_like(A)
    assert RGFDist(max_batch_size=max_batch_size, num_partitions=num_partitions).selected_inv(A, out, obc) is None
    ref = orc.selected_inv(L["diag"], L["upper"], L["lower"], L["obc_r"])
    nb = len(L["diag"])
    out = out.to("cpu")
    for i in range(nb):
        assert _rel(out.blocks[i, i], ref[0][i]) < TOL, i
    for i in range(nb - 1):
        assert _rel(out.blocks[i, i + 1], ref[1][i]) < TOL, i
        assert _rel(out.blocks[i + 1, i], ref[2][i]) < TOL, i


@pytest.mark.parametrize("num_partitions", [2, 3, 4])
@pytest.mark.parametrize("dsdb_type", [DSDBCOO, DSDBCSR], ids=["DSDBCOO", "DSDBCSR"])
def test_rgf_dist_selected_solve(num_partitions, dsdb_type):
    L, obc = _system(nb=12, b=5, seed=10 + num_partitions)
    A = dsdb_type.from_blocks(L["diag"], L["upper"], L["lower"], device="cuda")
    SL = dsdb_type.from_blocks(L["sl_d"], L["sl_u"], _lower_of(L["sl_u"]), device="cuda")
    SG = dsdb_type.from_blocks(L["sg_d"], L["sg_u"], _lower_of(L["sg_u"]), device="cuda")
    xl, xg, xr = (dsdb_type.zeros_like(A) for _ in range(3))
    RGFDist(max_batch_size=100, num_partitions=num_partitions).selected_solve(A, SL, SG, [xl, xg, xr], obc,
                                                                               return_retarded=True)
    ref = orc.selected_solve(L["diag"], L["upper"], L["lower"], L["sl_d"], L["sl_u"], L["sg_d"], L["sg_u"],
                             L["obc_r"], L["obc_l"], L["obc_g"])
    nb = len(L["diag"])
    for key, X in (("xl", xl.to("cpu")), ("xg", xg.to("cpu"))):
        for i in range(nb):
            assert _rel(X.blocks[i, i], ref[f"{key}_diag"][i]) < TOL, (key, i)
        for i in range(nb - 1):
            assert _rel(X.blocks[i, i + 1], ref[f"{key}_upper"][i]) < TOL, (key, i)
            assert _rel(X.blocks[i + 1, i], ref[f"{key}_lower"][i]) < TOL, (key, i)
    xr = xr.to("cpu")
    for i in range(nb):
        assert _rel(xr.blocks[i, i], ref["xr_diag"][i]) < TOL, i


def test_rgf_dist_equals_rgf_on_a_transport_device_with_host_data():
    """A seeded transport device (NumPy operands, mixed block sizes are not
    needed here) solved by RGF and by RGFDist with 4 partitions: the same
    G^<, G^> and diagonal G^R blocks at 1e-10."""
    dev = make_device(num_blocks=16, block_size=24, num_energies=5, seed=17)
    d, u, lo = dev.system_blocks()
    obc_d = orc.obc_self_energies(d, u, lo, dev.energies, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol,
                                  dev.sr_max_iter)
    nb = 16
    A = DSDBCOO.from_blocks(d, u, lo)
    Z = DSDBCOO.zeros_like(A)
    ob = OBCBlocks(nb)
    ob.retarded[0], ob.retarded[-1] = obc_d["retarded"]
    ob.lesser[0], ob.lesser[-1] = obc_d["lesser"]
    ob.greater[0], ob.greater[-1] = obc_d["greater"]
    ref = RGF().selected_solve(A, Z, Z, obc_blocks=ob, return_retarded=True)
    outs = [DSDBCOO.zeros_like(A) for _ in range(3)]
    RGFDist(num_partitions=4).selected_solve(A, Z, Z, outs, ob, return_retarded=True)
    assert isinstance(outs[0].data, np.ndarray)
    for got, want in zip(outs[:2], ref[:2]):
        for i in range(nb):
            assert _rel(got.blocks[i, i], want.blocks[i, i]) < TOL
        for i in range(nb - 1):
            assert _rel(got.blocks[i, i + 1], want.blocks[i, i + 1]) < TOL
    for i in range(nb):
        assert _rel(outs[2].blocks[i, i], ref[2].blocks[i, i]) < TOL


def test_rgf_dist_mixed_block_sizes_and_symmetric_outputs():
    sizes = [3, 4, 4, 2, 5, 3, 3, 4, 2]
    L, obc = _system(sizes=sizes, ne=3, seed=5)
    nb = len(sizes)
    A = DSDBCOO.from_blocks(L["diag"], L["upper"], L["lower"], device="cuda")
    SL = DSDBCOO.from_blocks(L["sl_d"], L["sl_u"], _lower_of(L["sl_u"]), device="cuda")
    SG = DSDBCOO.from_blocks(L["sg_d"], L["sg_u"], _lower_of(L["sg_u"]), device="cuda")
    neg_conj = lambda x: -np.conj(x)  # noqa: E731
    mask = DSDBCOO.from_blocks(L["diag"], L["upper"], L["lower"]).to_dense()[0] != 0
    pattern = sparse.coo_matrix(mask.astype(np.complex128))
    xl = DSDBCOO.from_sparray(pattern, np.array(sizes), (3,), symmetry=True,
                              symmetry_op=neg_conj, device="cuda")
    xl.data.zero_()
    xg = DSDBCOO.zeros_like(xl)
    RGFDist(num_partitions=3).selected_solve(A, SL, SG, [xl, xg], obc)
    ref = orc.selected_solve(L["diag"], L["upper"], L["lower"], L["sl_d"], L["sl_u"], L["sg_d"], L["sg_u"],
                             L["obc_r"], L["obc_l"], L["obc_g"])
    xl = xl.to("cpu")
    for i in range(nb):
        assert _rel(xl.blocks[i, i], ref["xl_diag"][i]) < TOL, i
    for i in range(nb - 1):
        assert _rel(xl.blocks[i, i + 1], ref["xl_upper"][i]) < TOL, i
        assert _rel(xl.blocks[i + 1, i], ref["xl_lower"][i]) < TOL, i


def test_rgf_dist_rejects_short_partitions():
    L, obc = _system(nb=5)
    A = DSDBCOO.from_blocks(L["diag"], L["upper"], L["lower"], device="cuda")
    with pytest.raises(ValueError):
        RGFDist(num_partitions=3).selected_inv(A, DSDBCOO.zeros_like(A))
    with pytest.raises(ValueError):
        RGFDist(num_partitions=1)


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _operands(ss):
    L, obc = _system(nb=11, b=5, seed=31)
    A = DSDBCOO.from_blocks(L["diag"], L["upper"], L["lower"], device="cuda")
    if not ss:
        return A, None, None, obc
    SL = DSDBCOO.from_blocks(L["sl_d"], L["sl_u"], _lower_of(L["sl_u"]), device="cuda")
    SG = DSDBCOO.from_blocks(L["sg_d"], L["sg_u"], _lower_of(L["sg_u"]), device="cuda")
    return A, SL, SG, obc


def _solve(solver, ss):
    A, SL, SG, obc = _operands(ss)
    if ss:
        outs = [DSDBCOO.zeros_like(A) for _ in range(3)]
        solver.selected_solve(A, SL, SG, outs, obc, return_retarded=True)
    else:
        outs = [DSDBCOO.zeros_like(A)]
        solver.selected_inv(A, outs[0], obc)
    return [o.to("cpu") for o in outs]


def _rank_worker(rank, world, port, ss, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        outs = _solve(RGFDist(max_batch_size=2, comm=dist.group.WORLD), ss)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), *[o.data for o in outs])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("ss", [False, True], ids=["inv", "solve"])
def test_rgf_dist_one_partition_per_rank(tmp_path, world, ss):
    mp.start_processes(_rank_worker, args=(world, _free_port(), ss, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    want = _solve(RGFDist(max_batch_size=2, num_partitions=world), ss)
    nb = len(want[0].block_sizes)
    bounds = [(0, 4), (4, 8), (8, 11)] if world == 3 else [(0, 6), (6, 11)]
    for rank, (s, e) in enumerate(bounds):
        got = np.load(tmp_path / f"r{rank}.npz")
        for k, w in enumerate(want):
            g = DSDBCOO.zeros_like(w)
            data = got[f"arr_{k}"]
            if isinstance(g.data, torch.Tensor):
                g.data.copy_(torch.from_numpy(data))
            else:
                g.data[...] = data
            keel = ss and k < 2
            for i in range(s, e):
                assert np.array_equal(g.blocks[i, i], w.blocks[i, i]), (rank, k, i)
                if i + 1 < nb and (keel or not ss):
                    assert np.array_equal(g.blocks[i, i + 1], w.blocks[i, i + 1]), (rank, k, i)
                    assert np.array_equal(g.blocks[i + 1, i], w.blocks[i + 1, i]), (rank, k, i)
