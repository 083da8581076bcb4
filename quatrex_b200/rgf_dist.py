"""Partitioned (nested-dissection) RGF: ``RGFDist``.

Mirrors ``qttools.greens_function_solver.RGFDist``
(``src/qttools/greens_function_solver/rgf_dist.py:16-384``, algorithm in
``src/qttools/greens_function_solver/_serinv.py``): the block axis is cut into
P partitions; the first partition eliminates its blocks downwards, the last
upwards, the middle ones with the permuted Schur complement that keeps their
first block coupled through buffer blocks; the 2 (P - 1) partition-boundary
blocks form a reduced block-tridiagonal system that is solved by RGF; the
results are mapped back and every partition finishes with its own selected
inversion.  Upstream gives each partition its own MPI rank.  Here the
partitions are either independent chains of block operations on their own
CUDA streams of one device (a long device with few energies keeps the GPU
busy with P chains of batched products in flight, and the reduced system is
the only sequential part), or, given a ``torch.distributed`` process group,
one partition per rank: the two boundary slots of every partition are
all-gathered (one collective per stack batch; NCCL over NVLink between GPUs)
and every rank solves the small reduced system itself, as upstream does.

Every block operation runs in ``libqtxrgf``: products and their
accumulations on the DMMA GEMM (``qtx_zgemm``, with its C epilogue), block
inverses on the batched Gauss-Jordan (``qtx_inv``), sums and conjugate
transposes on ``qtx_block_combine``.  There is no CPU path.

Differences from upstream, by design: the partition count is a constructor
argument or the size of the given process group (upstream takes it from its
MPI block communicator); upstream's
``permuted_selinv`` forms its product ``tmp2`` only when it solves for G^< /
G^> (``_serinv.py:1403``) yet uses it for G^R too (``:1515``), so upstream
``selected_inv`` fails with three or more partitions -- here it is formed in
both cases.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from quatrex_b200 import _lib
from quatrex_b200.datastructures import expand_symmetric, layout_of
from quatrex_b200.greens_function_solver import GFSolver, OBCBlocks

_N, _C = 0, 1


class _Ops:
    """Batched block operations on (batch, rows, cols) complex128 device tensors."""

    def __init__(self, dev: int, stream: torch.cuda.Stream):
        self.dev = dev
        self.stream = stream
        self.lib = _lib.load()
        self.ctx = _lib.context(dev)

    def _s(self):
        return self.stream.cuda_stream

    def empty(self, batch, rows, cols):
        with torch.cuda.stream(self.stream):
            return torch.empty((batch, rows, cols), dtype=torch.complex128, device=f"cuda:{self.dev}")

    def mm(self, a, b, op_a=_N, op_b=_N, alpha=1.0, c=None, beta=0.0):
        """alpha op(a) op(b) + beta c"""
        batch = a.shape[0]
        m = a.shape[-1] if op_a == _C else a.shape[-2]
        k = a.shape[-2] if op_a == _C else a.shape[-1]
        n = b.shape[-2] if op_b == _C else b.shape[-1]
        d = self.empty(batch, m, n)
        alpha, beta = complex(alpha), complex(beta)
        st = self.lib.qtx_zgemm(self.ctx, m, n, k, batch, alpha.real, alpha.imag, a.data_ptr(), a.stride(-2),
                                a.stride(0), op_a, b.data_ptr(), b.stride(-2), b.stride(0), op_b, beta.real, beta.imag,
                                c.data_ptr() if c is not None else None, c.stride(-2) if c is not None else n,
                                c.stride(0) if c is not None else 0,
                                d.data_ptr(), n, m * n, _lib.QTX_PREC_FP64, self._s())
        _lib.check(st, self.ctx, "RGFDist (block product)")
        return d

    def comb(self, x, y=None, alpha=1.0, beta=1.0, op_x=_N, op_y=_N):
        """alpha op(x) + beta op(y)"""
        batch = x.shape[0]
        rows = x.shape[-1] if op_x == _C else x.shape[-2]
        cols = x.shape[-2] if op_x == _C else x.shape[-1]
        out = self.empty(batch, rows, cols)
        alpha, beta = complex(alpha), complex(beta)
        st = self.lib.qtx_block_combine(self.ctx, rows, cols, batch, alpha.real, alpha.imag, x.data_ptr(),
                                        x.stride(-2), x.stride(0), op_x, beta.real, beta.imag,
                                        y.data_ptr() if y is not None else None,
                                        y.stride(-2) if y is not None else 0, y.stride(0) if y is not None else 0, op_y,
                                        out.data_ptr(), cols, rows * cols, self._s())
        _lib.check(st, self.ctx, "RGFDist (block combination)")
        return out

    def h(self, x):
        return self.comb(x, op_x=_C)

    def skew(self, x):
        """0.5 (x - x^H)"""
        return self.comb(x, x, alpha=0.5, beta=-0.5, op_y=_C)

    def inv(self, x):
        n = x.shape[-1]
        x = x.contiguous()
        out = self.empty(x.shape[0], n, n)
        st = self.lib.qtx_inv(self.ctx, n, x.shape[0], x.data_ptr(), n * n, out.data_ptr(), n * n, self._s())
        _lib.check(st, self.ctx, "RGFDist (block inverse)")
        return out


def _batch_offsets(num: int, max_batch: int) -> list[int]:
    """Stack batching of the solvers (``src/qttools/utils/solvers_utils.py:7-32``):
    num // min(max_batch, num) near-equal sections, the first ones larger."""
    n = num // min(max(1, int(max_batch)), num)
    base, rem = divmod(num, n)
    sizes = [base + 1 if k < rem else base for k in range(n)]
    return [0] + list(np.cumsum(sizes))


def partition_bounds(num_blocks: int, num_partitions: int) -> list[tuple[int, int]]:
    """Balanced contiguous partitions, the first ones one block larger
    (``src/qttools/utils/mpi_utils.py:16-67``); two blocks at least each."""
    base, rem = divmod(num_blocks, num_partitions)
    sizes = [base + 1 if p < rem else base for p in range(num_partitions)]
    if min(sizes) < 2:
        raise ValueError("RGFDist: every partition needs at least two blocks")
    starts = np.concatenate(([0], np.cumsum(sizes)))
    return [(int(starts[p]), int(starts[p + 1])) for p in range(num_partitions)]


class _Operand:
    """Dense (batch, bi, bj) views of the blocks of a DSDBSparse operand on
    the device (zero copy for dense blocks, a gather for sparse ones)."""

    def __init__(self, m, dev: int):
        if getattr(m, "symmetry", False):
            m = expand_symmetric(m, dev)
        self.lay = layout_of(m)
        data = m.data if isinstance(m.data, torch.Tensor) else torch.as_tensor(np.asarray(m.data))
        self.full = data.to(f"cuda:{dev}").reshape(-1, data.shape[-1])
        self.data = self.full

    def rows(self, e0: int, e1: int) -> "_Operand":
        view = object.__new__(_Operand)
        view.lay, view.full, view.data = self.lay, self.full, self.full[e0:e1]
        return view

    def block(self, i, j):
        lay = self.lay
        bi, bj = int(lay.block_sizes[i]), int(lay.block_sizes[j])
        k = 2 * i + j
        st, n = int(lay.block_offset[k]), int(lay.block_nnz[k])
        ne = self.data.shape[0]
        if st < 0 or n == 0:
            return torch.zeros((ne, bi, bj), dtype=torch.complex128, device=self.data.device)
        ix = lay.local_index[k]
        if ix is None:
            return self.data[:, st:st + n].reshape(ne, bi, bj)
        out = torch.zeros((ne, bi * bj), dtype=torch.complex128, device=self.data.device)
        out[:, torch.as_tensor(ix, dtype=torch.int64, device=self.data.device)] = self.data[:, st:st + n]
        return out.reshape(ne, bi, bj)


def _write_block(m, lay, data2d, i, j, value):
    """Store a dense (batch, bi, bj) block into block (i, j) of an output operand."""
    k = 2 * i + j
    if k < 0 or k >= len(lay.block_offset):
        return
    st, n = int(lay.block_offset[k]), int(lay.block_nnz[k])
    if st < 0 or n == 0:
        return
    ix = lay.local_index[k]
    v = value.reshape(value.shape[0], -1)
    if ix is None:
        data2d[:, st:st + n] = v
    else:
        data2d[:, st:st + n] = v[:, torch.as_tensor(ix, dtype=torch.int64, device=v.device)]


class RGFDist(GFSolver):
    """Partitioned selected inversion / selected solve (``rgf_dist.py:16-384``)
    with ``num_partitions`` partitions on the current CUDA device.

    ``selected_inv(a, out, obc_blocks=None)`` and
    ``selected_solve(a, sigma_lesser, sigma_greater, out, obc_blocks=None,
    return_retarded=False)`` take upstream's arguments (``out`` required) and
    write ``out`` in place."""

    def __init__(self, max_batch_size: int = 100, num_partitions: int = 2, comm=None) -> None:
        """``comm``: a ``torch.distributed`` process group; then every rank
        solves one partition (the partition count is the group size, as
        upstream takes it from its block communicator), every rank passes the
        same full operands, the reduced system is all-gathered (NCCL: device
        memory; gloo: through host memory) and solved on every rank, and each
        rank writes the blocks of its own partition (its block rows and the
        coupling to the next partition) into ``out``."""
        if comm is None and num_partitions < 2:
            raise ValueError("RGFDist needs at least two partitions (use RGF for one)")
        self.max_batch_size = max_batch_size
        self.num_partitions = num_partitions
        self.comm = comm

    # -- the shared driver ---------------------------------------------------
    def _run(self, a, sl, sg, outs, obc_blocks, ss: bool, return_retarded: bool):
        if not torch.cuda.is_available():
            raise RuntimeError("quatrex_b200 needs a CUDA device (B200, sm_100a); there is no CPU path")
        dev = torch.cuda.current_device()
        nb = a.num_blocks if hasattr(a, "num_blocks") else len(a.block_sizes)
        if self.comm is not None:
            import torch.distributed as dist

            rank, P = dist.get_rank(self.comm), dist.get_world_size(self.comm)
            if P < 2:
                raise ValueError("RGFDist needs at least two partitions (use RGF for one)")
            bounds = partition_bounds(nb, P)
            mine = [rank]
        else:
            bounds = partition_bounds(nb, self.num_partitions)
            P = len(bounds)
            mine = list(range(P))
        shapes = _slot_shapes(np.asarray(a.block_sizes), bounds)
        bmax = int(np.max(np.asarray(a.block_sizes)))
        if obc_blocks is None:
            obc_blocks = OBCBlocks(num_blocks=nb)
        stack = tuple(np.shape(a.data)[:-1])
        ne_all = int(math.prod(stack)) if stack else 1
        offs = _batch_offsets(ne_all, self.max_batch_size)
        # outputs: device working copies written back at the end
        out_dev = []
        for m in outs:
            if m is None:
                out_dev.append(None)
                continue
            t = m.data if isinstance(m.data, torch.Tensor) and m.data.is_cuda else None
            td = (t if t is not None else torch.as_tensor(np.asarray(m.data)).to(f"cuda:{dev}"))
            out_dev.append((m, layout_of(m), td.reshape(-1, td.shape[-1]), t is None))
        main = torch.cuda.current_stream(dev)
        streams = {p: torch.cuda.Stream(device=dev) for p in mine}
        A_all = _Operand(a, dev)
        SL_all = _Operand(sl, dev) if ss else None
        SG_all = _Operand(sg, dev) if ss else None
        for q in range(len(offs) - 1):
            e0, e1 = int(offs[q]), int(offs[q + 1])
            A = A_all.rows(e0, e1)
            SL = SL_all.rows(e0, e1) if ss else None
            SG = SG_all.rows(e0, e1) if ss else None

            def obc(which, i):
                lst = {"r": obc_blocks.retarded, "l": obc_blocks.lesser, "g": obc_blocks.greater}[which]
                x = lst[i] if lst is not None else None
                if x is None:
                    return None
                t = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(np.asarray(x)))
                t = t.to(device=f"cuda:{dev}", dtype=torch.complex128)
                return t.reshape(-1, t.shape[-2], t.shape[-1])[e0:e1]

            ev0 = torch.cuda.Event()
            ev0.record(main)
            parts = {}
            for p_idx in mine:
                s, e = bounds[p_idx]
                streams[p_idx].wait_event(ev0)
                part = _Part(p_idx, P, s, e, A, SL, SG, obc, _Ops(dev, streams[p_idx]), ss)
                with torch.cuda.stream(streams[p_idx]):
                    part.schur()
                parts[p_idx] = part
            # reduced system on the main stream once every partition is eliminated
            for st_ in streams.values():
                main.wait_stream(st_)
            ops = _Ops(dev, main)
            with torch.cuda.stream(main):
                if self.comm is None:
                    red = _gather_reduced([parts[p] for p in range(P)], ss)
                else:
                    part = parts[mine[0]]
                    buf = _pack_slots(_local_slots(part, ss), ss, e1 - e0, bmax, main.device)
                    red, neg_h = _reduced_from_gathered(_exchange_slots(buf, self.comm), shapes, P, ss)
                    for kind, i in neg_h:
                        red[kind][i] = ops.comb(red[kind][i], alpha=-1.0, op_x=_C)
                _reduced_solve(ops, red, ss)
                ev1 = torch.cuda.Event()
                ev1.record(main)
            blocks_out = []
            for p_idx, part in parts.items():
                streams[p_idx].wait_event(ev1)
                with torch.cuda.stream(streams[p_idx]):
                    part.map_back(red)
                    part.selinv()
                blocks_out.append(part.out)
            for st_ in streams.values():
                main.wait_stream(st_)
            # write the blocks of this stack batch into the outputs
            with torch.cuda.stream(main):
                keys = ("l", "g", "r") if ss else ("r",)
                for key, od in zip(keys, out_dev):
                    if od is None:
                        continue
                    m, lay, d2, _ = od
                    for part_out in blocks_out:
                        for (i, j), v in part_out[key].items():
                            _write_block(m, lay, d2[e0:e1], i, j, v)
                            if key != "r" and i != j and not getattr(m, "symmetry", False):
                                _write_block(m, lay, d2[e0:e1], j, i, -v.conj().transpose(-1, -2))
        torch.cuda.current_stream(dev).synchronize()
        for od in out_dev:
            if od is None:
                continue
            m, _, d2, host = od
            if host:
                m.data[...] = d2.reshape(np.shape(m.data)).cpu().numpy()

    def selected_inv(self, a, out, obc_blocks: OBCBlocks | None = None):
        """Selected inversion into ``out`` (``rgf_dist.py:37-131``)."""
        self._run(a, None, None, [out], obc_blocks, ss=False, return_retarded=True)

    def selected_solve(self, a, sigma_lesser, sigma_greater, out, obc_blocks: OBCBlocks | None = None,
                       return_retarded: bool = False):
        """Selected solve into ``out = (xl, xg[, xr])`` (``rgf_dist.py:133-384``)."""
        xl, xg, *xr = out
        if return_retarded:
            if len(xr) != 1:
                raise ValueError("Invalid number of output matrices.")
            xr = xr[0]
        else:
            xr = None
        self._run(a, sigma_lesser, sigma_greater, [xl, xg, xr], obc_blocks, ss=True,
                  return_retarded=return_retarded)


class _Part:
    """One partition: its blocks with local indices and its recursion state."""

    def __init__(self, idx, P, s, e, A, SL, SG, obc, ops: _Ops, ss: bool):
        self.idx, self.P, self.s, self.e, self.n = idx, P, s, e, e - s
        self.A, self.SL, self.SG, self.obc_fn, self.o, self.ss = A, SL, SG, obc, ops, ss
        self.kel = "lg" if ss else ""
        self.xr = [None] * self.n
        self.bl = [None] * self.n
        self.bu = [None] * self.n
        self.x = {c: [None] * self.n for c in "lg"}
        self.xb = {c: [None] * self.n for c in "lg"}
        self.out = {"r": {}, "l": {}, "g": {}}

    # block access with local indices
    def a(self, i, j):
        return self.A.block(self.s + i, self.s + j)

    def sigma(self, c, i, j):
        S = self.SL if c == "l" else self.SG
        gi, gj = self.s + i, self.s + j
        if gj == gi - 1:  # lower block of a skew-Hermitian operand: -upper^H
            return self.o.comb(S.block(gj, gi), alpha=-1.0, op_x=_C)
        return S.block(gi, gj)

    def a_obc(self, i):
        r = self.obc_fn("r", self.s + i)
        return self.a(i, i) if r is None else self.o.comb(self.a(i, i), r, beta=-1.0)

    def s_obc(self, c, i):
        o = self.obc_fn(c, self.s + i)
        return self.sigma(c, i, i) if o is None else self.o.comb(self.sigma(c, i, i), o)

    # X = x Y x^H
    def _sandwich(self, x, y):
        return self.o.mm(self.o.mm(x, y), x, op_b=_C)

    def schur(self):
        if self.idx == 0:
            self._downward_schur()
        elif self.idx == self.P - 1:
            self._upward_schur()
        else:
            self._permuted_schur()

    def _chain_step(self, i, j):
        """Downward / upward elimination of block i into block j (_serinv.py:797-864, 900-968)."""
        o = self.o
        self.xr[i] = o.inv(self.xr[i])
        for c in self.kel:
            self.x[c][i] = self._sandwich(self.xr[i], self.x[c][i])
        a_ji = self.a(j, i)
        a_ji_xr_ii = o.mm(a_ji, self.xr[i])
        self.xr[j] = o.mm(a_ji_xr_ii, self.a(i, j), alpha=-1.0, c=self.a_obc(j), beta=1.0)
        for c in self.kel:
            w = o.mm(a_ji_xr_ii, self.sigma(c, i, j))
            t = o.comb(w, w, alpha=-1.0, op_y=_C)  # w^H - w
            t = o.comb(t, self.s_obc(c, j))
            self.x[c][j] = o.mm(o.mm(a_ji, self.x[c][i]), a_ji, op_b=_C, c=t, beta=1.0)

    def _downward_schur(self):
        self.xr[0] = self.a_obc(0)
        for c in self.kel:
            self.x[c][0] = self.s_obc(c, 0)
        for i in range(self.n - 1):
            self._chain_step(i, i + 1)

    def _upward_schur(self):
        n = self.n - 1
        self.xr[n] = self.a_obc(n)
        for c in self.kel:
            self.x[c][n] = self.s_obc(c, n)
        for i in range(n, 0, -1):
            self._chain_step(i, i - 1)

    def _permuted_schur(self):
        """_serinv.py:971-1131."""
        o = self.o
        xr, bl, bu = self.xr, self.bl, self.bu
        bl[0] = self.a(0, 1)
        bu[0] = self.a(1, 0)
        xr[0] = self.a_obc(0)
        xr[1] = self.a_obc(1)
        for c in self.kel:
            self.xb[c][0] = self.sigma(c, 1, 0)
            self.x[c][0] = self.s_obc(c, 0)
            self.x[c][1] = self.s_obc(c, 1)
        for i in range(1, self.n - 1):
            j = i + 1
            xr[i] = o.inv(xr[i])
            a_ji = self.a(j, i)
            a_ij = self.a(i, j)
            xr_ii = xr[i]
            xr_ji_xr_ii = o.mm(bl[i - 1], xr_ii)
            a_ji_xr_ii = o.mm(a_ji, xr_ii)
            w = {c: o.mm(a_ji_xr_ii, self.sigma(c, i, j)) for c in self.kel}
            xr[j] = o.mm(a_ji_xr_ii, a_ij, alpha=-1.0, c=self.a_obc(j), beta=1.0)
            bl[i] = o.mm(xr_ji_xr_ii, a_ij, alpha=-1.0)
            bu[i] = o.mm(a_ji_xr_ii, bu[i - 1], alpha=-1.0)
            xr[0] = o.mm(xr_ji_xr_ii, bu[i - 1], alpha=-1.0, c=xr[0], beta=1.0)
            for c in self.kel:
                x, xb = self.x[c], self.xb[c]
                x[i] = self._sandwich(xr_ii, x[i])
                t = o.comb(w[c], w[c], alpha=-1.0, op_y=_C)
                t = o.comb(t, self.s_obc(c, j))
                x[j] = o.mm(o.mm(a_ji, x[i]), a_ji, op_b=_C, c=t, beta=1.0)
                # xb_i = a_ji x_i bl_{i-1}^H + S_ij^H (xr_ji xr_ii)^H - a_ji xr_ii xb_{i-1}
                t = o.mm(o.mm(a_ji, x[i]), bl[i - 1], op_b=_C)
                t = o.mm(self.sigma(c, i, j), xr_ji_xr_ii, op_a=_C, op_b=_C, c=t, beta=1.0)
                xb_new = o.mm(a_ji_xr_ii, xb[i - 1], alpha=-1.0, c=t, beta=1.0)
                # x_0 += bl_{i-1} x_i bl_{i-1}^H + xb_{i-1}^H (xr_ji xr_ii)^H - xr_ji xr_ii xb_{i-1}
                t = o.mm(o.mm(bl[i - 1], x[i]), bl[i - 1], op_b=_C, c=x[0], beta=1.0)
                t = o.mm(xb[i - 1], xr_ji_xr_ii, op_a=_C, op_b=_C, c=t, beta=1.0)
                x[0] = o.mm(xr_ji_xr_ii, xb[i - 1], alpha=-1.0, c=t, beta=1.0)
                xb[i] = xb_new

    def map_back(self, red):
        """_serinv.py:678-762: boundary blocks from the solved reduced system."""
        o = self.o
        p, n = self.idx, self.n
        if p > 0:
            k = 2 * p - 1
            self.xr[0] = red["xr"][k]
            for c in self.kel:
                self.x[c][0] = red["x" + c][k]
            if p < self.P - 1:
                self.bu[n - 2] = red["lo"][k]
                self.bl[n - 2] = red["up"][k]
                for c in self.kel:
                    self.xb[c][n - 2] = o.comb(red["x" + c + "_up"][k], alpha=-1.0, op_x=_C)
            self.out["r"][(self.s, self.s)] = self.xr[0]
            for c in self.kel:
                self.out[c][(self.s, self.s)] = self.x[c][0]
        if p < self.P - 1:
            k = 2 * p
            gi, gj = self.e - 1, self.e
            self.xr[n - 1] = red["xr"][k]
            self.out["r"][(gi, gi)] = red["xr"][k]
            self.out["r"][(gi, gj)] = red["up"][k]
            self.out["r"][(gj, gi)] = red["lo"][k]
            for c in self.kel:
                self.x[c][n - 1] = red["x" + c][k]
                self.out[c][(gi, gi)] = red["x" + c][k]
                self.out[c][(gi, gj)] = red["x" + c + "_up"][k]

    def selinv(self):
        if self.idx == 0:
            self._downward_selinv()
        elif self.idx == self.P - 1:
            self._upward_selinv()
        else:
            self._permuted_selinv()

    def _downward_selinv(self):
        """_serinv.py:1134-1225."""
        o, xr, s = self.o, self.xr, self.s
        for i in range(self.n - 2, -1, -1):
            j = i + 1
            xr_ii, xr_jj = xr[i], xr[j]
            xr_ii_a_ij = o.mm(xr_ii, self.a(i, j))
            xr_jj_a_ji = o.mm(xr_jj, self.a(j, i))
            p4 = o.mm(xr_ii_a_ij, xr_jj_a_ji)
            if self.kel:
                p3 = o.mm(xr_ii_a_ij, xr_jj)
            for c in self.kel:
                x = self.x[c]
                y = o.mm(xr_ii, self.sigma(c, i, j))
                t1 = o.mm(y, p3, op_b=_C, alpha=-1.0, c=o.mm(p4, x[i]), beta=1.0)
                t1 = o.comb(t1, t1, beta=-1.0, op_y=_C)
                t2 = o.mm(xr_ii_a_ij, x[j])
                x_ij = o.mm(x[i], xr_jj_a_ji, op_b=_C, alpha=-1.0, c=t2, beta=-1.0)
                x_ij = o.mm(y, xr_jj, op_b=_C, c=x_ij, beta=1.0)
                self.out[c][(i + s, j + s)] = x_ij
                x[i] = o.comb(o.mm(t2, xr_ii_a_ij, op_b=_C, c=x[i], beta=1.0), t1)
                self.out[c][(i + s, i + s)] = o.skew(x[i])
            self.out["r"][(j + s, i + s)] = o.mm(xr_jj_a_ji, xr_ii, alpha=-1.0)
            self.out["r"][(i + s, j + s)] = o.mm(xr_ii_a_ij, xr_jj, alpha=-1.0)
            xr[i] = o.mm(p4, xr_ii, c=xr_ii, beta=1.0)
            self.out["r"][(i + s, i + s)] = xr[i]

    def _upward_selinv(self):
        """_serinv.py:1228-1331."""
        o, xr, s = self.o, self.xr, self.s
        for i in range(1, self.n):
            j = i - 1
            xr_ii, xr_jj = xr[i], xr[j]
            xr_ii_a_ij = o.mm(xr_ii, self.a(i, j))
            xr_jj_a_ji = o.mm(xr_jj, self.a(j, i))
            p4 = o.mm(xr_ii_a_ij, xr_jj_a_ji)
            if self.kel:
                p3 = o.mm(xr_ii_a_ij, xr_jj)
            for c in self.kel:
                x = self.x[c]
                y = o.mm(xr_ii, self.sigma(c, i, j))
                t1 = o.mm(y, p3, op_b=_C)
                t1 = o.comb(t1, t1, beta=-1.0, op_y=_C)
                t_x = o.mm(xr_ii_a_ij, x[j])
                x_ij = o.mm(x[i], xr_jj_a_ji, op_b=_C, alpha=-1.0, c=t_x, beta=-1.0)
                x_ij = o.mm(y, xr_jj, op_b=_C, c=x_ij, beta=1.0)
                self.out[c][(j + s, i + s)] = o.comb(x_ij, alpha=-1.0, op_x=_C)
                t2 = o.mm(p4, x[i])
                acc = o.mm(t_x, xr_ii_a_ij, op_b=_C, c=x[i], beta=1.0)
                acc = o.comb(acc, t1, beta=-1.0)
                x[i] = o.comb(acc, o.comb(t2, t2, beta=-1.0, op_y=_C))
                self.out[c][(i + s, i + s)] = o.skew(x[i])
            self.out["r"][(j + s, i + s)] = o.mm(xr_jj_a_ji, xr_ii, alpha=-1.0)
            self.out["r"][(i + s, j + s)] = o.mm(xr_ii_a_ij, xr_jj, alpha=-1.0)
            xr[i] = o.mm(p4, xr_ii, c=xr_ii, beta=1.0)
            self.out["r"][(i + s, i + s)] = xr[i]

    def _permuted_selinv(self):
        """_serinv.py:1334-1531."""
        o, xr, bu, bl, s = self.o, self.xr, self.bu, self.bl, self.s
        for i in range(self.n - 2, 0, -1):
            xr_i, xr_ip1, xr_0 = xr[i], xr[i + 1], xr[0]
            a_i_ip1, a_ip1_i = self.a(i, i + 1), self.a(i + 1, i)
            bu_im1, bu_i, bl_im1, bl_i = bu[i - 1], bu[i], bl[i - 1], bl[i]
            xr_ip1_a_ip1_i = o.mm(xr_ip1, a_ip1_i)
            bu_i_bl_im1 = o.mm(bu_i, bl_im1)
            b1 = o.mm(bu_im1, bl_i, c=o.mm(a_i_ip1, xr_ip1), beta=1.0)
            b2 = o.mm(bu_im1, xr_0, c=o.mm(a_i_ip1, bu_i), beta=1.0)
            c1 = o.comb(xr_ip1_a_ip1_i, bu_i_bl_im1)
            c2 = o.mm(xr_0, bl_im1, c=o.mm(bl_i, a_ip1_i), beta=1.0)
            tmp2 = o.mm(xr_i, o.mm(b2, bl_im1, c=o.mm(b1, a_ip1_i), beta=1.0))
            if self.kel:
                tmp3 = o.h(c2)
                d1 = o.comb(xr_ip1_a_ip1_i, bu_i_bl_im1, op_x=_C, op_y=_C)  # (xr a)^H + (bu bl)^H
                tmp4 = o.mm(o.mm(tmp3, bu_im1, op_b=_C, c=o.mm(d1, a_i_ip1, op_b=_C), beta=1.0), xr_i, op_b=_C)
            for c in self.kel:
                x, xb = self.x[c], self.xb[c]
                x_i, x_ip1, x_0 = x[i], x[i + 1], x[0]
                s_i_ip1 = self.sigma(c, i, i + 1)
                tmp1 = o.mm(bu_im1, x_0, c=o.mm(a_i_ip1, xb[i]), beta=1.0)
                tmp5 = o.mm(xb[i - 1], xr_0, op_b=_C, c=o.mm(s_i_ip1, bl_i, op_b=_C), beta=1.0)
                tmp6 = o.mm(s_i_ip1, xr_ip1, op_b=_C)
                tmp6 = o.mm(xb[i - 1], bu_i, op_b=_C, c=tmp6, beta=1.0)
                tmp6 = o.mm(a_i_ip1, x_ip1, alpha=-1.0, c=tmp6, beta=1.0)
                tmp6 = o.mm(bu_im1, xb[i], op_b=_C, c=tmp6, beta=1.0)
                upper = o.mm(x_i, d1, alpha=-1.0, c=o.mm(xr_i, tmp6), beta=1.0)
                t51 = o.comb(tmp5, tmp1, beta=-1.0)
                # inner = b1 S_{i+1,i} + b2 (-xb_{i-1}^H) + (tmp5 - tmp1) bu_{i-1}^H + tmp6 a_{i,i+1}^H
                inner = o.mm(b1, self.sigma(c, i + 1, i))
                inner = o.mm(b2, xb[i - 1], op_b=_C, alpha=-1.0, c=inner, beta=1.0)
                inner = o.mm(t51, bu_im1, op_b=_C, c=inner, beta=1.0)
                inner = o.mm(tmp6, a_i_ip1, op_b=_C, c=inner, beta=1.0)
                acc = o.mm(tmp2, x_i, c=x_i, beta=1.0)
                acc = o.mm(x_i, tmp4, c=acc, beta=1.0)
                x[i] = o.mm(o.mm(xr_i, inner), xr_i, op_b=_C, alpha=-1.0, c=acc, beta=1.0)
                xb[i - 1] = o.mm(x_i, tmp3, alpha=-1.0, c=o.mm(xr_i, t51), beta=1.0)
                self.out[c][(i + s, i + 1 + s)] = upper
                self.out[c][(i + s, i + s)] = o.skew(x[i])
            self.out["r"][(i + s, i + 1 + s)] = o.mm(xr_i, b1, alpha=-1.0)
            self.out["r"][(i + 1 + s, i + s)] = o.mm(c1, xr_i, alpha=-1.0)
            bu[i - 1] = o.mm(xr_i, b2, alpha=-1.0)
            bl[i - 1] = o.mm(c2, xr_i, alpha=-1.0)
            xr[i] = o.mm(tmp2, xr_i, c=xr_i, beta=1.0)
            self.out["r"][(i + s, i + s)] = xr[i]
        self.out["r"][(1 + s, s)] = bu[0]
        self.out["r"][(s, 1 + s)] = bl[0]
        for c in self.kel:
            self.out[c][(s, 1 + s)] = o.comb(self.xb[c][0], alpha=-1.0, op_x=_C)


# -- the reduced system: slots, their order, and the exchange between ranks --
#
# Every partition p contributes the blocks of its first block row (slot 0,
# p > 0) and of its last block row (slot 1, p < P - 1) to the reduced system
# of the 2 (P - 1) partition-boundary blocks (_serinv.py:373-442; upstream
# all-gathers two slots per rank, :258-330).  Kinds per slot: the retarded
# diagonal "xr", the couplings "up" / "lo" and, for a selected solve, the
# Keldysh diagonals "xl" / "xg" and their upper couplings "xl_up" / "xg_up".
# Slot 0 of a middle partition couples its first block to its own last block
# through the buffer blocks; its "x?_up" entry is -(buffer)^H.

_KINDS_R = ("xr", "up", "lo")
_KINDS_SS = ("xr", "up", "lo", "xl", "xl_up", "xg", "xg_up")


def _kinds(ss):
    return _KINDS_SS if ss else _KINDS_R


def _reduced_order(P: int, ss: bool) -> list[tuple[int, int, str]]:
    """(partition, slot, kind) of every reduced-system entry, in the order of
    the reduced block lists: per kind, partition by partition, slot 0 before
    slot 1."""
    order = []
    kel = "lg" if ss else ""
    for p in range(P):
        if p > 0:
            order.append((p, 0, "xr"))
            order += [(p, 0, "x" + c) for c in kel]
            if p < P - 1:
                order += [(p, 0, "lo"), (p, 0, "up")]
                order += [(p, 0, "x" + c + "_up") for c in kel]
        if p < P - 1:
            order.append((p, 1, "xr"))
            order += [(p, 1, "x" + c) for c in kel]
            order += [(p, 1, "up"), (p, 1, "lo")]
            order += [(p, 1, "x" + c + "_up") for c in kel]
    return order


def _slot_shapes(block_sizes, bounds) -> dict:
    """(rows, cols) of every (partition, slot, kind) entry as exchanged
    (f, l: sizes of the partition's first and last block, nxt: the next
    partition's first block)."""
    bs = [int(b) for b in block_sizes]
    shapes = {}
    for p, (s, e) in enumerate(bounds):
        f, l = bs[s], bs[e - 1]
        nxt = bs[e] if e < len(bs) else 0
        for kind in _KINDS_SS:
            if kind in ("xr", "xl", "xg"):
                shapes[(p, 0, kind)], shapes[(p, 1, kind)] = (f, f), (l, l)
            elif kind == "lo":
                shapes[(p, 0, kind)], shapes[(p, 1, kind)] = (l, f), (nxt, l)
            elif kind == "up":
                shapes[(p, 0, kind)], shapes[(p, 1, kind)] = (f, l), (l, nxt)
            else:  # xl_up, xg_up: slot 0 holds the raw buffer block (l, f), its entry is -(.)^H
                shapes[(p, 0, kind)], shapes[(p, 1, kind)] = (l, f), (l, nxt)
    return shapes


def _local_slots(part, ss) -> dict:
    """The reduced-system entries of one eliminated partition, keyed by
    (slot, kind); slot 0's "x?_up" is the raw buffer block (negated and
    conjugate-transposed after the exchange)."""
    p, P, n = part.idx, part.P, part.n
    kel = "lg" if ss else ""
    out = {}
    if p > 0:
        out[(0, "xr")] = part.xr[0]
        for c in kel:
            out[(0, "x" + c)] = part.x[c][0]
        if p < P - 1:
            out[(0, "lo")] = part.bu[n - 2]
            out[(0, "up")] = part.bl[n - 2]
            for c in kel:
                out[(0, "x" + c + "_up")] = part.xb[c][n - 2]
    if p < P - 1:
        out[(1, "xr")] = part.xr[n - 1]
        for c in kel:
            out[(1, "x" + c)] = part.x[c][n - 1]
        out[(1, "up")] = part.a(n - 1, n)
        out[(1, "lo")] = part.a(n, n - 1)
        for c in kel:
            out[(1, "x" + c + "_up")] = part.sigma(c, n - 1, n)
    return out


def _pack_slots(slots: dict, ss: bool, batch: int, bmax: int, device) -> torch.Tensor:
    """One partition's entries in a (2, kinds, batch, bmax, bmax) buffer
    (zero padded; unused slots zero), the unit of the exchange."""
    kinds = _kinds(ss)
    buf = torch.zeros((2, len(kinds), batch, bmax, bmax), dtype=torch.complex128, device=device)
    for (slot, kind), t in slots.items():
        buf[slot, kinds.index(kind), :, :t.shape[-2], :t.shape[-1]] = t
    return buf


def _reduced_from(entry, P: int, ss: bool) -> tuple[dict, list]:
    """Reduced block lists from entry(p, slot, kind) -> (batch, rows, cols),
    plus the (kind, index) entries that must be replaced by -(.)^H."""
    red = {"xr": [], "up": [], "lo": []}
    for c in "lg":
        red["x" + c], red["x" + c + "_up"] = [], []
    neg_h = []
    for p, slot, kind in _reduced_order(P, ss):
        if slot == 0 and kind.endswith("_up") and kind != "up":
            neg_h.append((kind, len(red[kind])))
        red[kind].append(entry(p, slot, kind))
    return red, neg_h


def _reduced_from_gathered(gathered: torch.Tensor, shapes: dict, P: int, ss: bool) -> tuple[dict, list]:
    """Reduced block lists from the all-gathered (P, 2, kinds, batch, bmax,
    bmax) buffer: views of each entry at its own shape."""
    kinds = _kinds(ss)

    def entry(p, slot, kind):
        r, c = shapes[(p, slot, kind)]
        return gathered[p, slot, kinds.index(kind), :, :r, :c]

    return _reduced_from(entry, P, ss)


def _exchange_slots(buf: torch.Tensor, group) -> torch.Tensor:
    """All-gather one partition's slot buffer from every rank of ``group``:
    (P, 2, kinds, batch, bmax, bmax) on ``buf``'s device, rank order.  NCCL
    exchanges device memory; other backends (gloo) go through host memory
    (the stream is synchronised first)."""
    import torch.distributed as dist

    x = torch.view_as_real(buf)
    if dist.get_backend(group) != "nccl":
        if x.is_cuda:
            torch.cuda.current_stream(x.device).synchronize()
        x = x.cpu()
    recv = [torch.empty_like(x) for _ in range(dist.get_world_size(group))]
    dist.all_gather(recv, x, group=group)
    return torch.view_as_complex(torch.stack(recv).to(buf.device))


def _gather_reduced(parts, ss):
    """The reduced system of the partition boundary blocks (_serinv.py:373-442),
    all partitions in this process."""
    slots = [_local_slots(p, ss) for p in parts]
    red, neg_h = _reduced_from(lambda p, slot, kind: slots[p][(slot, kind)], len(parts), ss)
    o = parts[0].o
    for kind, i in neg_h:
        red[kind][i] = o.comb(red[kind][i], alpha=-1.0, op_x=_C)
    return red


def _reduced_solve(o: _Ops, red, ss):
    """RGF on the reduced system (_serinv.py:444-585)."""
    kel = "lg" if ss else ""
    xr, up, lo = red["xr"], red["up"], red["lo"]
    m = len(xr)

    def sandwich(x, y):
        return o.mm(o.mm(x, y), x, op_b=_C)

    for i in range(m - 1):
        xr[i] = o.inv(xr[i])
        for c in kel:
            red["x" + c][i] = sandwich(xr[i], red["x" + c][i])
        xr_ji_xr_ii = o.mm(lo[i], xr[i])
        xr[i + 1] = o.mm(xr_ji_xr_ii, up[i], alpha=-1.0, c=xr[i + 1], beta=1.0)
        for c in kel:
            w = o.mm(xr_ji_xr_ii, red["x" + c + "_up"][i])
            t = o.comb(o.comb(w, w, alpha=-1.0, op_y=_C), red["x" + c][i + 1])
            red["x" + c][i + 1] = o.mm(o.mm(lo[i], red["x" + c][i]), lo[i], op_b=_C, c=t, beta=1.0)
    xr[-1] = o.inv(xr[-1])
    for c in kel:
        red["x" + c][-1] = o.skew(sandwich(xr[-1], red["x" + c][-1]))
    for i in range(m - 2, -1, -1):
        xr_ii, xr_jj = xr[i], xr[i + 1]
        p1 = o.mm(xr_ii, up[i])
        p2 = o.mm(xr_jj, lo[i])
        p3 = o.mm(p1, xr_jj)
        p4 = o.mm(p1, p2)
        for c in kel:
            x, xu = red["x" + c], red["x" + c + "_up"]
            y = o.mm(xr_ii, xu[i])
            t1 = o.mm(y, p3, op_b=_C, alpha=-1.0, c=o.mm(p4, x[i]), beta=1.0)
            t1 = o.comb(t1, t1, beta=-1.0, op_y=_C)
            t2 = o.mm(p1, x[i + 1])
            u = o.mm(x[i], p2, op_b=_C, alpha=-1.0, c=t2, beta=-1.0)
            xu[i] = o.mm(y, xr_jj, op_b=_C, c=u, beta=1.0)
            x[i] = o.skew(o.comb(o.mm(t2, p1, op_b=_C, c=x[i], beta=1.0), t1))
        lo[i] = o.mm(p2, xr_ii, alpha=-1.0)
        up[i] = o.comb(p3, alpha=-1.0)
        xr[i] = o.mm(p4, xr_ii, c=xr_ii, beta=1.0)
