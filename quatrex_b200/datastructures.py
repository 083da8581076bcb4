"""DSDBSparse block layout on the device.

``DSDBCOO`` keeps the data layout of qttools' DSDBCOO
(``src/qttools/datastructures/dsdbcoo.py:23-1008``, base class
``src/qttools/datastructures/dsdbsparse.py:109-879``): a ``(*stack, nnz)``
complex array whose nonzeros are sorted block-row by block-row and, inside a
block row, block by block (``compute_block_sort_index``,
``src/qttools/kernels/datastructure/numba/dsdbcoo.py:172-236``), so block (i, j)
is one contiguous slice of every data row.  Inside a block the entries keep
canonical COO (row-major) order; a block whose every entry is present is
therefore a row-major dense tile and the kernels read and write it in place.

The data may live on a CUDA device (``torch`` tensor, the fast path) or on the
host (``numpy``); the solvers move host data to the device and back.  Only the
single-rank stack/block distribution is modelled (one GPU holds the whole
stack slice it is given).

``btd_layout`` also accepts any object with ``rows``, ``cols``,
``block_sizes`` and ``data`` attributes of that layout (an upstream qttools
DSDBCOO included).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from quatrex_b200 import _lib


@dataclass
class BtdLayout:
    """Block map of a block-tridiagonal DSDBSparse pattern (the qtx_btd_desc)."""

    block_sizes: np.ndarray  # int32 [nb]
    block_offset: np.ndarray  # int64 [3nb-2]
    block_nnz: np.ndarray  # int64 [3nb-2]
    local_index: list  # [3nb-2] of None (dense row-major / empty) or int32 numpy arrays
    nnz: int
    _dev_index: dict = field(default_factory=dict)

    @property
    def num_blocks(self) -> int:
        return int(len(self.block_sizes))

    def all_dense(self) -> bool:
        return all(ix is None for ix in self.local_index)

    def desc(self, stack_size: int, stack_stride: int, device: int | None) -> tuple[_lib.BtdDesc, list]:
        """ctypes descriptor plus the objects that must stay alive while it is used."""
        keep = []
        bs = np.ascontiguousarray(self.block_sizes, dtype=np.int32)
        bo = np.ascontiguousarray(self.block_offset, dtype=np.int64)
        bn = np.ascontiguousarray(self.block_nnz, dtype=np.int64)
        keep += [bs, bo, bn]
        idx_ptrs = None
        if not self.all_dense():
            if device is None:
                raise ValueError("sparse block patterns need a device for their index arrays")
            devs = self._dev_index.get(device)
            if devs is None:
                devs = [
                    None if ix is None else torch.as_tensor(ix, dtype=torch.int32).to(f"cuda:{device}")
                    for ix in self.local_index
                ]
                self._dev_index[device] = devs
            arr = (ctypes.c_void_p * len(devs))(*[0 if t is None else t.data_ptr() for t in devs])
            keep += [devs, arr]
            idx_ptrs = ctypes.cast(arr, ctypes.POINTER(ctypes.c_void_p))
        d = _lib.BtdDesc(
            num_blocks=len(bs),
            block_sizes=bs.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            block_offset=bo.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            block_nnz=bn.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            block_index=idx_ptrs,
            stack_size=int(stack_size),
            stack_stride=int(stack_stride),
        )
        return d, keep


def btd_layout_from_coords(rows: np.ndarray, cols: np.ndarray, block_sizes) -> BtdLayout:
    """Block map of block-sorted coordinates (raises if the pattern is not BTD or not block-sorted)."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    bsz = np.asarray(block_sizes, dtype=np.int64)
    nb = len(bsz)
    offs = np.concatenate(([0], np.cumsum(bsz)))
    br = np.searchsorted(offs, rows, side="right") - 1
    bc = np.searchsorted(offs, cols, side="right") - 1
    if rows.size and (np.abs(br - bc) > 1).any():
        raise ValueError("pattern is not block-tridiagonal for these block sizes")
    k = 2 * br + bc
    if rows.size and (np.diff(k) < 0).any():
        raise ValueError("nonzeros are not block-sorted (DSDBSparse layout expected)")
    nblk = 3 * nb - 2
    block_offset = np.full(nblk, -1, dtype=np.int64)
    block_nnz = np.zeros(nblk, dtype=np.int64)
    local_index: list = [None] * nblk
    if rows.size:
        uk, start, count = np.unique(k, return_index=True, return_counts=True)
        for kk, st, cn in zip(uk, start, count):
            kk = int(kk)
            # recover (i, j) from k = 2i + j with j in {i-1, i, i+1}
            i = (kk + 1) // 3
            j = kk - 2 * i
            bi, bj = int(bsz[i]), int(bsz[j])
            lin = (rows[st:st + cn] - offs[i]) * bj + (cols[st:st + cn] - offs[j])
            block_offset[kk] = st
            block_nnz[kk] = cn
            if not (cn == bi * bj and np.array_equal(lin, np.arange(cn))):
                local_index[kk] = lin.astype(np.int32)
    return BtdLayout(bsz.astype(np.int32), block_offset, block_nnz, local_index, int(rows.size))


def block_sort_index(rows: np.ndarray, cols: np.ndarray, block_sizes) -> np.ndarray:
    """Stable permutation sorting canonical COO entries block-row by block-row,
    then block by block (``compute_block_sort_index``,
    ``src/qttools/kernels/datastructure/numba/dsdbcoo.py:172-236``)."""
    offs = np.concatenate(([0], np.cumsum(np.asarray(block_sizes, dtype=np.int64))))
    br = np.searchsorted(offs, rows, side="right") - 1
    bc = np.searchsorted(offs, cols, side="right") - 1
    return np.lexsort((bc, br)).astype(np.int64)


def block_sort_index_device(rows, cols, block_sizes, device=None):
    """The same permutation as ``block_sort_index``, computed on the device
    (``qtx_block_sort_index``: block keys by binary search, stable radix sort);
    returns (sort_index as a device int64 tensor, per-block counts as a host
    (nb, nb) int64 array).  Raises ValueError for an index outside the matrix."""
    import ctypes

    from quatrex_b200 import _lib

    if not torch.cuda.is_available():
        raise RuntimeError("quatrex_b200 needs a CUDA device (B200, sm_100a); there is no CPU path")
    dev = torch.cuda.current_device() if device is None else torch.device(device).index or 0
    r = torch.as_tensor(rows, dtype=torch.int64).to(f"cuda:{dev}").contiguous()
    c = torch.as_tensor(cols, dtype=torch.int64).to(f"cuda:{dev}").contiguous()
    sizes = np.ascontiguousarray(np.asarray(block_sizes), dtype=np.int32)
    nb = len(sizes)
    out = torch.empty(r.shape[0], dtype=torch.int64, device=f"cuda:{dev}")
    counts = np.zeros(nb * nb, dtype=np.int64)
    lib = _lib.load()
    ctx = _lib.context(dev)
    st = lib.qtx_block_sort_index(ctx, int(r.shape[0]), r.data_ptr(), c.data_ptr(), nb,
                                  sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), out.data_ptr(),
                                  counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                  torch.cuda.current_stream(dev).cuda_stream)
    if st == _lib.QTX_E_INVAL:
        raise ValueError("qtx_block_sort_index: an index lies outside the matrix (or bad block sizes)")
    _lib.check(st, ctx, "qtx_block_sort_index")
    return out, counts.reshape(nb, nb)


def assemble_system(energies, eta: float, hamiltonian: "DSDBCOO", overlap: "DSDBCOO | None" = None,
                    potential=None, sigma: "DSDBCOO | None" = None) -> "DSDBCOO":
    """A(E) = (E + i eta) S - diag(V) - Sigma(E) - H on the device for every
    energy (``ElectronSolver._assemble_system_matrix``,
    ``src/quatrex/electron/solver.py:388-410``): S = I when ``overlap`` is None;
    H and S are energy independent (one data row), Sigma has one row per energy;
    all matrices share the entry order of ``hamiltonian``."""
    from quatrex_b200 import _lib

    if not torch.cuda.is_available():
        raise RuntimeError("quatrex_b200 needs a CUDA device (B200, sm_100a); there is no CPU path")
    dev = torch.cuda.current_device()
    cuda = f"cuda:{dev}"

    def row(m):
        d = m.data if isinstance(m.data, torch.Tensor) else torch.as_tensor(np.asarray(m.data))
        return d.to(cuda, dtype=torch.complex128).reshape(-1, d.shape[-1])

    e = torch.as_tensor(np.asarray(energies, dtype=np.float64)).to(cuda).contiguous()
    ne = int(e.shape[0])
    h = row(hamiltonian)[0].contiguous()
    nnz = int(h.shape[0])
    rows = torch.as_tensor(np.asarray(hamiltonian.rows, dtype=np.int64)).to(cuda)
    cols = torch.as_tensor(np.asarray(hamiltonian.cols, dtype=np.int64)).to(cuda)
    s = row(overlap)[0].contiguous() if overlap is not None else None
    v = torch.as_tensor(np.asarray(potential, dtype=np.float64)).to(cuda) if potential is not None else None
    sg = row(sigma).contiguous() if sigma is not None else None
    if sg is not None and sg.shape[0] != ne:
        raise ValueError("sigma needs one data row per energy")
    out = torch.empty((ne, nnz), dtype=torch.complex128, device=cuda)
    lib = _lib.load()
    ctx = _lib.context(dev)
    st = lib.qtx_assemble_system(ctx, nnz, ne, e.data_ptr(), float(eta), rows.data_ptr(), cols.data_ptr(),
                                 s.data_ptr() if s is not None else None, v.data_ptr() if v is not None else None,
                                 h.data_ptr(), sg.data_ptr() if sg is not None else None, nnz, out.data_ptr(), nnz,
                                 torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(st, ctx, "qtx_assemble_system")
    return DSDBCOO(out, hamiltonian.rows, hamiltonian.cols, hamiltonian.block_sizes, (ne,),
                   getattr(hamiltonian, "symmetry", False))


class _BlockIndexer:
    def __init__(self, m: "DSDBCOO"):
        self.m = m

    def __getitem__(self, ij):
        i, j = ij
        return self.m.get_block(i, j)

    def __setitem__(self, ij, value):
        i, j = ij
        self.m.set_block(i, j, value)


class DSDBCOO:
    """Stack of block-tridiagonal sparse matrices in the DSDBCOO layout."""

    def __init__(self, data, rows, cols, block_sizes, global_stack_shape, symmetry: bool = False):
        if isinstance(global_stack_shape, int):
            global_stack_shape = (global_stack_shape,)
        self.data = data
        self.rows = np.asarray(rows, dtype=np.int64)
        self.cols = np.asarray(cols, dtype=np.int64)
        self.global_stack_shape = tuple(global_stack_shape)
        self.symmetry = bool(symmetry)
        self.layout = btd_layout_from_coords(self.rows, self.cols, block_sizes)
        self.block_sizes = np.asarray(block_sizes, dtype=np.int64)
        self.block_offsets = np.concatenate(([0], np.cumsum(self.block_sizes)))
        self.num_blocks = len(self.block_sizes)
        self._blocks = _BlockIndexer(self)

    # -- shape -----------------------------------------------------------
    @property
    def stack_shape(self) -> tuple:
        return tuple(self.data.shape[:-1])

    @property
    def nnz(self) -> int:
        return int(self.data.shape[-1])

    @property
    def shape(self) -> tuple:
        n = int(self.block_offsets[-1])
        return self.stack_shape + (n, n)

    @property
    def dtype(self):
        return self.data.dtype

    @property
    def blocks(self) -> _BlockIndexer:
        return self._blocks

    @property
    def on_device(self) -> bool:
        return isinstance(self.data, torch.Tensor) and self.data.is_cuda

    # -- construction ----------------------------------------------------
    @classmethod
    def from_sparray(cls, sparray, block_sizes, global_stack_shape, symmetry: bool = False, device=None):
        """Same contract as ``DSDBCOO.from_sparray`` (``dsdbcoo.py:873-964``), single rank:
        the sparse matrix is broadcast over the stack."""
        from scipy import sparse

        if isinstance(global_stack_shape, int):
            global_stack_shape = (global_stack_shape,)
        coo = sparse.coo_matrix(sparray)
        if symmetry:
            coo = sparse.triu(coo, format="coo")
        coo.sum_duplicates()
        if device is not None and torch.device(device).type == "cuda":
            # block sorting and the broadcast over the stack on the device
            order, _ = block_sort_index_device(coo.row, coo.col, block_sizes, device)
            order_h = order.cpu().numpy()
            vals = torch.as_tensor(coo.data.astype(np.complex128)).to(order.device)[order]
            data = vals.expand(tuple(global_stack_shape) + (vals.shape[0],)).contiguous()
            return cls(data, coo.row[order_h], coo.col[order_h], block_sizes, global_stack_shape, symmetry)
        order = block_sort_index(coo.row, coo.col, block_sizes)
        rows, cols, vals = coo.row[order], coo.col[order], coo.data[order].astype(np.complex128)
        data = np.broadcast_to(vals, tuple(global_stack_shape) + (len(vals),)).copy()
        if device is not None:
            data = torch.as_tensor(data).to(device)
        return cls(data, rows, cols, block_sizes, global_stack_shape, symmetry)

    @classmethod
    def zeros_like(cls, other) -> "DSDBCOO":
        if isinstance(other.data, torch.Tensor):
            data = torch.zeros_like(other.data)
        else:
            data = np.zeros_like(other.data)
        return cls(data, other.rows, other.cols, other.block_sizes, getattr(other, "global_stack_shape", other.data.shape[:-1]),
                   getattr(other, "symmetry", False))

    @classmethod
    def from_blocks(cls, diag, upper, lower, device=None) -> "DSDBCOO":
        """Full block-tridiagonal matrix from dense block stacks (every block entry stored)."""
        sizes = np.array([d.shape[-1] for d in diag], dtype=np.int64)
        nb = len(sizes)
        offs = np.concatenate(([0], np.cumsum(sizes)))
        stack = tuple(diag[0].shape[:-2])
        rows_l, cols_l, chunks = [], [], []
        for i in range(nb):
            for j in range(max(0, i - 1), min(nb, i + 2)):
                blk = diag[i] if j == i else (upper[i] if j == i + 1 else lower[j])
                bi, bj = int(sizes[i]), int(sizes[j])
                r, c = np.meshgrid(np.arange(bi) + offs[i], np.arange(bj) + offs[j], indexing="ij")
                rows_l.append(r.ravel())
                cols_l.append(c.ravel())
                if isinstance(blk, torch.Tensor):
                    chunks.append(blk.reshape(stack + (bi * bj,)))
                else:
                    chunks.append(np.asarray(blk).reshape(stack + (bi * bj,)))
        if isinstance(chunks[0], torch.Tensor):
            data = torch.cat(chunks, dim=-1)
        else:
            data = np.concatenate(chunks, axis=-1)
            if device is not None:
                data = torch.as_tensor(data).to(device)
        return cls(data, np.concatenate(rows_l), np.concatenate(cols_l), sizes, stack)

    def to(self, device) -> "DSDBCOO":
        data = self.data if isinstance(self.data, torch.Tensor) else torch.as_tensor(self.data)
        return DSDBCOO(data.to(device), self.rows, self.cols, self.block_sizes, self.global_stack_shape, self.symmetry)

    def numpy_data(self) -> np.ndarray:
        if isinstance(self.data, torch.Tensor):
            return self.data.detach().cpu().numpy()
        return np.asarray(self.data)

    # -- block access (host-side convenience, not on the solver path) ------
    def _slice(self, i, j):
        k = 2 * i + j
        st = int(self.layout.block_offset[k])
        n = int(self.layout.block_nnz[k])
        return k, st, n

    def get_block(self, i: int, j: int) -> np.ndarray:
        nb = self.num_blocks
        i, j = i % nb, j % nb
        bi, bj = int(self.block_sizes[i]), int(self.block_sizes[j])
        if self.symmetry and j < i:
            return np.ascontiguousarray(np.conj(self.get_block(j, i).swapaxes(-1, -2)))
        out = np.zeros(self.stack_shape + (bi, bj), dtype=np.complex128)
        if abs(i - j) > 1:
            return out
        k, st, n = self._slice(i, j)
        if st < 0 or n == 0:
            return out
        vals = self.numpy_data()[..., st:st + n]
        ix = self.layout.local_index[k]
        lin = np.arange(n) if ix is None else ix
        flat = out.reshape(self.stack_shape + (bi * bj,))
        flat[..., lin] = vals
        if self.symmetry and i == j:
            out = out + np.conj(out.swapaxes(-1, -2))
            out[..., np.arange(bi), np.arange(bi)] /= 2
        return out

    def set_block(self, i: int, j: int, value) -> None:
        nb = self.num_blocks
        i, j = i % nb, j % nb
        if self.symmetry and j < i:
            self.set_block(j, i, np.conj(np.asarray(value).swapaxes(-1, -2)))
            return
        k, st, n = self._slice(i, j)
        if st < 0 or n == 0:
            return
        bi, bj = int(self.block_sizes[i]), int(self.block_sizes[j])
        value = np.broadcast_to(np.asarray(value), self.stack_shape + (bi, bj)).reshape(self.stack_shape + (bi * bj,))
        ix = self.layout.local_index[k]
        lin = np.arange(n) if ix is None else ix
        vals = value[..., lin]
        if isinstance(self.data, torch.Tensor):
            self.data[..., st:st + n] = torch.as_tensor(np.ascontiguousarray(vals)).to(self.data.device)
        else:
            self.data[..., st:st + n] = vals

    def to_dense(self) -> np.ndarray:
        n = int(self.block_offsets[-1])
        out = np.zeros(self.stack_shape + (n, n), dtype=np.complex128)
        out[..., self.rows, self.cols] = self.numpy_data()
        if self.symmetry:
            out = out + np.conj(out.swapaxes(-1, -2))
            out[..., np.arange(n), np.arange(n)] /= 2
        return out


def layout_of(m) -> BtdLayout:
    """Block map of a DSDBSparse-like object (ours or upstream)."""
    lay = getattr(m, "layout", None)
    if isinstance(lay, BtdLayout):
        return lay
    cached = getattr(m, "_qtx_layout", None)
    if cached is not None:
        return cached
    lay = btd_layout_from_coords(np.asarray(m.rows), np.asarray(m.cols), np.asarray(m.block_sizes))
    try:
        m._qtx_layout = lay
    except AttributeError:
        pass
    return lay
