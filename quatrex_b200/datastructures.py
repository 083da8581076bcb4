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

``DSDBCSR`` keeps qttools' DSDBCSR layout
(``src/qttools/datastructures/dsdbcsr.py:23-869``): the same block-sorted data
order (``compute_rowptr_map``,
``src/qttools/kernels/datastructure/numba/dsdbcsr.py:229-305``, block rows in
order, blocks of a block row in order, canonical COO order inside a block),
described by a row-pointer map ``{(i, j): rowptr}`` of absolute positions and
the column indices instead of row and column indices.

``layout_of`` accepts any object with ``rows``, ``cols``, ``block_sizes`` and
``data`` attributes (an upstream DSDBCOO) or with ``rowptr_map``, ``cols``,
``block_sizes`` and ``data`` (an upstream DSDBCSR).

Symmetric storage (``symmetry=True``, ``dsdbcoo.py:483-492``,
``dsdbcsr.py:262-339``) keeps the upper block triangle and the upper triangle
of each diagonal block; block (j, i) is ``symmetry_op(X_ij^T)`` and a diagonal
block is completed as ``U + symmetry_op(U^T)`` with its diagonal halved.  The
solvers expand symmetric-storage INPUTS on the device to full storage
(``expand_symmetric``) and write symmetric-storage OUTPUTS upper blocks only.
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


def rows_from_rowptr(rowptr_map: dict, nnz: int, block_sizes) -> np.ndarray:
    """Global row index of every stored entry of a DSDBCSR pattern."""
    offs = np.concatenate(([0], np.cumsum(np.asarray(block_sizes, dtype=np.int64))))
    rows = np.full(int(nnz), -1, dtype=np.int64)
    for (i, _j), rp in rowptr_map.items():
        rp = np.asarray(rp, dtype=np.int64)
        counts = np.diff(rp)
        rows[rp[0]:rp[-1]] = np.repeat(offs[int(i)] + np.arange(len(counts), dtype=np.int64), counts)
    if (rows < 0).any():
        raise ValueError("rowptr map does not cover every stored entry")
    return rows


def rowptr_map_from_coords(rows: np.ndarray, cols: np.ndarray, block_sizes) -> dict:
    """Row-pointer map of block-sorted coordinates (``compute_rowptr_map``,
    ``src/qttools/kernels/datastructure/numba/dsdbcsr.py:229-305``)."""
    bsz = np.asarray(block_sizes, dtype=np.int64)
    offs = np.concatenate(([0], np.cumsum(bsz)))
    br = np.searchsorted(offs, rows, side="right") - 1
    bc = np.searchsorted(offs, cols, side="right") - 1
    out = {}
    if rows.size == 0:
        return out
    key = br * len(bsz) + bc
    uk, start, count = np.unique(key, return_index=True, return_counts=True)
    for kk, st, cn in zip(uk, start, count):
        i, j = int(kk) // len(bsz), int(kk) % len(bsz)
        local = rows[st:st + cn] - offs[i]
        hist = np.bincount(local, minlength=int(bsz[i]))
        out[(i, j)] = np.concatenate(([0], np.cumsum(hist))).astype(np.int64) + st
    return out


def symmetry_kind(op) -> str:
    """Classify a qttools ``symmetry_op``: 'conj' (Hermitian storage, the
    default), 'neg_conj' (skew-Hermitian: G^<, G^>, Sigma^<, Sigma^>) or
    'identity' (complex symmetric: Sigma^R, the system matrix)."""
    if op is None:
        return "conj"
    probe = np.array([1.0 + 2.0j])
    r = np.asarray(op(probe))
    for kind, want in (("conj", 1.0 - 2.0j), ("neg_conj", -1.0 + 2.0j), ("identity", 1.0 + 2.0j)):
        if r.shape == (1,) and r[0] == want:
            return kind
    raise NotImplementedError("symmetry_op must be conj, -conj or the identity")


def _apply_sym(kind: str, x):
    """symmetry_op of `kind` applied to the transpose of x (numpy or torch)."""
    xt = x.swapaxes(-1, -2) if isinstance(x, np.ndarray) else x.transpose(-1, -2)
    if kind == "identity":
        return xt
    xc = xt.conj() if isinstance(x, np.ndarray) else xt.conj().resolve_conj()
    return xc if kind == "conj" else -xc


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

    def __init__(self, data, rows, cols, block_sizes, global_stack_shape, symmetry: bool = False,
                 symmetry_op=np.conj):
        if isinstance(global_stack_shape, int):
            global_stack_shape = (global_stack_shape,)
        self.data = data
        self.rows = np.asarray(rows, dtype=np.int64)
        self.cols = np.asarray(cols, dtype=np.int64)
        self.global_stack_shape = tuple(global_stack_shape)
        self.symmetry = bool(symmetry)
        self.symmetry_op = symmetry_op
        self._sym_kind = symmetry_kind(symmetry_op) if self.symmetry else "conj"
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
    def from_sparray(cls, sparray, block_sizes, global_stack_shape, symmetry: bool = False, device=None,
                     symmetry_op=np.conj):
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
            return cls._from_sorted(data, coo.row[order_h], coo.col[order_h], block_sizes, global_stack_shape,
                                    symmetry, symmetry_op)
        order = block_sort_index(coo.row, coo.col, block_sizes)
        rows, cols, vals = coo.row[order], coo.col[order], coo.data[order].astype(np.complex128)
        data = np.broadcast_to(vals, tuple(global_stack_shape) + (len(vals),)).copy()
        if device is not None:
            data = torch.as_tensor(data).to(device)
        return cls._from_sorted(data, rows, cols, block_sizes, global_stack_shape, symmetry, symmetry_op)

    @classmethod
    def _from_sorted(cls, data, rows, cols, block_sizes, global_stack_shape, symmetry, symmetry_op):
        return cls(data, rows, cols, block_sizes, global_stack_shape, symmetry, symmetry_op)

    @classmethod
    def zeros_like(cls, other) -> "DSDBCOO":
        if isinstance(other.data, torch.Tensor):
            data = torch.zeros_like(other.data)
        else:
            data = np.zeros_like(other.data)
        return cls(data, other.rows, other.cols, other.block_sizes, getattr(other, "global_stack_shape", other.data.shape[:-1]),
                   getattr(other, "symmetry", False), getattr(other, "symmetry_op", np.conj))

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
        return cls._from_sorted(data, np.concatenate(rows_l), np.concatenate(cols_l), sizes, stack, False, np.conj)

    def to(self, device) -> "DSDBCOO":
        data = self.data if isinstance(self.data, torch.Tensor) else torch.as_tensor(self.data)
        return DSDBCOO(data.to(device), self.rows, self.cols, self.block_sizes, self.global_stack_shape, self.symmetry,
                       self.symmetry_op)

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
            return np.ascontiguousarray(_apply_sym(self._sym_kind, self.get_block(j, i)))
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
            out = out + _apply_sym(self._sym_kind, out)
            out[..., np.arange(bi), np.arange(bi)] /= 2
        return out

    def set_block(self, i: int, j: int, value) -> None:
        nb = self.num_blocks
        i, j = i % nb, j % nb
        if self.symmetry and j < i:
            self.set_block(j, i, _apply_sym(self._sym_kind, np.asarray(value)))
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
            out = out + _apply_sym(self._sym_kind, out)
            out[..., np.arange(n), np.arange(n)] /= 2
        return out


class DSDBCSR(DSDBCOO):
    """Stack of block-tridiagonal sparse matrices in the DSDBCSR layout
    (``src/qttools/datastructures/dsdbcsr.py:23-869``): the block-sorted data
    order of DSDBCOO, described by ``rowptr_map`` and ``cols``."""

    def __init__(self, data, cols, rowptr_map, block_sizes, global_stack_shape, symmetry: bool = False,
                 symmetry_op=np.conj):
        nnz = int(data.shape[-1])
        self.rowptr_map = {tuple(int(v) for v in k): np.asarray(rp, dtype=np.int64) for k, rp in rowptr_map.items()}
        rows = rows_from_rowptr(self.rowptr_map, nnz, block_sizes)
        super().__init__(data, rows, cols, block_sizes, global_stack_shape, symmetry, symmetry_op)

    @classmethod
    def _from_sorted(cls, data, rows, cols, block_sizes, global_stack_shape, symmetry, symmetry_op):
        rp = rowptr_map_from_coords(np.asarray(rows, dtype=np.int64), np.asarray(cols, dtype=np.int64), block_sizes)
        return cls(data, cols, rp, block_sizes, global_stack_shape, symmetry, symmetry_op)

    @classmethod
    def zeros_like(cls, other) -> "DSDBCSR":
        data = torch.zeros_like(other.data) if isinstance(other.data, torch.Tensor) else np.zeros_like(other.data)
        return cls(data, other.cols, other.rowptr_map, other.block_sizes,
                   getattr(other, "global_stack_shape", other.data.shape[:-1]), getattr(other, "symmetry", False),
                   getattr(other, "symmetry_op", np.conj))

    def to(self, device) -> "DSDBCSR":
        data = self.data if isinstance(self.data, torch.Tensor) else torch.as_tensor(self.data)
        return DSDBCSR(data.to(device), self.cols, self.rowptr_map, self.block_sizes, self.global_stack_shape,
                       self.symmetry, self.symmetry_op)


def _dense_block_device(m, lay: "BtdLayout", data: torch.Tensor, i: int, j: int) -> torch.Tensor:
    """Block (i, j) of stored data as a dense (stack, bi, bj) tensor (zeros
    where the pattern has no entry)."""
    bi, bj = int(lay.block_sizes[i]), int(lay.block_sizes[j])
    k = 2 * i + j
    st, n = int(lay.block_offset[k]), int(lay.block_nnz[k])
    out = torch.zeros(data.shape[:-1] + (bi * bj,), dtype=data.dtype, device=data.device)
    if st >= 0 and n > 0:
        ix = lay.local_index[k]
        if ix is None:
            out[..., :n] = data[..., st:st + n]
        else:
            out[..., torch.as_tensor(ix, dtype=torch.int64, device=data.device)] = data[..., st:st + n]
    return out.reshape(data.shape[:-1] + (bi, bj))


def expand_symmetric(m, device: int) -> DSDBCOO:
    """Full-storage device copy of a symmetric-storage DSDBSparse (ours or
    upstream's): every block of the block-tridiagonal pattern dense, block
    (j, i) = symmetry_op(X_ij^T), diagonal blocks U + symmetry_op(U^T) with
    the diagonal halved (``dsdbcoo.py:321-400`` block access)."""
    lay = layout_of(m)
    kind = symmetry_kind(getattr(m, "symmetry_op", None))
    data = m.data if isinstance(m.data, torch.Tensor) else torch.as_tensor(np.asarray(m.data))
    data = data.to(device=f"cuda:{device}", dtype=torch.complex128)
    stack = tuple(data.shape[:-1])
    data = data.reshape(-1, data.shape[-1])
    nb = lay.num_blocks
    diag, upper, lower = [], [], []
    for i in range(nb):
        u = _dense_block_device(m, lay, data, i, i)
        d = u + _apply_sym(kind, u)
        idx = torch.arange(u.shape[-1], device=u.device)
        d[..., idx, idx] = d[..., idx, idx] / 2
        diag.append(d.reshape(stack + d.shape[-2:]))
        if i + 1 < nb:
            up = _dense_block_device(m, lay, data, i, i + 1)
            upper.append(up.reshape(stack + up.shape[-2:]))
            lo = _apply_sym(kind, up).contiguous()
            lower.append(lo.reshape(stack + lo.shape[-2:]))
    return DSDBCOO.from_blocks(diag, upper, lower)


def layout_of(m) -> BtdLayout:
    """Block map of a DSDBSparse-like object (ours or upstream)."""
    lay = getattr(m, "layout", None)
    if isinstance(lay, BtdLayout):
        return lay
    cached = getattr(m, "_qtx_layout", None)
    if cached is not None:
        return cached
    if getattr(m, "rows", None) is None and getattr(m, "rowptr_map", None) is not None:
        rows = rows_from_rowptr(m.rowptr_map, int(m.data.shape[-1]), np.asarray(m.block_sizes))
    else:
        rows = np.asarray(m.rows)
    lay = btd_layout_from_coords(rows, np.asarray(m.cols), np.asarray(m.block_sizes))
    try:
        m._qtx_layout = lay
    except AttributeError:
        pass
    return lay
