"""Drop-in RGF solver: qttools' ``GFSolver`` interface over libqtxrgf.so.

Mirrors ``src/qttools/greens_function_solver/solver.py`` (``OBCBlocks``
``:12-28``, ``GFSolver`` ``:31-113``) and ``rgf.py`` (``RGF`` ``:10-414``):
same class names, method signatures, argument meaning, return conventions and
errors.  Every call runs on the current CUDA device through the C ABI.  When every
operand is a host (NumPy) array the library streams the stack through the
device in energy batches (``QTX_FLAG_HOST_BUFFERS``: two device staging sets,
uploads and downloads overlapping the solve), so stacks larger than the
device memory work; mixed host/device operands are staged through the device
whole.  There is no CPU path: without the built library or a CUDA device the
calls raise.

Behaviour notes (upstream file:line):

* ``selected_inv`` returns a new matrix when ``out`` is None and writes ``out``
  in place otherwise (``rgf.py:59-62,112-113``).
* ``selected_solve`` returns ``(xl, xg)``, ``(xl, xg, xr)`` or
  ``(xl, xg, xr, current)`` without ``out``; with ``out=[xl, xg(, xr)]`` it
  returns ``current`` or None (``rgf.py:406-414``); a wrong ``out`` length with
  ``return_retarded`` raises ``ValueError`` (``rgf.py:184-186``).
* OBC lesser/greater blocks are added to the diagonal self-energy blocks and
  the retarded ones subtracted from the system matrix (``rgf.py:207-255``).
* Diagonal G^</G^> blocks are stored as 0.5 (X - X^H); the lower off-diagonal
  block as -X_ij^H unless the output stores the upper triangle only
  (``rgf.py:298-303,350-357``).
* The layer current uses the coupling of each interface (Meir-Wingreen).  The
  upstream loop reads a stale ``a_ji_dagger`` (the last forward step's,
  ``rgf.py:262`` vs ``:385,391``) for every interface but the last.
"""

from __future__ import annotations

import ctypes
import math
from abc import ABC, abstractmethod

import numpy as np
import torch

from quatrex_b200 import _lib
from quatrex_b200.datastructures import DSDBCOO, expand_symmetric, layout_of

_PRECISIONS = {"fp64": _lib.QTX_PREC_FP64, "mixed": _lib.QTX_PREC_MIXED}


class OBCBlocks:
    """Boundary blocks of the GF solvers (``solver.py:12-28``): lists of
    ``nb`` entries, each None or a ``(*stack, b_i, b_i)`` array."""

    def __init__(self, num_blocks: int):
        self.retarded: list = [None] * num_blocks
        self.lesser: list = [None] * num_blocks
        self.greater: list = [None] * num_blocks


class GFSolver(ABC):
    """Abstract base class of the Green's function solvers (``solver.py:31-113``)."""

    @abstractmethod
    def selected_inv(self, a, obc_blocks: OBCBlocks | None = None, out=None):
        ...

    @abstractmethod
    def selected_solve(self, a, sigma_lesser, sigma_greater, obc_blocks: OBCBlocks | None = None, out=None,
                       return_retarded: bool = False, return_current: bool = False):
        ...


def _device_index() -> int:
    if not torch.cuda.is_available():
        raise RuntimeError("quatrex_b200 needs a CUDA device (B200, sm_100a); there is no CPU path")
    return torch.cuda.current_device()


def _is_host(x) -> bool:
    if x is None:
        return True
    if isinstance(x, torch.Tensor):
        return not x.is_cuda
    return True


class _Operand:
    """A DSDBSparse-like matrix staged for one C call (``host``: passed as a
    host pointer for the streamed host-buffer mode)."""

    def __init__(self, m, device: int, writable: bool, host: bool = False):
        if not writable and getattr(m, "symmetry", False):
            # symmetric-storage input: full storage on the device (the lower
            # blocks and lower diagonal triangles are not stored)
            m = expand_symmetric(m, device)
            host = False
        self.m = m
        self.layout = layout_of(m)
        data = m.data
        self.host_array = None
        self.host = host
        if host:
            arr = data.numpy() if isinstance(data, torch.Tensor) else np.asarray(data)
            if arr.dtype != np.complex128:
                raise TypeError("DSDBSparse data must be complex128")
            self.host_array = arr
            self.h = np.ascontiguousarray(arr)  # the caller's array itself when contiguous
            self.orig = data
            self.writable = writable
            self.stack_shape = tuple(self.h.shape[:-1])
            self.stack_size = int(math.prod(self.stack_shape)) if self.stack_shape else 1
            self.nnz = int(self.h.shape[-1])
            self.desc, self.keep = self.layout.desc(self.stack_size, self.nnz, device)
            return
        if isinstance(data, torch.Tensor):
            if data.dtype != torch.complex128:
                raise TypeError("DSDBSparse data must be complex128")
            if data.is_cuda:
                self.t = data if data.is_contiguous() else data.contiguous()
            else:
                self.t = data.contiguous().to(f"cuda:{device}")
        else:
            arr = np.asarray(data)
            if arr.dtype != np.complex128:
                raise TypeError("DSDBSparse data must be complex128")
            self.host_array = arr
            self.t = torch.from_numpy(np.ascontiguousarray(arr)).to(f"cuda:{device}")
        self.orig = data
        self.writable = writable
        self.stack_shape = tuple(self.t.shape[:-1])
        self.stack_size = int(math.prod(self.stack_shape)) if self.stack_shape else 1
        self.nnz = int(self.t.shape[-1])
        self.desc, self.keep = self.layout.desc(self.stack_size, self.nnz, device)

    @property
    def ptr(self) -> int:
        return self.h.ctypes.data if self.host else self.t.data_ptr()

    def write_back(self) -> None:
        if not self.writable:
            return
        if self.host:
            if self.h is not self.host_array:
                self.host_array[...] = self.h.reshape(self.host_array.shape)
            return
        if self.host_array is not None:
            self.host_array[...] = self.t.cpu().numpy().reshape(self.host_array.shape)
        elif self.t is not self.orig:
            self.orig.copy_(self.t)


def _obc_ptrs(blocks, nb: int, stack_size: int, device: int, keep: list, host: bool = False):
    if blocks is None or all(b is None for b in blocks):
        return None
    if len(blocks) != nb:
        raise ValueError("OBC block list length differs from the number of blocks")
    ptrs = []
    for b in blocks:
        if b is None:
            ptrs.append(0)
            continue
        if host:
            h = np.ascontiguousarray(b.numpy() if isinstance(b, torch.Tensor) else np.asarray(b),
                                     dtype=np.complex128)
            if h.size // (h.shape[-1] * h.shape[-2]) != stack_size:
                raise ValueError("OBC block stack size differs from the system matrix")
            keep.append(h)
            ptrs.append(h.ctypes.data)
            continue
        t = b if isinstance(b, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(np.asarray(b)))
        t = t.to(device=f"cuda:{device}", dtype=torch.complex128).contiguous()
        if t.numel() // (t.shape[-1] * t.shape[-2]) != stack_size:
            raise ValueError("OBC block stack size differs from the system matrix")
        keep.append(t)
        ptrs.append(t.data_ptr())
    arr = (ctypes.c_void_p * nb)(*ptrs)
    keep.append(arr)
    return ctypes.cast(arr, ctypes.POINTER(ctypes.c_void_p))


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class RGF(GFSolver):
    """Selected inversion solver based on the Schur complement (``rgf.py:10-23``).

    Parameters
    ----------
    max_batch_size : int, optional
        Maximum number of stack entries solved together, by default 100.
    precision : {"fp64", "mixed"}
        "fp64": complex128 throughout.  "mixed": bulk block products as
        7-bit integer slice products on the INT8 tensor cores with exact
        accumulation (Ozaki scheme), inverses in FP64.
    """

    def __init__(self, max_batch_size: int = 100, precision: str = "fp64") -> None:
        self.max_batch_size = max_batch_size
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        self.precision = precision

    def _batch(self, op: _Operand) -> int:
        inner = op.stack_size // op.stack_shape[0] if op.stack_shape else 1
        return max(1, int(self.max_batch_size)) * max(1, inner)

    def selected_inv(self, a, obc_blocks: OBCBlocks | None = None, out=None):
        """Selected inversion of a block-tridiagonal matrix (``rgf.py:25-113``)."""
        dev = _device_index()
        lib = _lib.load()
        ctx = _lib.context(dev)
        if obc_blocks is None:
            obc_blocks = OBCBlocks(num_blocks=a.num_blocks)
        x = out if out is not None else _zeros_like(a)
        host = (all(_is_host(m.data) for m in (a, x)) and not getattr(a, "symmetry", False)
                and all(_is_host(b) for b in obc_blocks.retarded))
        A = _Operand(a, dev, writable=False, host=host)
        X = _Operand(x, dev, writable=True, host=host)
        keep: list = []
        obc_r = _obc_ptrs(obc_blocks.retarded, a.num_blocks, A.stack_size, dev, keep, host)
        flags = _lib.QTX_FLAG_HOST_BUFFERS if host else 0
        st = lib.qtx_selected_inv(ctx, ctypes.byref(A.desc), A.ptr, obc_r, ctypes.byref(X.desc), X.ptr,
                                  self._batch(A), _PRECISIONS[self.precision], flags, _stream())
        _lib.check(st, ctx, "RGF.selected_inv")
        X.write_back()
        if out is None:
            return x
        return None

    def selected_solve(self, a, sigma_lesser, sigma_greater, obc_blocks: OBCBlocks | None = None, out=None,
                       return_retarded: bool = False, return_current: bool = False):
        """Selected solve X^< = A^-1 Sigma^< A^-H, X^> likewise (``rgf.py:115-414``)."""
        dev = _device_index()
        lib = _lib.load()
        ctx = _lib.context(dev)
        nb = a.num_blocks
        if obc_blocks is None:
            obc_blocks = OBCBlocks(num_blocks=nb)
        if out is not None:
            xl, xg, *xr = out
            if return_retarded:
                if len(xr) != 1:
                    raise ValueError("Invalid number of output matrices.")
                xr = xr[0]
            else:
                xr = None
        else:
            xl = _zeros_like(a)
            xg = _zeros_like(a)
            xr = _zeros_like(a) if return_retarded else None
        mats = [a, sigma_lesser, sigma_greater, xl, xg] + ([xr] if xr is not None else [])
        host = all(_is_host(m.data) for m in mats) and not any(
            getattr(m, "symmetry", False) for m in (a, sigma_lesser, sigma_greater)) and all(
            _is_host(b) for blocks in (obc_blocks.retarded, obc_blocks.lesser, obc_blocks.greater) for b in blocks)
        A = _Operand(a, dev, writable=False, host=host)
        SL = _Operand(sigma_lesser, dev, writable=False, host=host)
        SG = _Operand(sigma_greater, dev, writable=False, host=host)
        XL = _Operand(xl, dev, writable=True, host=host)
        XG = _Operand(xg, dev, writable=True, host=host)
        XR = _Operand(xr, dev, writable=True, host=host) if xr is not None else None
        keep: list = []
        obc = _lib.Obc(
            retarded=_obc_ptrs(obc_blocks.retarded, nb, A.stack_size, dev, keep, host),
            lesser=_obc_ptrs(obc_blocks.lesser, nb, A.stack_size, dev, keep, host),
            greater=_obc_ptrs(obc_blocks.greater, nb, A.stack_size, dev, keep, host),
        )
        flags = _lib.QTX_FLAG_HOST_BUFFERS if host else 0
        if return_retarded:
            flags |= _lib.QTX_FLAG_RETURN_RETARDED
        if getattr(xl, "symmetry", False):
            flags |= _lib.QTX_FLAG_SYMMETRIC_OUT
        current = None
        if return_current:
            flags |= _lib.QTX_FLAG_RETURN_CURRENT
            if host:
                current = np.zeros(A.stack_shape + (nb - 1,), dtype=np.complex128)
            else:
                current = torch.zeros(A.stack_shape + (nb - 1,), dtype=torch.complex128, device=f"cuda:{dev}")
        cur_ptr = None
        if current is not None:
            cur_ptr = current.ctypes.data if host else current.data_ptr()
        st = lib.qtx_selected_solve(
            ctx, ctypes.byref(A.desc), A.ptr, ctypes.byref(SL.desc), SL.ptr, ctypes.byref(SG.desc), SG.ptr,
            ctypes.byref(obc), ctypes.byref(XL.desc), XL.ptr, ctypes.byref(XG.desc), XG.ptr,
            ctypes.byref(XR.desc) if XR else None, XR.ptr if XR else None,
            cur_ptr, self._batch(A), _PRECISIONS[self.precision], flags, _stream())
        _lib.check(st, ctx, "RGF.selected_solve")
        for op in (XL, XG, XR):
            if op is not None:
                op.write_back()
        if current is not None and not host and A.host_array is not None:
            current = current.cpu().numpy()
        if out is None:
            if return_retarded:
                if return_current:
                    return xl, xg, xr, current
                return xl, xg, xr
            return xl, xg
        if return_current:
            return current
        return None


def _zeros_like(a):
    zl = getattr(type(a), "zeros_like", None)
    if zl is not None:
        return zl(a)
    return DSDBCOO.zeros_like(a)
