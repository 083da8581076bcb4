"""Non-linear eigenvalue problems of the lead blocks on the device.

``Beyn`` mirrors ``qttools.nevp.Beyn`` (``src/qttools/nevp/beyn.py:14-379``):
the same constructor, the same probe block (``numpy.random.default_rng(42)``
drawn at construction, real parts then imaginary parts per call,
``beyn.py:96,310-313``), the same quadrature and the same SVD (or QR)
projection.  The contour integral -- one n x n inverse per quadrature point
and energy, the bulk of the work -- and the moment products run in
``qtx_beyn_moments`` (DMMA GEMM and batched inverse), the products of the
projection on the device.  The two small dense factorisations follow
upstream's ``project_compute_location`` / ``eig_compute_location``: with
upstream's default ``"numpy"`` the n x m0 SVD (or QR) and the m0 x m0
eigenproblem run in NumPy/LAPACK on the host, as upstream does
(``beyn.py:120-125, 265-272``), split over host threads; any other value runs
them through ``torch.linalg`` on the device.  Measured on B200 for 148
energies (b = 256, m0 = 64): ``torch.linalg.svd`` 1.38 s and
``torch.linalg.eig`` 0.49 s on the device (batched small factorisations are
not what those routines are built for; the latter's hybrid path iterates on
the host anyway) against the 69 ms contour; the whole Spectral call takes
0.20 s with the host factorisations and 1.97 s with the device ones.
"""

from __future__ import annotations

import math
import os
from abc import ABC, abstractmethod
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from quatrex_b200 import _lib


class NEVP(ABC):
    """Solver of sum_n w^n a_n v = 0 for the coefficient blocks a_xx
    (lowest order first), ``src/qttools/nevp/nevp.py``."""

    @abstractmethod
    def __call__(self, a_xx):
        ...


def _device_tensor(x, dev: int) -> tuple[torch.Tensor, bool]:
    host = not (isinstance(x, torch.Tensor) and x.is_cuda)
    t = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(np.asarray(x)))
    return t.to(device=f"cuda:{dev}", dtype=torch.complex128).contiguous(), host


def _batched(t: torch.Tensor) -> tuple[int, int]:
    """(batch, stride) of a (..., n, n) block; a 2-D block is shared (stride 0)."""
    n = t.shape[-1]
    if t.dim() == 2:
        return 1, 0
    return int(math.prod(t.shape[:-2])), n * n


def _host_batched(fn, x: np.ndarray, nout: int):
    """fn over the leading (batch) axis of x in chunks on host threads (the
    NumPy linear-algebra loops release the GIL), each chunk with a
    single-threaded BLAS so the threads do not oversubscribe the cores; nout
    stacked results."""
    batch = x.shape[0]
    workers = max(1, min(batch, os.cpu_count() or 1, 16))
    if workers == 1:
        return fn(x)
    bounds = np.linspace(0, batch, workers + 1).astype(int)
    try:
        from threadpoolctl import threadpool_limits
        limit = threadpool_limits(limits=1)
    except ImportError:
        limit = None
    try:
        with ThreadPoolExecutor(max_workers=workers) as ex:
            parts = list(ex.map(lambda q: fn(x[bounds[q]:bounds[q + 1]]), range(workers)))
    finally:
        if limit is not None:
            limit.restore_original_limits()
    return tuple(np.concatenate([p[k] for p in parts]) for k in range(nout))


def _on_host(location: str) -> bool:
    return location == "numpy"


class Beyn(NEVP):
    """Beyn's contour-integral method for the eigenpairs inside the annulus
    r_i < |w| < r_o (``beyn.py:14-95``).  ``eig_compute_location`` and
    ``project_compute_location`` choose where the small factorisations run
    ("numpy": the host, as upstream's default; otherwise the device);
    ``num_threads_contour``, ``contour_batch_size`` and ``use_pinned_memory``
    are accepted for signature compatibility (the device path sizes its own
    passes)."""

    def __init__(self, r_o: float, r_i: float, m_0: int, num_quad_points: int, num_threads_contour: int = 1024,
                 eig_compute_location: str = "numpy", project_compute_location: str = "numpy", use_qr: bool = False,
                 contour_batch_size: int | None = None, use_pinned_memory: bool = True):
        self.r_o = float(r_o)
        self.r_i = float(r_i)
        self.m_0 = int(m_0)
        self.num_quad_points = int(num_quad_points)
        self.num_threads_contour = num_threads_contour
        self.eig_compute_location = eig_compute_location
        self.project_compute_location = project_compute_location
        self.use_qr = use_qr
        self.contour_batch_size = contour_batch_size
        self.use_pinned_memory = use_pinned_memory
        self.rng = np.random.default_rng(42)

    def moments(self, a_ji: torch.Tensor, a_ii: torch.Tensor, a_ij: torch.Tensor, y: torch.Tensor):
        """p0 = q0 y, p1 = q1 y on the device (``beyn.py:187-239, 316-317``)."""
        dev = a_ii.device.index
        n = a_ii.shape[-1]
        batch, s_ii = _batched(a_ii)
        _, s_ij = _batched(a_ij)
        _, s_ji = _batched(a_ji)
        m0 = y.shape[-1]
        p0 = torch.empty((batch, n, m0), dtype=torch.complex128, device=a_ii.device)
        p1 = torch.empty_like(p0)
        lib = _lib.load()
        ctx = _lib.context(dev)
        st = lib.qtx_beyn_moments(ctx, n, batch, a_ii.data_ptr(), s_ii, a_ij.data_ptr(), s_ij, a_ji.data_ptr(), s_ji,
                                  self.r_o, self.r_i, self.num_quad_points, y.data_ptr(), m0, p0.data_ptr(),
                                  p1.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(st, ctx, "Beyn (contour moments)")
        return p0, p1

    def _project(self, p0: torch.Tensor, p1: torch.Tensor):
        """Projected m0 x m0 problem and the back-projection (``beyn.py:99-185``).
        Singular values below s_max m0 eps are dropped (``:131-136``); the
        dropped rows and columns are zero, so the padded problem's extra
        eigenvalues are exactly 0 and never chosen as lead modes."""
        m0 = p0.shape[-1]
        host = _on_host(self.project_compute_location)
        if self.use_qr:
            if host:
                q, r = _host_batched(lambda x: np.linalg.qr(x), p0.cpu().numpy(), 2)
                q, r = torch.from_numpy(q).to(p0.device), torch.from_numpy(r).to(p0.device)
            else:
                q, r = torch.linalg.qr(p0)
            a = q.mH @ p1 @ torch.linalg.inv(r)
            return a, q
        if host:
            u, s, vh = _host_batched(lambda x: np.linalg.svd(x, full_matrices=False), p0.cpu().numpy(), 3)
            u, s, vh = (torch.from_numpy(t).to(p0.device) for t in (u, s, vh))
        else:
            u, s, vh = torch.linalg.svd(p0, full_matrices=False)
        keep = s > s.amax(dim=-1, keepdim=True) * m0 * torch.finfo(torch.float64).eps
        s_safe = torch.where(keep, s, torch.ones_like(s))
        a = (u.mH @ p1 @ vh.mH) / s_safe[..., None, :].to(p1.dtype)
        km = keep.to(p1.dtype)
        a = a * km[..., :, None] * km[..., None, :]
        return a, u * km[..., None, :]

    def __call__(self, a_xx):
        """Eigenpairs (ws (batch, m0), vs (batch, n, m0)) of
        (a_ji / w + a_ii + a_ij w) v = 0 inside the annulus; device tensors."""
        if len(a_xx) != 3:
            raise NotImplementedError("Beyn on the device handles three coefficient blocks (block_sections = 1)")
        dev = torch.cuda.current_device()
        a_ji, _ = _device_tensor(a_xx[0], dev)
        a_ii, _ = _device_tensor(a_xx[1], dev)
        a_ij, _ = _device_tensor(a_xx[2], dev)
        if a_ii.dim() == 2:
            a_ii = a_ii[None]
        batch_shape = tuple(a_ii.shape[:-2])
        n = a_ii.shape[-1]
        batch = int(math.prod(batch_shape))
        a_ii = a_ii.reshape(batch, n, n)
        a_ji = a_ji.reshape(-1, n, n) if a_ji.dim() > 2 else a_ji
        a_ij = a_ij.reshape(-1, n, n) if a_ij.dim() > 2 else a_ij
        y_h = self.rng.random((batch, n, self.m_0)) + 1j * self.rng.random((batch, n, self.m_0))
        y = torch.from_numpy(y_h).to(f"cuda:{dev}")
        p0, p1 = self.moments(a_ji, a_ii, a_ij, y)
        a, back = self._project(p0, p1)
        if _on_host(self.eig_compute_location):
            w, v = _host_batched(lambda x: np.linalg.eig(x), a.cpu().numpy(), 2)
            w, v = torch.from_numpy(w).to(a.device), torch.from_numpy(v).to(a.device)
        else:
            w, v = torch.linalg.eig(a)
        vs = back @ v
        return w.reshape(batch_shape + (self.m_0,)), vs.reshape(batch_shape + (n, self.m_0))
