"""Non-linear eigenvalue problems of the lead blocks on the device.

``Beyn`` mirrors ``qttools.nevp.Beyn`` (``src/qttools/nevp/beyn.py:14-379``):
the same constructor, the same probe block (``numpy.random.default_rng(42)``
drawn at construction, real parts then imaginary parts per call,
``beyn.py:96,310-313``), the same quadrature and the same SVD (or QR)
projection.  The contour integral -- one n x n inverse per quadrature point
and energy, the bulk of the work -- and the moment products run in
``qtx_beyn_moments`` (DMMA GEMM and batched inverse); the projection onto the
subspace and the small m0 x m0 eigenproblem use the dense SVD / QR / eig of
``torch.linalg`` on the device (cuSOLVER), in place of upstream's LAPACK
calls (``eig_compute_location`` / ``project_compute_location``).
"""

from __future__ import annotations

import ctypes
import math
from abc import ABC, abstractmethod

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


class Beyn(NEVP):
    """Beyn's contour-integral method for the eigenpairs inside the annulus
    r_i < |w| < r_o (``beyn.py:14-95``).  ``num_threads_contour``,
    ``eig_compute_location``, ``project_compute_location``,
    ``contour_batch_size`` and ``use_pinned_memory`` are accepted for
    signature compatibility; the device path sizes its own passes."""

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
        if self.use_qr:
            q, r = torch.linalg.qr(p0)
            a = q.mH @ p1 @ torch.linalg.inv(r)
            return a, q
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
        w, v = torch.linalg.eig(a)
        vs = back @ v
        return w.reshape(batch_shape + (self.m_0,)), vs.reshape(batch_shape + (n, self.m_0))
