"""Open-boundary conditions on the device: Sancho-Rubio decimation and the
contact self-energy assembly.

``SanchoRubio`` mirrors ``src/qttools/boundary_conditions/obc/sancho_rubio.py``
(``__init__`` ``:28-31``, ``__call__`` ``:33-86``): same defaults, same
arguments, the same RuntimeWarning when ``max_iterations`` is reached.  Each
energy stops iterating once its own convergence measure
``|| |alpha| + |beta| ||_F / 2`` is below the tolerance (the upstream loop
stops when the maximum over the batch is); converged entries change by
O(tol^2) per extra iteration, far below the parity tolerance.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from quatrex_b200 import _lib


def _as_device(x, device: int) -> tuple[torch.Tensor, bool]:
    was_host = not (isinstance(x, torch.Tensor) and x.is_cuda)
    t = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(np.asarray(x)))
    return t.to(device=f"cuda:{device}", dtype=torch.complex128).contiguous(), was_host


def _batch_view(t: torch.Tensor) -> tuple[int, int]:
    """(batch, stride) of a (..., n, n) tensor; a 2-D tensor is broadcast (stride 0)."""
    n = t.shape[-1]
    if t.dim() == 2:
        return 1, 0
    return int(math.prod(t.shape[:-2])), n * n


class SanchoRubio:
    """Surface Green's function by Sancho-Rubio decimation on the GPU.

    Parameters
    ----------
    max_iterations : int, optional
        The maximum number of iterations, by default 100.
    convergence_tol : float, optional
        Convergence tolerance on the Frobenius norm of |alpha| + |beta|, by
        default 1e-6.
    """

    def __init__(self, max_iterations: int = 100, convergence_tol: float = 1e-6):
        self.max_iterations = max_iterations
        self.convergence_tol = convergence_tol
        self.last_iterations = None

    def __call__(self, a_ii, a_ij, a_ji, contact: str = ""):
        """Returns the surface Green's function x = inv(a_ii - a_ji x a_ij)."""
        dev = torch.cuda.current_device() if torch.cuda.is_available() else None
        if dev is None:
            raise RuntimeError("quatrex_b200 needs a CUDA device (B200, sm_100a); there is no CPU path")
        lib = _lib.load()
        ctx = _lib.context(dev)
        tii, host = _as_device(a_ii, dev)
        tij, _ = _as_device(a_ij, dev)
        tji, _ = _as_device(a_ji, dev)
        n = tii.shape[-1]
        shapes = [t.shape[:-2] for t in (tii, tij, tji) if t.dim() > 2]
        batch_shape = shapes[0] if shapes else ()
        batch = int(math.prod(batch_shape)) if batch_shape else 1
        _, sii = _batch_view(tii)
        _, sij = _batch_view(tij)
        _, sji = _batch_view(tji)
        x = torch.empty(batch_shape + (n, n), dtype=torch.complex128, device=f"cuda:{dev}")
        its = torch.zeros(batch, dtype=torch.int32, device=f"cuda:{dev}")
        st = lib.qtx_sancho_rubio(ctx, n, batch, tii.data_ptr(), sii, tij.data_ptr(), sij, tji.data_ptr(), sji,
                                  float(self.convergence_tol), int(self.max_iterations), x.data_ptr(),
                                  its.data_ptr(), torch.cuda.current_stream().cuda_stream)
        _lib.check(st, ctx, "SanchoRubio")
        self.last_iterations = its.cpu().numpy()
        if host:
            return x.cpu().numpy()
        return x


def contact_self_energies(g, m_ji, m_ij, occupancy):
    """Sigma^R = m_ji g m_ij, Gamma = i (Sigma - Sigma^H), Sigma^< = i f Gamma,
    Sigma^> = i (f - 1) Gamma (``src/quatrex/electron/solver.py:318-337``)."""
    dev = torch.cuda.current_device()
    lib = _lib.load()
    ctx = _lib.context(dev)
    tg, host = _as_device(g, dev)
    tji, _ = _as_device(m_ji, dev)
    tij, _ = _as_device(m_ij, dev)
    n = tg.shape[-1]
    batch, _ = _batch_view(tg)
    _, sji = _batch_view(tji)
    _, sij = _batch_view(tij)
    occ = torch.as_tensor(np.asarray(occupancy, dtype=np.float64)).to(f"cuda:{dev}").contiguous()
    out = [torch.empty_like(tg) for _ in range(3)]
    st = lib.qtx_obc_assemble(ctx, n, batch, tg.data_ptr(), tji.data_ptr(), sji, tij.data_ptr(), sij,
                              occ.data_ptr(), out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(),
                              torch.cuda.current_stream().cuda_stream)
    _lib.check(st, ctx, "contact_self_energies")
    if host:
        return tuple(o.cpu().numpy() for o in out)
    return tuple(out)
