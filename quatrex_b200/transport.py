"""Generator-form transport solve on the device (qtx_transport_solve).

The energy-independent Hamiltonian blocks stay resident on the GPU; for each
energy batch the library forms A(E) = (E + i eta) I - H on the fly (inside the
GEMM epilogues), computes both contact self-energies by Sancho-Rubio, runs
the selected solve and writes the requested Green's-function blocks and
observables.  This is the device-resident form of
``ElectronSolver.solve`` (``src/quatrex/electron/solver.py:456-604``) for a
device whose leads repeat its end cells and whose interior scattering
self-energies vanish.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from quatrex_b200 import _lib
from quatrex_b200.workloads import TransportDevice

_PRECISIONS = {"fp64": _lib.QTX_PREC_FP64, "mixed": _lib.QTX_PREC_MIXED}

OUTPUT_KEYS = ("gr_diag", "gr_upper", "gr_lower", "gl_diag", "gl_upper", "gg_diag", "gg_upper", "density",
               "hole_density", "transmission", "current_left", "current_right", "sr_iterations", "dos",
               "layer_current")


def allocate_outputs(num_blocks: int, block_size: int, num_energies: int, keys=OUTPUT_KEYS,
                     cuda_device: int = 0) -> dict:
    """Device output arrays of qtx_transport_solve for the given keys."""
    nb, b, ne = int(num_blocks), int(block_size), int(num_energies)
    dev = f"cuda:{cuda_device}"
    shapes = {
        "gr_diag": (ne, nb, b, b), "gr_upper": (ne, nb - 1, b, b), "gr_lower": (ne, nb - 1, b, b),
        "gl_diag": (ne, nb, b, b), "gl_upper": (ne, nb - 1, b, b),
        "gg_diag": (ne, nb, b, b), "gg_upper": (ne, nb - 1, b, b),
    }
    out = {}
    for k in keys:
        if k in shapes:
            out[k] = torch.empty(shapes[k], dtype=torch.complex128, device=dev)
        elif k in ("density", "hole_density", "dos"):
            out[k] = torch.empty((ne, nb), dtype=torch.float64, device=dev)
        elif k == "layer_current":
            out[k] = torch.empty((ne, nb - 1), dtype=torch.complex128, device=dev)
        elif k == "transmission":
            out[k] = torch.empty((ne,), dtype=torch.float64, device=dev)
        elif k in ("current_left", "current_right"):
            out[k] = torch.empty((ne,), dtype=torch.complex128, device=dev)
        elif k == "sr_iterations":
            out[k] = torch.empty((ne, 2), dtype=torch.int32, device=dev)
    return out


class TransportSolver:
    """Device-resident transport solver for one ``TransportDevice``."""

    def __init__(self, device: TransportDevice, max_batch_size: int = 128, precision: str = "fp64",
                 cuda_device: int | None = None, h_diag=None, h_upper=None, ctx: int | None = None,
                 stream=None, use_graph: bool = False):
        if not torch.cuda.is_available():
            raise RuntimeError("quatrex_b200 needs a CUDA device (B200, sm_100a); there is no CPU path")
        self.dev = device
        self.cuda = torch.cuda.current_device() if cuda_device is None else cuda_device
        self.max_batch_size = int(max_batch_size)
        self.precision = precision
        self.nb = device.num_blocks
        self.b = device.block_size
        # H may be handed in already on the device (e.g. shared by several solvers)
        self.h_diag = h_diag if h_diag is not None else torch.from_numpy(device.h_diag).to(f"cuda:{self.cuda}")
        self.h_upper = h_upper if h_upper is not None else torch.from_numpy(device.h_upper).to(f"cuda:{self.cuda}")
        self.ctx = ctx
        self.stream = stream
        # CUDA-graph replay needs the same buffers every call: a fixed energy buffer
        self.use_graph = use_graph
        self._e_buf = None

    @staticmethod
    def footprint_bytes(num_blocks: int, block_size: int, energies_per_call: int, keys=OUTPUT_KEYS,
                        precision: str = "fp64") -> int:
        """Device bytes one call holds: H and couplings, the library's work
        space for one energy batch (sweep, Sancho-Rubio, the scratch of the
        block inverse and of the mixed-precision products:
        ``qtx_transport_footprint``) and the requested outputs (used for
        admission control)."""
        nb, b, ne = int(num_blocks), int(block_size), int(energies_per_call)
        bb = 16 * b * b
        h = bb * (nb + 3 * max(nb - 1, 1))
        lib = _lib.load()
        prec = _lib.QTX_PREC_MIXED if precision == "mixed" else _lib.QTX_PREC_FP64
        ws = int(lib.qtx_transport_footprint(nb, b, ne, prec))
        blocks = {"gr_diag": nb, "gr_upper": nb - 1, "gr_lower": nb - 1, "gl_diag": nb, "gl_upper": nb - 1,
                  "gg_diag": nb, "gg_upper": nb - 1}
        out = sum(bb * ne * blocks[k] for k in keys if k in blocks) + 64 * ne * nb
        return int(h + ws + out)

    def allocate_outputs(self, num_energies: int, keys=OUTPUT_KEYS) -> dict:
        return allocate_outputs(self.nb, self.b, num_energies, keys, self.cuda)

    def release_graphs(self, stream=None) -> None:
        """Drop the captured sweeps of this solver's context (stream-ordered free)."""
        lib = _lib.load()
        ctx = self.ctx if self.ctx is not None else _lib.context(self.cuda)
        s = self._stream_handle(stream)
        _lib.check(lib.qtx_ctx_release_graphs(ctx, s), ctx, "ctx_release_graphs")

    def _stream_handle(self, stream=None):
        if stream is None:
            stream = self.stream
        if stream is None:
            return torch.cuda.current_stream(self.cuda).cuda_stream
        return stream.cuda_stream if hasattr(stream, "cuda_stream") else stream

    def solve(self, energies, outputs: dict | None = None, keys=OUTPUT_KEYS, stream=None) -> dict:
        """Solve at the given energies (device or host array); returns the output dict."""
        e = energies if isinstance(energies, torch.Tensor) else torch.as_tensor(np.asarray(energies, dtype=np.float64))
        e = e.to(device=f"cuda:{self.cuda}", dtype=torch.float64).contiguous()
        ne = int(e.shape[0])
        flags = 0
        if self.use_graph and ne <= self.max_batch_size:
            if self._e_buf is None or self._e_buf.shape[0] != ne:
                self._e_buf = torch.empty(ne, dtype=torch.float64, device=f"cuda:{self.cuda}")
            self._e_buf.copy_(e, non_blocking=True)
            e = self._e_buf
            flags |= _lib.QTX_FLAG_GRAPH
        if outputs is None:
            outputs = self.allocate_outputs(ne, keys)
        lib = _lib.load()
        ctx = self.ctx if self.ctx is not None else _lib.context(self.cuda)
        p = _lib.TransportProblem(
            num_blocks=self.nb, block_size=self.b, num_energies=ne, h_diag=self.h_diag.data_ptr(),
            h_upper=self.h_upper.data_ptr(), energies=e.data_ptr(), eta=self.dev.eta, mu_left=self.dev.mu_left,
            mu_right=self.dev.mu_right, kt=self.dev.kt, sr_tol=self.dev.sr_tol,
            sr_max_iterations=self.dev.sr_max_iter, max_batch_size=self.max_batch_size)
        o = _lib.TransportOutputs(**{k: (outputs[k].data_ptr() if k in outputs else None) for k in OUTPUT_KEYS})
        s = self._stream_handle(stream)
        st = lib.qtx_transport_solve(ctx, ctypes.byref(p), ctypes.byref(o), _PRECISIONS[self.precision], flags, s)
        _lib.check(st, ctx, "transport_solve")
        return outputs


GROUPED_MAX_BLOCK_SIZE = 64


def grouped_footprint_bytes(num_blocks, num_energies, block_size: int) -> int:
    """Device bytes of one qtx_transport_solve_grouped call (descriptors and
    the per-CTA work spaces; H and outputs not included)."""
    nbs = (ctypes.c_int32 * len(num_blocks))(*[int(x) for x in num_blocks])
    nes = (ctypes.c_int64 * len(num_energies))(*[int(x) for x in num_energies])
    return int(_lib.load().qtx_transport_grouped_footprint(len(nbs), nbs, nes, int(block_size)))


def solve_grouped(devices: list[TransportDevice], energies: list, keys=OUTPUT_KEYS, cuda_device: int | None = None,
                  hamiltonians: list | None = None, ctx: int | None = None, stream=None) -> list[dict]:
    """Solve every energy of several devices that share one block size
    (<= 64) in one persistent launch (qtx_transport_solve_grouped).

    ``energies[q]`` is the energy grid of ``devices[q]``; ``hamiltonians[q]``
    may hand in its (h_diag, h_upper) already on the device.  Returns one
    output dict (device tensors) per device, in input order."""
    if not torch.cuda.is_available():
        raise RuntimeError("quatrex_b200 needs a CUDA device (B200, sm_100a); there is no CPU path")
    if len(devices) != len(energies) or not devices:
        raise ValueError("solve_grouped: one energy grid per device")
    cuda = torch.cuda.current_device() if cuda_device is None else cuda_device
    dev = f"cuda:{cuda}"
    b = devices[0].block_size
    if any(d.block_size != b for d in devices):
        raise ValueError("solve_grouped: every device must have the same block size")
    keep, probs, outs, results = [], [], [], []
    for q, d in enumerate(devices):
        if hamiltonians is not None:
            h_diag, h_upper = hamiltonians[q]
        else:
            h_diag = torch.from_numpy(d.h_diag).to(dev)
            h_upper = torch.from_numpy(d.h_upper).to(dev)
        e = energies[q]
        e = e if isinstance(e, torch.Tensor) else torch.as_tensor(np.asarray(e, dtype=np.float64))
        e = e.to(device=dev, dtype=torch.float64).contiguous()
        out = allocate_outputs(d.num_blocks, b, int(e.shape[0]), keys, cuda)
        keep.append((h_diag, h_upper, e))
        results.append(out)
        probs.append(_lib.TransportProblem(
            num_blocks=d.num_blocks, block_size=b, num_energies=int(e.shape[0]), h_diag=h_diag.data_ptr(),
            h_upper=h_upper.data_ptr(), energies=e.data_ptr(), eta=d.eta, mu_left=d.mu_left, mu_right=d.mu_right,
            kt=d.kt, sr_tol=d.sr_tol, sr_max_iterations=d.sr_max_iter, max_batch_size=0))
        outs.append(_lib.TransportOutputs(**{k: (out[k].data_ptr() if k in out else None) for k in OUTPUT_KEYS}))
    p_arr = (_lib.TransportProblem * len(probs))(*probs)
    o_arr = (_lib.TransportOutputs * len(outs))(*outs)
    lib = _lib.load()
    ctx = ctx if ctx is not None else _lib.context(cuda)
    if stream is None:
        s = torch.cuda.current_stream(cuda).cuda_stream
    else:
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
    st = lib.qtx_transport_solve_grouped(ctx, len(probs), p_arr, o_arr, _lib.QTX_PREC_FP64, 0, None, s)
    _lib.check(st, ctx, "transport_solve_grouped")
    return results


# outputs derived from the Green's functions of an energy (zero when those are)
_G_DERIVED_KEYS = ("gr_diag", "gr_upper", "gr_lower", "gl_diag", "gl_upper", "gg_diag", "gg_upper", "density",
                   "hole_density", "transmission", "current_left", "current_right", "layer_current")


def peak_mask(dos, energies, dos_peak_limit: float = 100.0):
    """Energies whose Green's functions ``ElectronSolver._filter_peaks``
    (``src/quatrex/electron/solver.py:412-454``) sets to zero: the largest
    slope |d dos / dE| over the blocks above ``dos_peak_limit``, or the largest
    block DOS above 10.  ``dos`` is the (num_energies, nb) 'dos' output over
    the whole energy grid (a slope needs the neighbouring energies); the slope
    is taken as numpy.gradient takes it: second-order central differences
    inside the grid, one-sided differences at its ends."""
    e = torch.as_tensor(np.asarray(energies, dtype=np.float64) if not isinstance(energies, torch.Tensor)
                        else energies, dtype=torch.float64, device=dos.device)
    slope = torch.gradient(dos, spacing=(e,), dim=0)[0].abs()
    return (slope.amax(dim=1) > dos_peak_limit) | (dos.amax(dim=1) > 10)


def filter_peaks(outputs: dict, mask) -> None:
    """Zero, in place, the Green's-function blocks of the masked energies and
    the observables formed from them (upstream filters G before its
    observables are computed, so they vanish there too); 'dos' and
    'sr_iterations' are kept."""
    for k in _G_DERIVED_KEYS:
        if k in outputs:
            outputs[k][mask.to(outputs[k].device)] = 0
