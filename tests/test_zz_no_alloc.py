"""The allocation-free Sancho-Rubio entry point.

qtx_sancho_rubio_noalloc exists for callers that cannot let a library allocate
device memory (their own allocator owns the device memory, their host forbids
library allocations, or a cudaMalloc / cudaFree would stall a latency-critical
loop).  It keeps its work arrays in one fixed 16 MiB device array of the
library.  These tests call it through the C ABI, twice in a row on the same
inputs, and compare each result with the regular qtx_sancho_rubio entry point
(which allocates from its context's pool) within the 1e-12 relative tolerance
used for single kernels; they also check that a request larger than the fixed
array is refused with a message.  The file is named to run last.
"""

import ctypes

import numpy as np
import pytest
import torch

from quatrex_b200 import _lib
from quatrex_b200.workloads import make_device

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def _inputs(n=32, ne=6, seed=17):
    dev = make_device(num_blocks=2, block_size=n, num_energies=ne, seed=seed)
    d, u, lo = dev.system_blocks()
    to = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    return to(d[0]), to(u[0]), to(lo[0])


def _regular(a_ii, a_ij, a_ji, tol=1e-12, max_it=200):
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    n, ne = a_ii.shape[-1], a_ii.shape[0]
    x = torch.empty_like(a_ii)
    its = torch.zeros(ne, dtype=torch.int32, device="cuda")
    st = lib.qtx_sancho_rubio(ctx, n, ne, a_ii.data_ptr(), n * n, a_ij.data_ptr(), n * n, a_ji.data_ptr(), n * n,
                              tol, max_it, x.data_ptr(), its.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == _lib.QTX_OK
    return x, its


def _noalloc(a_ii, a_ij, a_ji, tol=1e-12, max_it=200, batch=None):
    lib = _lib.load()
    n = a_ii.shape[-1]
    ne = a_ii.shape[0] if batch is None else batch
    x = torch.empty_like(a_ii)
    its = torch.zeros(a_ii.shape[0], dtype=torch.int32, device="cuda")
    err = ctypes.create_string_buffer(512)
    st = lib.qtx_sancho_rubio_noalloc(n, ne, a_ii.data_ptr(), n * n, a_ij.data_ptr(), n * n, a_ji.data_ptr(),
                                      n * n, tol, max_it, x.data_ptr(), its.data_ptr(),
                                      torch.cuda.current_stream().cuda_stream, err, len(err))
    return st, x, its, err.value.decode()


def test_noalloc_matches_regular_entry_point_twice():
    a_ii, a_ij, a_ji = _inputs()
    x_ref, its_ref = _regular(a_ii, a_ij, a_ji)
    for _ in range(2):  # the second call reuses the shared array left by the first
        st, x, its, msg = _noalloc(a_ii, a_ij, a_ji)
        assert st == _lib.QTX_OK, msg
        assert _rel(x, x_ref) < 1e-12
        assert torch.equal(its, its_ref)


def test_noalloc_different_inputs_back_to_back():
    """A second call with different data is not affected by the first call's leftovers."""
    first = _inputs(n=24, ne=5, seed=3)
    second = _inputs(n=16, ne=9, seed=4)
    for a in (first, second, first):
        x_ref, _ = _regular(*a)
        st, x, _, msg = _noalloc(*a)
        assert st == _lib.QTX_OK, msg
        assert _rel(x, x_ref) < 1e-12


def test_noalloc_rejects_oversize_request():
    a_ii, a_ij, a_ji = _inputs(n=32, ne=2)
    # 9 * 16 * 32^2 * batch bytes > 16 MiB for batch >= 114; claim a batch of 200
    lib = _lib.load()
    err = ctypes.create_string_buffer(512)
    st = lib.qtx_sancho_rubio_noalloc(32, 200, a_ii.data_ptr(), 0, a_ij.data_ptr(), 0, a_ji.data_ptr(), 0, 1e-12,
                                      10, a_ii.data_ptr(), None, torch.cuda.current_stream().cuda_stream, err,
                                      len(err))
    assert st == _lib.QTX_E_INVAL
    assert "bytes" in err.value.decode()
