"""The allocation-free Sancho-Rubio entry point.

qtx_sancho_rubio_noalloc exists for callers that cannot let a library allocate
device memory (their own allocator owns the device memory, their host forbids
library allocations, or a cudaMalloc / cudaFree would stall a latency-critical
loop).  It keeps its work arrays in one fixed 16 MiB device array of the
library.  These tests call it through the C ABI, twice in a row on the same
inputs, and compare each result with the regular qtx_sancho_rubio entry point
(which allocates from its context's pool) within the 1e-12 relative tolerance
used for single kernels, and with the oracle within the 1e-10 bar of the other
Sancho-Rubio tests; they check that a call leaves the device's free memory,
the stream-ordered pool and torch's allocator exactly as they were, that a
request larger than the fixed array is refused with a message, that a run out
of iterations reports QTX_E_NOT_CONVERGED with its message and still writes
x, and that an exactly singular decimation block reports QTX_E_SINGULAR.  The
file is named to run last.
"""

import ctypes

import numpy as np
import pytest
import torch

from oracle import rgf_oracle as orc
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


def _pool_counters():
    """(reserved, used) bytes of the device's default stream-ordered pool (the
    pool the regular entry points allocate from), via the driver API."""
    cu = ctypes.CDLL("libcuda.so.1")
    dev = ctypes.c_int()
    assert cu.cuDeviceGet(ctypes.byref(dev), torch.cuda.current_device()) == 0
    pool = ctypes.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(ctypes.byref(pool), dev) == 0
    out = []
    for attr in (5, 7):  # CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT, CU_MEMPOOL_ATTR_USED_MEM_CURRENT
        v = ctypes.c_uint64()
        assert cu.cuMemPoolGetAttribute(pool, attr, ctypes.byref(v)) == 0
        out.append(v.value)
    return tuple(out)


def _memory_state():
    """Device free memory, the stream-ordered pool's counters and torch's
    cached reservation.  (torch's count of live tensors is left out: a tensor
    of an earlier test may be collected at any moment, and the library never
    allocates through torch.)"""
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info()
    return {"free": free, "pool": _pool_counters(), "torch_reserved": torch.cuda.memory_reserved()}


def test_noalloc_matches_oracle():
    dev = make_device(num_blocks=3, block_size=24, num_energies=9, seed=11)
    d, u, lo = dev.system_blocks()
    x_ref, it_ref = orc.sancho_rubio(d[0], u[0], lo[0], 200, 1e-12)
    to = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    for _ in range(2):
        st, x, its, msg = _noalloc(to(d[0]), to(u[0]), to(lo[0]))
        assert st == _lib.QTX_OK, msg
        assert _rel(x.cpu(), torch.from_numpy(x_ref)) < 1e-10
        assert int(its.max()) == it_ref


def test_noalloc_allocates_nothing():
    a_ii, a_ij, a_ji = _inputs(n=32, ne=8, seed=21)
    st, _, _, msg = _noalloc(a_ii, a_ij, a_ji)  # loads every kernel the call launches
    assert st == _lib.QTX_OK, msg
    x = torch.empty_like(a_ii)
    its = torch.zeros(a_ii.shape[0], dtype=torch.int32, device="cuda")
    err = ctypes.create_string_buffer(512)
    lib = _lib.load()
    before = _memory_state()
    for _ in range(2):
        st = lib.qtx_sancho_rubio_noalloc(32, 8, a_ii.data_ptr(), 32 * 32, a_ij.data_ptr(), 32 * 32,
                                          a_ji.data_ptr(), 32 * 32, 1e-12, 200, x.data_ptr(), its.data_ptr(),
                                          torch.cuda.current_stream().cuda_stream, err, len(err))
        assert st == _lib.QTX_OK, err.value.decode()
    after = _memory_state()
    assert after == before


def test_noalloc_not_converged_reports_and_writes_x():
    a_ii, a_ij, a_ji = _inputs(n=16, ne=4, seed=5)
    lib = _lib.load()
    x = torch.full_like(a_ii, float("nan"))
    its = torch.zeros(4, dtype=torch.int32, device="cuda")
    err = ctypes.create_string_buffer(512)
    st = lib.qtx_sancho_rubio_noalloc(16, 4, a_ii.data_ptr(), 256, a_ij.data_ptr(), 256, a_ji.data_ptr(), 256,
                                      1e-12, 1, x.data_ptr(), its.data_ptr(),
                                      torch.cuda.current_stream().cuda_stream, err, len(err))
    torch.cuda.synchronize()
    assert st == _lib.QTX_E_NOT_CONVERGED
    assert "did not converge" in err.value.decode()
    assert bool(torch.isfinite(torch.view_as_real(x)).all())
    assert int(its.max()) == 1
    # the same as the regular entry point with one iteration
    x_ref = torch.empty_like(a_ii)
    ctx = _lib.context(torch.cuda.current_device())
    st_ref = lib.qtx_sancho_rubio(ctx, 16, 4, a_ii.data_ptr(), 256, a_ij.data_ptr(), 256, a_ji.data_ptr(), 256,
                                  1e-12, 1, x_ref.data_ptr(), None, torch.cuda.current_stream().cuda_stream)
    assert st_ref == _lib.QTX_E_NOT_CONVERGED
    assert _rel(x, x_ref) < 1e-12


def test_noalloc_singular_decimation_block():
    n, ne = 8, 2
    a_ii = torch.zeros(ne, n, n, dtype=torch.complex128, device="cuda")  # exactly singular first block
    a_ij = torch.eye(n, dtype=torch.complex128, device="cuda").repeat(ne, 1, 1)
    st, _, _, msg = _noalloc(a_ii, a_ij, a_ij.clone(), max_it=3)
    assert st == _lib.QTX_E_SINGULAR
    assert "singular" in msg
    # the shared array is cleared again by the next call
    good = _inputs(n=8, ne=2, seed=9)
    x_ref, _ = _regular(*good)
    st, x, _, msg = _noalloc(*good)
    assert st == _lib.QTX_OK, msg
    assert _rel(x, x_ref) < 1e-12
