"""Edge cases at the C ABI and the Python entry points: empty energy batches
are no-ops, a block size beyond the inverse's limit is refused with a status
(the context stays usable), the smallest devices solve."""


import numpy as np
import pytest
import torch

from quatrex_b200 import _lib
from quatrex_b200.obc import SanchoRubio
from quatrex_b200.transport import TransportSolver
from quatrex_b200.workloads import make_device

pytestmark = pytest.mark.gpu


def test_empty_batches_are_no_ops():
    lib = _lib.load()
    ctx = _lib.context(0)
    a = torch.zeros(1, 8, 8, dtype=torch.complex128, device="cuda")
    x = torch.full_like(a, 7.0)
    assert lib.qtx_inv(ctx, 8, 0, a.data_ptr(), 64, x.data_ptr(), 64, 0) == _lib.QTX_OK
    assert lib.qtx_zgemm(ctx, 8, 8, 8, 0, 1.0, 0.0, a.data_ptr(), 8, 64, 0, a.data_ptr(), 8, 64, 0, 0.0, 0.0, None, 8,
                         0, x.data_ptr(), 8, 64, _lib.QTX_PREC_FP64, 0) == _lib.QTX_OK
    assert lib.qtx_sancho_rubio(ctx, 8, 0, a.data_ptr(), 64, a.data_ptr(), 64, a.data_ptr(), 64, 1e-12, 10,
                                x.data_ptr(), None, 0) == _lib.QTX_OK
    torch.cuda.synchronize()
    assert torch.all(x == 7.0)


def test_transport_with_no_energies():
    dev = make_device(num_blocks=4, block_size=8, num_energies=3, seed=2)
    out = TransportSolver(dev, max_batch_size=4).solve(np.zeros(0), keys=("density", "transmission", "gr_diag"))
    assert out["density"].shape == (0, 4) and out["transmission"].shape == (0,)
    assert out["gr_diag"].shape == (0, 4, 8, 8)


def test_sancho_rubio_with_no_energies():
    dev = make_device(num_blocks=3, block_size=6, num_energies=2, seed=4)
    d, u, lo = dev.system_blocks()
    x = SanchoRubio(max_iterations=50, convergence_tol=1e-12)(d[0][:0], u[0], lo[0])
    assert tuple(x.shape) == (0, 6, 6)


def test_inverse_refuses_oversize_blocks_and_stays_usable():
    lib = _lib.load()
    ctx = _lib.context(0)
    a = torch.eye(513, dtype=torch.complex128, device="cuda")[None].contiguous()
    x = torch.empty_like(a)
    st = lib.qtx_inv(ctx, 513, 1, a.data_ptr(), 513 * 513, x.data_ptr(), 513 * 513, 0)
    assert st == _lib.QTX_E_UNSUPPORTED
    b = torch.eye(16, dtype=torch.complex128, device="cuda")[None].contiguous() * 2
    y = torch.empty_like(b)
    _lib.check(lib.qtx_inv(ctx, 16, 1, b.data_ptr(), 256, y.data_ptr(), 256, 0), ctx, "inv")
    assert torch.allclose(y, b / 4)


def test_two_block_device_every_energy_batching():
    """The smallest generator device (two blocks, both contacts) with one
    energy per call and all in one call: identical results."""
    dev = make_device(num_blocks=2, block_size=12, num_energies=5, seed=6)
    keys = ("gr_diag", "gl_diag", "density", "transmission")
    one = TransportSolver(dev, max_batch_size=1).solve(dev.energies, keys=keys)
    all_ = TransportSolver(dev, max_batch_size=5).solve(dev.energies, keys=keys)
    for k in keys:
        assert torch.equal(one[k], all_[k]), k
