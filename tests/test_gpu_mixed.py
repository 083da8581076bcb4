"""Mixed-precision form: complex products from 7-bit integer slices on the
INT8 tensor cores (tcgen05 kind::i8, exact INT32 accumulation), inverses and
Sancho-Rubio in FP64.

Bars: a single mixed GEMM within 1e-12 relative Frobenius error of the
complex128 product; the transport observables (per-block density,
transmission, contact current) within 1e-8 of the complex128 solve; the
drop-in selected solve within 1e-8 per block of the oracle."""

import numpy as np
import pytest
import torch

from oracle import rgf_oracle as orc
from quatrex_b200 import _lib
from quatrex_b200.datastructures import DSDBCOO
from quatrex_b200.greens_function_solver import RGF, OBCBlocks
from quatrex_b200.transport import TransportSolver
from quatrex_b200.workloads import make_device

pytestmark = pytest.mark.gpu


def _crand(g, *shape):
    return torch.complex(torch.randn(*shape, generator=g, dtype=torch.float64),
                         torch.randn(*shape, generator=g, dtype=torch.float64)).cuda()


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (128, 32, 32), (37, 53, 71), (256, 256, 256), (300, 200, 100)])
@pytest.mark.parametrize("op_a,op_b", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_mixed_gemm_matches_complex128(m, n, k, op_a, op_b):
    g = torch.Generator().manual_seed(m + 7 * n + 13 * k + op_a + 2 * op_b)
    batch = 3
    a = _crand(g, batch, *((m, k) if op_a == 0 else (k, m)))
    b = _crand(g, batch, *((k, n) if op_b == 0 else (n, k)))
    c = _crand(g, batch, m, n)
    d = torch.empty(batch, m, n, dtype=torch.complex128, device="cuda")
    lib = _lib.load()
    ctx = _lib.context(0)
    st = lib.qtx_zgemm(ctx, m, n, k, batch, 0.5, 0.25, a.data_ptr(), a.shape[-1], a.shape[-1] * a.shape[-2], op_a,
                       b.data_ptr(), b.shape[-1], b.shape[-1] * b.shape[-2], op_b, -1.0, 0.0, c.data_ptr(), n, m * n,
                       d.data_ptr(), n, m * n, _lib.QTX_PREC_MIXED, torch.cuda.current_stream().cuda_stream)
    _lib.check(st, ctx, "zgemm mixed")
    aa = a if op_a == 0 else a.conj().transpose(-1, -2)
    bb = b if op_b == 0 else b.conj().transpose(-1, -2)
    prod = aa @ bb
    ref = complex(0.5, 0.25) * prod - c
    err = float(torch.linalg.norm(d - ref) / torch.linalg.norm(prod))
    assert err < 1e-12, err


def test_mixed_gemm_wide_dynamic_range_rows():
    """Per-row / per-column power-of-two scales: rows of very different magnitude stay accurate."""
    g = torch.Generator().manual_seed(5)
    a = _crand(g, 1, 64, 64)
    a[0, :32] *= 1e8
    a[0, 32:] *= 1e-8
    b = _crand(g, 1, 64, 64)
    d = torch.empty(1, 64, 64, dtype=torch.complex128, device="cuda")
    lib = _lib.load()
    ctx = _lib.context(0)
    st = lib.qtx_zgemm(ctx, 64, 64, 64, 1, 1.0, 0.0, a.data_ptr(), 64, 4096, 0, b.data_ptr(), 64, 4096, 0, 0.0, 0.0,
                       None, 64, 4096, d.data_ptr(), 64, 4096, _lib.QTX_PREC_MIXED, 0)
    _lib.check(st, ctx, "zgemm mixed")
    ref = a @ b
    rel_rows = torch.linalg.norm(d - ref, dim=-1) / torch.linalg.norm(ref, dim=-1)
    assert float(rel_rows.max()) < 1e-12


def test_mixed_transport_observables_within_1e8():
    dev = make_device(num_blocks=8, block_size=64, num_energies=12, seed=77)
    keys = ("gl_diag", "density", "hole_density", "transmission", "current_left", "current_right")
    f = TransportSolver(dev, precision="fp64").solve(dev.energies, keys=keys)
    m = TransportSolver(dev, precision="mixed").solve(dev.energies, keys=keys)
    dens_err = (torch.abs(m["density"] - f["density"]) / torch.abs(f["density"]).amax(dim=1, keepdim=True)).max()
    assert float(dens_err) < 1e-8
    t_err = torch.abs(m["transmission"] - f["transmission"]) / torch.clamp(torch.abs(f["transmission"]), min=1e-12)
    assert float(t_err.max()) < 1e-8
    c_err = torch.abs(m["current_left"] - f["current_left"]) / torch.abs(f["current_left"]).max()
    assert float(c_err.max()) < 1e-8


def test_mixed_selected_solve_against_oracle():
    dev = make_device(num_blocks=5, block_size=32, num_energies=4, seed=12)
    d, u, lo = dev.system_blocks()
    obc = orc.obc_self_energies(d, u, lo, dev.energies, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol,
                                dev.sr_max_iter)
    nb = 5
    A = DSDBCOO.from_blocks(d, u, lo, device="cuda")
    Z = DSDBCOO.from_blocks([np.zeros_like(x) for x in d], [np.zeros_like(x) for x in u],
                            [np.zeros_like(x) for x in lo], device="cuda")
    ob = OBCBlocks(nb)
    ob.retarded[0], ob.retarded[-1] = obc["retarded"]
    ob.lesser[0], ob.lesser[-1] = obc["lesser"]
    ob.greater[0], ob.greater[-1] = obc["greater"]
    xl, xg, xr = RGF(precision="mixed").selected_solve(A, Z, Z, obc_blocks=ob, return_retarded=True)
    pad = [None] * (nb - 2)
    z = [np.zeros_like(x) for x in d]
    zu = [np.zeros_like(x) for x in u]
    ref = orc.selected_solve(d, u, lo, z, zu, z, zu, [obc["retarded"][0], *pad, obc["retarded"][1]],
                             [obc["lesser"][0], *pad, obc["lesser"][1]], [obc["greater"][0], *pad, obc["greater"][1]])
    for i in range(nb):
        for key, X in (("xl", xl), ("xg", xg), ("xr", xr)):
            want = ref[f"{key}_diag"][i]
            got = X.blocks[i, i]
            assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-8, (key, i)
