"""Kernel-level parity on the GPU: the batched complex GEMM against a torch
complex128 matmul, the batched inverse against NumPy/LAPACK, Sancho-Rubio
against the oracle.  Tolerances: relative Frobenius error 1e-12 for a single
GEMM, 1e-10 for inverses of well-conditioned blocks."""


import numpy as np
import pytest
import torch

from oracle import rgf_oracle as orc
from quatrex_b200 import _lib
from quatrex_b200.obc import SanchoRubio, contact_self_energies
from quatrex_b200.workloads import make_device

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else a
    b = b.cpu().numpy() if isinstance(b, torch.Tensor) else b
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _crand(g, *shape):
    return torch.complex(torch.randn(*shape, generator=g, dtype=torch.float64),
                         torch.randn(*shape, generator=g, dtype=torch.float64)).cuda()


def _zgemm(m, n, k, batch, alpha, a, op_a, b, op_b, beta, c, d, sa=None, sb=None):
    lib = _lib.load()
    ctx = _lib.context(0)
    lda = a.shape[-1]
    ldb = b.shape[-1]
    sa = a.shape[-1] * a.shape[-2] if sa is None else sa
    sb = b.shape[-1] * b.shape[-2] if sb is None else sb
    st = lib.qtx_zgemm(ctx, m, n, k, batch, alpha.real, alpha.imag, a.data_ptr(), lda, sa, op_a, b.data_ptr(), ldb,
                       sb, op_b, beta.real, beta.imag, c.data_ptr() if c is not None else None, n, m * n,
                       d.data_ptr(), n, m * n, 0, torch.cuda.current_stream().cuda_stream)
    _lib.check(st, ctx, "zgemm")
    torch.cuda.synchronize()


@pytest.mark.parametrize("m,n,k", [(64, 64, 64), (1, 1, 1), (2, 4, 2), (37, 53, 71), (128, 96, 200), (256, 256, 256)])
@pytest.mark.parametrize("op_a", [0, 1])
@pytest.mark.parametrize("op_b", [0, 1])
def test_zgemm_matches_torch(m, n, k, op_a, op_b):
    g = torch.Generator().manual_seed(m * 1000 + n * 10 + k)
    batch = 3
    a = _crand(g, batch, *((m, k) if op_a == 0 else (k, m)))
    b = _crand(g, batch, *((k, n) if op_b == 0 else (n, k)))
    c = _crand(g, batch, m, n)
    d = torch.empty(batch, m, n, dtype=torch.complex128, device="cuda")
    alpha, beta = complex(0.7, -0.2), complex(-1.0, 0.5)
    _zgemm(m, n, k, batch, alpha, a, op_a, b, op_b, beta, c, d)
    aa = a if op_a == 0 else a.conj().transpose(-1, -2)
    bb = b if op_b == 0 else b.conj().transpose(-1, -2)
    ref = alpha * (aa @ bb) + beta * c
    assert _rel(d, ref) < 1e-13


def test_zgemm_broadcast_operand():
    g = torch.Generator().manual_seed(5)
    a = _crand(g, 1, 48, 48)
    b = _crand(g, 4, 48, 48)
    d = torch.empty(4, 48, 48, dtype=torch.complex128, device="cuda")
    _zgemm(48, 48, 48, 4, 1.0 + 0j, a, 0, b, 0, 0j, None, d, sa=0)
    assert _rel(d, a @ b) < 1e-13


@pytest.mark.parametrize("n", [1, 2, 3, 4, 8, 16, 24, 31, 48, 64, 96, 100, 128, 129, 161, 200, 250, 255, 256, 257, 300,
                               512])
def test_inverse_matches_lapack(n):
    rng = np.random.default_rng(n)
    batch = 5
    a = rng.standard_normal((batch, n, n)) + 1j * rng.standard_normal((batch, n, n))
    a += np.sqrt(n) * np.eye(n)  # keep the condition number moderate
    ta = torch.from_numpy(a).cuda()
    x = torch.empty_like(ta)
    lib = _lib.load()
    ctx = _lib.context(0)
    st = lib.qtx_inv(ctx, n, batch, ta.data_ptr(), n * n, x.data_ptr(), n * n, torch.cuda.current_stream().cuda_stream)
    _lib.check(st, ctx, "inv")
    ref = np.linalg.inv(a)
    assert _rel(x, ref) < 1e-10
    # in place
    st = lib.qtx_inv(ctx, n, batch, ta.data_ptr(), n * n, ta.data_ptr(), n * n, torch.cuda.current_stream().cuda_stream)
    _lib.check(st, ctx, "inv")
    assert _rel(ta, ref) < 1e-10


@pytest.mark.parametrize("n", [96, 200, 256, 300])
def test_inverse_split_and_fused_paths_agree(n):
    """Small batches take the split path (one launch per panel elimination and
    one per rank-w update over the whole GPU), large batches the fused kernel
    (one CTA per matrix); both apply the same operations in the same order,
    so the first entries of a 130-matrix batch equal a 5-matrix call bit for
    bit, and both match LAPACK."""
    rng = np.random.default_rng(n + 7)
    a = rng.standard_normal((130, n, n)) + 1j * rng.standard_normal((130, n, n))
    a[:, np.arange(n), np.arange(n)] += np.sqrt(n)
    ta = torch.from_numpy(a).cuda()
    big, small = torch.empty_like(ta), torch.empty_like(ta[:5])
    lib = _lib.load()
    ctx = _lib.context(0)
    _lib.check(lib.qtx_inv(ctx, n, 130, ta.data_ptr(), n * n, big.data_ptr(), n * n, 0), ctx, "inv")
    _lib.check(lib.qtx_inv(ctx, n, 5, ta.data_ptr(), n * n, small.data_ptr(), n * n, 0), ctx, "inv")
    assert torch.equal(small, big[:5])
    assert _rel(small, np.linalg.inv(a[:5])) < 1e-10


@pytest.mark.parametrize("n", [200, 256])
@pytest.mark.parametrize("batch", [5, 130], ids=["split", "fused"])
def test_inverse_output_sixteen_bytes_off(n, batch):
    """The split path reads and writes adjacent column pairs in one 32-byte
    access only when the matrices start 32-byte aligned; an output batch that
    starts one complex element (16 bytes) into its buffer takes the 16-byte
    accesses and returns the same bits as an aligned one."""
    rng = np.random.default_rng(n + batch)
    a = rng.standard_normal((batch, n, n)) + 1j * rng.standard_normal((batch, n, n))
    a[:, np.arange(n), np.arange(n)] += np.sqrt(n)
    ta = torch.from_numpy(a).cuda()
    aligned = torch.empty_like(ta)
    buf = torch.empty(batch * n * n + 1, dtype=torch.complex128, device="cuda")
    off = buf[1:].view(batch, n, n)
    assert off.data_ptr() % 32 == 16
    lib = _lib.load()
    ctx = _lib.context(0)
    _lib.check(lib.qtx_inv(ctx, n, batch, ta.data_ptr(), n * n, aligned.data_ptr(), n * n, 0), ctx, "inv")
    _lib.check(lib.qtx_inv(ctx, n, batch, ta.data_ptr(), n * n, off.data_ptr(), n * n, 0), ctx, "inv")
    assert torch.equal(off, aligned)
    assert _rel(aligned[:3], np.linalg.inv(a[:3])) < 1e-10


def test_inverse_needs_pivoting():
    # zero leading diagonal entries: fails without row interchanges
    a = np.array([[0, 1, 2], [1, 0, 3], [4, 5, 0]], dtype=np.complex128)[None]
    ta = torch.from_numpy(a).cuda()
    x = torch.empty_like(ta)
    lib = _lib.load()
    ctx = _lib.context(0)
    _lib.check(lib.qtx_inv(ctx, 3, 1, ta.data_ptr(), 9, x.data_ptr(), 9, 0), ctx, "inv")
    assert _rel(x, np.linalg.inv(a)) < 1e-14


@pytest.mark.parametrize("n", [64, 200, 256])
def test_inverse_pivoting_large_blocks(n):
    """Row-permuted, well-conditioned blocks with a zero diagonal: every
    column needs a row interchange, across panels (the 129-256 kernel keeps
    the next panel's elimination under the current panel's update)."""
    rng = np.random.default_rng(n + 1)
    batch = 6
    base = rng.standard_normal((batch, n, n)) + 1j * rng.standard_normal((batch, n, n))
    base += 2 * np.sqrt(n) * np.eye(n)
    perm = np.roll(np.arange(n), n // 3 + 1)
    a = np.ascontiguousarray(base[:, perm, :])
    assert np.all(np.abs(np.diagonal(a, axis1=1, axis2=2)) < 2 * np.sqrt(n) - 1e-9)
    ta = torch.from_numpy(a).cuda()
    x = torch.empty_like(ta)
    lib = _lib.load()
    ctx = _lib.context(0)
    _lib.check(lib.qtx_inv(ctx, n, batch, ta.data_ptr(), n * n, x.data_ptr(), n * n, 0), ctx, "inv")
    assert _rel(x, np.linalg.inv(a)) < 1e-12


@pytest.mark.parametrize("n", [4, 200])
def test_inverse_singular_block_flags_its_energy(n):
    """A block with a zero column in the middle of a batch returns
    QTX_E_SINGULAR; the other blocks are still inverted correctly."""
    rng = np.random.default_rng(7)
    a = rng.standard_normal((3, n, n)) + 1j * rng.standard_normal((3, n, n)) + np.sqrt(n) * np.eye(n)
    a[1, :, n // 2] = 0
    ta = torch.from_numpy(a).cuda()
    x = torch.empty_like(ta)
    lib = _lib.load()
    ctx = _lib.context(0)
    st = lib.qtx_inv(ctx, n, 3, ta.data_ptr(), n * n, x.data_ptr(), n * n, 0)
    assert st == _lib.QTX_E_SINGULAR
    torch.cuda.synchronize()
    xc = x.cpu().numpy()
    for e in (0, 2):
        assert _rel(xc[e], np.linalg.inv(a[e])) < 1e-10


def test_inverse_singular_block_raises():
    a = np.zeros((2, 4, 4), dtype=np.complex128)
    a[0] = np.eye(4)
    ta = torch.from_numpy(a).cuda()
    x = torch.empty_like(ta)
    lib = _lib.load()
    ctx = _lib.context(0)
    st = lib.qtx_inv(ctx, 4, 2, ta.data_ptr(), 16, x.data_ptr(), 16, 0)
    assert st == _lib.QTX_E_SINGULAR
    with pytest.raises(np.linalg.LinAlgError):
        _lib.check(st, ctx, "inv")
    # the context stays usable
    st = lib.qtx_inv(ctx, 4, 1, ta.data_ptr(), 16, x.data_ptr(), 16, 0)
    assert st == _lib.QTX_OK


def test_sancho_rubio_matches_oracle():
    dev = make_device(num_blocks=3, block_size=24, num_energies=9, seed=11)
    d, u, lo = dev.system_blocks()
    x_ref, it_ref = orc.sancho_rubio(d[0], u[0], lo[0], 200, 1e-12)
    sr = SanchoRubio(max_iterations=200, convergence_tol=1e-12)
    x = sr(d[0], u[0], lo[0], "left")
    assert _rel(x, x_ref) < 1e-10
    assert sr.last_iterations.max() == it_ref
    # fixed point of the upstream test criterion
    assert _rel(x, np.linalg.inv(d[0] - lo[0] @ x @ u[0])) < 1e-6
    # broadcast couplings (2-D a_ij / a_ji)
    x2 = sr(d[0], u[0][0], lo[0][0], "left")
    assert _rel(x2, x_ref) < 1e-10


def test_sancho_rubio_not_converged_warns():
    dev = make_device(num_blocks=2, block_size=8, num_energies=3, seed=3)
    d, u, lo = dev.system_blocks()
    with pytest.warns(RuntimeWarning):
        SanchoRubio(max_iterations=1, convergence_tol=1e-12)(d[0], u[0], lo[0], "left")


def test_sancho_rubio_singular_decimation_block():
    """An exactly singular decimation block is reported (QTX_E_SINGULAR ->
    LinAlgError), not passed on as silent NaN; the context stays usable."""
    n, ne = 8, 2
    a_ii = torch.zeros(ne, n, n, dtype=torch.complex128, device="cuda")
    a_ij = torch.eye(n, dtype=torch.complex128, device="cuda").repeat(ne, 1, 1)
    x = torch.empty_like(a_ii)
    lib = _lib.load()
    ctx = _lib.context(0)
    st = lib.qtx_sancho_rubio(ctx, n, ne, a_ii.data_ptr(), n * n, a_ij.data_ptr(), n * n, a_ij.data_ptr(), n * n,
                              1e-12, 3, x.data_ptr(), None, 0)
    assert st == _lib.QTX_E_SINGULAR
    with pytest.raises(np.linalg.LinAlgError):
        SanchoRubio(max_iterations=3, convergence_tol=1e-12)(a_ii, a_ij, a_ij, "left")
    dev = make_device(num_blocks=2, block_size=8, num_energies=2, seed=3)
    d, u, lo = dev.system_blocks()
    x_ok = SanchoRubio(max_iterations=200, convergence_tol=1e-12)(d[0], u[0], lo[0], "left")
    x_ref, _ = orc.sancho_rubio(d[0], u[0], lo[0], 200, 1e-12)
    assert _rel(x_ok, x_ref) < 1e-10


def test_contact_self_energies_match_oracle():
    dev = make_device(num_blocks=3, block_size=16, num_energies=5, seed=2)
    d, u, lo = dev.system_blocks()
    ref = orc.obc_self_energies(d, u, lo, dev.energies, dev.mu_left, dev.mu_right, dev.kt)
    f = orc.fermi_dirac(dev.energies - dev.mu_left, dev.kt)
    sr, sl, sg = contact_self_energies(ref["surface"][0], lo[0], u[0], f)
    assert _rel(sr, ref["retarded"][0]) < 1e-12
    assert _rel(sl, ref["lesser"][0]) < 1e-12
    assert _rel(sg, ref["greater"][0]) < 1e-12


@pytest.mark.parametrize("sizes", [[3, 5, 4, 6], [8] * 12, [1, 2, 1, 3, 2]])
def test_block_sort_index_device_matches_host(sizes):
    """DSDBCOO construction on the device: the same stable block-sorting
    permutation as the host rule (and upstream's compute_block_sort_index),
    per-block counts, and an index outside the matrix refused."""
    from quatrex_b200.datastructures import block_sort_index, block_sort_index_device

    rng = np.random.default_rng(len(sizes))
    n = int(np.sum(sizes))
    # random pattern with entries in every block pair (not only the band), shuffled order
    m = (rng.random((n, n)) < 0.3).astype(np.complex128)
    r, c = np.nonzero(m)
    perm = rng.permutation(len(r))
    r, c = r[perm], c[perm]
    got, counts = block_sort_index_device(r, c, sizes)
    want = block_sort_index(r, c, sizes)
    assert np.array_equal(got.cpu().numpy(), want)
    offs = np.concatenate(([0], np.cumsum(sizes)))
    br = np.searchsorted(offs, r, side="right") - 1
    bc = np.searchsorted(offs, c, side="right") - 1
    ref = np.zeros((len(sizes), len(sizes)), dtype=np.int64)
    np.add.at(ref, (br, bc), 1)
    assert np.array_equal(counts, ref)
    with pytest.raises(ValueError):
        block_sort_index_device(np.array([0, n]), np.array([0, 0]), sizes)


@pytest.mark.parametrize("with_overlap", [False, True])
def test_assemble_system_matches_formula(with_overlap):
    """A(E) = (E + i eta) S - diag(V) - Sigma(E) - H on the data rows."""
    from scipy import sparse

    from quatrex_b200.datastructures import DSDBCOO, assemble_system

    rng = np.random.default_rng(3)
    sizes = np.array([3, 4, 3])
    n = int(sizes.sum())
    band = np.abs(np.subtract.outer(np.arange(n), np.arange(n))) <= 3
    hm = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) * band
    hm = hm + hm.conj().T + np.eye(n)
    H = DSDBCOO.from_sparray(sparse.coo_matrix(hm), sizes, (1,))
    S = None
    sm = np.eye(n)
    if with_overlap:
        sm = np.eye(n) + 0.1 * band * rng.standard_normal((n, n))
        S = DSDBCOO(np.asarray(sm[H.rows, H.cols], dtype=np.complex128)[None], H.rows, H.cols, sizes, (1,))
    e = np.array([-0.5, 0.1, 0.7])
    v = rng.standard_normal(n)
    sig = (rng.standard_normal((3, H.rows.size)) + 1j * rng.standard_normal((3, H.rows.size)))
    SG = DSDBCOO(sig, H.rows, H.cols, sizes, (3,))
    A = assemble_system(e, 1e-3, H, overlap=S, potential=v, sigma=SG)
    got = A.data.cpu().numpy()
    for k in range(3):
        full = (e[k] + 1e-3j) * sm - np.diag(v) - hm
        want = full[H.rows, H.cols] - sig[k]
        assert np.allclose(got[k], want, rtol=0, atol=1e-13)


@pytest.mark.skipif(not torch.cuda.is_available() or torch.cuda.device_count() < 2,
                    reason="needs two visible CUDA devices")
def test_two_devices_in_one_process():
    """The large shared-memory opt-in of the GEMM and inverse kernels is a
    per-device attribute: a solve on a second device after the first has used
    the library must still launch (and agree with the oracle)."""
    dev = make_device(num_blocks=3, block_size=64, num_energies=4, seed=7)
    d, u, lo = dev.system_blocks()
    x_ref, _ = orc.sancho_rubio(d[0], u[0], lo[0], 200, 1e-12)
    for k in (0, 1):
        with torch.cuda.device(k):
            x = SanchoRubio(max_iterations=200, convergence_tol=1e-12)(d[0], u[0], lo[0], "left")
            assert _rel(x, x_ref) < 1e-10
