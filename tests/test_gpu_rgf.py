"""Parity of the drop-in RGF solver (CUDA path through the C ABI) with the
oracle and the upstream fixtures.

Bar: relative Frobenius error <= 1e-10 per returned block against the oracle
(complex128), and the upstream unit-test criterion (dense inverse / congruence
with numpy.allclose defaults) on the upstream-style sparse BTD matrices for
every combination the upstream conftest parametrises: constant and mixed block
sizes, batching 1 / 2 / 100, out on/off, return_retarded on/off, stack shapes
(10,), (7, 2), (9, 2, 4).
"""

import os

import numpy as np
import pytest
import torch
from scipy import sparse

from oracle import rgf_oracle as orc
from quatrex_b200.datastructures import DSDBCOO, DSDBCSR
from quatrex_b200.greens_function_solver import RGF, OBCBlocks
from quatrex_b200.workloads import make_device

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-10


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _bt_dense(rng, block_sizes):
    """Seeded upstream-style random BTD matrix (50 % dense blocks, diagonally dominant)."""
    offs = np.hstack(([0], np.cumsum(block_sizes)))
    n = offs[-1]
    arr = np.zeros((n, n), dtype=np.complex128)

    def blk(m, k):
        mask = rng.random((m, k)) < 0.5
        return mask * (rng.random((m, k)) + 1j * rng.random((m, k)))

    for i in range(len(block_sizes)):
        arr[offs[i]:offs[i + 1], offs[i]:offs[i + 1]] = blk(block_sizes[i], block_sizes[i]) + np.eye(block_sizes[i])
        if i > 0:
            arr[offs[i]:offs[i + 1], offs[i - 1]:offs[i]] = blk(block_sizes[i], block_sizes[i - 1])
            arr[offs[i - 1]:offs[i], offs[i]:offs[i + 1]] = blk(block_sizes[i - 1], block_sizes[i])
    for i in range(n):
        arr[i, i] = (1 + 1j) + complex(np.sum(arr[i, :]))
    return arr


BLOCK_SIZES = [np.array([2] * 10), np.array([2] * 3 + [4] * 2 + [2] * 3)]
STACKS = [(10,), (7, 2), (9, 2, 4)]
# both storage layouts, as the upstream solver tests parametrise them
# (tests/qttools/greens_function_solver/conftest.py:12)
DSDB_TYPES = [DSDBCOO, DSDBCSR]


@pytest.mark.parametrize("block_sizes", BLOCK_SIZES, ids=["constant", "mixed"])
@pytest.mark.parametrize("max_batch_size", [1, 2, 100])
@pytest.mark.parametrize("use_out", [True, False])
@pytest.mark.parametrize("stack", STACKS, ids=["1D", "2D", "3D"])
@pytest.mark.parametrize("on_device", [True, False])
@pytest.mark.parametrize("dsdb_type", DSDB_TYPES, ids=["DSDBCOO", "DSDBCSR"])
def test_selected_inv_upstream_criterion(block_sizes, max_batch_size, use_out, stack, on_device, dsdb_type):
    rng = np.random.default_rng(len(block_sizes) * 7 + max_batch_size)
    bt = _bt_dense(rng, block_sizes)
    mask = bt.astype(bool)
    ref = np.linalg.inv(bt) * mask
    a = dsdb_type.from_sparray(sparse.coo_matrix(bt), block_sizes, stack, device="cuda" if on_device else None)
    assert type(a) is dsdb_type
    solver = RGF(max_batch_size=max_batch_size)
    if use_out:
        x = dsdb_type.zeros_like(a)
        assert solver.selected_inv(a, out=x) is None
    else:
        x = solver.selected_inv(a)
    got = x.to_dense() * mask
    assert np.allclose(np.broadcast_to(ref, stack + ref.shape), got)
    assert _rel(got, np.broadcast_to(ref, got.shape)) < 1e-12


@pytest.mark.parametrize("block_sizes", BLOCK_SIZES, ids=["constant", "mixed"])
@pytest.mark.parametrize("max_batch_size", [1, 2, 100])
@pytest.mark.parametrize("use_out", [True, False])
@pytest.mark.parametrize("return_retarded", [True, False])
@pytest.mark.parametrize("stack", STACKS, ids=["1D", "2D", "3D"])
@pytest.mark.parametrize("dsdb_type", DSDB_TYPES, ids=["DSDBCOO", "DSDBCSR"])
def test_selected_solve_upstream_criterion(block_sizes, max_batch_size, use_out, return_retarded, stack, dsdb_type):
    rng = np.random.default_rng(len(block_sizes) * 11 + max_batch_size)
    bt = _bt_dense(rng, block_sizes)
    bl = bt - bt.conj().T
    bg = bt - bt.conj().T
    ref_r = np.linalg.inv(bt)
    ref_l = ref_r @ bl @ ref_r.conj().T
    ref_g = ref_r @ bg @ ref_r.conj().T
    A = dsdb_type.from_sparray(sparse.coo_matrix(bt), block_sizes, stack, device="cuda")
    BL = dsdb_type.from_sparray(sparse.coo_matrix(bl), block_sizes, stack, device="cuda")
    BG = dsdb_type.from_sparray(sparse.coo_matrix(bg), block_sizes, stack, device="cuda")
    solver = RGF(max_batch_size=max_batch_size)
    if use_out:
        XR, XL, XG = (dsdb_type.zeros_like(A) for _ in range(3))
        assert solver.selected_solve(A, BL, BG, out=[XL, XG, XR], return_retarded=return_retarded) is None
    elif return_retarded:
        XL, XG, XR = solver.selected_solve(A, BL, BG, return_retarded=True)
    else:
        XL, XG = solver.selected_solve(A, BL, BG)
    if return_retarded:
        m = XR.to_dense().astype(bool)
        assert np.allclose(np.broadcast_to(ref_r, stack + ref_r.shape) * m, XR.to_dense() * m)
    for X, ref in ((XL, ref_l), (XG, ref_g)):
        m = X.to_dense().astype(bool)
        assert np.allclose(np.broadcast_to(ref, stack + ref.shape) * m, X.to_dense() * m)


def test_selected_solve_wrong_out_length_raises():
    bt = _bt_dense(np.random.default_rng(0), BLOCK_SIZES[0])
    A = DSDBCOO.from_sparray(sparse.coo_matrix(bt), BLOCK_SIZES[0], (2,), device="cuda")
    with pytest.raises(ValueError):
        RGF().selected_solve(A, A, A, out=[DSDBCOO.zeros_like(A), DSDBCOO.zeros_like(A)], return_retarded=True)


@pytest.mark.parametrize("case", ["constant", "mixed"])
def test_against_upstream_fixture(case):
    g = np.load(os.path.join(GOLDEN, f"btd_{case}.npz"))
    sizes = g["block_sizes"]
    stack = int(g["stack"])
    mask = g["a"] != 0
    A = DSDBCOO.from_sparray(sparse.coo_matrix(g["a"]), sizes, (stack,), device="cuda")
    BL = DSDBCOO.from_sparray(sparse.coo_matrix(g["sigma_lesser"]), sizes, (stack,), device="cuda")
    BG = DSDBCOO.from_sparray(sparse.coo_matrix(g["sigma_greater"]), sizes, (stack,), device="cuda")
    solver = RGF(max_batch_size=2)
    x = solver.selected_inv(A).to_dense()[3] * mask
    assert _rel(x, g["inv"] * mask) < 1e-12
    xl, xg, xr = solver.selected_solve(A, BL, BG, return_retarded=True)
    for key, got in (("xl", xl), ("xg", xg)):
        m = g[key] != 0
        assert _rel(got.to_dense()[0] * m, g[key] * m) < 1e-12
    m = g["xr"] != 0
    assert _rel(xr.to_dense()[0] * m, g["xr"] * m) < 1e-12


def _transport_inputs(dev, energies=None, device="cuda"):
    e = dev.energies if energies is None else energies
    d, u, lo = dev.system_blocks(e)
    obc = orc.obc_self_energies(d, u, lo, e, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol, dev.sr_max_iter)
    nb = len(d)
    A = DSDBCOO.from_blocks(d, u, lo, device=device)
    z = DSDBCOO.from_blocks([np.zeros_like(x) for x in d], [np.zeros_like(x) for x in u],
                            [np.zeros_like(x) for x in lo], device=device)
    ob = OBCBlocks(nb)
    ob.retarded[0], ob.retarded[-1] = obc["retarded"]
    ob.lesser[0], ob.lesser[-1] = obc["lesser"]
    ob.greater[0], ob.greater[-1] = obc["greater"]
    return d, u, lo, obc, A, z, ob


def _blocks(m, nb):
    return ([m.blocks[i, i] for i in range(nb)], [m.blocks[i, i + 1] for i in range(nb - 1)],
            [m.blocks[i + 1, i] for i in range(nb - 1)])


def test_transport_small_against_upstream_fixture():
    g = np.load(os.path.join(GOLDEN, "transport_small.npz"))
    dev = make_device(num_blocks=4, block_size=8, num_energies=6, seed=7)
    d, u, lo, obc, A, Z, ob = _transport_inputs(dev)
    xl, xg, xr, cur = RGF().selected_solve(A, Z, Z, obc_blocks=ob, return_retarded=True, return_current=True)
    nb = 4
    for key, X in (("xl", xl), ("xg", xg)):
        dd, uu, ll = _blocks(X, nb)
        assert _rel(np.stack(dd, 1), g[f"{key}_diag"]) < TOL
        assert _rel(np.stack(uu, 1), g[f"{key}_upper"]) < TOL
        assert _rel(np.stack(ll, 1), g[f"{key}_lower"]) < TOL
    assert _rel(np.stack(_blocks(xr, nb)[0], 1), g["xr_diag"]) < TOL
    cur = cur.cpu().numpy()
    # the last interface is where upstream reads the right coupling
    assert _rel(cur[:, -1], g["current"][:, -1]) < 1e-9
    x = RGF().selected_inv(A, obc_blocks=ob)
    dd, uu, ll = _blocks(x, nb)
    assert _rel(np.stack(dd, 1), g["inv_diag"]) < TOL
    assert _rel(np.stack(uu, 1), g["inv_upper"]) < TOL
    assert _rel(np.stack(ll, 1), g["inv_lower"]) < TOL


@pytest.mark.parametrize("max_batch_size", [1, 3, 100])
def test_transport_per_block_against_oracle(max_batch_size):
    dev = make_device(num_blocks=6, block_size=24, num_energies=7, seed=21)
    d, u, lo, obc, A, Z, ob = _transport_inputs(dev)
    nb = 6
    pad = [None] * (nb - 2)
    ref = orc.selected_solve(d, u, lo, [np.zeros_like(x) for x in d], [np.zeros_like(x) for x in u],
                             [np.zeros_like(x) for x in d], [np.zeros_like(x) for x in u],
                             [obc["retarded"][0], *pad, obc["retarded"][1]], [obc["lesser"][0], *pad, obc["lesser"][1]],
                             [obc["greater"][0], *pad, obc["greater"][1]], return_current=True)
    xl, xg, xr, cur = RGF(max_batch_size=max_batch_size).selected_solve(
        A, Z, Z, obc_blocks=ob, return_retarded=True, return_current=True)
    for key, X in (("xl", xl), ("xg", xg)):
        dd, uu, ll = _blocks(X, nb)
        for i in range(nb):
            assert _rel(dd[i], ref[f"{key}_diag"][i]) < TOL, (key, i)
        for i in range(nb - 1):
            assert _rel(uu[i], ref[f"{key}_upper"][i]) < TOL
            assert _rel(ll[i], ref[f"{key}_lower"][i]) < TOL
    for i in range(nb):
        assert _rel(xr.blocks[i, i], ref["xr_diag"][i]) < TOL
    assert _rel(cur.cpu().numpy(), ref["current"]) < 1e-9


def test_host_numpy_inputs_roundtrip():
    """NumPy (host) matrices: copied to the device and the outputs written back."""
    dev = make_device(num_blocks=4, block_size=16, num_energies=3, seed=4)
    d, u, lo, obc, A, Z, ob = _transport_inputs(dev, device=None)
    assert isinstance(A.data, np.ndarray)
    xl, xg = RGF().selected_solve(A, Z, Z, obc_blocks=ob)
    assert isinstance(xl.data, np.ndarray)
    pad = [None] * 2
    ref = orc.selected_solve(d, u, lo, [np.zeros_like(x) for x in d], [np.zeros_like(x) for x in u],
                             [np.zeros_like(x) for x in d], [np.zeros_like(x) for x in u],
                             [obc["retarded"][0], *pad, obc["retarded"][1]], [obc["lesser"][0], *pad, obc["lesser"][1]],
                             [obc["greater"][0], *pad, obc["greater"][1]])
    assert _rel(xl.blocks[2, 2], ref["xl_diag"][2]) < TOL


def test_single_block_device():
    """nb = 1: no sweep, x_0 = inv(A_00 - Sigma_0)."""
    rng = np.random.default_rng(9)
    a = rng.standard_normal((5, 5)) + 1j * rng.standard_normal((5, 5)) + 5 * np.eye(5)
    A = DSDBCOO.from_sparray(sparse.coo_matrix(a), np.array([5]), (2,), device="cuda")
    x = RGF().selected_inv(A)
    assert _rel(x.to_dense()[0], np.linalg.inv(a)) < 1e-12
    sl = a - a.conj().T
    SL = DSDBCOO.from_sparray(sparse.coo_matrix(sl), np.array([5]), (2,), device="cuda")
    xl, xg = RGF().selected_solve(A, SL, SL)
    ref = np.linalg.inv(a) @ sl @ np.linalg.inv(a).conj().T
    assert _rel(xl.to_dense()[1], 0.5 * (ref - ref.conj().T)) < 1e-12


@pytest.mark.parametrize("max_batch_size", [2, 100])
def test_host_buffer_streaming_equals_device_path(max_batch_size):
    """NumPy operands go through QTX_FLAG_HOST_BUFFERS (streamed in energy
    batches through two device staging sets); the results equal the
    device-resident call bit for bit, entries the solver does not write keep
    their values, and the layer current comes back as a host array."""
    dev = make_device(num_blocks=5, block_size=12, num_energies=7, seed=31)
    _, _, _, _, Ah, Zh, ob = _transport_inputs(dev, device=None)
    _, _, _, _, Ad, Zd, _ = _transport_inputs(dev, device="cuda")
    assert isinstance(Ah.data, np.ndarray)
    solver = RGF(max_batch_size=max_batch_size)
    # host: out= with a pre-filled retarded output (its off-diagonal blocks are not written)
    xl_h, xg_h, xr_h = (DSDBCOO.zeros_like(Ah) for _ in range(3))
    xr_h.data[...] = 7.0 + 3.0j
    cur_h = solver.selected_solve(Ah, Zh, Zh, obc_blocks=ob, out=[xl_h, xg_h, xr_h], return_retarded=True,
                                  return_current=True)
    assert isinstance(cur_h, np.ndarray)
    xl_d, xg_d, xr_d = (DSDBCOO.zeros_like(Ad) for _ in range(3))
    xr_d.data[...] = 7.0 + 3.0j
    cur_d = solver.selected_solve(Ad, Zd, Zd, obc_blocks=ob, out=[xl_d, xg_d, xr_d], return_retarded=True,
                                  return_current=True)
    for h, d in ((xl_h, xl_d), (xg_h, xg_d), (xr_h, xr_d)):
        assert np.array_equal(h.data, d.data.cpu().numpy())
    assert np.array_equal(cur_h, cur_d.cpu().numpy())
    assert np.all(xr_h.blocks[0, 1] == 7.0 + 3.0j)
    # selected inversion
    x_h = solver.selected_inv(Ah, obc_blocks=ob)
    x_d = solver.selected_inv(Ad, obc_blocks=ob)
    assert isinstance(x_h.data, np.ndarray)
    assert np.array_equal(x_h.data, x_d.data.cpu().numpy())


def test_coulomb_screening_call_pattern():
    """The second upstream caller of the same solver, CoulombScreeningSolver.solve
    (src/quatrex/coulomb_screening/solver.py:466-489): out=(W^<, W^>) of length
    two with return_retarded=False, sources L^< and L^> on every block of the
    pattern, mixed block sizes, and contact blocks (retarded, lesser, greater,
    different per energy) at both ends.  Reference: the dense
    W^R = (A - OBC^R)^-1 and W^≶ = W^R (L^≶ + OBC^≶) W^R^H per energy."""
    rng = np.random.default_rng(77)
    sizes = np.array([3, 5, 4, 4, 2])
    ne = 6
    offs = np.hstack(([0], np.cumsum(sizes)))
    bt = _bt_dense(rng, sizes)
    s = _bt_dense(rng, sizes)
    srcs = {"lesser": s - s.conj().T, "greater": 2.0 * (s.conj().T - s)}
    A = DSDBCOO.from_sparray(sparse.coo_matrix(bt), sizes, (ne,), device="cuda")
    L = {k: DSDBCOO.from_sparray(sparse.coo_matrix(v), sizes, (ne,), device="cuda") for k, v in srcs.items()}
    ob = OBCBlocks(len(sizes))

    def rnd(b):
        return 0.3 * (rng.standard_normal((ne, b, b)) + 1j * rng.standard_normal((ne, b, b)))

    r0, rn = rnd(sizes[0]), rnd(sizes[-1])
    ob.retarded[0], ob.retarded[-1] = r0, rn
    obc_src = {}
    for k in ("lesser", "greater"):
        a0, an = rnd(sizes[0]), rnd(sizes[-1])
        obc_src[k] = (a0 - a0.conj().swapaxes(-1, -2), an - an.conj().swapaxes(-1, -2))
    ob.lesser[0], ob.lesser[-1] = obc_src["lesser"]
    ob.greater[0], ob.greater[-1] = obc_src["greater"]
    out = (DSDBCOO.zeros_like(A), DSDBCOO.zeros_like(A))
    assert RGF(max_batch_size=4).selected_solve(A, L["lesser"], L["greater"], obc_blocks=ob, out=out,
                                                return_retarded=False) is None
    first, last = slice(offs[0], offs[1]), slice(offs[-2], offs[-1])
    mask = np.broadcast_to(bt != 0, (ne,) + bt.shape)
    for (k, src), x in zip(srcs.items(), out):
        ref = np.empty((ne,) + bt.shape, dtype=np.complex128)
        for e in range(ne):
            a = bt.copy()
            a[first, first] -= r0[e]
            a[last, last] -= rn[e]
            sig = src.copy()
            sig[first, first] += obc_src[k][0][e]
            sig[last, last] += obc_src[k][1][e]
            wr = np.linalg.inv(a)
            ref[e] = wr @ sig @ wr.conj().T
        got = x.to_dense()
        got = got.cpu().numpy() if isinstance(got, torch.Tensor) else got
        assert _rel(got[mask], ref[mask]) < TOL, k
        assert np.allclose(got[mask], ref[mask])


@pytest.mark.parametrize("return_current", [False, True])
def test_partially_zero_self_energies(return_current):
    """Interior Sigma^< / Sigma^> that vanish on some blocks only: the solver
    skips every product with a zero block (and shares W = x_j A_ji between the
    two components where block j injects nothing); every returned block still
    meets 1e-10 against the oracle's full component recursion."""
    dev = make_device(num_blocks=7, block_size=16, num_energies=5, seed=44)
    d, u, lo, obc, A, Z, ob = _transport_inputs(dev)
    nb = 7
    rng = np.random.default_rng(3)

    def skew(shape):
        x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        return x - x.conj().swapaxes(-1, -2)

    # Sigma^<: diagonal blocks 1 and 4, upper block (2, 3); Sigma^>: diagonal 2 only
    sl_d = [np.zeros_like(x) for x in d]
    sl_u = [np.zeros_like(x) for x in u]
    sg_d = [np.zeros_like(x) for x in d]
    sg_u = [np.zeros_like(x) for x in u]
    sl_d[1] = 0.1 * skew(d[1].shape)
    sl_d[4] = 0.1 * skew(d[4].shape)
    sl_u[2] = 0.05 * (rng.standard_normal(u[2].shape) + 1j * rng.standard_normal(u[2].shape))
    sg_d[2] = 0.1 * skew(d[2].shape)
    sl_lo = [-x.conj().swapaxes(-1, -2) for x in sl_u]
    sg_lo = [-x.conj().swapaxes(-1, -2) for x in sg_u]
    SL = DSDBCOO.from_blocks(sl_d, sl_u, sl_lo, device="cuda")
    SG = DSDBCOO.from_blocks(sg_d, sg_u, sg_lo, device="cuda")
    pad = [None] * (nb - 2)
    ref = orc.selected_solve(d, u, lo, sl_d, sl_u, sg_d, sg_u, [obc["retarded"][0], *pad, obc["retarded"][1]],
                             [obc["lesser"][0], *pad, obc["lesser"][1]], [obc["greater"][0], *pad, obc["greater"][1]],
                             return_current=return_current)
    res = RGF(max_batch_size=3).selected_solve(A, SL, SG, obc_blocks=ob, return_retarded=True,
                                               return_current=return_current)
    xl, xg, xr = res[:3]
    for key, X in (("xl", xl), ("xg", xg)):
        dd, uu, ll = _blocks(X, nb)
        for i in range(nb):
            assert _rel(dd[i], ref[f"{key}_diag"][i]) < TOL, (key, i)
        for i in range(nb - 1):
            assert _rel(uu[i], ref[f"{key}_upper"][i]) < TOL, (key, i)
            assert _rel(ll[i], ref[f"{key}_lower"][i]) < TOL, (key, i)
    for i in range(nb):
        assert _rel(xr.blocks[i, i], ref["xr_diag"][i]) < TOL
    if return_current:
        assert _rel(res[3].cpu().numpy(), ref["current"]) < 1e-9


@pytest.mark.parametrize("dsdb_type", DSDB_TYPES, ids=["DSDBCOO", "DSDBCSR"])
def test_symmetric_storage_against_upstream_fixture(dsdb_type):
    """Symmetric storage as quatrex's SCBA uses it (upper block triangle and
    upper triangle of each diagonal block): a complex-symmetric system matrix
    (symmetry_op = identity), skew-Hermitian self-energies and outputs
    (symmetry_op = -conj), G^R diagonal stored complex-symmetric.  Against
    upstream RGF.selected_solve on the same symmetric-storage operands
    (tests/golden/dsdb_layouts.npz), on the stored entries and the completed
    dense matrices."""
    g = np.load(os.path.join(GOLDEN, "dsdb_layouts.npz"))
    sizes = g["block_sizes"]
    ident = lambda x: x  # noqa: E731
    neg_conj = lambda x: -x.conj()  # noqa: E731
    stack = (3,)
    A = dsdb_type.from_sparray(sparse.coo_matrix(g["sym_a"]), sizes, stack, symmetry=True, symmetry_op=ident,
                               device="cuda")
    SL = dsdb_type.from_sparray(sparse.coo_matrix(g["sym_sigma_lesser"]), sizes, stack, symmetry=True,
                                symmetry_op=neg_conj, device="cuda")
    SG = dsdb_type.from_sparray(sparse.coo_matrix(g["sym_sigma_greater"]), sizes, stack, symmetry=True,
                                symmetry_op=neg_conj, device="cuda")
    XL, XG = dsdb_type.zeros_like(SL), dsdb_type.zeros_like(SL)
    XR = dsdb_type.zeros_like(A)
    assert RGF(max_batch_size=2).selected_solve(A, SL, SG, out=[XL, XG, XR], return_retarded=True) is None
    assert _rel(XL.numpy_data()[1], g["sym_xl_data"]) < 1e-12
    assert _rel(XR.numpy_data()[1], g["sym_xr_data"]) < 1e-12
    for X, key in ((XL, "sym_xl"), (XG, "sym_xg"), (XR, "sym_xr")):
        m = g[key] != 0
        assert _rel(X.to_dense()[2] * m, g[key] * m) < 1e-12, key
    # and against the dense definition on full storage
    a = g["sym_a"]
    ref_r = np.linalg.inv(a)
    ref_l = ref_r @ g["sym_sigma_lesser"] @ ref_r.conj().T
    m = XL.to_dense()[0] != 0
    assert np.allclose(XL.to_dense()[0] * m, ref_l * m)


class _UpstreamDSDBCOOStandIn:
    """An object carrying only the attributes an upstream qttools DSDBCOO
    exposes to a solver: data, rows, cols, block_sizes, num_blocks,
    symmetry, symmetry_op (no method of this package's classes)."""

    def __init__(self, data, rows, cols, block_sizes):
        self.data = data
        self.rows = rows
        self.cols = cols
        self.block_sizes = block_sizes
        self.num_blocks = len(block_sizes)
        self.symmetry = False
        self.symmetry_op = np.conj


def test_upstream_attribute_stand_in():
    """The boundary reads only the upstream layout attributes: a stand-in
    with rows / cols / block_sizes / data (NumPy data, as the upstream NumPy
    backend holds it) is solved and written in place."""
    g = np.load(os.path.join(GOLDEN, "dsdb_layouts.npz"))
    sizes = g["block_sizes"]
    a = g["a"]
    stack = 4
    data = np.broadcast_to(g["coo_full_data"], (stack, len(g["coo_full_data"]))).copy()
    A = _UpstreamDSDBCOOStandIn(data, g["coo_full_rows"], g["coo_full_cols"], sizes)
    out = _UpstreamDSDBCOOStandIn(np.zeros_like(data), g["coo_full_rows"], g["coo_full_cols"], sizes)
    assert RGF(max_batch_size=3).selected_inv(A, out=out) is None
    ref = np.linalg.inv(a)[g["coo_full_rows"], g["coo_full_cols"]]
    assert _rel(out.data[2], ref) < 1e-12
