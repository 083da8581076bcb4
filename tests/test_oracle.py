"""The CPU oracle against the fixtures produced by the upstream implementation."""

import os

import numpy as np
import pytest

from oracle import rgf_oracle as orc
from quatrex_b200.workloads import make_device

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _blocks_from_dense(dense, sizes, stack):
    offs = np.hstack(([0], np.cumsum(sizes)))
    nb = len(sizes)
    d = [np.broadcast_to(dense[offs[i]:offs[i + 1], offs[i]:offs[i + 1]], (stack, sizes[i], sizes[i])).copy() for i in range(nb)]
    u = [np.broadcast_to(dense[offs[i]:offs[i + 1], offs[i + 1]:offs[i + 2]], (stack, sizes[i], sizes[i + 1])).copy() for i in range(nb - 1)]
    lo = [np.broadcast_to(dense[offs[i + 1]:offs[i + 2], offs[i]:offs[i + 1]], (stack, sizes[i + 1], sizes[i])).copy() for i in range(nb - 1)]
    return d, u, lo


@pytest.mark.parametrize("case", ["constant", "mixed"])
def test_oracle_btd_against_upstream(case):
    g = np.load(os.path.join(GOLDEN, f"btd_{case}.npz"))
    sizes = g["block_sizes"]
    stack = int(g["stack"])
    offs = np.hstack(([0], np.cumsum(sizes)))
    mask = g["a"] != 0
    d, u, lo = _blocks_from_dense(g["a"], sizes, stack)
    sld, slu, _ = _blocks_from_dense(g["sigma_lesser"], sizes, stack)
    sgd, sgu, _ = _blocks_from_dense(g["sigma_greater"], sizes, stack)
    xd, xu, xl_ = orc.selected_inv(d, u, lo, max_batch_size=3)
    dense = orc.dense_from_blocks(xd, xu, xl_)[0] * mask
    assert _rel(dense, g["inv"] * mask) < 1e-12
    res = orc.selected_solve(d, u, lo, sld, slu, sgd, sgu, max_batch_size=3)
    for key in ("xl", "xg"):
        got = orc.dense_from_blocks(res[f"{key}_diag"], res[f"{key}_upper"], res[f"{key}_lower"])[0] * mask
        assert _rel(got, g[key] * mask) < 1e-12
    ref_r = g["xr"]
    for i in range(len(sizes)):
        blk = ref_r[offs[i]:offs[i + 1], offs[i]:offs[i + 1]]
        m = mask[offs[i]:offs[i + 1], offs[i]:offs[i + 1]]
        assert _rel(res["xr_diag"][i][0] * m, blk * m) < 1e-12
    # the reference test criterion: dense inverse / congruence
    a_inv = np.linalg.inv(g["a"])
    assert np.allclose(dense, a_inv * mask)


def test_oracle_transport_small_against_upstream():
    g = np.load(os.path.join(GOLDEN, "transport_small.npz"))
    dev = make_device(num_blocks=4, block_size=8, num_energies=6, seed=7)
    assert np.array_equal(dev.h_diag, g["h_diag"]) and np.array_equal(dev.h_upper, g["h_upper"])
    d, u, lo = dev.system_blocks()
    obc = orc.obc_self_energies(d, u, lo, dev.energies, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol, dev.sr_max_iter)
    assert _rel(obc["surface"][0], g["g_surface_left"]) < 1e-12
    assert _rel(obc["surface"][1], g["g_surface_right"]) < 1e-12
    for side, k in (("left", 0), ("right", 1)):
        assert _rel(obc["retarded"][k], g[f"sigma_r_{side}"]) < 1e-12
        assert _rel(obc["lesser"][k], g[f"sigma_l_{side}"]) < 1e-12
        assert _rel(obc["greater"][k], g[f"sigma_g_{side}"]) < 1e-12
    nb = 4
    obc_r = [obc["retarded"][0], None, None, obc["retarded"][1]]
    obc_l = [obc["lesser"][0], None, None, obc["lesser"][1]]
    obc_g = [obc["greater"][0], None, None, obc["greater"][1]]
    zd = [np.zeros_like(x) for x in d]
    zu = [np.zeros_like(x) for x in u]
    res = orc.selected_solve(d, u, lo, zd, zu, zd, zu, obc_r, obc_l, obc_g, return_current=True,
                             current_stale_coupling=True)
    for key in ("xl", "xg"):
        for part in ("diag", "upper", "lower"):
            got = np.stack(res[f"{key}_{part}"], axis=1)
            assert _rel(got, g[f"{key}_{part}"]) < 1e-11, (key, part)
    assert _rel(np.stack(res["xr_diag"], axis=1), g["xr_diag"]) < 1e-11
    assert _rel(res["current"], g["current"]) < 1e-10
    xd, xu, xlo = orc.selected_inv(d, u, lo, obc_r)
    assert _rel(np.stack(xd, axis=1), g["inv_diag"]) < 1e-11
    assert _rel(np.stack(xu, axis=1), g["inv_upper"]) < 1e-11
    assert _rel(np.stack(xlo, axis=1), g["inv_lower"]) < 1e-11
    assert nb == len(d)


def test_oracle_observables_against_upstream():
    """Layer current (upstream observables.device_current with the Hamiltonian),
    per-block DOS and the energies upstream ElectronSolver._filter_peaks zeroes,
    on the oracle's own solve of the fixture's device."""
    g = np.load(os.path.join(GOLDEN, "observables_small.npz"))
    dev = make_device(num_blocks=5, block_size=8, num_energies=40, seed=21)
    assert np.array_equal(dev.h_diag, g["h_diag"]) and np.array_equal(dev.h_upper, g["h_upper"])
    d, u, lo = dev.system_blocks()
    obc = orc.obc_self_energies(d, u, lo, dev.energies, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol, dev.sr_max_iter)
    pad = [None] * 3
    zd = [np.zeros_like(x) for x in d]
    zu = [np.zeros_like(x) for x in u]
    res = orc.selected_solve(d, u, lo, zd, zu, zd, zu, [obc["retarded"][0], *pad, obc["retarded"][1]],
                             [obc["lesser"][0], *pad, obc["lesser"][1]], [obc["greater"][0], *pad, obc["greater"][1]])
    cur = orc.layer_current(res["xl_upper"], dev.h_upper)
    assert cur.shape == g["layer_current"].shape == (40, 4)
    assert np.abs(cur - g["layer_current"]).max() <= 1e-10 * np.abs(g["layer_current"]).max()
    dos = orc.block_dos(res["xr_diag"])
    assert _rel(dos, g["dos"]) < 1e-11
    assert np.array_equal(orc.peak_mask(g["dos"], dev.energies, float(g["peak_limit"])), g["peak_mask"])
    assert np.array_equal(orc.peak_mask(dos, dev.energies, float(g["peak_limit"])), g["peak_mask"])
    assert 0 < g["peak_mask"].sum() < len(dev.energies)


def test_oracle_transport_cfg_small_subset():
    g = np.load(os.path.join(GOLDEN, "transport_cfg_small_subset.npz"))
    dev = make_device(num_blocks=16, block_size=64, num_energies=32, seed=1234)
    e = dev.energies[g["energy_index"]]
    d, u, lo = dev.system_blocks(e)
    obc = orc.obc_self_energies(d, u, lo, e, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol, dev.sr_max_iter)
    nb = 16
    pad = [None] * (nb - 2)
    res = orc.selected_solve(
        d, u, lo, [np.zeros_like(x) for x in d], [np.zeros_like(x) for x in u],
        [np.zeros_like(x) for x in d], [np.zeros_like(x) for x in u],
        [obc["retarded"][0], *pad, obc["retarded"][1]],
        [obc["lesser"][0], *pad, obc["lesser"][1]],
        [obc["greater"][0], *pad, obc["greater"][1]], return_current=True, return_extras=True)
    for key in ("xl", "xg", "xr"):
        dd = np.stack(res[f"{key}_diag"], axis=1)
        assert _rel(np.linalg.norm(dd, axis=(-2, -1)), g[f"{key}_diag_fro"]) < 1e-10
        assert _rel(orc.block_density(res[f"{key}_diag"]), g[f"{key}_block_density"]) < 1e-10
        assert _rel(dd[:, 0], g[f"{key}_first_block"]) < 1e-10
    # upstream reads a stale coupling for every interface but the last
    assert _rel(res["current"][:, -1], g["current"][:, -1]) < 1e-9
    # Meir-Wingreen with the interface's own coupling conserves the current
    # through a ballistic device: every interface carries the left contact
    # current, up to the leakage of the eta = 1e-6 broadening (< 1e-2 here;
    # the stale upstream coupling is off by O(1) on these interfaces)
    for k in range(nb - 1):
        assert np.allclose(res["current"][:, k], g["i_left"], rtol=1e-2, atol=1e-9 * np.abs(g["i_left"]).max())
    i_l, i_r = orc.contact_currents(res["xl_diag"][0], res["xg_diag"][0], res["xl_diag"][-1], res["xg_diag"][-1], obc)
    assert _rel(i_l, g["i_left"]) < 1e-9 and _rel(i_r, g["i_right"]) < 1e-9
    # Caroli transmission against the contact current (ballistic device)
    t = orc.caroli_transmission(res["xr_corner"], obc["gamma"][0], obc["gamma"][1])
    f_l = orc.fermi_dirac(e - dev.mu_left, dev.kt)
    f_r = orc.fermi_dirac(e - dev.mu_right, dev.kt)
    sel = np.abs(f_l - f_r) > 1e-3
    if sel.any():
        t_cur = (-g["i_left"][sel] / (f_l[sel] - f_r[sel])).real
        assert np.allclose(t[sel], t_cur, rtol=1e-7, atol=1e-9)


def test_oracle_selected_inv_matches_dense_inverse():
    dev = make_device(num_blocks=5, block_size=6, num_energies=3, seed=3)
    d, u, lo = dev.system_blocks()
    xd, xu, xlo = orc.selected_inv(d, u, lo)
    full = np.linalg.inv(orc.dense_from_blocks(d, u, lo))
    got = orc.dense_from_blocks(xd, xu, xlo)
    mask = orc.dense_from_blocks([np.ones_like(x) for x in d], [np.ones_like(x) for x in u], [np.ones_like(x) for x in lo]) != 0
    assert _rel(got * mask, full * mask) < 1e-10


def test_oracle_sancho_rubio_fixed_point():
    """The upstream SR test criterion: x = inv(a_ii - a_ji x a_ij)."""
    dev = make_device(num_blocks=2, block_size=10, num_energies=5, seed=5)
    d, u, lo = dev.system_blocks()
    x, it = orc.sancho_rubio(d[0], u[0], lo[0], 200, 1e-12)
    assert it < 200
    assert _rel(x, np.linalg.inv(d[0] - lo[0] @ x @ u[0])) < 1e-6
    with pytest.warns(RuntimeWarning):
        orc.sancho_rubio(d[0], u[0], lo[0], 1, 1e-12)


def test_get_batches_matches_upstream_rule():
    assert orc.get_batches(10, 3)[0] == [4, 3, 3]
    assert orc.get_batches(10, 100)[0] == [10]
    assert orc.get_batches(7, 1)[0] == [1] * 7
    assert list(orc.get_batches(10, 2)[1]) == [0, 2, 4, 6, 8, 10]


def test_keldysh_recursion_is_linear_in_the_contact_sources():
    """The identity the generator-form kernels use: with the contacts as the
    only sources (Sigma^<_c = i f_c Gamma_c, Sigma^>_c = i (f_c - 1) Gamma_c),
    the recursion run once per contact source (i Gamma_L at the first block,
    i Gamma_R at the last) and mixed with the occupations gives the G^< and
    G^> of the component recursion, block for block."""
    dev = make_device(num_blocks=5, block_size=8, num_energies=6, seed=17)
    d, u, lo = dev.system_blocks()
    obc = orc.obc_self_energies(d, u, lo, dev.energies, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol,
                                dev.sr_max_iter)
    nb = len(d)
    zd = [np.zeros_like(x) for x in d]
    zu = [np.zeros_like(x) for x in u]
    pad = [None] * (nb - 2)
    obc_r = [obc["retarded"][0], *pad, obc["retarded"][1]]

    def solve(src0, srcn):
        return orc.selected_solve(d, u, lo, zd, zu, zd, zu, obc_r, [src0, *pad, srcn], [src0, *pad, srcn])

    full = orc.selected_solve(d, u, lo, zd, zu, zd, zu, obc_r, [obc["lesser"][0], *pad, obc["lesser"][1]],
                              [obc["greater"][0], *pad, obc["greater"][1]])
    zero_l, zero_r = np.zeros_like(obc["gamma"][0]), np.zeros_like(obc["gamma"][1])
    x_l = solve(1j * obc["gamma"][0], zero_r)
    x_r = solve(zero_l, 1j * obc["gamma"][1])
    f_l = orc.fermi_dirac(dev.energies - dev.mu_left, dev.kt)[:, None, None]
    f_r = orc.fermi_dirac(dev.energies - dev.mu_right, dev.kt)[:, None, None]
    for part in ("diag", "upper"):
        for i in range(len(full[f"xl_{part}"])):
            want_l = full[f"xl_{part}"][i]
            want_g = full[f"xg_{part}"][i]
            got_l = f_l * x_l[f"xl_{part}"][i] + f_r * x_r[f"xl_{part}"][i]
            got_g = (f_l - 1) * x_l[f"xl_{part}"][i] + (f_r - 1) * x_r[f"xl_{part}"][i]
            assert _rel(got_l, want_l) < 1e-12, (part, i)
            assert _rel(got_g, want_g) < 1e-12, (part, i)


def test_spectral_oracle_against_upstream():
    """The spectral-OBC restatement (Beyn + Spectral, block_sections = 1)
    reproduces upstream's surface Green's functions and eigenvalues on the
    fixture written by upstream Spectral(Beyn(...)) (tests/golden/spectral_small.npz)."""
    from oracle import spectral_oracle as so

    g = np.load(os.path.join(GOLDEN, "spectral_small.npz"))
    x, info = so.spectral(g["a_ii"], g["a_ij"], g["a_ji"], r_o=float(g["r_o"]), r_i=float(g["r_i"]),
                          m_0=int(g["m_0"]), num_quad_points=int(g["num_quad_points"]), rng=np.random.default_rng(42))
    rel = np.linalg.norm(x - g["x"], axis=(-2, -1)) / np.linalg.norm(g["x"], axis=(-2, -1))
    assert rel.max() < 1e-12
    # the eigenvalues of the first call (same probe block), as sets
    for e in range(len(g["energies"])):
        assert np.allclose(np.sort_complex(info["ws"][e]), np.sort_complex(g["ws"][e]), rtol=0, atol=1e-12)
    # on this lead (rank-4 coupling) the spectral OBC agrees with Sancho-Rubio
    rel_sr = np.linalg.norm(x - g["x_sancho_rubio"], axis=(-2, -1)) / np.linalg.norm(g["x_sancho_rubio"], axis=(-2, -1))
    assert rel_sr.max() < 2e-9


@pytest.mark.parametrize("num_partitions", [2, 3, 4, 6])
def test_partitioned_oracle_equals_rgf_oracle(num_partitions):
    """The nested-dissection restatement (RGFDist / _serinv) returns the
    blocks of the plain RGF restatement -- pinned to upstream fixtures -- to
    rounding, for selected inversion and selected solve with contact blocks
    and interior self-energies (upstream RGFDist needs several MPI ranks and
    cannot run in this container, so it is pinned through this equality)."""
    from oracle import rgf_dist_oracle as rd

    rng = np.random.default_rng(num_partitions)

    def rnd(*s):
        return rng.standard_normal(s) + 1j * rng.standard_normal(s)

    def skew(x):
        return x - x.conj().swapaxes(-1, -2)

    nb, b, ne = 13, 4, 3
    diag = [rnd(ne, b, b) + 6 * np.eye(b) for _ in range(nb)]
    upper = [rnd(ne, b, b) for _ in range(nb - 1)]
    lower = [rnd(ne, b, b) for _ in range(nb - 1)]
    sl_d, sl_u = [skew(rnd(ne, b, b)) for _ in range(nb)], [rnd(ne, b, b) for _ in range(nb - 1)]
    sg_d, sg_u = [skew(rnd(ne, b, b)) for _ in range(nb)], [rnd(ne, b, b) for _ in range(nb - 1)]
    pad = [None] * (nb - 2)
    obc_r = [rnd(ne, b, b), *pad, rnd(ne, b, b)]
    obc_l = [skew(rnd(ne, b, b)), *pad, skew(rnd(ne, b, b))]
    obc_g = [skew(rnd(ne, b, b)), *pad, skew(rnd(ne, b, b))]

    def rel(a, r):
        return np.linalg.norm(a - r) / np.linalg.norm(r)

    ref_inv = orc.selected_inv(diag, upper, lower, obc_r)
    got_inv = rd.selected_inv(diag, upper, lower, obc_r, num_partitions=num_partitions)
    for k in range(3):
        assert max(rel(a, r) for a, r in zip(got_inv[k], ref_inv[k])) < 1e-12
    ref = orc.selected_solve(diag, upper, lower, sl_d, sl_u, sg_d, sg_u, obc_r, obc_l, obc_g)
    got = rd.selected_solve(diag, upper, lower, sl_d, sl_u, sg_d, sg_u, obc_r, obc_l, obc_g,
                            num_partitions=num_partitions)
    for key in ("xl_diag", "xl_upper", "xl_lower", "xg_diag", "xg_upper", "xg_lower", "xr_diag"):
        assert max(rel(a, r) for a, r in zip(got[key], ref[key])) < 1e-12, key
    with pytest.raises(ValueError):
        rd.partition_bounds(5, 3)


def test_partitioned_oracle_accuracy_on_a_transport_device():
    """On a transport device (energies inside the bands, no diagonal
    dominance: make_device(64, 32, 4)) two partitions still reproduce the RGF
    restatement to 1e-10 of the largest entry, but the deviation grows with
    the number of partitions: with P = 8 (partitions of 8 blocks) the G^R
    diagonal moves by ~3e-7.  A property of the partitioned elimination
    (middle partitions carry their first block's coupling across the
    partition), recorded here; the GPU solver follows the same algorithm."""
    from oracle import rgf_dist_oracle as rd

    nb, b, ne = 64, 32, 4
    dev = make_device(num_blocks=nb, block_size=b, num_energies=ne, seed=3)
    d, u, lo = dev.system_blocks()
    obc = orc.obc_self_energies(d, u, lo, dev.energies, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol,
                                dev.sr_max_iter)
    z, zu = [np.zeros_like(x) for x in d], [np.zeros_like(x) for x in u]
    pad = [None] * (nb - 2)
    r = [obc["retarded"][0], *pad, obc["retarded"][1]]
    lg = ([obc["lesser"][0], *pad, obc["lesser"][1]], [obc["greater"][0], *pad, obc["greater"][1]])
    ref = orc.selected_solve(d, u, lo, z, zu, z, zu, r, *lg)

    def dev_max(got, key):
        return max(np.abs(a - c).max() for a, c in zip(got[key], ref[key])) / max(np.abs(c).max() for c in ref[key])

    two = rd.selected_solve(d, u, lo, z, zu, z, zu, r, *lg, num_partitions=2)
    eight = rd.selected_solve(d, u, lo, z, zu, z, zu, r, *lg, num_partitions=8)
    for key in ("xr_diag", "xl_diag", "xl_upper"):
        assert dev_max(two, key) < 1e-10, key
        assert dev_max(eight, key) < 1e-5, key
    assert dev_max(eight, "xr_diag") > 100 * dev_max(two, "xr_diag")
