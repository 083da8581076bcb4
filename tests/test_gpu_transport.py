"""Generator-form transport solve (qtx_transport_solve) against the oracle and
the upstream fixtures.

Every returned block must be within 1e-10 relative Frobenius error of the
oracle, density / contact currents / transmission within 1e-9 -- except at
energies where the problem itself is that sensitive: Sancho-Rubio decimation
can pass through nearly singular intermediate blocks (cond ~1e6 at some
energies), so a 1e-16 relative perturbation of H moves the oracle's own result
by up to ~1e-7 there.  The bound at each energy is therefore
max(1e-10, 20 x the oracle's spread under three 1e-16 perturbations of H)."""

import os

import numpy as np
import pytest
import torch

from oracle import rgf_oracle as orc
from quatrex_b200.transport import TransportSolver
from quatrex_b200.workloads import make_device

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _rel(a, b):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else a
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _oracle(dev, energies):
    return _oracle_h(dev, dev.h_diag, energies)


def _oracle_h(dev, h_diag, energies):
    saved = dev.h_diag
    dev.h_diag = h_diag
    try:
        d, u, lo = dev.system_blocks(energies)
    finally:
        dev.h_diag = saved
    obc = orc.obc_self_energies(d, u, lo, energies, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol, dev.sr_max_iter)
    nb = len(d)
    pad = [None] * (nb - 2)
    z = [np.zeros_like(x) for x in d]
    zu = [np.zeros_like(x) for x in u]
    ref = orc.selected_solve(d, u, lo, z, zu, z, zu, [obc["retarded"][0], *pad, obc["retarded"][1]],
                             [obc["lesser"][0], *pad, obc["lesser"][1]], [obc["greater"][0], *pad, obc["greater"][1]],
                             return_extras=True)
    return ref, obc


def _per_energy_rel(a, b):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else a
    b = np.asarray(b)
    ax = tuple(range(1, b.ndim))
    if not ax:
        return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    return np.sqrt((np.abs(a - b) ** 2).sum(ax)) / np.maximum(np.sqrt((np.abs(b) ** 2).sum(ax)), 1e-300)


def _oracle_spread(dev, energies, ref, trials=3):
    """Per-energy relative spread of the oracle's G^R diagonal under 1e-16 perturbations of H."""
    rng = np.random.default_rng(123)
    want = np.stack(ref["xr_diag"], axis=1)
    spread = np.zeros(len(energies))
    for _ in range(trials):
        h = dev.h_diag * (1 + 1e-16 * rng.standard_normal(dev.h_diag.shape))
        h = 0.5 * (h + h.conj().swapaxes(-1, -2))
        r2, _ = _oracle_h(dev, h, energies)
        spread = np.maximum(spread, _per_energy_rel(np.stack(r2["xr_diag"], axis=1), want))
    return spread



def _layer_err(got, want, gl_upper, h_upper):
    """Per-energy error of the layer currents (E, nb - 1), each against the size
    of the terms its trace sums, ||G^<_ij||_F ||H_ij||_F: wherever f_L ~ f_R a
    layer current is rounding noise of order one of those terms, so neither
    its own size nor the device's largest current is a scale."""
    got = got.cpu().numpy() if isinstance(got, torch.Tensor) else got
    gl = gl_upper.cpu().numpy() if isinstance(gl_upper, torch.Tensor) else np.stack(gl_upper, axis=1)
    scale = np.linalg.norm(gl, axis=(-2, -1)) * np.linalg.norm(h_upper, axis=(-2, -1))[None, :]
    return (np.abs(got - want) / np.maximum(scale, 1e-300)).max(axis=1)

@pytest.mark.parametrize("max_batch_size", [2, 100])
def test_transport_blocks_and_observables(max_batch_size):
    dev = make_device(num_blocks=5, block_size=24, num_energies=6, seed=31)
    ref, obc = _oracle(dev, dev.energies)
    bound = np.maximum(1e-10, 20 * _oracle_spread(dev, dev.energies, ref))
    out = TransportSolver(dev, max_batch_size=max_batch_size).solve(dev.energies)
    nb = 5

    def check(got, want, scale=1.0):
        err = _per_energy_rel(got, want)
        assert (err <= scale * bound).all(), (err, bound)

    for i in range(nb):
        check(out["gr_diag"][:, i], ref["xr_diag"][i])
        check(out["gl_diag"][:, i], ref["xl_diag"][i])
        check(out["gg_diag"][:, i], ref["xg_diag"][i])
    for i in range(nb - 1):
        check(out["gr_upper"][:, i], ref["xr_upper"][i])
        check(out["gr_lower"][:, i], ref["xr_lower"][i])
        check(out["gl_upper"][:, i], ref["xl_upper"][i])
        check(out["gg_upper"][:, i], ref["xg_upper"][i])
    check(out["density"], orc.block_density(ref["xl_diag"]), 10)
    check(out["hole_density"], -orc.block_density(ref["xg_diag"]), 10)
    t_ref = orc.caroli_transmission(ref["xr_corner"], obc["gamma"][0], obc["gamma"][1])
    check(out["transmission"], t_ref, 10)
    i_l, i_r = orc.contact_currents(ref["xl_diag"][0], ref["xg_diag"][0], ref["xl_diag"][-1], ref["xg_diag"][-1], obc)
    check(out["current_left"], i_l, 10)
    check(out["current_right"], i_r, 10)
    check(out["dos"], orc.block_dos(ref["xr_diag"]), 10)
    err = _layer_err(out["layer_current"], orc.layer_current(ref["xl_upper"], dev.h_upper), ref["xl_upper"],
                     dev.h_upper)
    assert (err <= 10 * bound).all(), (err, bound)
    # the well-conditioned energies meet the plain 1e-10 bar
    assert (bound == 1e-10).sum() >= 4
    its = out["sr_iterations"].cpu().numpy()
    assert its.min() >= 1 and its.max() <= max(obc["iterations"]) + 1


def test_transport_against_upstream_subset():
    g = np.load(os.path.join(GOLDEN, "transport_cfg_small_subset.npz"))
    dev = make_device(num_blocks=16, block_size=64, num_energies=32, seed=1234)
    e = dev.energies[g["energy_index"]]
    out = TransportSolver(dev).solve(e)
    assert _rel(out["density"], g["xl_block_density"]) < 1e-9
    assert _rel(out["hole_density"], -g["xg_block_density"]) < 1e-9
    assert _rel(out["current_left"], g["i_left"]) < 1e-9
    assert _rel(out["current_right"], g["i_right"]) < 1e-9
    assert _rel(np.linalg.norm(out["gl_diag"].cpu().numpy(), axis=(-2, -1)), g["xl_diag_fro"]) < 1e-9
    assert _rel(out["gr_diag"][:, 0], g["xr_first_block"]) < 1e-9


def test_transport_ballistic_transmission_matches_current():
    """Caroli transmission equals -I_left / (f_L - f_R) in the ballistic device."""
    dev = make_device(num_blocks=4, block_size=16, num_energies=9, seed=8, e_min=-0.2, e_max=0.2)
    out = TransportSolver(dev).solve(dev.energies)
    f_l = orc.fermi_dirac(dev.energies - dev.mu_left, dev.kt)
    f_r = orc.fermi_dirac(dev.energies - dev.mu_right, dev.kt)
    t_cur = (-out["current_left"].cpu().numpy() / (f_l - f_r)).real
    assert np.allclose(out["transmission"].cpu().numpy(), t_cur, rtol=1e-6, atol=1e-9)
    # current conservation: every interface carries the same layer current, up
    # to the leakage of the eta = 1e-6 broadening (< 1e-2 here, as for the
    # interface currents of the selected solve in tests/test_oracle.py)
    lay = out["layer_current"].cpu().numpy()
    assert np.allclose(lay, lay[:, :1], rtol=1e-2, atol=1e-9 * np.abs(lay).max())
