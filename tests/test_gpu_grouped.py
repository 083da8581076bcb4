"""Grouped transport solve (qtx_transport_solve_grouped): every energy of
several devices of one block size in one persistent launch.

Each device's blocks and observables must meet the generator-form bar against
the oracle: 1e-10 relative per block, or 20 x the oracle's own spread under
1e-16 perturbations of H at energies where the problem is that sensitive
(ill-conditioned Sancho-Rubio steps, or a lead's Gamma cancelling outside its
band).  They must also equal the layered qtx_transport_solve of the same
device within twice that bound (bit for bit at b <= 32, where the block
inverses coincide)."""

import ctypes
import warnings

import numpy as np
import pytest
import torch

from oracle import rgf_oracle as orc
from quatrex_b200 import _lib
from quatrex_b200.transport import TransportSolver, grouped_footprint_bytes, solve_grouped
from quatrex_b200.workloads import make_device
from test_gpu_transport import _layer_err, _oracle, _oracle_h, _per_energy_rel

pytestmark = pytest.mark.gpu

OBS = ("density", "hole_density", "transmission", "current_left", "current_right", "sr_iterations")


def _spread(dev, energies, ref, trials=3):
    """Per-energy relative spread of the oracle's G^R, G^< and G^> diagonal
    blocks under 1e-16 perturbations of H.  G^< and G^> are included because
    outside a lead's band Gamma = i (Sigma - Sigma^H) is a small difference of
    nearly Hermitian terms, which G^R alone does not show."""
    rng = np.random.default_rng(123)
    spread = np.zeros(len(energies))
    for _ in range(trials):
        h = dev.h_diag * (1 + 1e-16 * rng.standard_normal(dev.h_diag.shape))
        h = 0.5 * (h + h.conj().swapaxes(-1, -2))
        r2, _ = _oracle_h(dev, h, energies)
        for k in ("xr_diag", "xl_diag", "xg_diag"):
            spread = np.maximum(spread, _per_energy_rel(np.stack(r2[k], axis=1), np.stack(ref[k], axis=1)))
    return spread


def _check_oracle(dev, energies, out):
    ref, obc = _oracle(dev, energies)
    bound = np.maximum(1e-10, 20 * _spread(dev, energies, ref))
    nb = dev.num_blocks

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
    check(out["transmission"], orc.caroli_transmission(ref["xr_corner"], obc["gamma"][0], obc["gamma"][1]), 10)
    i_l, i_r = orc.contact_currents(ref["xl_diag"][0], ref["xg_diag"][0], ref["xl_diag"][-1], ref["xg_diag"][-1], obc)
    check(out["current_left"], i_l, 10)
    check(out["current_right"], i_r, 10)
    check(out["dos"], orc.block_dos(ref["xr_diag"]), 10)
    err = _layer_err(out["layer_current"], orc.layer_current(ref["xl_upper"], dev.h_upper), ref["xl_upper"],
                     dev.h_upper)
    assert (err <= 10 * bound).all(), (err, bound)
    its = out["sr_iterations"].cpu().numpy()
    assert its.min() >= 1 and its.max() <= max(obc["iterations"]) + 1
    return bound


@pytest.mark.parametrize("b", [24, 64])
def test_grouped_blocks_against_oracle(b):
    """Uneven devices of one block size, each with its own energies, in one call."""
    devs = [make_device(num_blocks=nb, block_size=b, num_energies=ne, seed=31 + q)
            for q, (nb, ne) in enumerate([(5, 6), (2, 3), (7, 4)])]
    outs = solve_grouped(devs, [d.energies for d in devs])
    well = 0
    for d, out in zip(devs, outs):
        well += int((_check_oracle(d, d.energies, out) == 1e-10).sum())
    assert well >= 4


def _obs_err(k, got, want):
    """Per-energy error of an observable.  A contact current is a small
    difference of two traces of order one wherever f_L ~ f_R, so its rounding
    is measured against the device's largest current, not the current itself
    (as density errors are measured against the largest block of the energy)."""
    if k.startswith("current"):
        got = got.cpu().numpy() if isinstance(got, torch.Tensor) else got
        return np.abs(got - want) / max(np.abs(want).max(), 1e-300)
    return _per_energy_rel(got, want)


def _pair_bound(dev):
    """Per-energy bound for two FP64 evaluations of the same solve: each is
    within max(1e-10, 20 x the oracle's spread) of the exact result."""
    ref, _ = _oracle(dev, dev.energies)
    return np.maximum(1e-10, 40 * _spread(dev, dev.energies, ref))


@pytest.mark.parametrize("b", [8, 32, 48, 64])
def test_grouped_equals_layered(b):
    devs = [make_device(num_blocks=nb, block_size=b, num_energies=ne, seed=100 + 7 * q)
            for q, (nb, ne) in enumerate([(6, 5), (3, 9), (9, 2), (4, 4)])]
    outs = solve_grouped(devs, [d.energies for d in devs])
    for d, out in zip(devs, outs):
        ref = TransportSolver(d, max_batch_size=3).solve(d.energies)
        bound = _pair_bound(d)
        assert torch.equal(out["sr_iterations"], ref["sr_iterations"])
        for k in ("gr_diag", "gr_upper", "gr_lower", "gl_diag", "gl_upper", "gg_diag", "gg_upper"):
            if b <= 32:
                # same products in the same order, same single-panel inverse
                assert torch.equal(out[k], ref[k]), k
            err = _per_energy_rel(out[k], ref[k].cpu().numpy())
            assert (err <= bound).all(), (k, err, bound)
        for k in ("density", "hole_density", "transmission", "current_left", "current_right", "dos"):
            err = _obs_err(k, out[k], ref[k].cpu().numpy())
            assert (err <= 10 * bound).all(), (k, err, bound)
        err = _layer_err(out["layer_current"], ref["layer_current"].cpu().numpy(), ref["gl_upper"], d.h_upper)
        assert (err <= 10 * bound).all(), ("layer_current", err, bound)


def test_grouped_is_one_launch_for_uneven_devices():
    rng = np.random.default_rng(5)
    devs = []
    for q in range(12):
        nb = int(rng.integers(2, 14))
        ne = int(rng.integers(1, 9))
        devs.append(make_device(num_blocks=nb, block_size=32, num_energies=ne, seed=500 + q))
    ctx = _lib.new_context(torch.cuda.current_device())
    try:
        before = _lib.load().qtx_launch_count(ctx)
        outs = solve_grouped(devs, [d.energies for d in devs], keys=OBS, ctx=ctx)
        assert _lib.load().qtx_launch_count(ctx) - before == 1
    finally:
        torch.cuda.synchronize()
        _lib.destroy_context(ctx)
    for d, out in zip(devs, outs):
        ref = TransportSolver(d).solve(d.energies, keys=OBS)
        bound = _pair_bound(d)
        assert torch.equal(out["sr_iterations"], ref["sr_iterations"])
        for k in ("density", "hole_density", "transmission", "current_left", "current_right"):
            err = _obs_err(k, out[k], ref[k].cpu().numpy())
            assert (err <= 10 * bound).all(), (k, err, bound)


def test_grouped_not_converged_and_refusals():
    d = make_device(num_blocks=3, block_size=16, num_energies=3, seed=2)
    d.sr_max_iter = 1
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        out = solve_grouped([d], [d.energies], keys=OBS)[0]
    assert any(issubclass(x.category, RuntimeWarning) for x in w)
    assert (out["sr_iterations"].cpu().numpy() == 1).all()
    big = make_device(num_blocks=2, block_size=65, num_energies=1, seed=3)
    with pytest.raises(NotImplementedError):
        solve_grouped([big], [big.energies], keys=OBS)
    a = make_device(num_blocks=3, block_size=16, num_energies=2, seed=4)
    c = make_device(num_blocks=3, block_size=32, num_energies=2, seed=4)
    with pytest.raises(ValueError):
        solve_grouped([a, c], [a.energies, c.energies], keys=OBS)
    # the INT8 split products are not offered on this path
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    h = torch.from_numpy(a.h_diag).cuda()
    u = torch.from_numpy(a.h_upper).cuda()
    e = torch.from_numpy(a.energies).cuda()
    p = _lib.TransportProblem(num_blocks=3, block_size=16, num_energies=2, h_diag=h.data_ptr(), h_upper=u.data_ptr(),
                              energies=e.data_ptr(), eta=a.eta, mu_left=a.mu_left, mu_right=a.mu_right, kt=a.kt,
                              sr_tol=a.sr_tol, sr_max_iterations=a.sr_max_iter, max_batch_size=0)
    o = _lib.TransportOutputs()
    assert lib.qtx_transport_solve_grouped(ctx, 1, ctypes.byref(p), ctypes.byref(o), _lib.QTX_PREC_MIXED, 0,
                                           None, None) == _lib.QTX_E_UNSUPPORTED
    assert grouped_footprint_bytes([3, 9], [4, 100], 64) > grouped_footprint_bytes([3, 9], [4, 100], 32) > 0
    assert grouped_footprint_bytes([3], [4], 65) == 0
