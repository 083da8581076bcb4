"""Parity on the benchmark configurations themselves, per returned block.

* nb=16, b=64, all 32 energies on [-2, 2] (the CPU-runnable case);
* nb=64, b=256 (the single-GPU scale-up) at three of its 1024 energies;
* the mixed-precision form on the nb=16, b=64 inputs.

The bar is 1e-10 relative Frobenius error per returned block and energy.
Where it applies, and why the test is split in two:

The selected solve itself is well conditioned on these devices: a 1e-16
relative perturbation of the diagonal blocks moves the oracle's G^R, G^< and
G^> blocks by at most 1.6e-11 (with the contact self-energies held fixed).
The Sancho-Rubio surface Green's function is not: at a few energies (near
band edges of the leads) the same perturbation moves the oracle's own surface
Green's function, and through it every block, by up to 6e-9.  So

1. the CUDA path is compared with the oracle's selected solve fed with the
   surface Green's functions that the CUDA Sancho-Rubio produced (the contact
   self-energies, Fermi functions and every RGF product are still the
   oracle's): 1e-10 per block at EVERY energy of the nb=16, b=64 device; at
   nb=64, b=256 the selected solve's own sensitivity reaches 6e-10 in the G^<
   blocks at one energy, so G^< and G^> are held there to 20 x that measured
   spread and G^R to the plain bar;
2. it is compared with the oracle end to end (the oracle's own Sancho-Rubio)
   with the per-energy bound max(1e-10, 20 x the oracle's spread under two
   1e-16 perturbations of H), and the plain 1e-10 bar holds at every energy
   whose spread is below 5e-12.

The drop-in ``RGF.selected_solve`` / ``selected_inv`` (the qttools plugin
API on DSDBCOO operands) takes the contact blocks as inputs, so it is held to
1e-10 per block at every energy directly.
"""

import numpy as np
import pytest
import torch

from oracle import rgf_oracle as orc
from quatrex_b200.datastructures import DSDBCOO
from quatrex_b200.greens_function_solver import RGF, OBCBlocks
from quatrex_b200.obc import SanchoRubio
from quatrex_b200.transport import TransportSolver
from quatrex_b200.workloads import CONFIG_LARGE, CONFIG_SMALL, make_device

pytestmark = pytest.mark.gpu

BAR = 1e-10
CFG2_ENERGY_INDEX = np.array([100, 500, 900])


def _np(x):
    return x.cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)


def _block_rel(got, want):
    """Relative Frobenius error per energy of a (E, b, b) block stack; an
    exactly zero reference block (G^> below every lead band) compares in
    absolute terms."""
    got, want = _np(got), _np(want)
    num = np.sqrt((np.abs(got - want) ** 2).sum((-2, -1)))
    den = np.sqrt((np.abs(want) ** 2).sum((-2, -1)))
    return np.where(den > 0, num / np.maximum(den, 1e-300), num)


def _obc_from_surface(d, u, lo, energies, dev, g_l, g_r):
    """The oracle's contact assembly (electron/solver.py:305-386) on given
    surface Green's functions."""
    sig_l = lo[0] @ g_l @ u[0]
    sig_r = u[-1] @ g_r @ lo[-1]
    f_l = orc.fermi_dirac(energies - dev.mu_left, dev.kt)[:, None, None]
    f_r = orc.fermi_dirac(energies - dev.mu_right, dev.kt)[:, None, None]
    gam_l = 1j * (sig_l - sig_l.conj().swapaxes(-2, -1))
    gam_r = 1j * (sig_r - sig_r.conj().swapaxes(-2, -1))
    return {"retarded": [sig_l, sig_r], "lesser": [1j * f_l * gam_l, 1j * f_r * gam_r],
            "greater": [1j * (f_l - 1) * gam_l, 1j * (f_r - 1) * gam_r], "gamma": [gam_l, gam_r]}


def _oracle_solve(d, u, lo, obc, return_current=False):
    nb = len(d)
    pad = [None] * (nb - 2)
    z = [np.zeros_like(x) for x in d]
    zu = [np.zeros_like(x) for x in u]
    return orc.selected_solve(d, u, lo, z, zu, z, zu, [obc["retarded"][0], *pad, obc["retarded"][1]],
                              [obc["lesser"][0], *pad, obc["lesser"][1]],
                              [obc["greater"][0], *pad, obc["greater"][1]], return_extras=True,
                              return_current=return_current)


def _gpu_surfaces(dev, d, u, lo):
    sr = SanchoRubio(dev.sr_max_iter, dev.sr_tol)
    return sr(d[0], u[0], lo[0], "left"), sr(d[-1], lo[-1], u[-1], "right")


def _oracle_spread(dev, energies, ref, trials=2):
    rng = np.random.default_rng(123)
    spread = np.zeros(len(energies))
    for _ in range(trials):
        h = dev.h_diag * (1 + 1e-16 * rng.standard_normal(dev.h_diag.shape))
        h = 0.5 * (h + h.conj().swapaxes(-1, -2))
        saved, dev.h_diag = dev.h_diag, h
        try:
            d, u, lo = dev.system_blocks(energies)
        finally:
            dev.h_diag = saved
        obc = orc.obc_self_energies(d, u, lo, energies, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol,
                                    dev.sr_max_iter)
        r2 = _oracle_solve(d, u, lo, obc)
        for key in ("xr_diag", "xl_diag", "xg_diag"):
            for i in range(len(d)):
                spread = np.maximum(spread, _block_rel(r2[key][i], ref[key][i]))
    return spread


# returned blocks of the generator form: (output key, oracle key, block class)
_BLOCKS = (("gr_diag", "xr_diag", "r"), ("gr_upper", "xr_upper", "r"), ("gr_lower", "xr_lower", "r"),
           ("gl_diag", "xl_diag", "l"), ("gl_upper", "xl_upper", "l"), ("gg_diag", "xg_diag", "g"),
           ("gg_upper", "xg_upper", "g"))


def _worst_per_class(out, ref):
    """Per energy and block class (G^R, G^<, G^>), the worst relative error
    over every returned block of that class."""
    ne = len(ref["xr_diag"][0])
    worst = {c: np.zeros(ne) for c in "rlg"}
    for key, rkey, cls in _BLOCKS:
        for i in range(len(ref[rkey])):
            worst[cls] = np.maximum(worst[cls], _block_rel(out[key][:, i], ref[rkey][i]))
    return worst


def _check_transport_blocks(out, ref, nb, bound):
    """Every returned block of the generator form against an oracle result;
    `bound` is one per-energy array for every block, or one per block class."""
    worst = _worst_per_class(out, ref)
    bounds = bound if isinstance(bound, dict) else {c: bound for c in "rlg"}
    for c in "rlg":
        assert (worst[c] <= bounds[c]).all(), (c, worst[c], bounds[c])
    return np.maximum(np.maximum(worst["r"], worst["l"]), worst["g"])


def _rgf_spread(d, u, lo, obc, ref, trials=1):
    """Per energy and block class, the relative change of the oracle's own
    selected solve under a 1e-16 relative perturbation of the diagonal blocks
    of A, with the contact blocks held fixed."""
    rng = np.random.default_rng(7)
    spread = {c: np.zeros(len(d[0])) for c in "rlg"}
    for _ in range(trials):
        d2 = [x * (1 + 1e-16 * rng.standard_normal(x.shape)) for x in d]
        r2 = _oracle_solve(d2, u, lo, obc)
        out2 = {key: np.stack(r2[rkey], axis=1) for key, rkey, _ in _BLOCKS}
        w = _worst_per_class(out2, ref)
        for c in "rlg":
            spread[c] = np.maximum(spread[c], w[c])
    return spread


def _check_observables(out, ref, obc, bound):
    dens_ref = orc.block_density(ref["xl_diag"])
    dens = _np(out["density"])
    scale = np.abs(dens_ref).max(axis=1)
    assert (np.abs(dens - dens_ref).max(axis=1) <= bound * np.maximum(scale, 1e-300)).all()
    t_ref = orc.caroli_transmission(ref["xr_corner"], obc["gamma"][0], obc["gamma"][1])
    t = _np(out["transmission"])
    assert (np.abs(t - t_ref) <= bound * np.maximum(np.abs(t_ref), 1e-12)).all(), (t, t_ref)


def _config_run(cfg, energy_index=None, precision="fp64"):
    dev = make_device(**cfg)
    e = dev.energies if energy_index is None else dev.energies[energy_index]
    d, u, lo = dev.system_blocks(e)
    out = TransportSolver(dev, max_batch_size=len(e), precision=precision).solve(e)
    out = {k: _np(v) for k, v in out.items()}
    g_l, g_r = _gpu_surfaces(dev, d, u, lo)
    obc_gpu = _obc_from_surface(d, u, lo, e, dev, g_l, g_r)
    ref_gpu = _oracle_solve(d, u, lo, obc_gpu)
    return dev, e, d, u, lo, out, obc_gpu, ref_gpu


def test_config_small_transport_every_block_every_energy():
    """nb=16, b=64, all 32 energies: every returned block (G^R diagonal, upper,
    lower; G^< and G^> diagonal and upper) at 1e-10 against the oracle's
    selected solve on the CUDA surface Green's functions; density and
    transmission at 1e-10."""
    dev, e, d, u, lo, out, obc_gpu, ref_gpu = _config_run(CONFIG_SMALL)
    bound = np.full(len(e), BAR)
    _check_transport_blocks(out, ref_gpu, dev.num_blocks, bound)
    _check_observables(out, ref_gpu, obc_gpu, bound)
    # the CUDA surface Green's functions themselves against the oracle's
    # Sancho-Rubio (same tolerance and iteration cap) at 1e-10 wherever the
    # oracle is stable to 5e-12, and within its spread elsewhere
    obc_ref = orc.obc_self_energies(d, u, lo, e, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol, dev.sr_max_iter)
    ref = _oracle_solve(d, u, lo, obc_ref)
    spread = _oracle_spread(dev, e, ref)
    bound_e2e = np.maximum(BAR, 20 * spread)
    worst = _check_transport_blocks(out, ref, dev.num_blocks, bound_e2e)
    stable = spread < 5e-12  # 7 of the 32 energies of this device
    assert stable.sum() >= 5
    assert (worst[stable] <= BAR).all()


def test_config_small_dropin_every_block_every_energy():
    """The plugin call RGF.selected_solve(return_retarded, return_current) and
    RGF.selected_inv on DSDBCOO operands of the nb=16, b=64 device at all 32
    energies, with the oracle's contact blocks as OBC inputs: every block of
    G^< and G^> (diagonal, upper and lower), the diagonal of G^R, the layer
    current and every block of the selected inverse at 1e-10."""
    dev = make_device(**CONFIG_SMALL)
    e = dev.energies
    d, u, lo = dev.system_blocks(e)
    nb = dev.num_blocks
    obc = orc.obc_self_energies(d, u, lo, e, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol, dev.sr_max_iter)
    ref = _oracle_solve(d, u, lo, obc, return_current=True)
    A = DSDBCOO.from_blocks(d, u, lo, device="cuda")
    Z = DSDBCOO.zeros_like(A)
    ob = OBCBlocks(nb)
    ob.retarded[0], ob.retarded[-1] = obc["retarded"]
    ob.lesser[0], ob.lesser[-1] = obc["lesser"]
    ob.greater[0], ob.greater[-1] = obc["greater"]
    xl, xg, xr, cur = RGF(max_batch_size=32).selected_solve(A, Z, Z, obc_blocks=ob, return_retarded=True,
                                                            return_current=True)
    xl, xg, xr = xl.to("cpu"), xg.to("cpu"), xr.to("cpu")
    for i in range(nb):
        assert _block_rel(xl.blocks[i, i], ref["xl_diag"][i]).max() <= BAR
        assert _block_rel(xg.blocks[i, i], ref["xg_diag"][i]).max() <= BAR
        assert _block_rel(xr.blocks[i, i], ref["xr_diag"][i]).max() <= BAR
    for i in range(nb - 1):
        assert _block_rel(xl.blocks[i, i + 1], ref["xl_upper"][i]).max() <= BAR
        assert _block_rel(xl.blocks[i + 1, i], ref["xl_lower"][i]).max() <= BAR
        assert _block_rel(xg.blocks[i, i + 1], ref["xg_upper"][i]).max() <= BAR
        assert _block_rel(xg.blocks[i + 1, i], ref["xg_lower"][i]).max() <= BAR
    # layer currents: relative to the largest current of the grid (outside the
    # bias window a layer current is a difference of two nearly equal traces)
    cur_ref = ref["current"]
    cur = _np(cur)
    assert np.abs(cur - cur_ref).max() <= BAR * np.abs(cur_ref).max()
    # selected inversion of the same system (with the retarded contact blocks)
    inv_ref = orc.selected_inv(d, u, lo, [obc["retarded"][0], *([None] * (nb - 2)), obc["retarded"][1]])
    ob_r = OBCBlocks(nb)
    ob_r.retarded[0], ob_r.retarded[-1] = obc["retarded"]
    X = RGF(max_batch_size=32).selected_inv(A, obc_blocks=ob_r).to("cpu")
    for i in range(nb):
        assert _block_rel(X.blocks[i, i], inv_ref[0][i]).max() <= BAR
    for i in range(nb - 1):
        assert _block_rel(X.blocks[i, i + 1], inv_ref[1][i]).max() <= BAR
        assert _block_rel(X.blocks[i + 1, i], inv_ref[2][i]).max() <= BAR


def test_config_large_three_energies_every_block():
    """nb=64, b=256 at energies 100, 500 and 900 of its 1024-point grid,
    against the oracle's selected solve on the CUDA surface Green's functions:
    every G^R block (diagonal, upper, lower) at 1e-10; every G^< and G^> block
    at max(1e-10, 20 x the oracle's own spread).  At this size the oracle's
    selected solve is itself stable only to ~6e-10 in the G^< blocks at the
    energy where G^< is a small difference of nearly equal terms (index 900,
    f_L ~ f_R ~ 0), and to ~2e-11 in G^R.  Then against the oracle end to end
    within the Sancho-Rubio conditioning bound."""
    dev, e, d, u, lo, out, obc_gpu, ref_gpu = _config_run(CONFIG_LARGE, CFG2_ENERGY_INDEX)
    spread = _rgf_spread(d, u, lo, obc_gpu, ref_gpu)
    assert (spread["r"] < 5e-11).all(), spread["r"]
    bounds = {"r": np.full(len(e), BAR), "l": np.maximum(BAR, 20 * spread["l"]),
              "g": np.maximum(BAR, 20 * spread["g"])}
    _check_transport_blocks(out, ref_gpu, dev.num_blocks, bounds)
    _check_observables(out, ref_gpu, obc_gpu, np.maximum(BAR, 20 * spread["l"]))
    obc_ref = orc.obc_self_energies(d, u, lo, e, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol, dev.sr_max_iter)
    ref = _oracle_solve(d, u, lo, obc_ref)
    spread_e2e = _oracle_spread(dev, e, ref, trials=1)
    worst_rgf = np.maximum(np.maximum(spread["r"], spread["l"]), spread["g"])
    _check_transport_blocks(out, ref, dev.num_blocks, np.maximum(BAR, 20 * np.maximum(spread_e2e, worst_rgf)))


def test_config_mixed_precision_on_small_inputs():
    """The precision form (INT8 split products in the sweep; inverses and
    Sancho-Rubio in FP64) on the nb=16, b=64 inputs at all 32 energies: G^R
    diagonal blocks, G^< diagonal blocks (relative Frobenius per block),
    per-block density (relative to the energy's largest block) and
    transmission (relative), each at most 1e-8 against the FP64 oracle -- its
    selected solve on the surface Green's functions of the (FP64) CUDA
    Sancho-Rubio, which is what the mixed form keeps in FP64."""
    dev, e, d, u, lo, out, obc_gpu, ref = _config_run(CONFIG_SMALL, precision="mixed")
    nb = dev.num_blocks
    err = {"gr_diag": 0.0, "gl_diag": 0.0}
    for i in range(nb):
        err["gr_diag"] = max(err["gr_diag"], _block_rel(out["gr_diag"][:, i], ref["xr_diag"][i]).max())
        err["gl_diag"] = max(err["gl_diag"], _block_rel(out["gl_diag"][:, i], ref["xl_diag"][i]).max())
    dens_ref = orc.block_density(ref["xl_diag"])
    err["density"] = float((np.abs(out["density"] - dens_ref).max(axis=1) /
                            np.abs(dens_ref).max(axis=1).clip(1e-300)).max())
    t_ref = orc.caroli_transmission(ref["xr_corner"], obc_gpu["gamma"][0], obc_gpu["gamma"][1])
    err["transmission"] = float((np.abs(out["transmission"] - t_ref) / np.maximum(np.abs(t_ref), 1e-12)).max())
    assert all(v <= 1e-8 for v in err.values()), err
