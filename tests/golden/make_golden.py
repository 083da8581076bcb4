"""Generate the golden fixtures under tests/golden/ by running the UPSTREAM code.

This script is run by hand in a container where the upstream repository is
checked out (its root given by the required ``QTX_UPSTREAM`` variable); it
never runs on the GPU machine and nothing imports it.  It imports the upstream
``qttools`` package (NumPy backend) through a single-rank ``mpi4py`` stand-in
(``tests/golden/_mpi_shim``) and records, for seeded inputs:

* ``btd_<case>.npz``  -- the upstream unit-test construction (random 50 %-dense
  complex blocks made diagonally dominant,
  ``tests/qttools/greens_function_solver/conftest.py:58-104``) for constant and
  mixed block sizes; outputs of upstream ``RGF.selected_inv`` and
  ``RGF.selected_solve(return_retarded=True)`` on a DSDBCOO of that pattern.
* ``transport_small.npz`` -- nb=4, b=8, 6 energies of the seeded transport
  generator; upstream ``SanchoRubio`` (tol 1e-12) for both contacts, the OBC
  assembly of ``ElectronSolver._compute_obc`` and upstream
  ``RGF.selected_solve(..., return_retarded=True, return_current=True)``; all
  blocks stored.
* ``transport_cfg_small_subset.npz`` -- nb=16, b=64 at 4 of its 32 energies;
  reduced outputs (per-block density, per-block Frobenius norms, contact
  currents, traces) so the file stays small.
* ``observables_small.npz`` -- nb=5, b=8, 40 energies of the seeded transport
  generator: upstream ``observables.device_current`` on the upstream G^< with
  the Hamiltonian as the operator, the per-block density of states of
  upstream G^R and the energies that upstream ``ElectronSolver._filter_peaks``
  zeroes for a peak limit set to the median of the largest DOS slopes.

* ``spectral_small.npz`` -- upstream ``Spectral(Beyn(...))`` surface Green's
  functions of a seeded b=16 lead with a rank-4 coupling at 8 energies, with
  the NEVP eigenpairs of the first call and upstream Sancho-Rubio's result.
* ``dsdb_layouts.npz`` -- upstream DSDBCOO and DSDBCSR layouts (full and
  symmetric storage) of one seeded sparse BTD pattern with mixed block sizes,
  and upstream ``RGF.selected_solve`` on symmetric-storage operands.

Usage:  QTX_UPSTREAM=<upstream checkout> python tests/golden/make_golden.py [generator ...]
"""

from __future__ import annotations

import os
import sys
import tempfile
import warnings

import numpy as np

sys.dont_write_bytecode = True  # nothing is written next to the upstream sources
HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
UPSTREAM = os.environ.get("QTX_UPSTREAM")
if not UPSTREAM or not os.path.isdir(os.path.join(UPSTREAM, "src", "qttools")):
    sys.exit("make_golden.py: set QTX_UPSTREAM to the root of an upstream quatrex checkout "
             "(the directory that holds src/qttools)")

os.environ["QTX_ARRAY_MODULE"] = "numpy"
os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "qtx_numba_cache"))
sys.path.insert(0, os.path.join(HERE, "_mpi_shim"))
sys.path.insert(0, os.path.join(UPSTREAM, "src"))
sys.path.insert(0, REPO)

from scipy import sparse  # noqa: E402

from qttools.comm import comm  # noqa: E402

_cfg = {k: "device_mpi" for k in ("all_to_all", "all_gather", "all_reduce", "bcast")}
comm.configure(block_comm_size=1, block_comm_config=_cfg, stack_comm_config=_cfg, override=True)

from qttools.boundary_conditions.obc import SanchoRubio  # noqa: E402
from qttools.datastructures import DSDBCOO, DSDBCSR  # noqa: E402
from qttools.greens_function_solver import RGF  # noqa: E402
from qttools.greens_function_solver.solver import OBCBlocks  # noqa: E402

from quatrex_b200.workloads import make_device  # noqa: E402


def random_block(rng, m, n):
    """Seeded form of the upstream ``_random_block`` (50 % density, complex)."""
    coo = sparse.random(int(m), int(n), density=0.5, format="coo", random_state=rng).astype(np.complex128)
    coo.data += 1j * rng.uniform(size=coo.nnz)
    return coo.toarray()


def bt_dense(rng, block_sizes):
    """Seeded form of the upstream ``bt_dense`` fixture."""
    offs = np.hstack(([0], np.cumsum(block_sizes)))
    nb = len(block_sizes)
    n = int(offs[-1])
    arr = np.zeros((n, n), dtype=np.complex128)
    for i in range(nb):
        arr[offs[i]:offs[i + 1], offs[i]:offs[i + 1]] = random_block(rng, block_sizes[i], block_sizes[i]) + np.eye(block_sizes[i])
        if i > 0:
            arr[offs[i]:offs[i + 1], offs[i - 1]:offs[i]] = random_block(rng, block_sizes[i], block_sizes[i - 1])
            arr[offs[i - 1]:offs[i], offs[i]:offs[i + 1]] = random_block(rng, block_sizes[i - 1], block_sizes[i])
    for i in range(n):
        arr[i, i] = (1 + 1j) + complex(np.sum(arr[i, :]))
    return arr


def btd_case(name, block_sizes, stack, seed):
    rng = np.random.default_rng(seed)
    block_sizes = np.asarray(block_sizes)
    dense = bt_dense(rng, block_sizes)
    coo_a = sparse.coo_matrix(dense)
    coo_bl = sparse.coo_matrix(dense)
    coo_bl = coo_bl - coo_bl.conj().T
    coo_bg = sparse.coo_matrix(dense)
    coo_bg = coo_bg - coo_bg.conj().T
    a = DSDBCOO.from_sparray(coo_a, block_sizes, (stack,))
    bl = DSDBCOO.from_sparray(sparse.coo_matrix(coo_bl), block_sizes, (stack,))
    bg = DSDBCOO.from_sparray(sparse.coo_matrix(coo_bg), block_sizes, (stack,))
    solver = RGF(max_batch_size=2)
    x_inv = solver.selected_inv(a)
    xl, xg, xr = solver.selected_solve(a, bl, bg, return_retarded=True)
    np.savez_compressed(
        os.path.join(HERE, f"btd_{name}.npz"),
        block_sizes=block_sizes,
        stack=np.int64(stack),
        a=dense,
        sigma_lesser=coo_bl.toarray(),
        sigma_greater=coo_bg.toarray(),
        inv=x_inv.to_dense()[0],
        xl=xl.to_dense()[0],
        xg=xg.to_dense()[0],
        xr=xr.to_dense()[0],
    )
    print(f"btd_{name}: n={dense.shape[0]} nnz={coo_a.nnz}")


def dsdbcoo_from_blocks(diag, upper, lower):
    """Full BTD DSDBCOO over the energy stack with the given dense blocks."""
    sizes = np.array([d.shape[-1] for d in diag])
    offs = np.hstack(([0], np.cumsum(sizes)))
    n = int(offs[-1])
    ne = diag[0].shape[0]
    pattern = np.zeros((n, n), dtype=np.complex128)
    for i in range(len(diag)):
        pattern[offs[i]:offs[i + 1], max(offs[i - 1] if i > 0 else 0, 0):offs[min(i + 2, len(diag))]] = 1.0
    coo = sparse.coo_matrix(pattern)
    m = DSDBCOO.from_sparray(coo, sizes, (ne,))
    for i in range(len(diag)):
        m.blocks[i, i] = diag[i]
        if i + 1 < len(diag):
            m.blocks[i, i + 1] = upper[i]
            m.blocks[i + 1, i] = lower[i]
    return m


def transport_reference(dev, energies):
    diag, upper, lower = dev.system_blocks(energies)
    nb = len(diag)
    sr = SanchoRubio(max_iterations=dev.sr_max_iter, convergence_tol=dev.sr_tol)
    g_l = sr(diag[0], upper[0], lower[0], contact="left")
    g_r = sr(diag[-1], lower[-1], upper[-1], contact="right")
    sig_l = lower[0] @ g_l @ upper[0]
    sig_r = upper[-1] @ g_r @ lower[-1]
    f_l = 1.0 / (1.0 + np.exp((energies - dev.mu_left) / dev.kt))
    f_r = 1.0 / (1.0 + np.exp((energies - dev.mu_right) / dev.kt))
    gam_l = 1j * (sig_l - sig_l.conj().swapaxes(-2, -1))
    gam_r = 1j * (sig_r - sig_r.conj().swapaxes(-2, -1))
    obc = OBCBlocks(num_blocks=nb)
    obc.retarded[0], obc.retarded[-1] = sig_l, sig_r
    obc.lesser[0] = 1j * f_l[:, None, None] * gam_l
    obc.lesser[-1] = 1j * f_r[:, None, None] * gam_r
    obc.greater[0] = 1j * (f_l - 1)[:, None, None] * gam_l
    obc.greater[-1] = 1j * (f_r - 1)[:, None, None] * gam_r
    a = dsdbcoo_from_blocks(diag, upper, lower)
    zero = [np.zeros_like(d) for d in diag]
    zu = [np.zeros_like(u) for u in upper]
    zl = [np.zeros_like(l_) for l_ in lower]
    s_l = dsdbcoo_from_blocks(zero, zu, zl)
    s_g = dsdbcoo_from_blocks(zero, zu, zl)
    solver = RGF(max_batch_size=100)
    xl, xg, xr, cur = solver.selected_solve(a, s_l, s_g, obc_blocks=obc, return_retarded=True, return_current=True)
    x_inv = solver.selected_inv(a, obc_blocks=obc)
    return dict(diag=diag, upper=upper, lower=lower, obc=obc, g_l=g_l, g_r=g_r, xl=xl, xg=xg, xr=xr,
                current=cur, inv=x_inv, f_l=f_l, f_r=f_r)


def blocks_of(m, nb):
    d = np.stack([m.blocks[i, i] for i in range(nb)], axis=1)
    u = np.stack([m.blocks[i, i + 1] for i in range(nb - 1)], axis=1)
    lo = np.stack([m.blocks[i + 1, i] for i in range(nb - 1)], axis=1)
    return d, u, lo


def transport_small():
    dev = make_device(num_blocks=4, block_size=8, num_energies=6, seed=7)
    r = transport_reference(dev, dev.energies)
    nb = 4
    out = dict(h_diag=dev.h_diag, h_upper=dev.h_upper, energies=dev.energies,
               sigma_r_left=r["obc"].retarded[0], sigma_r_right=r["obc"].retarded[-1],
               sigma_l_left=r["obc"].lesser[0], sigma_l_right=r["obc"].lesser[-1],
               sigma_g_left=r["obc"].greater[0], sigma_g_right=r["obc"].greater[-1],
               g_surface_left=r["g_l"], g_surface_right=r["g_r"], current=r["current"])
    for key in ("xl", "xg", "xr", "inv"):
        d, u, lo = blocks_of(r[key], nb)
        out[f"{key}_diag"], out[f"{key}_upper"], out[f"{key}_lower"] = d, u, lo
    np.savez_compressed(os.path.join(HERE, "transport_small.npz"), **out)
    print("transport_small written")


def transport_cfg_small_subset():
    dev = make_device(num_blocks=16, block_size=64, num_energies=32, seed=1234)
    idx = np.array([0, 9, 17, 31])
    r = transport_reference(dev, dev.energies[idx])
    nb = 16
    out = dict(energy_index=idx, energies=dev.energies[idx], current=r["current"])
    for key in ("xl", "xg", "xr"):
        d, u, lo = blocks_of(r[key], nb)
        out[f"{key}_diag_fro"] = np.linalg.norm(d, axis=(-2, -1))
        out[f"{key}_diag_trace"] = np.trace(d, axis1=-2, axis2=-1)
        if key != "xr":
            out[f"{key}_upper_fro"] = np.linalg.norm(u, axis=(-2, -1))
        out[f"{key}_block_density"] = np.diagonal(d, axis1=-2, axis2=-1).imag.sum(-1)
        out[f"{key}_first_block"] = d[:, 0]
    out["sigma_r_left_fro"] = np.linalg.norm(r["obc"].retarded[0], axis=(-2, -1))
    out["sigma_r_right_fro"] = np.linalg.norm(r["obc"].retarded[-1], axis=(-2, -1))
    xl_d, _, _ = blocks_of(r["xl"], nb)
    xg_d, _, _ = blocks_of(r["xg"], nb)
    i_left = np.trace(r["obc"].greater[0] @ xl_d[:, 0] - xg_d[:, 0] @ r["obc"].lesser[0], axis1=-2, axis2=-1)
    i_right = np.trace(r["obc"].greater[-1] @ xl_d[:, -1] - xg_d[:, -1] @ r["obc"].lesser[-1], axis1=-2, axis2=-1)
    out["i_left"], out["i_right"] = i_left, i_right
    np.savez_compressed(os.path.join(HERE, "transport_cfg_small_subset.npz"), **out)
    print("transport_cfg_small_subset written")


def observables_small():
    from quatrex.core.observables import device_current
    from quatrex.electron.solver import ElectronSolver

    dev = make_device(num_blocks=5, block_size=8, num_energies=40, seed=21)
    r = transport_reference(dev, dev.energies)
    nb, b = 5, 8
    n = nb * b
    h = np.zeros((n, n), dtype=np.complex128)
    for i in range(nb):
        h[i * b:(i + 1) * b, i * b:(i + 1) * b] = dev.h_diag[i]
        if i + 1 < nb:
            h[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] = dev.h_upper[i]
            h[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] = dev.h_upper[i].conj().T
    current = device_current(r["xl"], sparse.coo_matrix(h))
    # per-block DOS of upstream G^R, the quantity _filter_peaks differentiates
    diag = r["xr"].diagonal()
    dos = np.stack([-diag[..., i * b:(i + 1) * b].imag.mean(-1) for i in range(nb)], axis=-1)
    slopes = np.abs(np.gradient(dos, dev.energies, axis=0)).max(axis=1)
    limit = float(np.median(slopes))

    class _Solver:  # the two attributes _filter_peaks reads
        energies = dev.energies
        dos_peak_limit = limit

    xl, xg, xr = r["xl"], r["xg"], r["xr"]
    before = np.abs(xr.data).sum(axis=-1)
    ElectronSolver._filter_peaks(_Solver(), (xl, xg, xr))
    mask = (np.abs(xr.data).sum(axis=-1) == 0) & (before > 0)
    np.savez_compressed(os.path.join(HERE, "observables_small.npz"), h_diag=dev.h_diag, h_upper=dev.h_upper,
                        energies=dev.energies, layer_current=np.asarray(current), dos=dos, peak_limit=limit,
                        peak_mask=mask)
    print("observables_small written", int(mask.sum()), "of", len(mask), "energies masked")


def spectral_small():
    """Upstream Spectral(Beyn) surface Green's functions of a seeded lead
    whose cells couple through 4 of their 16 orbitals (workloads.make_lead,
    8 energies; Beyn with r_o=10, r_i=0.8, m_0=16, 20 quadrature points, the
    other Spectral parameters at their defaults), with the eigenpairs of the
    first call and the Sancho-Rubio result of the same lead."""
    from qttools.boundary_conditions.obc import Spectral
    from qttools.nevp import Beyn

    from quatrex_b200.workloads import make_lead

    a_ii, a_ij, a_ji, energies = make_lead(16, 4, 8, seed=5)
    out = {"energies": energies, "r_o": 10.0, "r_i": 0.8, "m_0": 16, "num_quad_points": 20,
           "a_ii": a_ii, "a_ij": a_ij, "a_ji": a_ji}
    bij = np.broadcast_to(a_ij, a_ii.shape).copy()
    bji = np.broadcast_to(a_ji, a_ii.shape).copy()
    nevp = Beyn(r_o=10.0, r_i=0.8, m_0=16, num_quad_points=20)
    ws, vs = nevp((bji, a_ii, bij))
    nevp.rng = np.random.default_rng(42)  # the probe block of a first call again
    out["x"] = Spectral(nevp=nevp)(a_ii, bij, bji, contact="left")
    out["ws"], out["vs"] = ws, vs
    out["x_sancho_rubio"] = SanchoRubio(max_iterations=200, convergence_tol=1e-12)(a_ii, bij, bji, contact="left")
    np.savez_compressed(os.path.join(HERE, "spectral_small.npz"), **out)
    print("spectral_small written")


def _rowptr_arrays(m):
    keys = sorted(m.rowptr_map.keys())
    ptrs = [np.asarray(m.rowptr_map[k], dtype=np.int64) for k in keys]
    return (np.array(keys, dtype=np.int64).reshape(-1, 2), np.concatenate(ptrs),
            np.array([len(p) for p in ptrs], dtype=np.int64))


def dsdb_layouts():
    """Upstream DSDBCOO / DSDBCSR layouts (full and symmetric storage) of one
    seeded sparse BTD pattern with mixed block sizes, and upstream
    RGF.selected_solve on symmetric-storage operands: a complex-symmetric
    system matrix (symmetry_op = identity), skew-Hermitian self-energies and
    outputs (symmetry_op = -conj), G^R diagonal stored complex-symmetric, as
    quatrex's SCBA stores them (src/quatrex/core/scba.py:164-183)."""
    rng = np.random.default_rng(21)
    block_sizes = np.array([3, 3, 5, 4, 4, 3])
    dense = bt_dense(rng, block_sizes)
    out = {"block_sizes": block_sizes, "a": dense}
    for sym in (False, True):
        tag = "sym" if sym else "full"
        coo = DSDBCOO.from_sparray(sparse.coo_matrix(dense), block_sizes, (1,), symmetry=sym)
        out[f"coo_{tag}_rows"] = np.asarray(coo.rows)
        out[f"coo_{tag}_cols"] = np.asarray(coo.cols)
        out[f"coo_{tag}_data"] = np.asarray(coo.data[0])
        csr = DSDBCSR.from_sparray(sparse.coo_matrix(dense), block_sizes, (1,), symmetry=sym)
        keys, ptrs, lens = _rowptr_arrays(csr)
        out[f"csr_{tag}_cols"] = np.asarray(csr.cols)
        out[f"csr_{tag}_data"] = np.asarray(csr.data[0])
        out[f"csr_{tag}_keys"], out[f"csr_{tag}_ptrs"], out[f"csr_{tag}_lens"] = keys, ptrs, lens
    # symmetric-storage selected solve
    a_sym = 0.5 * (dense + dense.T)
    s = random_block(rng, dense.shape[0], dense.shape[0]) * (np.abs(dense) > 0)
    sl = s - s.conj().T
    s = random_block(rng, dense.shape[0], dense.shape[0]) * (np.abs(dense) > 0)
    sg = s - s.conj().T
    stack = 3
    ident = lambda x: x  # noqa: E731
    neg_conj = lambda x: -x.conj()  # noqa: E731
    A = DSDBCOO.from_sparray(sparse.coo_matrix(a_sym), block_sizes, (stack,), symmetry=True, symmetry_op=ident)
    SL = DSDBCOO.from_sparray(sparse.coo_matrix(sl), block_sizes, (stack,), symmetry=True, symmetry_op=neg_conj)
    SG = DSDBCOO.from_sparray(sparse.coo_matrix(sg), block_sizes, (stack,), symmetry=True, symmetry_op=neg_conj)
    xl = DSDBCOO.zeros_like(SL)
    xg = DSDBCOO.zeros_like(SL)
    xr = DSDBCOO.zeros_like(A)
    RGF(max_batch_size=2).selected_solve(A, SL, SG, out=[xl, xg, xr], return_retarded=True)
    out.update(sym_a=a_sym, sym_sigma_lesser=sl, sym_sigma_greater=sg, sym_xl=xl.to_dense()[0],
               sym_xg=xg.to_dense()[0], sym_xr=xr.to_dense()[0], sym_xl_data=np.asarray(xl.data[0]),
               sym_xr_data=np.asarray(xr.data[0]))
    np.savez_compressed(os.path.join(HERE, "dsdb_layouts.npz"), **out)
    print("dsdb_layouts written: nnz", len(out["coo_full_rows"]), "(symmetric", len(out["coo_sym_rows"]), ")")


if __name__ == "__main__":
    warnings.simplefilter("ignore", FutureWarning)
    if len(sys.argv) > 1:
        for name in sys.argv[1:]:
            globals()[name]()
        sys.exit(0)
    btd_case("constant", [2] * 10, 10, seed=11)
    btd_case("mixed", [2, 2, 2, 4, 4, 2, 2, 2], 10, seed=12)
    transport_small()
    transport_cfg_small_subset()
    observables_small()
    dsdb_layouts()
    spectral_small()
