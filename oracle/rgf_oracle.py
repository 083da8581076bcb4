"""CPU oracle for the RGF selected inversion / selected solve path.

TEST INFRASTRUCTURE ONLY.  This module is the checker the CUDA path is compared
against; it is imported by ``tests/``, by ``__graft_entry__.smoke()`` and by the
CPU-baseline leg of ``bench.py``, and by nothing else.  The product package
(``quatrex_b200``) never imports it and has no CPU fallback.

It restates, in plain NumPy on dense block stacks, the algorithms of the
upstream qttools / quatrex code (paths relative to the upstream repository):

* ``selected_inv``   -- ``src/qttools/greens_function_solver/rgf.py:25-113``
* ``selected_solve`` -- ``src/qttools/greens_function_solver/rgf.py:115-414``
* ``sancho_rubio``   -- ``src/qttools/boundary_conditions/obc/sancho_rubio.py:33-86``
* ``obc_self_energies`` -- ``src/quatrex/electron/solver.py:305-386`` with
  ``src/qttools/utils/stack_utils.py:6-30`` and
  ``src/quatrex/core/statistics.py:7-23``
* ``get_batches``    -- ``src/qttools/utils/solvers_utils.py:7-32`` with
  ``src/qttools/utils/mpi_utils.py:16-67``
* ``layer_current``  -- ``src/quatrex/core/observables.py:192-237``
* ``block_dos``, ``peak_mask`` -- ``src/quatrex/electron/solver.py:412-454``

Parity of this restatement is pinned against the upstream implementation run
in the build container: ``tests/golden/make_golden.py`` imports the upstream
package and writes the fixtures under ``tests/golden/``; ``tests/test_oracle.py``
checks this module against them.

Block-stack convention used throughout: a block-tridiagonal matrix with ``nb``
blocks is given as three lists of arrays with a leading stack (energy) axis:
``diag[i] = A[i, i]`` (E, b_i, b_i), ``upper[i] = A[i, i+1]`` (E, b_i, b_{i+1})
and ``lower[i] = A[i+1, i]`` (E, b_{i+1}, b_i).
"""

from __future__ import annotations

import warnings

import numpy as np


def _h(x: np.ndarray) -> np.ndarray:
    """Conjugate transpose of the last two axes."""
    return x.conj().swapaxes(-2, -1)


def inv(a: np.ndarray) -> np.ndarray:
    """Batched dense inverse (``src/qttools/kernels/linalg/inv.py:6-40``)."""
    return np.linalg.inv(a)


def get_batches(num_sections: int, max_batch_size: int) -> tuple[list[int], np.ndarray]:
    """Stack batching of ``RGF`` (``src/qttools/utils/solvers_utils.py:7-32``).

    ``num_sections // min(max_batch_size, num_sections)`` near-equal sections,
    the first ``num_sections % n`` of them one larger
    (``src/qttools/utils/mpi_utils.py:16-67``, balanced strategy).
    """
    n = num_sections // min(max_batch_size, num_sections)
    base, rem = divmod(num_sections, n)
    sizes = [base + 1 if k < rem else base for k in range(n)]
    return sizes, np.hstack(([0], np.cumsum(sizes)))


def _with_obc(block: np.ndarray, obc: list | None, idx: int, sl: slice, sign: float) -> np.ndarray:
    if obc is None or obc[idx] is None:
        return block
    return block + sign * obc[idx][sl]


def selected_inv(diag, upper, lower, obc_retarded=None, max_batch_size: int = 100):
    """Selected inverse on the block-tridiagonal pattern.

    Follows ``src/qttools/greens_function_solver/rgf.py:25-113``:
    x_0 = inv(A_00 - S_0); forward x_j = inv(A_jj - S_j - A_ji x_i A_ij)
    (``:79-92``); backward X_ji = -X_jj A_ji x_i, X_ij = -x_i A_ij X_jj,
    X_ii = x_i - x_i A_ij X_ji (``:98-110``).  ``obc_retarded`` is a list of
    ``nb`` entries (None or (E, b, b)) that are subtracted from the diagonal.

    Returns (x_diag, x_upper, x_lower) lists with the layout of the input.
    """
    nb = len(diag)
    ne = diag[0].shape[0]
    sizes, offs = get_batches(ne, max_batch_size)
    x_diag = [np.zeros_like(d) for d in diag]
    x_upper = [np.zeros_like(u) for u in upper]
    x_lower = [np.zeros_like(l_) for l_ in lower]
    for bi in range(len(sizes)):
        sl = slice(int(offs[bi]), int(offs[bi + 1]))
        xd = [None] * nb
        xd[0] = inv(_with_obc(diag[0][sl], obc_retarded, 0, sl, -1.0))
        for i in range(nb - 1):
            j = i + 1
            a_jj = _with_obc(diag[j][sl], obc_retarded, j, sl, -1.0)
            xd[j] = inv(a_jj - lower[i][sl] @ xd[i] @ upper[i][sl])
        x_diag[nb - 1][sl] = xd[nb - 1]
        for i in range(nb - 2, -1, -1):
            j = i + 1
            x_ii, x_jj = xd[i], xd[j]
            x_ji = -x_jj @ lower[i][sl] @ x_ii
            x_lower[i][sl] = x_ji
            x_upper[i][sl] = -x_ii @ upper[i][sl] @ x_jj
            xd[i] = x_ii - x_ii @ upper[i][sl] @ x_ji
            x_diag[i][sl] = xd[i]
    return x_diag, x_upper, x_lower


def selected_solve(
    diag,
    upper,
    lower,
    sl_diag,
    sl_upper,
    sg_diag,
    sg_upper,
    obc_retarded=None,
    obc_lesser=None,
    obc_greater=None,
    max_batch_size: int = 100,
    return_current: bool = False,
    return_extras: bool = False,
    current_stale_coupling: bool = False,
):
    """Selected solve X^< = A^-1 S^< A^-H (and X^>), plus diagonal X^R.

    Follows ``src/qttools/greens_function_solver/rgf.py:115-414``:

    * first block ``:207-231`` and forward Keldysh recursion ``:233-295``, the
      OBC lesser/greater blocks are *added* to the diagonal self-energy
      (``:214-225``, ``:244-255``) and the retarded OBC block subtracted from A;
    * last diagonal blocks stored anti-Hermitian-symmetrised ``0.5 (X - X^H)``
      (``:297-305``);
    * backward sweep ``:307-404``; diagonal G^</G^> stored as ``0.5 (X - X^H)``
      (``:355-357``, ``:377-379``), lower off-diagonal ``-X_ij^H``
      (``:351-352``), diagonal G^R update ``:402``;
    * optional Meir-Wingreen layer current ``:381-400``.  The upstream code
      reads ``a_ji_dagger`` there, a name that the backward loop never assigns:
      it still holds ``A[nb-1, nb-2]^H`` from the last forward step (``:262``),
      so upstream interfaces other than the last use the wrong coupling.  This
      restatement uses the coupling of the interface itself (Meir-Wingreen as
      documented at ``:152-154``); ``current_stale_coupling=True`` reproduces
      the upstream behaviour bit for bit and exists only to pin this oracle
      against the upstream fixtures.

    ``sl_upper[i]``/``sg_upper[i]`` are the (i, i+1) blocks of Sigma^</Sigma^>.

    Returns a dict with ``xl_diag, xl_upper, xl_lower, xg_diag, xg_upper,
    xg_lower, xr_diag`` and, if requested, ``current`` (E, nb-1).  With
    ``return_extras`` it also holds the retarded off-diagonal blocks
    ``xr_upper`` (X_ij = -x_i A_ij X_jj, the product the upstream code forms as
    ``xr_ii_a_ij_xr_jj`` at ``:331``), ``xr_lower`` (X_ji = -X_jj A_ji x_i) and
    the corner block ``xr_corner`` = G^R[0, nb-1] built by the backward chain
    G_{i,N-1} = -x_i A_{i,i+1} G_{i+1,N-1}.
    """
    nb = len(diag)
    ne = diag[0].shape[0]
    sizes, offs = get_batches(ne, max_batch_size)
    out = {
        "xl_diag": [np.zeros_like(d) for d in diag],
        "xg_diag": [np.zeros_like(d) for d in diag],
        "xr_diag": [np.zeros_like(d) for d in diag],
        "xl_upper": [np.zeros_like(u) for u in upper],
        "xg_upper": [np.zeros_like(u) for u in upper],
        "xl_lower": [np.zeros_like(l_) for l_ in lower],
        "xg_lower": [np.zeros_like(l_) for l_ in lower],
    }
    if return_extras:
        out["xr_upper"] = [np.zeros_like(u) for u in upper]
        out["xr_lower"] = [np.zeros_like(l_) for l_ in lower]
        out["xr_corner"] = np.zeros((ne, diag[0].shape[1], diag[-1].shape[2]), dtype=diag[0].dtype)
    if return_current:
        out["current"] = np.zeros((ne, nb - 1), dtype=diag[0].dtype)

    for bi in range(len(sizes)):
        sl = slice(int(offs[bi]), int(offs[bi + 1]))
        xr = [None] * nb
        xl = [None] * nb
        xg = [None] * nb

        a_jj = _with_obc(diag[0][sl], obc_retarded, 0, sl, -1.0)
        sl_jj = _with_obc(sl_diag[0][sl], obc_lesser, 0, sl, +1.0)
        sg_jj = _with_obc(sg_diag[0][sl], obc_greater, 0, sl, +1.0)
        xr_jj = inv(a_jj)
        xr[0] = xr_jj
        xl[0] = xr_jj @ sl_jj @ _h(xr_jj)
        xg[0] = xr_jj @ sg_jj @ _h(xr_jj)

        for i in range(nb - 1):
            j = i + 1
            a_jj = _with_obc(diag[j][sl], obc_retarded, j, sl, -1.0)
            sl_jj = _with_obc(sl_diag[j][sl], obc_lesser, j, sl, +1.0)
            sg_jj = _with_obc(sg_diag[j][sl], obc_greater, j, sl, +1.0)
            a_ji = lower[i][sl]
            a_ji_h = _h(a_ji)
            a_ji_xr_ii = a_ji @ xr[i]
            xr_jj = inv(a_jj - a_ji_xr_ii @ upper[i][sl])
            xr_jj_h = _h(xr_jj)
            xr[j] = xr_jj
            w = a_ji_xr_ii @ sl_upper[i][sl]
            xl[j] = xr_jj @ (sl_jj + a_ji @ xl[i] @ a_ji_h + _h(w) - w) @ xr_jj_h
            w = a_ji_xr_ii @ sg_upper[i][sl]
            xg[j] = xr_jj @ (sg_jj + a_ji @ xg[i] @ a_ji_h + _h(w) - w) @ xr_jj_h

        n = nb - 1
        out["xl_diag"][n][sl] = 0.5 * (xl[n] - _h(xl[n]))
        out["xg_diag"][n][sl] = 0.5 * (xg[n] - _h(xg[n]))
        out["xr_diag"][n][sl] = xr[n]
        if return_extras:
            corner = xr[n]

        for i in range(nb - 2, -1, -1):
            j = i + 1
            xr_ii, xr_jj = xr[i], xr[j]
            a_ij, a_ji = upper[i][sl], lower[i][sl]
            xl_ii, xl_jj = xl[i], xl[j]
            xg_ii, xg_jj = xg[i], xg[j]
            s_l_ij, s_g_ij = sl_upper[i][sl], sg_upper[i][sl]

            xr_jj_h = _h(xr_jj)
            xr_ii_a_ij = xr_ii @ a_ij
            a_ij_h_xr_ii_h = _h(xr_ii_a_ij)
            xr_jj_a_ji = xr_jj @ a_ji
            a_ji_h_xr_jj_h = _h(xr_jj_a_ji)
            xr_ii_a_ij_xr_jj = xr_ii_a_ij @ xr_jj
            xr_jj_h_a_ij_h_xr_ii_h = _h(xr_ii_a_ij_xr_jj)
            xr_ii_a_ij_xr_jj_a_ji = xr_ii_a_ij @ xr_jj_a_ji

            if return_extras:
                out["xr_upper"][i][sl] = -xr_ii_a_ij_xr_jj
                out["xr_lower"][i][sl] = -xr_jj_a_ji @ xr_ii
                corner = -xr_ii_a_ij @ corner

            t1 = xr_ii_a_ij_xr_jj_a_ji @ xl_ii - xr_ii @ s_l_ij @ xr_jj_h_a_ij_h_xr_ii_h
            t1 = t1 - _h(t1)
            t2 = xr_ii_a_ij @ xl_jj
            xl_ij = -t2 - xl_ii @ a_ji_h_xr_jj_h + xr_ii @ s_l_ij @ xr_jj_h
            out["xl_upper"][i][sl] = xl_ij
            out["xl_lower"][i][sl] = -_h(xl_ij)
            xl[i] = xl_ii + t2 @ a_ij_h_xr_ii_h + t1
            out["xl_diag"][i][sl] = 0.5 * (xl[i] - _h(xl[i]))

            t1 = xr_ii_a_ij_xr_jj_a_ji @ xg_ii - xr_ii @ s_g_ij @ xr_jj_h_a_ij_h_xr_ii_h
            t1 = t1 - _h(t1)
            t2 = xr_ii_a_ij @ xg_jj
            xg_ij = -t2 - xg_ii @ a_ji_h_xr_jj_h + xr_ii @ s_g_ij @ xr_jj_h
            out["xg_upper"][i][sl] = xg_ij
            out["xg_lower"][i][sl] = -_h(xg_ij)
            xg[i] = xg_ii + t2 @ a_ij_h_xr_ii_h + t1
            out["xg_diag"][i][sl] = 0.5 * (xg[i] - _h(xg[i]))

            if return_current:
                a_ji_xr_ii = a_ji @ xr_ii
                a_ji_h = _h(lower[nb - 2][sl]) if current_stale_coupling else _h(a_ji)
                w = a_ji_xr_ii @ s_l_ij
                s_l_tilde = a_ji @ xl_ii @ a_ji_h + _h(w) - w
                w = a_ji_xr_ii @ s_g_ij
                s_g_tilde = a_ji @ xg_ii @ a_ji_h + _h(w) - w
                out["current"][sl, i] = np.trace(
                    s_g_tilde @ xl[j] - xg[j] @ s_l_tilde, axis1=-2, axis2=-1
                )

            xr[i] = xr_ii + xr_ii_a_ij_xr_jj_a_ji @ xr_ii
            out["xr_diag"][i][sl] = xr[i]

        if return_extras:
            out["xr_corner"][sl] = corner
    return out


def sancho_rubio(a_ii, a_ij, a_ji, max_iterations: int = 100, convergence_tol: float = 1e-6):
    """Sancho-Rubio surface Green's function.

    Follows ``src/qttools/boundary_conditions/obc/sancho_rubio.py:33-86``:
    eps <- eps - a inv(eps) b - b inv(eps) a, eps_s <- eps_s - a inv(eps) b,
    a <- a inv(eps) a, b <- b inv(eps) b with a = a_ji, b = a_ij, until
    max_E ||(|a| + |b|)||_F / 2 < tol; returns (inv(eps_s), iterations).
    A RuntimeWarning is raised when ``max_iterations`` is reached (``:81-82``).
    """
    eps = a_ii.copy()
    eps_s = a_ii.copy()
    alpha = a_ji.copy()
    beta = a_ij.copy()
    it = 0
    for it in range(1, max_iterations + 1):
        inverse = inv(eps)
        a_inv_b = alpha @ inverse @ beta
        eps = eps - a_inv_b - beta @ inverse @ alpha
        eps_s = eps_s - a_inv_b
        alpha = alpha @ inverse @ alpha
        beta = beta @ inverse @ beta
        delta = np.linalg.norm(np.abs(alpha) + np.abs(beta), axis=(-2, -1)).max() / 2
        if delta < convergence_tol:
            break
    else:
        warnings.warn("Surface Green's function did not converge.", RuntimeWarning)
    return inv(eps_s), it


def fermi_dirac(energy, kt: float):
    """Fermi-Dirac occupancy 1 / (1 + exp(E / kT)) (``src/quatrex/core/statistics.py:7-23``,
    with k_B T given directly in the energy unit)."""
    return 1.0 / (1.0 + np.exp(energy / kt))


def obc_self_energies(diag, upper, lower, energies, mu_left, mu_right, kt, tol=1e-12, max_iterations=200):
    """Contact self-energies of a device whose leads repeat its end cells.

    Follows ``src/quatrex/electron/solver.py:305-386`` with
    ``get_periodic_superblocks`` as the identity (``block_sections=1``,
    ``src/quatrex/core/utils.py:157-212``) and no extra OBC broadening:

    * left: g = SR(A_00, A_01, A_10); Sigma^R = A_10 g A_01 (``:318-326``);
    * right: g = SR(A_nn, A_nm, A_mn) (the upstream flips are a permutation
      similarity and cancel, ``:340-370``); Sigma^R = A_mn g A_nm (``:375``);
    * Gamma = i (Sigma - Sigma^H); Sigma^< = i f Gamma; Sigma^> = i (f - 1) Gamma
      (``:328-337``, ``:377-386``; ``scale_stack`` multiplies per energy).

    Returns dict with retarded/lesser/greater [left, right], the surface
    Green's functions and the Sancho-Rubio iteration counts.
    """
    g_l, it_l = sancho_rubio(diag[0], upper[0], lower[0], max_iterations, tol)
    g_r, it_r = sancho_rubio(diag[-1], lower[-1], upper[-1], max_iterations, tol)
    sig_l = lower[0] @ g_l @ upper[0]
    sig_r = upper[-1] @ g_r @ lower[-1]
    f_l = fermi_dirac(energies - mu_left, kt)[:, None, None]
    f_r = fermi_dirac(energies - mu_right, kt)[:, None, None]
    gam_l = 1j * (sig_l - _h(sig_l))
    gam_r = 1j * (sig_r - _h(sig_r))
    return {
        "retarded": [sig_l, sig_r],
        "lesser": [1j * f_l * gam_l, 1j * f_r * gam_r],
        "greater": [1j * (f_l - 1) * gam_l, 1j * (f_r - 1) * gam_r],
        "gamma": [gam_l, gam_r],
        "surface": [g_l, g_r],
        "iterations": [it_l, it_r],
    }


def caroli_transmission(gr_corner, gamma_left, gamma_right):
    """T(E) = Tr[Gamma_L G^R_{0,N-1} Gamma_R (G^R_{0,N-1})^H] (Caroli).

    The upstream NEGF path has no transmission output; this definition is
    cross-checked against its contact current
    (``src/quatrex/core/observables.py:130-189``) in the ballistic case,
    T = -I_left / (f_L - f_R).
    """
    prod = gamma_left @ gr_corner @ gamma_right @ _h(gr_corner)
    return np.trace(prod, axis1=-2, axis2=-1).real


def block_density(x_diag):
    """Per-block sum of Im diag(X_ii) (``src/quatrex/core/observables.py:57-82``,
    summed over the orbitals of each block); returns (E, nb)."""
    return np.stack([np.diagonal(x, axis1=-2, axis2=-1).imag.sum(-1) for x in x_diag], axis=-1)


def contact_currents(xl_first, xg_first, xl_last, xg_last, obc):
    """Contact currents (``src/quatrex/core/observables.py:130-189``)."""
    i_left = np.trace(obc["greater"][0] @ xl_first - xg_first @ obc["lesser"][0], axis1=-2, axis2=-1)
    i_right = np.trace(obc["greater"][1] @ xl_last - xg_last @ obc["lesser"][1], axis1=-2, axis2=-1)
    return i_left, i_right


def block_dos(xr_diag):
    """Per-block mean of -Im diag(G^R_ii): the local density of states that
    ``ElectronSolver._filter_peaks`` builds (``src/quatrex/electron/solver.py:428-434``);
    returns (E, nb)."""
    return np.stack([-np.diagonal(x, axis1=-2, axis2=-1).imag.mean(-1) for x in xr_diag], axis=-1)


def layer_current(xl_upper, h_upper):
    """``observables.device_current`` (``src/quatrex/core/observables.py:192-237``)
    with the Hamiltonian as the operator: for interface i (j = i + 1),
    sum(H_ij * (G^<_ji)^T - G^<_ij * (H_ji)^T) over the block, with the stored
    lower block G^<_ji = -(G^<_ij)^H and H_ji = H_ij^H; returns (E, nb - 1)."""
    out = []
    for g, h in zip(xl_upper, h_upper):
        g_ji = -_h(g)
        h_ji = _h(h)
        out.append((h * g_ji.swapaxes(-2, -1) - g * h_ji.swapaxes(-2, -1)).sum(axis=(-1, -2)))
    return np.stack(out, axis=-1)


def peak_mask(dos, energies, dos_peak_limit):
    """Energies at which ``ElectronSolver._filter_peaks`` zeroes G^<, G^>, G^R
    (``src/quatrex/electron/solver.py:436-454``): the largest |d dos / dE| over
    the blocks above ``dos_peak_limit``, or the largest dos above 10.  ``dos``
    is (E, nb); the derivative is numpy.gradient along the energy grid."""
    grad = np.abs(np.gradient(dos, energies, axis=0))
    return (grad.max(axis=1) > dos_peak_limit) | (dos.max(axis=1) > 10)


def dense_from_blocks(diag, upper, lower):
    """Dense (E, N, N) matrix from the block lists (for cross-checks)."""
    sizes = [d.shape[-1] for d in diag]
    offs = np.hstack(([0], np.cumsum(sizes)))
    ne = diag[0].shape[0]
    out = np.zeros((ne, offs[-1], offs[-1]), dtype=diag[0].dtype)
    for i, d in enumerate(diag):
        out[:, offs[i]:offs[i + 1], offs[i]:offs[i + 1]] = d
    for i in range(len(diag) - 1):
        out[:, offs[i]:offs[i + 1], offs[i + 1]:offs[i + 2]] = upper[i]
        out[:, offs[i + 1]:offs[i + 2], offs[i]:offs[i + 1]] = lower[i]
    return out
