"""CPU oracle for the spectral open-boundary condition (Beyn contour NEVP).

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` and by nothing in the
product package.  A plain NumPy restatement, on batched dense blocks, of the
upstream algorithms (paths relative to the upstream repository):

* ``beyn``        -- ``src/qttools/nevp/beyn.py:14-379`` (one-sided Beyn with
  the SVD projector, ``_contour_integrate`` ``:187-239``, ``_project_svd``
  ``:99-144``, ``_solve_reduced_system`` ``:241-289``, ``_one_sided``
  ``:291-330``) with the contour operator of
  ``src/qttools/kernels/operator.py:122-179``;
* ``spectral``    -- ``src/qttools/boundary_conditions/obc/spectral.py:15-526``
  for ``block_sections = 1``: mode filtering ``_find_reflected_modes``
  ``:196-322``, group velocity ``_compute_dE_dk`` ``:156-194``, normalisation
  ``_upscale_eigenmodes`` ``:324-372``, surface Green's function
  ``_compute_x_ii`` ``:374-418`` and the refinement iterations of ``__call__``
  ``:420-526``.

Parity of this restatement is pinned to fixtures written by the upstream code
(``tests/golden/make_golden.py`` -> ``tests/golden/spectral_small.npz``).
"""

from __future__ import annotations

import warnings

import numpy as np


def contour_points(r_o: float, r_i: float, num_quad_points: int):
    """Quadrature points on the outer and inner circle and their weight
    (``beyn.py:203-209``): phases exp(2 pi i (q + 1.5) / N), q = 0..N-1."""
    zeta = np.arange(num_quad_points) + 1
    phase = np.exp(2j * np.pi * (zeta + 0.5) / num_quad_points)
    return r_o * phase, r_i * phase, 1.0 / num_quad_points


def beyn_moments(a_ji, a_ii, a_ij, r_o, r_i, num_quad_points):
    """q0 = sum_q w (z_o T(z_o)^-1 - z_i T(z_i)^-1), q1 the same with z^2,
    T(z) = a_ji / z + a_ii + a_ij z (``beyn.py:187-239``, ``operator.py:122-179``)."""
    z_o, z_i, w = contour_points(r_o, r_i, num_quad_points)
    z_o = z_o.reshape(1, -1, 1, 1)
    z_i = z_i.reshape(1, -1, 1, 1)
    a_xx = [a[:, None] for a in (a_ji, a_ii, a_ij)]

    def inverse(z):
        # the contour operator sum_n z^n a_n, n = -1, 0, 1 (operator.py:155-157)
        return np.linalg.inv(sum(z ** n * a_x for a_x, n in zip(a_xx, range(-1, 2))))

    inv_o, inv_i = inverse(z_o), inverse(z_i)
    q0 = np.sum(w * z_o * inv_o - w * z_i * inv_i, axis=1)
    q1 = np.sum(w * z_o ** 2 * inv_o - w * z_i ** 2 * inv_i, axis=1)
    return q0, q1


def beyn_subspace(batch: int, d: int, m_0: int, rng: np.random.Generator):
    """The random probe block Y (``beyn.py:310-313``): real parts, then
    imaginary parts, from the solver's generator (seeded 42 at construction)."""
    return rng.random((batch, d, m_0)) + 1j * rng.random((batch, d, m_0))


def beyn(a_ji, a_ii, a_ij, r_o, r_i, m_0, num_quad_points, y):
    """Eigenpairs inside the annulus r_i < |w| < r_o of
    (a_ji / w + a_ii + a_ij w) v = 0; ws (batch, m_0) padded with zeros and vs
    (batch, d, m_0) padded with the columns of y (``beyn.py:241-330``)."""
    batch, d = a_ii.shape[0], a_ii.shape[-1]
    q0, q1 = beyn_moments(a_ji, a_ii, a_ij, r_o, r_i, num_quad_points)
    p0 = q0 @ y
    p1 = q1 @ y
    u, s, vh = np.linalg.svd(p0, full_matrices=False)
    ws = np.zeros((batch, m_0), dtype=np.complex128)
    vs = y.copy()
    for e in range(batch):
        keep = s[e] > s[e].max() * m_0 * np.finfo(p0.dtype).eps
        ui, si, vhi = u[e][:, keep], s[e][keep], vh[e][keep, :]
        a = ui.conj().T @ p1[e] @ vhi.conj().T / si
        w, v = np.linalg.eig(a)
        ws[e, : len(w)] = w
        vs[e, :, : len(w)] = ui @ v
    return ws, vs


def group_velocity(ws, vs, a_xx):
    """dE/dk = -sum_n (i n) diag(V^H a_n V) w^n over n = -1, 0, 1
    (``spectral.py:156-194``)."""
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        return -sum((1j * n) * np.diagonal(vs.conj().swapaxes(-1, -2) @ a_x @ vs, axis1=-2, axis2=-1) * ws ** n
                    for a_x, n in zip(a_xx, range(-1, 2)))


def reflected_modes(ws, vs, a_xx, min_decay=1e-3, max_decay=6.9, min_propagation=0.01, residual_tolerance=1e-3,
                    residual_normalization=True, eta_decay=1e-14):
    """Mask of the modes that propagate or decay into the lead
    (``spectral.py:196-322``)."""
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        products = sum(a_x @ vs * ws[..., None, :] ** (i - 1) for i, a_x in enumerate(a_xx))
        residuals = np.linalg.norm(products, axis=-2) / np.linalg.norm(vs, axis=-2)
        if residual_normalization:
            residuals = residuals / np.abs(ws)
        dedk = group_velocity(ws, vs, a_xx)
        ks = -1j * np.log(ws)
    dedk = np.nan_to_num(dedk, nan=0, posinf=0, neginf=0)
    ks = np.nan_to_num(ks, nan=0, posinf=0, neginf=0)
    eps = np.finfo(dedk.dtype).eps
    speed = np.abs(dedk.real) / (np.abs(dedk.imag) + eps)
    propagating = (np.abs(ks.imag) < min_decay) & (min_propagation < speed) & (dedk.real < 0)
    decaying = ks.imag < -min_decay
    decaying |= (min_propagation >= speed) & (ks.imag < -eta_decay)
    decaying &= ks.imag > -max_decay
    return (propagating | decaying) & (residuals < residual_tolerance)


def spectral(a_ii, a_ij, a_ji, r_o=10.0, r_i=0.8, m_0=10, num_quad_points=20, rng=None, y=None,
             num_ref_iterations=2, **filter_kw):
    """Surface Green's function of the spectral OBC (``spectral.py:420-526``,
    block_sections = 1).  Either ``y`` (the probe block) or ``rng`` (the Beyn
    solver's generator) must be given."""
    if a_ii.ndim == 2:
        a_ii, a_ij, a_ji = a_ii[None], a_ij[None], a_ji[None]
    batch, d = a_ii.shape[0], a_ii.shape[-1]
    a_ij = np.broadcast_to(a_ij, a_ii.shape)
    a_ji = np.broadcast_to(a_ji, a_ii.shape)
    if y is None:
        y = beyn_subspace(batch, d, m_0, rng)
    ws, vs = beyn(a_ji, a_ii, a_ij, r_o, r_i, m_0, num_quad_points, y)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        vs = vs / np.linalg.norm(vs, axis=-2, keepdims=True)
    mask = reflected_modes(ws, vs, (a_ji, a_ii, a_ij), **filter_kw)
    x_ii_a_ij = np.zeros_like(a_ii)
    for e in range(batch):
        vr = vs[e][:, mask[e]]
        w = ws[e][mask[e]]
        v_inv = np.linalg.inv(vr.conj().T @ vr) @ vr.conj().T
        x_ii_a_ij[e] = vr / w @ v_inv
    x = np.linalg.inv(a_ii + a_ji @ x_ii_a_ij)
    for _ in range(num_ref_iterations - 1):
        x = np.linalg.inv(a_ii - a_ji @ x @ a_ij)
    x = np.linalg.inv(a_ii - a_ji @ x @ a_ij)
    return x, {"ws": ws, "vs": vs, "mask": mask, "y": y}
