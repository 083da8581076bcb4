"""CPU emulation of the 3xTF32 precision form of the transport solve.

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` and by nothing in the
product package.  It answers one question by emulation on the host: how
accurate are density and transmission when the bulk block products of the
recursion run as 3xTF32 split products with FP32 accumulation (the precision
form the specification names), with the diagonal-block inverses, the contact
self-energies and an iterative-refinement residual in FP64?

* ``tf32``: round-to-nearest of FP32 values to TF32 (10 explicit mantissa
  bits; the 13 low bits of the FP32 mantissa are rounded away).
* ``mm3``: A B for complex128 operands as four real products, each the sum
  of three TF32 products hi*hi + hi*lo + lo*hi with FP32 accumulation, where
  hi = tf32(fp32(x)), lo = tf32(fp32(x) - hi) (the usual 3xTF32 split).
* ``transport_plain``: the per-source Keldysh recursion of the generator form
  with every block product through ``mm``: G^R blocks and the two contact
  responses X_L, X_R -> density and Caroli transmission.
* ``transport_refined``: block-column form.  The block columns of G^R at the
  two contacts, Y_0 = A^-1 E_0 and Y_N = A^-1 E_N, are solved with the
  Schur-complement factorisation built from ``mm`` products and FP64
  inverses; then one refinement pass R = E - A Y in FP64 (A is
  block-tridiagonal: three FP64 block products per block row), Y += A^-1 R
  with the same low-precision factorisation.  Density
  sum_r Im (f_L Y_0 Gamma_L Y_0^H + f_R Y_N Gamma_R Y_N^H)_rr and the
  transmission Tr[Gamma_L Y_N,0 Gamma_R Y_N,0^H] follow in FP64.

``fp64_units`` counts, per energy, the FP64 block operations each form keeps
(products and inverses, one unit = one b x b x b complex product): the floor
under any speed-up the low-precision products can give.
"""

from __future__ import annotations

import numpy as np


def tf32(x32: np.ndarray) -> np.ndarray:
    """Round FP32 values to TF32 (round half away from zero on the dropped bits)."""
    u = np.ascontiguousarray(x32, dtype=np.float32).view(np.uint32)
    r = ((u + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).astype(np.uint32)
    return r.view(np.float32)


def _split(x: np.ndarray):
    x32 = x.astype(np.float32)
    hi = tf32(x32)
    lo = tf32((x32 - hi).astype(np.float32))
    return hi, lo


def _real3(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    ah, al = _split(a)
    bh, bl = _split(b)
    acc = np.matmul(ah, bh)  # float32 accumulation
    acc = acc + np.matmul(ah, bl)
    acc = acc + np.matmul(al, bh)
    return acc.astype(np.float64)


def mm3(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Complex product with every real product in 3xTF32 / FP32 accumulation."""
    ar, ai, br, bi = a.real, a.imag, b.real, b.imag
    return (_real3(ar, br) - _real3(ai, bi)) + 1j * (_real3(ar, bi) + _real3(ai, br))


def mm64(a, b):
    return a @ b


def _h(x):
    return x.conj().swapaxes(-1, -2)


def transport_plain(diag, upper, lower, obc, f_l, f_r, mm=mm3):
    """Per-source recursion (the generator form's sweep) with products via
    ``mm`` and FP64 inverses; returns (density (E, nb), transmission (E,))."""
    nb = len(diag)
    s_r = [obc["retarded"][0]] + [None] * (nb - 2) + [obc["retarded"][1]]
    gam_l, gam_r = obc["gamma"]
    x = [None] * nb
    xl = [None] * nb
    m0 = diag[0] - s_r[0]
    x[0] = np.linalg.inv(m0)
    xl[0] = mm(mm(x[0], 1j * gam_l), _h(x[0]))
    for i in range(nb - 1):
        j = i + 1
        m = diag[j] - mm(mm(lower[i], x[i]), upper[i])
        if s_r[j] is not None:
            m = m - s_r[j]
        x[j] = np.linalg.inv(m)
        w = mm(x[j], lower[i])
        xl[j] = mm(mm(w, xl[i]), _h(w))
    # backward: full G^R diagonal, the corner G_{0,N} and the two responses
    g = [None] * nb
    yl = [None] * nb
    yr = [None] * nb
    g[-1] = x[-1]
    yl[-1] = xl[-1]
    yr[-1] = mm(mm(x[-1], 1j * gam_r), _h(x[-1]))
    corner = x[-1]  # G_{N,N}; G_{i,N} = -x_i A_{i,i+1} G_{i+1,N}
    col = [None] * nb
    col[-1] = x[-1]
    for i in range(nb - 2, -1, -1):
        j = i + 1
        p1 = mm(x[i], upper[i])  # x_i A_ij
        p4 = mm(p1, mm(g[j], lower[i]))  # x_i A_ij G_jj A_ji
        col[i] = -mm(p1, col[j])
        g[i] = x[i] + mm(p4, x[i])
        # X_L,i = X_L,i + P1 X_L,j P1^H + (P4 X_L,i - (P4 X_L,i)^H); X_R,i = P1 X_R,j P1^H
        t2 = mm(p1, yl[j])
        t1 = mm(p4, xl[i])
        t1 = t1 - _h(t1)
        yl[i] = xl[i] + mm(t2, _h(p1)) + t1
        yr[i] = mm(mm(p1, yr[j]), _h(p1))
    corner = col[0]
    density = np.stack([np.diagonal(f_l[:, None, None] * yl[i] + f_r[:, None, None] * yr[i], axis1=-2,
                                    axis2=-1).imag.sum(-1) for i in range(nb)], axis=-1)
    trans = np.trace(gam_l @ corner @ gam_r @ _h(corner), axis1=-2, axis2=-1).real
    return density, trans


def _factor(diag, upper, lower, s_r, mm):
    """Forward Schur complements (low-precision products, FP64 inverses)."""
    nb = len(diag)
    x = [None] * nb
    m = diag[0] - s_r[0]
    x[0] = np.linalg.inv(m)
    for i in range(nb - 1):
        j = i + 1
        m = diag[j] - mm(mm(lower[i], x[i]), upper[i])
        if s_r[j] is not None:
            m = m - s_r[j]
        x[j] = np.linalg.inv(m)
    return x


def _solve(x, upper, lower, rhs, mm):
    """A Y = rhs (block column, list of (E, b, b)) with the factorisation x:
    forward z_j = x_j (r_j - A_ji z_i), backward y_i = z_i - x_i A_ij y_j."""
    nb = len(x)
    z = [None] * nb
    z[0] = mm(x[0], rhs[0])
    for i in range(nb - 1):
        j = i + 1
        z[j] = mm(x[j], rhs[j] - mm(lower[i], z[i]))
    y = [None] * nb
    y[-1] = z[-1]
    for i in range(nb - 2, -1, -1):
        y[i] = z[i] - mm(mm(x[i], upper[i]), y[i + 1])
    return y


def _residual(diag, upper, lower, s_r, y, rhs):
    """R = rhs - (A - S) Y in FP64 on the block-tridiagonal pattern."""
    nb = len(diag)
    r = []
    for i in range(nb):
        a_ii = diag[i] - s_r[i] if s_r[i] is not None else diag[i]
        acc = a_ii @ y[i]
        if i > 0:
            acc = acc + lower[i - 1] @ y[i - 1]
        if i + 1 < nb:
            acc = acc + upper[i] @ y[i + 1]
        r.append(rhs[i] - acc)
    return r


def transport_refined(diag, upper, lower, obc, f_l, f_r, mm=mm3, refinements=1):
    """Block-column solves with low-precision factorisation and FP64
    refinement; returns (density, transmission)."""
    nb = len(diag)
    s_r = [obc["retarded"][0]] + [None] * (nb - 2) + [obc["retarded"][1]]
    gam_l, gam_r = obc["gamma"]
    ne, b = diag[0].shape[0], diag[0].shape[-1]
    eye = np.broadcast_to(np.eye(b, dtype=np.complex128), (ne, b, b))
    zero = np.zeros((ne, b, b), dtype=np.complex128)
    x = _factor(diag, upper, lower, s_r, mm)
    cols = []
    for src in (0, nb - 1):
        rhs = [eye if k == src else zero for k in range(nb)]
        y = _solve(x, upper, lower, rhs, mm)
        for _ in range(refinements):
            r = _residual(diag, upper, lower, s_r, y, rhs)
            d = _solve(x, upper, lower, r, mm)
            y = [a + c for a, c in zip(y, d)]
        cols.append(y)
    y0, yn = cols
    density = np.stack([np.diagonal(f_l[:, None, None] * (y0[i] @ (1j * gam_l) @ _h(y0[i]))
                                    + f_r[:, None, None] * (yn[i] @ (1j * gam_r) @ _h(yn[i])), axis1=-2,
                                    axis2=-1).imag.sum(-1) for i in range(nb)], axis=-1)
    corner = yn[0]
    trans = np.trace(gam_l @ corner @ gam_r @ _h(corner), axis1=-2, axis2=-1).real
    return density, trans


def fp64_units(nb: int, refinements: int = 1) -> dict:
    """FP64 block operations per energy that each form keeps (units of one
    b x b x b complex product; an inverse counts one), Sancho-Rubio excluded.
    plain 3xTF32: the nb inverses.  Refined block columns: the nb inverses,
    per refinement and contact column the residual (3 products per block
    row), and per contact column and block the product Y Gamma whose
    diagonal against Y^H gives the density (O(b^2) once Y Gamma exists)."""
    return {"fp64_form_products": 3 + 2 + (nb - 1) * 17 + 6,
            "plain_3xtf32_fp64": nb,
            "refined_fp64": nb + refinements * 2 * 3 * nb + 2 * nb}
