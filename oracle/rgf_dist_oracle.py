"""CPU oracle for the partitioned (nested-dissection) RGF, ``RGFDist``.

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` and by nothing in the
product package.  A plain NumPy restatement of the upstream algorithm with
the P block partitions (one per MPI rank upstream) held in one process
(paths relative to the upstream repository):

* ``src/qttools/greens_function_solver/rgf_dist.py:16-384`` -- the driver:
  per partition a Schur elimination, the reduced system of the partition
  boundary blocks, its solve, the scatter back and the per-partition
  selected inversion;
* ``src/qttools/greens_function_solver/_serinv.py`` -- ``downward_schur``
  ``:765-864`` (first partition), ``upward_schur`` ``:867-968`` (last),
  ``permuted_schur`` ``:971-1131`` (middle partitions, keeping their first
  block coupled through buffer blocks), ``ReducedSystem`` ``:41-762``
  (map ``:373-442``, solve ``:444-585``, map back ``:678-762``),
  ``downward_selinv`` ``:1134-1225``, ``upward_selinv`` ``:1228-1331``,
  ``permuted_selinv`` ``:1334-1531``.

Upstream RGFDist needs several MPI ranks, which the build container cannot
provide, so this restatement is pinned through its results: it returns the
same blocks as ``rgf_oracle.selected_inv`` / ``selected_solve`` (pinned to
upstream-written fixtures) to rounding (``tests/test_oracle.py``).

Block-stack convention as ``rgf_oracle``: ``diag[i]`` (E, b, b),
``upper[i] = A[i, i+1]``, ``lower[i] = A[i+1, i]``; Sigma^< / Sigma^> are
given by their diagonal and upper blocks (skew-Hermitian: lower = -upper^H).
"""

from __future__ import annotations

import numpy as np


def _h(x):
    return x.conj().swapaxes(-2, -1)


def _inv(x):
    return np.linalg.inv(x)


def partition_bounds(num_blocks: int, num_partitions: int) -> list[tuple[int, int]]:
    """Balanced contiguous partitions of the block axis, the first ones one
    block larger (``src/qttools/utils/mpi_utils.py:16-67``); every partition
    needs two blocks at least."""
    base, rem = divmod(num_blocks, num_partitions)
    sizes = [base + 1 if p < rem else base for p in range(num_partitions)]
    if min(sizes) < 2:
        raise ValueError("every partition needs at least two blocks")
    starts = np.concatenate(([0], np.cumsum(sizes)))
    return [(int(starts[p]), int(starts[p + 1])) for p in range(num_partitions)]


class _Part:
    """Blocks of one partition seen with local indices (global = s + local)."""

    def __init__(self, s, e, diag, upper, lower, sl, sg, obc):
        self.s, self.e, self.n = s, e, e - s
        self._d, self._u, self._lo = diag, upper, lower
        self._sl, self._sg = sl, sg
        self._obc = obc

    def a(self, i, j):
        gi, gj = self.s + i, self.s + j
        if gi == gj:
            return self._d[gi]
        return self._u[gi] if gj == gi + 1 else self._lo[gj]

    def sigma(self, which, i, j):
        d, u = self._sl if which == "l" else self._sg
        gi, gj = self.s + i, self.s + j
        if gi == gj:
            return d[gi]
        return u[gi] if gj == gi + 1 else -_h(u[gj])

    def a_obc(self, i):
        r = self._obc[0][self.s + i] if self._obc[0] is not None else None
        return self.a(i, i) if r is None else self.a(i, i) - r

    def s_obc(self, which, i):
        k = 1 if which == "l" else 2
        o = self._obc[k][self.s + i] if self._obc[k] is not None else None
        return self.sigma(which, i, i) if o is None else self.sigma(which, i, i) + o


def _downward_schur(p: _Part, st, ss):
    n = p.n
    xr = st["xr"]
    xr[0] = p.a_obc(0)
    if ss:
        for c in "lg":
            st["x" + c][0] = p.s_obc(c, 0)
    for i in range(n - 1):
        j = i + 1
        xr[i] = _inv(xr[i])
        if ss:
            for c in "lg":
                st["x" + c][i] = xr[i] @ st["x" + c][i] @ _h(xr[i])
        a_ji = p.a(j, i)
        a_ji_xr_ii = a_ji @ xr[i]
        xr[j] = p.a_obc(j) - a_ji_xr_ii @ p.a(i, j)
        if ss:
            for c in "lg":
                w = a_ji_xr_ii @ p.sigma(c, i, j)
                st["x" + c][j] = p.s_obc(c, j) + a_ji @ st["x" + c][i] @ _h(a_ji) + _h(w) - w


def _upward_schur(p: _Part, st, ss):
    n = p.n - 1
    xr = st["xr"]
    xr[n] = p.a_obc(n)
    if ss:
        for c in "lg":
            st["x" + c][n] = p.s_obc(c, n)
    for i in range(n, 0, -1):
        j = i - 1
        xr[i] = _inv(xr[i])
        if ss:
            for c in "lg":
                st["x" + c][i] = xr[i] @ st["x" + c][i] @ _h(xr[i])
        a_ji = p.a(j, i)
        a_ji_xr_ii = a_ji @ xr[i]
        xr[j] = p.a_obc(j) - a_ji_xr_ii @ p.a(i, j)
        if ss:
            for c in "lg":
                w = a_ji_xr_ii @ p.sigma(c, i, j)
                st["x" + c][j] = p.s_obc(c, j) + a_ji @ st["x" + c][i] @ _h(a_ji) + _h(w) - w


def _permuted_schur(p: _Part, st, ss):
    xr, bl, bu = st["xr"], st["xr_bl"], st["xr_bu"]
    bl[0] = p.a(0, 1)
    bu[0] = p.a(1, 0)
    xr[0] = p.a_obc(0)
    xr[1] = p.a_obc(1)
    if ss:
        for c in "lg":
            st["x" + c + "_bu"][0] = p.sigma(c, 1, 0)
            st["x" + c][0] = p.s_obc(c, 0)
            st["x" + c][1] = p.s_obc(c, 1)
    for i in range(1, p.n - 1):
        j = i + 1
        xr[i] = _inv(xr[i])
        a_ji = p.a(j, i)
        xr_ii = xr[i]
        xr_ji_xr_ii = bl[i - 1] @ xr_ii
        a_ji_xr_ii = a_ji @ xr_ii
        if ss:
            w = {c: a_ji_xr_ii @ p.sigma(c, i, j) for c in "lg"}
        xr[j] = p.a_obc(j) - a_ji_xr_ii @ p.a(i, j)
        bl[i] = -xr_ji_xr_ii @ p.a(i, j)
        bu[i] = -a_ji_xr_ii @ bu[i - 1]
        xr[0] = xr[0] - xr_ji_xr_ii @ bu[i - 1]
        if ss:
            for c in "lg":
                x = st["x" + c]
                xb = st["x" + c + "_bu"]
                x[i] = xr_ii @ x[i] @ _h(xr_ii)
                x[j] = p.s_obc(c, j) + a_ji @ x[i] @ _h(a_ji) + _h(w[c]) - w[c]
                # upstream writes the source term as Sigma^<_ij^H for the lesser
                # and -Sigma^>_ji for the greater component: the same block of
                # a skew-Hermitian operand
                xb[i] = a_ji @ x[i] @ _h(bl[i - 1]) + _h(p.sigma(c, i, j)) @ _h(xr_ji_xr_ii) - a_ji_xr_ii @ xb[i - 1]
                x[0] = x[0] + bl[i - 1] @ x[i] @ _h(bl[i - 1]) + _h(xb[i - 1]) @ _h(xr_ji_xr_ii) - xr_ji_xr_ii @ xb[i - 1]


def _reduced_solve(red, ss):
    """RGF on the reduced system (``_serinv.py:444-585``)."""
    xr, up, lo = red["xr"], red["up"], red["lo"]
    m = len(xr)
    for i in range(m - 1):
        xr[i] = _inv(xr[i])
        if ss:
            for c in "lg":
                red["x" + c][i] = xr[i] @ red["x" + c][i] @ _h(xr[i])
        xr_ji_xr_ii = lo[i] @ xr[i]
        xr[i + 1] = xr[i + 1] - xr_ji_xr_ii @ up[i]
        if ss:
            for c in "lg":
                w = xr_ji_xr_ii @ red["x" + c + "_up"][i]
                red["x" + c][i + 1] = red["x" + c][i + 1] + lo[i] @ red["x" + c][i] @ _h(lo[i]) + _h(w) - w
    xr[-1] = _inv(xr[-1])
    if ss:
        for c in "lg":
            x = red["x" + c]
            x[-1] = xr[-1] @ x[-1] @ _h(xr[-1])
            x[-1] = 0.5 * (x[-1] - _h(x[-1]))
    for i in range(m - 2, -1, -1):
        xr_ii, xr_jj, xr_ij, xr_ji = xr[i], xr[i + 1], up[i], lo[i]
        p1 = xr_ii @ xr_ij
        p2 = xr_jj @ xr_ji
        p3 = p1 @ xr_jj
        p4 = p1 @ p2
        if ss:
            for c in "lg":
                x, xu = red["x" + c], red["x" + c + "_up"]
                t1 = p4 @ x[i] - xr_ii @ xu[i] @ _h(p3)
                t1 = t1 - _h(t1)
                t2 = p1 @ x[i + 1]
                xu[i] = -t2 - x[i] @ _h(p2) + xr_ii @ xu[i] @ _h(xr_jj)
                x[i] = x[i] + t2 @ _h(p1) + t1
                x[i] = 0.5 * (x[i] - _h(x[i]))
        lo[i] = -p2 @ xr_ii
        up[i] = -p3
        xr[i] = xr_ii + p4 @ xr_ii


def _downward_selinv(p: _Part, st, out, ss):
    xr = st["xr"]
    for i in range(p.n - 2, -1, -1):
        j = i + 1
        xr_ii, xr_jj = xr[i], xr[j]
        a_ij, a_ji = p.a(i, j), p.a(j, i)
        xr_ii_a_ij = xr_ii @ a_ij
        xr_jj_a_ji = xr_jj @ a_ji
        p4 = xr_ii_a_ij @ xr_jj_a_ji
        if ss:
            for c in "lg":
                x = st["x" + c]
                s_ij = p.sigma(c, i, j)
                t1 = p4 @ x[i] - xr_ii @ s_ij @ _h(xr_ii_a_ij @ xr_jj)
                t1 = t1 - _h(t1)
                t2 = xr_ii_a_ij @ x[j]
                x_ij = -t2 - x[i] @ _h(xr_jj_a_ji) + xr_ii @ s_ij @ _h(xr_jj)
                out["x" + c][(i + p.s, j + p.s)] = x_ij
                x[i] = x[i] + t2 @ _h(xr_ii_a_ij) + t1
                out["x" + c][(i + p.s, i + p.s)] = 0.5 * (x[i] - _h(x[i]))
        out["xr"][(j + p.s, i + p.s)] = -xr_jj_a_ji @ xr_ii
        out["xr"][(i + p.s, j + p.s)] = -xr_ii_a_ij @ xr_jj
        xr[i] = xr_ii + p4 @ xr_ii
        out["xr"][(i + p.s, i + p.s)] = xr[i]


def _upward_selinv(p: _Part, st, out, ss):
    xr = st["xr"]
    for i in range(1, p.n):
        j = i - 1
        xr_ii, xr_jj = xr[i], xr[j]
        a_ij, a_ji = p.a(i, j), p.a(j, i)
        xr_ii_a_ij = xr_ii @ a_ij
        xr_jj_a_ji = xr_jj @ a_ji
        p4 = xr_ii_a_ij @ xr_jj_a_ji
        if ss:
            for c in "lg":
                x = st["x" + c]
                s_ij = p.sigma(c, i, j)
                t1 = xr_ii @ s_ij @ _h(xr_ii_a_ij @ xr_jj)
                t1 = t1 - _h(t1)
                t_x = xr_ii_a_ij @ x[j]
                x_ij = -t_x - x[i] @ _h(xr_jj_a_ji) + xr_ii @ s_ij @ _h(xr_jj)
                # block (j, i) of the output is the upper block of (j, j + 1)
                out["x" + c][(j + p.s, i + p.s)] = -_h(x_ij)
                t2 = p4 @ x[i]
                x[i] = x[i] + t_x @ _h(xr_ii_a_ij) - t1 + (t2 - _h(t2))
                out["x" + c][(i + p.s, i + p.s)] = 0.5 * (x[i] - _h(x[i]))
        out["xr"][(j + p.s, i + p.s)] = -xr_jj_a_ji @ xr_ii
        out["xr"][(i + p.s, j + p.s)] = -xr_ii_a_ij @ xr_jj
        xr[i] = xr_ii + p4 @ xr_ii
        out["xr"][(i + p.s, i + p.s)] = xr[i]


def _permuted_selinv(p: _Part, st, out, ss):
    xr, bu, bl = st["xr"], st["xr_bu"], st["xr_bl"]
    s = p.s
    for i in range(p.n - 2, 0, -1):
        xr_i, xr_ip1, xr_0 = xr[i], xr[i + 1], xr[0]
        a_i_ip1, a_ip1_i = p.a(i, i + 1), p.a(i + 1, i)
        bu_im1, bu_i, bl_im1, bl_i = bu[i - 1], bu[i], bl[i - 1], bl[i]
        xr_ip1_a_ip1_i = xr_ip1 @ a_ip1_i
        bu_i_bl_im1 = bu_i @ bl_im1
        b1 = a_i_ip1 @ xr_ip1 + bu_im1 @ bl_i
        b2 = a_i_ip1 @ bu_i + bu_im1 @ xr_0
        c1 = xr_ip1_a_ip1_i + bu_i_bl_im1
        c2 = bl_i @ a_ip1_i + xr_0 @ bl_im1
        tmp2 = xr_i @ (b1 @ a_ip1_i + b2 @ bl_im1)
        if ss:
            tmp3 = _h(c2)
            tmp4 = ((_h(xr_ip1_a_ip1_i) + _h(bu_i_bl_im1)) @ _h(a_i_ip1) + tmp3 @ _h(bu_im1)) @ _h(xr_i)
            for c in "lg":
                x, xb = st["x" + c], st["x" + c + "_bu"]
                x_i, x_ip1, x_0 = x[i], x[i + 1], x[0]
                s_i_ip1 = p.sigma(c, i, i + 1)
                tmp1 = a_i_ip1 @ xb[i] + bu_im1 @ x_0
                tmp5 = s_i_ip1 @ _h(bl_i) + xb[i - 1] @ _h(xr_0)
                tmp6 = s_i_ip1 @ _h(xr_ip1) + xb[i - 1] @ _h(bu_i) - a_i_ip1 @ x_ip1 + bu_im1 @ _h(xb[i])
                b31 = -_h(xb[i - 1])
                upper = xr_i @ tmp6 - x_i @ (_h(xr_ip1_a_ip1_i) + _h(bu_i_bl_im1))
                x[i] = (x_i + tmp2 @ x_i + x_i @ tmp4
                        - xr_i @ (b1 @ p.sigma(c, i + 1, i) + b2 @ b31 + (tmp5 - tmp1) @ _h(bu_im1)
                                  + tmp6 @ _h(a_i_ip1)) @ _h(xr_i))
                xb[i - 1] = xr_i @ (tmp5 - tmp1) - x_i @ tmp3
                out["x" + c][(i + s, i + 1 + s)] = upper
                out["x" + c][(i + s, i + s)] = 0.5 * (x[i] - _h(x[i]))
        out["xr"][(i + s, i + 1 + s)] = -xr_i @ b1
        out["xr"][(i + 1 + s, i + s)] = -c1 @ xr_i
        bu[i - 1] = -xr_i @ b2
        bl[i - 1] = -c2 @ xr_i
        xr[i] = xr_i + tmp2 @ xr_i
        out["xr"][(i + s, i + s)] = xr[i]
    out["xr"][(1 + s, s)] = bu[0]
    out["xr"][(s, 1 + s)] = bl[0]
    if ss:
        for c in "lg":
            out["x" + c][(s, 1 + s)] = -_h(st["x" + c + "_bu"][0])


def _run(diag, upper, lower, sl, sg, obc, num_partitions, ss):
    nb = len(diag)
    bounds = partition_bounds(nb, num_partitions)
    P = len(bounds)
    parts = [_Part(s, e, diag, upper, lower, sl, sg, obc) for s, e in bounds]
    states = []
    for p_idx, p in enumerate(parts):
        st = {"xr": [None] * p.n, "xr_bl": [None] * p.n, "xr_bu": [None] * p.n}
        for c in "lg":
            st["x" + c] = [None] * p.n
            st["x" + c + "_bu"] = [None] * p.n
        if p_idx == 0:
            _downward_schur(p, st, ss)
        elif p_idx == P - 1:
            _upward_schur(p, st, ss)
        else:
            _permuted_schur(p, st, ss)
        states.append(st)
    # reduced system of the 2 (P - 1) partition boundary blocks (_serinv.py:373-442)
    red = {"xr": [], "up": [], "lo": []}
    for c in "lg":
        red["x" + c], red["x" + c + "_up"] = [], []
    kel = "lg" if ss else ""
    for p_idx, (p, st) in enumerate(zip(parts, states)):
        if p_idx > 0:
            red["xr"].append(st["xr"][0])
            for c in kel:
                red["x" + c].append(st["x" + c][0])
            if p_idx < P - 1:
                red["lo"].append(st["xr_bu"][p.n - 2])
                red["up"].append(st["xr_bl"][p.n - 2])
                for c in kel:
                    red["x" + c + "_up"].append(-_h(st["x" + c + "_bu"][p.n - 2]))
        if p_idx < P - 1:
            red["xr"].append(st["xr"][p.n - 1])
            for c in kel:
                red["x" + c].append(st["x" + c][p.n - 1])
            red["up"].append(p.a(p.n - 1, p.n))
            red["lo"].append(p.a(p.n, p.n - 1))
            for c in kel:
                red["x" + c + "_up"].append(p.sigma(c, p.n - 1, p.n))
    _reduced_solve(red, ss)
    # map back (_serinv.py:678-762) and the per-partition selected inversion
    out = {"xr": {}, "xl": {}, "xg": {}}
    for p_idx, (p, st) in enumerate(zip(parts, states)):
        if p_idx > 0:
            k = 2 * p_idx - 1
            st["xr"][0] = red["xr"][k]
            for c in kel:
                st["x" + c][0] = red["x" + c][k]
            if p_idx < P - 1:
                st["xr_bu"][p.n - 2] = red["lo"][k]
                st["xr_bl"][p.n - 2] = red["up"][k]
                for c in kel:
                    st["x" + c + "_bu"][p.n - 2] = -_h(red["x" + c + "_up"][k])
        if p_idx < P - 1:
            k = 2 * p_idx
            st["xr"][p.n - 1] = red["xr"][k]
            gi, gj = p.e - 1, p.e
            out["xr"][(gi, gi)] = red["xr"][k]
            out["xr"][(gi, gj)] = red["up"][k]
            out["xr"][(gj, gi)] = red["lo"][k]
            for c in kel:
                st["x" + c][p.n - 1] = red["x" + c][k]
                out["x" + c][(gi, gi)] = red["x" + c][k]
                out["x" + c][(gi, gj)] = red["x" + c + "_up"][k]
        if p_idx > 0:
            out["xr"][(p.s, p.s)] = st["xr"][0]
            for c in kel:
                out["x" + c][(p.s, p.s)] = st["x" + c][0]
        if p_idx == 0:
            _downward_selinv(p, st, out, ss)
        elif p_idx == P - 1:
            _upward_selinv(p, st, out, ss)
        else:
            _permuted_selinv(p, st, out, ss)
    return out


def selected_inv(diag, upper, lower, obc_retarded=None, num_partitions: int = 2):
    """Selected inverse by P partitions (``rgf_dist.py:37-131``); returns
    (x_diag, x_upper, x_lower) lists like ``rgf_oracle.selected_inv``."""
    nb = len(diag)
    zero = [np.zeros_like(d) for d in diag]
    zu = [np.zeros_like(u) for u in upper]
    out = _run(diag, upper, lower, (zero, zu), (zero, zu), (obc_retarded, None, None), num_partitions, False)
    xr = out["xr"]
    return ([xr[(i, i)] for i in range(nb)], [xr[(i, i + 1)] for i in range(nb - 1)],
            [xr[(i + 1, i)] for i in range(nb - 1)])


def selected_solve(diag, upper, lower, sl_diag, sl_upper, sg_diag, sg_upper, obc_retarded=None, obc_lesser=None,
                   obc_greater=None, num_partitions: int = 2):
    """Selected solve by P partitions (``rgf_dist.py:133-384``); returns the
    dict layout of ``rgf_oracle.selected_solve`` (diagonal G^< / G^> stored
    0.5 (X - X^H), lower blocks -upper^H, diagonal and off-diagonal G^R)."""
    nb = len(diag)
    out = _run(diag, upper, lower, (sl_diag, sl_upper), (sg_diag, sg_upper), (obc_retarded, obc_lesser, obc_greater),
               num_partitions, True)
    res = {}
    for c in "lg":
        res[f"x{c}_diag"] = [out["x" + c][(i, i)] for i in range(nb)]
        res[f"x{c}_upper"] = [out["x" + c][(i, i + 1)] for i in range(nb - 1)]
        res[f"x{c}_lower"] = [-_h(u) for u in res[f"x{c}_upper"]]
    res["xr_diag"] = [out["xr"][(i, i)] for i in range(nb)]
    res["xr_upper"] = [out["xr"][(i, i + 1)] for i in range(nb - 1)]
    res["xr_lower"] = [out["xr"][(i + 1, i)] for i in range(nb - 1)]
    return res
