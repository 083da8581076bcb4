"""OBC memoizer (OBCSystem) and the fixed-point step on the GPU, following the
upstream Sancho-Rubio tests (tests/qttools/boundary_conditions/obc/test_sancho_rubio.py:9-50)
on synthetic leads (the upstream fixture data are Git-LFS pointers)."""

import numpy as np
import pytest
import torch

from oracle import rgf_oracle as orc
from quatrex_b200.obc import OBCMemoizer, SanchoRubio, fixed_point_step, inverse
from quatrex_b200.workloads import make_device

pytestmark = pytest.mark.gpu


def _lead(seed=6, b=20, ne=7):
    dev = make_device(num_blocks=2, block_size=b, num_energies=ne, seed=seed)
    d, u, lo = dev.system_blocks()
    return d[0], u[0], lo[0]


def test_fixed_point_step_matches_oracle():
    a_ii, a_ij, a_ji = _lead()
    x, _ = orc.sancho_rubio(a_ii, a_ij, a_ji, 200, 1e-12)
    rel, ab, x_ref = fixed_point_step(a_ii, a_ij, a_ji, x)
    want = np.linalg.inv(a_ii - a_ji @ x @ a_ij)
    assert np.linalg.norm(x_ref - want) / np.linalg.norm(want) < 1e-10
    # residuals at the roundoff level differ between any two implementations;
    # compare them on the scale of 1e-10 |x|
    scale = np.linalg.norm(x, axis=(-2, -1))
    assert np.allclose(ab, np.linalg.norm(want - x, axis=(-2, -1)), rtol=1e-6, atol=1e-10 * scale.max())
    assert rel.max() < 1e-6


def test_inverse_wrapper():
    a_ii, _, _ = _lead()
    assert np.linalg.norm(inverse(a_ii) - np.linalg.inv(a_ii)) / np.linalg.norm(np.linalg.inv(a_ii)) < 1e-12


def test_memoizer_reuses_after_small_perturbation():
    """Upstream: a second call with a 1e-6 perturbation reuses the memoized
    solution and still satisfies the fixed-point equation."""
    a_ii, a_ij, a_ji = _lead()
    memo = OBCMemoizer(SanchoRubio(max_iterations=200, convergence_tol=1e-12))
    x1, rel1, ab1 = memo((a_ii, a_ij, a_ji), "left")
    assert not memo.last_reused
    assert rel1.max() < 1e-6
    x_ref, _ = orc.sancho_rubio(a_ii, a_ij, a_ji, 200, 1e-12)
    assert np.linalg.norm(x1 - x_ref) / np.linalg.norm(x_ref) < 1e-8
    a2 = a_ii + 1e-6 * np.eye(a_ii.shape[-1])
    x2, rel2, ab2 = memo((a2, a_ij, a_ji), "left")
    assert memo.last_reused
    want = np.linalg.inv(a2 - a_ji @ x2 @ a_ij)
    assert np.linalg.norm(x2 - want) / np.linalg.norm(want) < 0.2


def test_memoizer_off_always_solves():
    a_ii, a_ij, a_ji = _lead()
    memo = OBCMemoizer(SanchoRubio(max_iterations=200, convergence_tol=1e-12), memoization_mode="off")
    memo((a_ii, a_ij, a_ji), "right")
    memo((a_ii, a_ij, a_ji), "right")
    assert not memo.last_reused


def test_memoizer_warns_on_high_residual():
    a_ii, a_ij, a_ji = _lead()
    memo = OBCMemoizer(SanchoRubio(max_iterations=1, convergence_tol=1e-12), memoization_mode="off")
    with pytest.warns(RuntimeWarning, match="High error"):
        memo((a_ii, a_ij, a_ji), "left")


def test_memoizer_device_tensors():
    a_ii, a_ij, a_ji = (torch.from_numpy(x).cuda() for x in _lead())
    memo = OBCMemoizer(SanchoRubio(max_iterations=200, convergence_tol=1e-12))
    x, rel, ab = memo((a_ii, a_ij, a_ji), "left")
    assert isinstance(x, torch.Tensor) and x.is_cuda
    assert float(rel.max()) < 1e-6
