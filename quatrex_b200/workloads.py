"""Seeded synthetic transport devices (the inputs of the RGF benchmarks and tests).

The upstream project has no public benchmark dataset for this path, so every
workload is drawn from one seeded generator:

* ``H_ii = (X + X^H) / (2 sqrt(b)) + diag(U)``, X complex normal (real and
  imaginary parts N(0, 1/2)), U ~ N(0, 0.25) (standard deviation 0.5);
* ``H_i,i+1 = Y / (2 sqrt(b))``, Y complex normal, ``H_i+1,i = H_i,i+1^H``;
* S = I, ``A_ii(E) = (E + i eta) I - H_ii``, ``A_i,i+1 = -H_i,i+1``,
  ``A_i+1,i = -H_i,i+1^H`` (``src/quatrex/electron/solver.py:388-410`` with
  no potential and no scattering self-energy);
* energies uniform on [-2, 2] (``linspace``), eta = 1e-6;
* leads repeat the first and last cells; the contact self-energies come from
  Sancho-Rubio at tol 1e-12; Fermi occupancies at kT = 0.025 with
  mu_L = +0.1, mu_R = -0.1.

Draw order (fixed): X for all diagonal blocks (real then imaginary parts),
U, then Y (real then imaginary parts), all from ``numpy.random.default_rng(seed)``.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class TransportDevice:
    """A block-tridiagonal tight-binding device (energy independent part)."""

    h_diag: np.ndarray  # (nb, b, b) complex128
    h_upper: np.ndarray  # (nb-1, b, b) complex128, H[i, i+1]
    energies: np.ndarray  # (NE,) float64
    eta: float = 1e-6
    mu_left: float = 0.1
    mu_right: float = -0.1
    kt: float = 0.025
    sr_tol: float = 1e-12
    sr_max_iter: int = 200
    extra: dict = field(default_factory=dict)

    @property
    def num_blocks(self) -> int:
        return self.h_diag.shape[0]

    @property
    def block_size(self) -> int:
        return self.h_diag.shape[1]

    def system_blocks(self, energies: np.ndarray | None = None):
        """Dense block lists of A(E): (diag, upper, lower), each with a stack axis."""
        e = self.energies if energies is None else np.asarray(energies)
        b = self.block_size
        z = (e + 1j * self.eta)[:, None, None]
        eye = np.eye(b)
        diag = [z * eye - self.h_diag[i][None] for i in range(self.num_blocks)]
        upper = [np.broadcast_to(-self.h_upper[i], (len(e), b, b)).copy() for i in range(self.num_blocks - 1)]
        lower = [np.broadcast_to(-self.h_upper[i].conj().T, (len(e), b, b)).copy() for i in range(self.num_blocks - 1)]
        return diag, upper, lower


def make_device(num_blocks: int, block_size: int, num_energies: int, seed: int = 0,
                e_min: float = -2.0, e_max: float = 2.0, **kw) -> TransportDevice:
    """Draw one device with the seeded Hamiltonian generator."""
    nb, b = int(num_blocks), int(block_size)
    rng = np.random.default_rng(seed)
    xr = rng.standard_normal((nb, b, b))
    xi = rng.standard_normal((nb, b, b))
    x = (xr + 1j * xi) / np.sqrt(2.0)
    u = rng.normal(0.0, 0.5, size=(nb, b))
    yr = rng.standard_normal((max(nb - 1, 0), b, b))
    yi = rng.standard_normal((max(nb - 1, 0), b, b))
    y = (yr + 1j * yi) / np.sqrt(2.0)
    h_diag = (x + x.conj().swapaxes(-2, -1)) / (2.0 * np.sqrt(b))
    h_diag[:, np.arange(b), np.arange(b)] += u
    h_upper = y / (2.0 * np.sqrt(b))
    energies = np.linspace(e_min, e_max, int(num_energies))
    return TransportDevice(h_diag=h_diag, h_upper=h_upper, energies=energies, **kw)


# The workloads the benchmarks are quoted on.
CONFIG_SMALL = dict(num_blocks=16, block_size=64, num_energies=32, seed=1234)
"""nb=16, b=64, 32 energies: the CPU-runnable case."""

CONFIG_LARGE = dict(num_blocks=64, block_size=256, num_energies=1024, seed=1234)
"""nb=64, b=256, 1024 energies, complex128: the single-GPU scale-up."""


def uneven_instances(count: int, seed: int = 4321):
    """Size draw of the uneven batch: b log-uniform over {32,...,512},
    nb uniform in [8, 128], 64-512 energies; one seed per instance."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        b = int(2 ** rng.integers(5, 10))
        nb = int(rng.integers(8, 129))
        ne = int(rng.integers(64, 513))
        out.append(dict(num_blocks=nb, block_size=b, num_energies=ne, seed=seed + 1 + k))
    return out


def make_lead(block_size: int, coupling_rank: int, num_energies: int, seed: int = 0, e_min: float = -1.0,
              e_max: float = 1.0, eta: float = 1e-6):
    """Boundary blocks of a semi-infinite lead whose cells couple through
    their last / first ``coupling_rank`` orbitals only (as the boundary
    orbitals of a real wire do), for the spectral OBC: the quadratic
    eigenproblem (a_ji / w + a_ii + a_ij w) v = 0 then has 2 coupling_rank
    finite nonzero eigenvalues.  H_00 as in ``make_device``; the coupling
    block Y / sqrt(k) sits in rows b-k.., columns ..k.  Returns
    (a_ii (E, b, b), a_ij (b, b), a_ji (b, b), energies)."""
    b, k = int(block_size), int(coupling_rank)
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal((b, b)) + 1j * rng.standard_normal((b, b))) / np.sqrt(2.0)
    h = (x + x.conj().T) / (2.0 * np.sqrt(b)) + np.diag(rng.normal(0.0, 0.5, b))
    y = (rng.standard_normal((k, k)) + 1j * rng.standard_normal((k, k))) / np.sqrt(2.0)
    t = np.zeros((b, b), dtype=np.complex128)
    t[b - k:, :k] = y / np.sqrt(k)
    energies = np.linspace(e_min, e_max, int(num_energies))
    a_ii = (energies[:, None, None] + 1j * eta) * np.eye(b) - h[None]
    return a_ii, -t, -t.conj().T, energies
