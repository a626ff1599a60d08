"""Tabulated EAM potentials for the misa_b200 library (host side).

``fe_analytic`` builds the synthetic Fe potential the benchmarks use:
phi(r) = A (rc - r)^2 (1 + B r), f(r) = (rc - r)^2, F(rho) = -sqrt(rho),
tabulated on uniform knots r in [0, rc] and rho in [0, rho_max].
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import _abi


@dataclasses.dataclass
class EamTables:
    n_types: int
    dr: float
    drho: float
    cutoff: float
    f: np.ndarray    # [n_types, nr]
    F: np.ndarray    # [n_types, nrho]
    phi: np.ndarray  # [n_types*(n_types+1)//2, nr]

    @property
    def nr(self) -> int:
        return self.f.shape[1]

    @property
    def nrho(self) -> int:
        return self.F.shape[1]

    def as_c(self) -> _abi.MbEamTables:
        """ctypes view; keeps references to the arrays on the returned struct."""
        f = np.ascontiguousarray(self.f, dtype=np.float64)
        F = np.ascontiguousarray(self.F, dtype=np.float64)
        phi = np.ascontiguousarray(self.phi, dtype=np.float64)
        t = _abi.MbEamTables(self.n_types, f.shape[1], F.shape[1], 0, self.dr, self.drho, self.cutoff,
                             _abi.dptr(f), _abi.dptr(F), _abi.dptr(phi))
        t._keep = (f, F, phi)
        return t


def fe_analytic(nr: int = 5000, nrho: int = 5000, cutoff: float = 5.6, rho_max: float = 50.0,
                A: float = 0.8, B: float = -0.2) -> EamTables:
    r = np.linspace(0.0, cutoff, nr)
    rho = np.linspace(0.0, rho_max, nrho)
    f = (cutoff - r) ** 2
    phi = A * (cutoff - r) ** 2 * (1.0 + B * r)
    F = -np.sqrt(rho)
    return EamTables(1, cutoff / (nr - 1), rho_max / (nrho - 1), cutoff, f[None, :], F[None, :], phi[None, :])


def alloy_analytic(n_types: int = 3, nr: int = 2000, nrho: int = 2000, cutoff: float = 5.6,
                   rho_max: float = 200.0) -> EamTables:
    """A multi-type variant of the same analytic family (types differ by scale)."""
    r = np.linspace(0.0, cutoff, nr)
    rho = np.linspace(0.0, rho_max, nrho)
    f = np.stack([(1.0 + 0.15 * a) * (cutoff - r) ** 2 for a in range(n_types)])
    F = np.stack([-(1.0 + 0.1 * a) * np.sqrt(rho) for a in range(n_types)])
    rows = []
    for a in range(n_types):
        for b in range(a, n_types):
            rows.append((0.8 + 0.05 * (a + b)) * (cutoff - r) ** 2 * (1.0 - 0.2 * r))
    return EamTables(n_types, cutoff / (nr - 1), rho_max / (nrho - 1), cutoff, f, F, np.stack(rows))
