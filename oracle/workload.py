"""Seeded synthetic workloads for the CPU oracle — TEST INFRASTRUCTURE ONLY.

The lattice set-up MISA-MD's host does before it calls the plugin (BCC box in the
doubled-x index, vacancies, octahedral interstitials, Maxwell-Boltzmann velocities,
the periodic ghost fill of the ext array) and the analytic Fe potential tabulated at
5000 knots, restated in numpy so that the CPU reference arm of the benchmark and the
oracle-side parity checks build their inputs without loading the product library.
tests/test_oracle.py checks that these arrays are byte-for-byte the ones the product
package builds from the same seeds.

Index convention (MISA-MD's, which the reference kernels assume,
src/kernels/kernel_itl.hpp:21-46): x is doubled, unit cell (cx, cy, cz) holds sites
gx = 2 cx and 2 cx + 1; the ideal position of site (gx, gy, gz) is
(gx a0 / 2, (gy + (gx & 1) / 2) a0, (gz + (gx & 1) / 2) a0).  Box order is
((gz ny) + gy) (2 nx) + gx.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import oracle as orc

KB_EV = 8.617333262e-5    # eV / K
FTM2V = 9.64853321233e-3  # (eV/A)/amu -> A/fs^2
MVV2E = 1.0 / FTM2V       # amu A^2/fs^2 -> eV

A0, MASS, RC, SKIN, DT = 2.855, 55.845, 5.6, 0.7, 1.0

# the six octahedral sites of a BCC unit cell, in units of a0
OCTAHEDRAL = np.array([[0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5],
                       [0.5, 0.0, 0.0], [0.0, 0.5, 0.0], [0.0, 0.0, 0.5]])


@dataclasses.dataclass
class Tables:
    n_types: int
    dr: float
    drho: float
    cutoff: float
    f: np.ndarray
    F: np.ndarray
    phi: np.ndarray


def fe_tables(nr: int = 5000, nrho: int = 5000, cutoff: float = RC, rho_max: float = 50.0, A: float = 0.8,
              B: float = -0.2) -> Tables:
    """phi(r) = A (rc - r)^2 (1 + B r), f(r) = (rc - r)^2, F(rho) = -sqrt(rho), tabulated
    on uniform knots r in [0, rc] and rho in [0, rho_max]."""
    r = np.linspace(0.0, cutoff, nr)
    rho = np.linspace(0.0, rho_max, nrho)
    f = (cutoff - r) ** 2
    phi = A * (cutoff - r) ** 2 * (1.0 + B * r)
    F = -np.sqrt(rho)
    return Tables(1, cutoff / (nr - 1), rho_max / (nrho - 1), cutoff, f[None, :], F[None, :], phi[None, :])


def bcc_box(cells, a0: float = A0) -> np.ndarray:
    nx, ny, nz = cells
    gz, gy, gx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(2 * nx), indexing="ij")
    h = 0.5 * (gx & 1)
    pos = np.stack([0.5 * a0 * gx, a0 * (gy + h), a0 * (gz + h)], axis=-1).reshape(-1, 3)
    a = np.zeros(pos.shape[0], dtype=orc.ATOM)
    a["id"] = np.arange(1, pos.shape[0] + 1)
    a["x"] = pos
    return a


def add_vacancies(box: np.ndarray, fraction: float, seed: int) -> None:
    rng = np.random.default_rng(seed)
    n = int(round(fraction * box.shape[0]))
    idx = rng.choice(box.shape[0], size=n, replace=False) if n else np.zeros(0, dtype=np.int64)
    box["type"][idx] = -1
    box["v"][idx] = 0.0


def octahedral_interstitials(n: int, cells, a0: float, seed: int, first_id: int = 1 << 40) -> np.ndarray:
    rng = np.random.default_rng(seed)
    nx, ny, nz = cells
    pick = rng.choice(nx * ny * nz * 6, size=n, replace=False) if n else np.zeros(0, dtype=np.int64)
    kind, cell = pick % 6, pick // 6
    c = np.stack([cell % nx, (cell // nx) % ny, cell // (nx * ny)], axis=-1)
    itl = np.zeros(n, dtype=orc.ATOM)
    itl["id"] = first_id + np.arange(n)
    itl["x"] = (c + OCTAHEDRAL[kind]) * a0
    return itl


def maxwell_boltzmann(box: np.ndarray, itl: np.ndarray | None, temperature: float, mass: float, seed: int) -> None:
    """Gaussian velocities, zero net momentum, scaled to (3N - 3)/2 kB T exactly."""
    rng = np.random.default_rng(seed)
    live = box["type"] >= 0
    n_live = int(live.sum())
    n_itl = 0 if itl is None else itl.shape[0]
    v = rng.normal(0.0, np.sqrt(KB_EV * temperature * FTM2V / mass), size=(n_live + n_itl, 3))
    v -= v.mean(axis=0)
    n = n_live + n_itl
    ke = 0.5 * mass * np.sum(v * v) * MVV2E
    if ke > 0 and temperature > 0:
        v *= np.sqrt(0.5 * (3 * n - 3) * KB_EV * temperature / ke)
    box["v"][live] = v[:n_live]
    box["v"][~live] = 0.0
    if n_itl:
        itl["v"] = v[n_live:]


def ghost_for_reach(a0: float, reach: float) -> tuple[int, int, int]:
    """Ghost widths (doubled x, y, z) that cover the oracle's stencil of this reach: the
    largest |dx|, |dy|, |dz| of its linear offsets (dx rounded up to even)."""
    ex, ey = 1 << 20, 1 << 10
    big = orc.Domain(0, 0, 0, ex, ey, 1, ex, ey, 1, 0, 0, 0, 0)
    e, o = orc.stencil(big, a0, reach)
    offs = np.concatenate([e, o])
    dz = np.rint(offs / float(ex * ey)).astype(np.int64)
    rem = offs - dz * ex * ey
    dy = np.rint(rem / float(ex)).astype(np.int64)
    dx = rem - dy * ex
    gx = int(np.abs(dx).max())
    return gx + (gx & 1), int(np.abs(dy).max()), int(np.abs(dz).max())


def box_to_ext(box: np.ndarray, cells, ghost, a0: float = A0) -> np.ndarray:
    """The host's ghost-extended AoS array: every ext record is its periodic box image."""
    bx, by, bz = 2 * cells[0], cells[1], cells[2]
    gx, gy, gz = ghost
    ex, ey, ez = bx + 2 * gx, by + 2 * gy, bz + 2 * gz
    zz, yy, xx = np.meshgrid(np.arange(ez) - gz, np.arange(ey) - gy, np.arange(ex) - gx, indexing="ij")
    sx, sy, sz = np.mod(xx, bx), np.mod(yy, by), np.mod(zz, bz)
    ext = box[((sz * by + sy) * bx + sx).reshape(-1)]
    L = np.array([cells[0] * a0, cells[1] * a0, cells[2] * a0])
    ext["x"] += np.stack([(xx - sx) // bx * L[0], (yy - sy) // by * L[1], (zz - sz) // bz * L[2]],
                         axis=-1).reshape(-1, 3)
    return ext


def ext_to_box(ext: np.ndarray, cells, ghost) -> np.ndarray:
    bx, by, bz = 2 * cells[0], cells[1], cells[2]
    gx, gy, gz = ghost
    e = ext.reshape(bz + 2 * gz, by + 2 * gy, bx + 2 * gx)
    return np.ascontiguousarray(e[gz:gz + bz, gy:gy + by, gx:gx + bx]).reshape(-1)


# The benchmark configurations, by name.  velocity_seed is the seed of the Maxwell-
# Boltzmann draw; seed the one of the vacancies and the interstitial sites.
CONFIGS = {
    # 20^3 cells, 16,000 atoms, 600 K from seed 42, 100 steps (the CPU-runnable case)
    "fe20": dict(cells=(20, 20, 20), temperature=600.0, vacancy=0.0, n_itl=0, seed=42, velocity_seed=42),
    # 128^3 cells (4,194,304 sites), 0.5% vacancies and 200 octahedral interstitials
    # from seed 7, 300 K
    "fe128": dict(cells=(128, 128, 128), temperature=300.0, vacancy=0.005, n_itl=200, seed=7, velocity_seed=1007),
    # 200^3 cells (16,000,000 sites), the same defect densities (763 interstitials), 900 K
    "fe200": dict(cells=(200, 200, 200), temperature=900.0, vacancy=0.005, n_itl=763, seed=7, velocity_seed=1007),
}


def build_state(cells, temperature: float, vacancy: float, n_itl: int, seed: int, velocity_seed: int,
                a0: float = A0, mass: float = MASS):
    """Box-order records and interstitials of a workload (no forces yet)."""
    box = bcc_box(cells, a0)
    add_vacancies(box, vacancy, seed)
    itl = octahedral_interstitials(n_itl, cells, a0, seed)
    maxwell_boltzmann(box, itl, temperature, mass, velocity_seed)
    return box, itl


def config_state(name: str, cells=None):
    """State of a named configuration, optionally on a different lattice size with the
    defect counts scaled to it."""
    c = dict(CONFIGS[name])
    full = c["cells"]
    cells = tuple(cells or full)
    n_itl = int(round(c["n_itl"] * np.prod(cells) / float(np.prod(full))))
    return build_state(cells, c["temperature"], c["vacancy"], n_itl, c["seed"], c["velocity_seed"])


class OracleRun:
    """The reference algorithm's state for a workload: ext array with its ghost fill,
    the interstitial list, the parity stencils and the potential, ready for
    oracle.md_run (forces at the starting positions already computed)."""

    def __init__(self, box: np.ndarray, itl: np.ndarray, cells, reach: float = RC + SKIN, a0: float = A0,
                 mass: float = MASS, dt: float = DT, cutoff: float = RC, tables: Tables | None = None):
        self.cells = tuple(cells)
        self.ghost = ghost_for_reach(a0, reach)
        self.dom = orc.make_domain(self.cells, self.ghost)
        self.even, self.odd = orc.stencil(self.dom, a0, reach)
        self.ext = box_to_ext(box, self.cells, self.ghost, a0)
        self.itl = np.ascontiguousarray(itl).copy() if itl is not None and itl.shape[0] else None
        self.pot = orc.Pot.from_tables(tables or fe_tables(cutoff=cutoff))
        self.mp = orc.md_params(a0, mass, dt, cutoff)
        self.n_atoms = int((box["type"] >= 0).sum()) + (0 if self.itl is None else self.itl.shape[0])
        self.pe, self.ke = orc.compute_forces(self.pot, self.dom, self.ext, self.itl, self.even, self.odd, self.mp)

    def steps(self, n: int, record: bool = False):
        """n velocity-Verlet steps; with record=True the (n + 1, 2) energies (pe, ke)."""
        return orc.md_run(self.pot, self.dom, self.ext, self.itl, self.even, self.odd, self.mp, n, record=record)

    def box(self) -> np.ndarray:
        return ext_to_box(self.ext, self.cells, self.ghost)
