"""Seeded lattice scenarios shared by the tests (host-side set-up only)."""
from __future__ import annotations

import dataclasses

import numpy as np

import misa_b200 as mb
from oracle import oracle as orc

A0 = 2.855
MASS = 55.845
RC = 5.6
SKIN = 0.7


@dataclasses.dataclass
class Scenario:
    cells: tuple
    box: np.ndarray
    itl: np.ndarray
    tables: object
    ghost: tuple
    a0: float = A0
    mass: float = MASS
    dt: float = 1.0
    cutoff: float = RC
    skin: float = SKIN

    @property
    def reach(self) -> float:
        return self.cutoff + self.skin

    def ext(self) -> np.ndarray:
        return mb.lattice.box_to_ext(self.box, self.cells, self.ghost, self.a0)

    def domain(self):
        return mb.lattice.domain(self.cells, self.ghost)

    def orc_domain(self):
        return orc.make_domain(self.cells, self.ghost)

    def stencil(self):
        d = self.domain()
        return mb.lattice.stencil_linear(self.a0, self.reach, d.ext_size_x, d.ext_size_y)

    def orc_pot(self):
        return orc.Pot.from_tables(self.tables)

    def md_params(self):
        return orc.md_params(self.a0, self.mass, self.dt, self.cutoff, 1.0)


def make(cells=(5, 5, 5), temperature=600.0, vacancy=0.0, n_itl=0, seed=1, jitter=0.05, tables=None,
         n_types=1, skin=SKIN) -> Scenario:
    tables = tables or (mb.potential.fe_analytic() if n_types == 1 else mb.potential.alloy_analytic(n_types))
    box = mb.lattice.bcc_box(cells, A0)
    rng = np.random.default_rng(seed + 100)
    if n_types > 1:
        box["type"] = rng.integers(0, n_types, size=box.shape[0])
    mb.lattice.add_vacancies(box, vacancy, seed)
    itl = mb.lattice.octahedral_interstitials(n_itl, cells, A0, seed + 1)
    if n_types > 1 and n_itl:
        itl["type"] = rng.integers(0, n_types, size=n_itl)
    mb.lattice.maxwell_boltzmann(box, itl, temperature, MASS, seed + 2)
    live = box["type"] >= 0
    box["x"][live] += rng.normal(0.0, jitter, size=(int(live.sum()), 3))
    ghost = mb.lattice.ghost_for_reach(A0, RC + skin)
    return Scenario(tuple(cells), box, itl, tables, ghost, skin=skin)


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """max |a-b| / max(|b|, floor) over rows (vectors: per-row norm)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.ndim == 1:
        return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
    d = np.linalg.norm(a - b, axis=-1)
    return float(np.max(d) / max(np.max(np.linalg.norm(b, axis=-1)), 1e-300))
