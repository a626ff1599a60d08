"""Generates tests/golden/small_md.npz from the CPU oracle.

Scenario: 5x5x5 BCC Fe cells (250 sites), 2% vacancies, 3 octahedral
interstitials, 900 K Maxwell-Boltzmann velocities plus 0.05 A positional jitter
(seeds 11..14), the analytic Fe tables of misa_b200.potential.fe_analytic, a
stencil reach of cutoff + 0.7 A; one force evaluation at the start and 5
velocity-Verlet steps of dt = 1 fs.  Run from the repository root:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parents[1]))
import conftest  # noqa: E402,F401  (registers misa_b200)
import misa_b200 as mb  # noqa: E402
from oracle import oracle as orc  # noqa: E402
from scenarios import make  # noqa: E402


def main() -> None:
    orc.set_threads(1)
    sc = make(cells=(5, 5, 5), temperature=900.0, vacancy=0.02, n_itl=3, seed=11, jitter=0.05)
    pot = sc.orc_pot()
    dom = sc.orc_domain()
    even, odd = orc.stencil(dom, sc.a0, sc.reach)
    ext = sc.ext().view(orc.ATOM)
    itl = sc.itl.view(orc.ATOM).copy()
    ext0, itl0 = ext.copy(), itl.copy()
    orc.compute_forces(pot, dom, ext0, itl0, even, odd, sc.md_params())
    nsteps = 5
    e = orc.md_run(pot, dom, ext, itl, even, odd, sc.md_params(), nsteps)
    t = sc.tables
    np.savez_compressed(
        HERE / "small_md.npz",
        cells=np.array(sc.cells), ghost=np.array(sc.ghost), a0=sc.a0, mass=sc.mass, dt=sc.dt, cutoff=sc.cutoff,
        skin=sc.skin, dr=t.dr, drho=t.drho, f_tab=t.f, F_tab=t.F, phi_tab=t.phi,
        box_in=sc.box.view(np.uint8).reshape(-1, 104), itl_in=sc.itl.view(np.uint8).reshape(-1, 104),
        box_f0=mb.lattice.ext_to_box(ext0, sc.cells, sc.ghost).view(np.uint8).reshape(-1, 104),
        itl_f0=itl0.view(np.uint8).reshape(-1, 104),
        box_out=mb.lattice.ext_to_box(ext, sc.cells, sc.ghost).view(np.uint8).reshape(-1, 104),
        itl_out=itl.view(np.uint8).reshape(-1, 104), energies=e, even=even, odd=odd, nsteps=nsteps)
    print("wrote", HERE / "small_md.npz", "energies", e[:, 0] + e[:, 1])


if __name__ == "__main__":
    main()
