"""Edge cases of the FP64 path against the oracle: lattices with no atoms, with a single
atom, the smallest box the device-resident run takes, the smallest domain the hooks
take, every atom an interstitial neighbour, and lattices right at the size limits."""
from __future__ import annotations

import numpy as np
import pytest

import misa_b200 as mb
from oracle import oracle as orc
from scenarios import A0, MASS, RC, SKIN, make, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hooks():
    h = mb.Hooks(0)
    yield h
    mb.Hooks.clean()


def _hooks_setup(hooks, sc):
    dom = mb.lattice.domain(sc.cells, sc.ghost)
    hooks.domain_init(dom)
    even, odd = mb.lattice.stencil_linear(A0, sc.reach, dom.ext_size_x, dom.ext_size_y)
    hooks.nei_offset_init(even, odd)
    hooks.pot_init(sc.tables)
    return orc.make_domain(sc.cells, sc.ghost), even, odd


def _hook_passes(hooks, sc, ext):
    L = [c * A0 for c in sc.cells]
    odom = orc.make_domain(sc.cells, sc.ghost)
    hooks.rho_calc(ext, sc.cutoff)
    orc.ghost_fill(odom, ext.view(orc.ATOM), L, 2)
    hooks.force_calc(ext, sc.cutoff)


def test_all_vacant_lattice_leaves_every_record_as_it_was(hooks):
    sc = make(cells=(6, 6, 6), seed=3)
    _hooks_setup(hooks, sc)
    ext = sc.ext()
    ext["type"] = -1
    ext["rho"] = 7.0
    ext["f"] = 3.0
    before = ext.copy()
    _hook_passes(hooks, sc, ext)
    assert ext.tobytes() == before.tobytes()


def test_single_atom_in_a_vacant_lattice_feels_nothing(hooks):
    # one atom alone: no neighbour inside the cutoff, so rho = 0, df = F'(0), f = 0
    sc = make(cells=(6, 6, 6), seed=3, jitter=0.0)
    odom, even, odd = _hooks_setup(hooks, sc)
    box = sc.box.copy()
    box["type"] = -1
    box["type"][len(box) // 2] = 0
    ext = mb.lattice.box_to_ext(box, sc.cells, sc.ghost, A0)
    eo = ext.copy().view(orc.ATOM)
    _hook_passes(hooks, sc, ext)
    pot = sc.orc_pot()
    orc.rho_pass(pot, odom, eo, even, odd, sc.cutoff)
    bg = mb.lattice.ext_to_box(ext, sc.cells, sc.ghost)
    bo = mb.lattice.ext_to_box(eo.view(mb.ATOM_DTYPE), sc.cells, sc.ghost)
    k = len(box) // 2
    assert bg["rho"][k] == 0.0 and bo["rho"][k] == 0.0
    assert bg["df"][k] == bo["df"][k]
    assert np.all(bg["f"][k] == 0.0)


def test_smallest_hook_domain_matches_oracle(hooks):
    # box as thin as the ghost along every axis (2 x 2 x 2 cells, ghost (4, 2, 2)): every
    # neighbour of a box site may be a ghost record
    sc = make(cells=(2, 2, 2), temperature=900.0, seed=5, jitter=0.1)
    odom, even, odd = _hooks_setup(hooks, sc)
    ext = sc.ext()
    eo = ext.copy().view(orc.ATOM)
    _hook_passes(hooks, sc, ext)
    pot = sc.orc_pot()
    L = [c * A0 for c in sc.cells]
    orc.rho_pass(pot, odom, eo, even, odd, sc.cutoff)
    orc.ghost_fill(odom, eo, L, 2)
    orc.force_pass(pot, odom, eo, even, odd, sc.cutoff)
    bg = mb.lattice.ext_to_box(ext, sc.cells, sc.ghost)
    bo = mb.lattice.ext_to_box(eo.view(mb.ATOM_DTYPE), sc.cells, sc.ghost)
    assert rel_err(bg["rho"], bo["rho"]) < 1e-12
    assert rel_err(bg["f"], bo["f"]) < 1e-10


def test_smallest_device_resident_box_matches_oracle():
    # 5 cells = 14.3 A per edge: just over two interaction spheres (2 x 6.3 A)
    sc = make(cells=(5, 5, 5), temperature=600.0, vacancy=0.02, n_itl=1, seed=7, jitter=0.05)
    odom = sc.orc_domain()
    even, odd = orc.stencil(odom, A0, sc.reach)
    ext = sc.ext().view(orc.ATOM)
    itl = sc.itl.view(orc.ATOM).copy()
    eo = orc.md_run(sc.orc_pot(), odom, ext, itl, even, odd, sc.md_params(), 5)
    bo = mb.lattice.ext_to_box(ext.view(mb.ATOM_DTYPE), sc.cells, sc.ghost)
    with mb.Sim(sc.cells, sc.tables, lattice_const=A0, mass=MASS, dt=1.0, cutoff=RC, stencil_skin=SKIN,
                max_interstitials=1) as sim:
        sim.upload(sc.box, sc.itl)
        sim.run(5, energy_every=1)
        bg, ig = sim.download()
        eg = sim.energies()
    live = bo["type"] >= 0
    assert rel_err(bg["f"][live], bo["f"][live]) < 1e-10
    assert rel_err(ig["f"], itl["f"]) < 1e-10
    n = int(live.sum()) + 1
    assert np.max(np.abs(eg[:, 1] - eo[:, 0])) / n < 1e-12
    with pytest.raises(mb.MbError, match="2 \\* \\(cutoff"):
        mb.Sim((4, 5, 5), sc.tables, lattice_const=A0, cutoff=RC, stencil_skin=SKIN)


def test_every_site_within_reach_of_an_interstitial_matches_oracle():
    # a small box crowded with interstitials: every lattice site is flagged and computed
    # by the warp-per-item passes
    sc = make(cells=(5, 5, 6), temperature=300.0, n_itl=12, seed=13, jitter=0.02)
    odom = sc.orc_domain()
    even, odd = orc.stencil(odom, A0, sc.reach)
    ext = sc.ext().view(orc.ATOM)
    itl = sc.itl.view(orc.ATOM).copy()
    orc.md_run(sc.orc_pot(), odom, ext, itl, even, odd, sc.md_params(), 3)
    bo = mb.lattice.ext_to_box(ext.view(mb.ATOM_DTYPE), sc.cells, sc.ghost)
    with mb.Sim(sc.cells, sc.tables, lattice_const=A0, mass=MASS, dt=1.0, cutoff=RC, stencil_skin=SKIN,
                max_interstitials=12) as sim:
        sim.upload(sc.box, sc.itl)
        sim.run(3)
        bg, ig = sim.download()
    live = bo["type"] >= 0
    assert rel_err(bg["f"][live], bo["f"][live]) < 1e-10
    assert rel_err(ig["f"], itl["f"]) < 1e-10


def test_size_limits_are_refused_with_a_message():
    t = mb.potential.fe_analytic()
    with pytest.raises(mb.MbError, match="32-bit"):
        mb.Sim((1000, 1000, 600), t)  # 1.2 G sites: beyond the 32-bit split-layout offsets
    with pytest.raises(mb.MbError, match="edges"):
        mb.Ensemble(t).add((3000, 10, 10), np.zeros(2 * 3000 * 100, dtype=mb.ATOM_DTYPE))
