"""Lattice <-> interstitial conversion on the device (FP64 path) against the oracle.

MISA-MD keeps atoms that have left their lattice site in its interstitial list; the
device-resident run does the same bookkeeping after every step (atoms farther than the
conversion distance from their site join the list in box order, interstitials within
the recombination distance of a vacant site take it in list order).  The oracle applies
the same rule (oracle/eam_oracle.c orc_convert) after each of its steps."""
from __future__ import annotations

import numpy as np
import pytest

import misa_b200 as mb
from oracle import oracle as orc
from scenarios import A0, MASS, RC, SKIN, rel_err

pytestmark = pytest.mark.gpu
D_CONV, D_REC = SKIN, 0.5 * SKIN


def _octahedral(cells, n_itl, seed, vac, temperature):
    """Interstitials at octahedral sites: they push neighbours off their sites."""
    box = mb.lattice.bcc_box(cells, A0)
    mb.lattice.add_vacancies(box, vac, seed)
    itl = mb.lattice.octahedral_interstitials(n_itl, cells, A0, seed)
    mb.lattice.maxwell_boltzmann(box, itl, temperature, MASS, seed + 4)
    return box, itl


def _oracle_run(box, itl0, cells, steps, dt, cap, conv=True):
    ghost = mb.lattice.ghost_for_reach(A0, RC + SKIN)
    dom = orc.make_domain(cells, ghost)
    even, odd = orc.stencil(dom, A0, RC + SKIN)
    ext = mb.lattice.box_to_ext(box, cells, ghost, A0).view(orc.ATOM)
    pot = orc.Pot.from_tables(mb.potential.fe_analytic())
    mp = orc.md_params(A0, MASS, dt, RC, SKIN)
    itl = np.zeros(cap, dtype=orc.ATOM)
    n = itl0.shape[0]
    itl[:n] = itl0.view(orc.ATOM)
    cnt = np.zeros(3, dtype=np.int64)
    orc.compute_forces(pot, dom, ext, itl[:n] if n else None, even, odd, mp)
    if conv:  # bookkeeping after every drift, before the new forces (the device's order)
        n = orc.md_run_convert(pot, dom, ext, itl, n, even, odd, mp, steps, D_CONV, D_REC, cnt)
    else:
        orc.md_run(pot, dom, ext, itl[:n] if n else None, even, odd, mp, steps, record=False)
    return mb.lattice.ext_to_box(ext.view(mb.ATOM_DTYPE), cells, ghost), itl[:n].view(mb.ATOM_DTYPE).copy(), cnt


def _sim(cells, cap, dt):
    return mb.Sim(cells, mb.potential.fe_analytic(), lattice_const=A0, mass=MASS, dt=dt, cutoff=RC,
                  stencil_skin=SKIN, max_interstitials=cap)


def test_conversion_matches_oracle_step_by_step():
    cells, steps, dt, cap = (7, 7, 7), 200, 1.0, 64
    box, itl0 = _octahedral(cells, 2, 7, 0.01, 900.0)
    bo, io, cnt = _oracle_run(box, itl0, cells, steps, dt, cap)
    assert cnt[0] >= 5 and cnt[1] >= 1 and cnt[2] == 0  # both directions of the bookkeeping ran
    with _sim(cells, cap, dt) as sim:
        sim.upload(box, itl0)
        sim.set_conversion(D_CONV, D_REC)
        sim.run(steps)
        st = sim.conversion_stats()
        bg, ig = sim.download()
    # The device also converts after the drift that ends its last step (the state it
    # reports is that step's start), so it may be one bookkeeping pass ahead of the oracle.
    assert st["converted"] >= cnt[0] and st["recombined"] >= cnt[1] and st["refused"] == 0
    assert st["n_itl"] == ig.shape[0]

    def by_id(b, i):
        a = np.concatenate([b[b["type"] >= 0], i])
        assert np.unique(a["id"]).size == a.shape[0]  # every atom once, on a site or in the list
        return a[np.argsort(a["id"])]

    ag, ao = by_id(bg, ig), by_id(bo, io)
    assert np.array_equal(ag["id"], ao["id"]) and np.array_equal(ag["type"], ao["type"])
    assert np.abs(ag["x"] - ao["x"]).max() < 1e-9
    assert np.abs(ag["v"] - ao["v"]).max() < 1e-9
    assert rel_err(ag["f"], ao["f"]) < 1e-9


def test_conversion_keeps_energy_with_octahedral_interstitials():
    # two octahedral interstitials at 900 K: the atoms they push off their sites break
    # the fixed stencil unless they are moved to the interstitial list
    cells, dt, steps = (8, 8, 8), 1.0, 1500
    box, itl = _octahedral(cells, 2, 7, 0.005, 900.0)
    n = int((box["type"] >= 0).sum()) + 2
    drift = {}
    for conv in (False, True):
        with _sim(cells, 64, dt) as sim:
            sim.upload(box, itl)
            if conv:
                sim.set_conversion(D_CONV, D_REC)
            sim.run(steps, energy_every=50)
            e = sim.energies()
            st = sim.conversion_stats()
        tot = e[:, 1] + e[:, 2]
        drift[conv] = np.abs(tot - tot[0]).max() / n
        if conv:
            assert st["converted"] > 0 and st["recombined"] > 0 and st["refused"] == 0
    assert drift[True] < 2e-5, drift
    assert drift[False] > 10 * drift[True], drift


def test_conversion_arguments_are_checked():
    with _sim((6, 6, 6), 0, 1.0) as sim:
        with pytest.raises(mb.MbError, match="max_interstitials"):
            sim.set_conversion(D_CONV, D_REC)
    with _sim((6, 6, 6), 8, 1.0) as sim:
        with pytest.raises(mb.MbError, match="recombine_distance"):
            sim.set_conversion(0.5, 0.5)
        sim.set_conversion(0.0, 0.0)  # off


def test_mixed_conversion_keeps_energy_with_octahedral_interstitials():
    # the same bookkeeping in the mixed-precision ensemble kernels
    cells, dt, steps = (8, 8, 8), 1.0, 1500
    box, itl = _octahedral(cells, 2, 7, 0.005, 900.0)
    n = int((box["type"] >= 0).sum()) + 2
    drift = {}
    for conv in (False, True):
        with mb.Sim(cells, mb.potential.fe_analytic(), lattice_const=A0, mass=MASS, dt=dt, cutoff=RC,
                    stencil_skin=SKIN, precision=mb.MB_PREC_MIXED, max_interstitials=64) as sim:
            sim.upload(box, itl)
            if conv:
                sim.set_conversion(D_CONV, D_REC)
            sim.run(steps, energy_every=50)
            e = sim.energies()
            st = sim.conversion_stats() if conv else None
            bg, ig = sim.download()
        tot = e[:, 1] + e[:, 2]
        drift[conv] = np.abs(tot - tot[0]).max() / n
        if conv:
            assert st["converted"] > 0 and st["recombined"] > 0 and st["refused"] == 0
            assert st["n_itl"] == ig.shape[0]
            a = np.concatenate([bg[bg["type"] >= 0], ig])
            assert np.unique(a["id"]).size == a.shape[0] == n  # every atom once
    assert drift[True] < 2e-5, drift
    assert drift[False] > 10 * drift[True], drift


def test_mixed_conversion_batched_equals_alone():
    # the bookkeeping of one lattice does not depend on what else is in the batch
    cells, steps = (8, 8, 8), 300
    box, itl = _octahedral(cells, 2, 7, 0.005, 900.0)
    other, oitl = _octahedral((9, 8, 10), 1, 3, 0.01, 600.0)

    def ens():
        return mb.Ensemble(mb.potential.fe_analytic(), lattice_const=A0, mass=MASS, dt=1.0, cutoff=RC,
                           stencil_skin=SKIN)

    with ens() as e:
        slot = e.add(cells, box, itl, steps=steps, max_interstitials=64)
        e.set_conversion(D_CONV, D_REC)
        e.run(steps)
        alone = e.download(slot)
        st_alone = e.conversion_stats(slot)
    with ens() as e:
        e.add((9, 8, 10), other, oitl, steps=steps, max_interstitials=32)
        slot = e.add(cells, box, itl, steps=steps, max_interstitials=64)
        e.set_conversion(D_CONV, D_REC)
        e.run(steps)
        mixed = e.download(slot)
        st_mixed = e.conversion_stats(slot)
    assert st_alone == st_mixed and st_alone["converted"] > 0
    for a, b in zip(alone, mixed):
        assert np.array_equal(a["id"], b["id"]) and np.array_equal(a["type"], b["type"])
        assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["f"], b["f"])
