"""z-slab decomposition on one device: two and three slabs of one lattice, each a
separate slab sim, their ghost layers handed over between launches (LocalRing), give
bitwise the positions, velocities, forces, rho and df of the whole lattice advanced in
one piece, and the same energies (1e-12 eV/atom).  The slabs' kernels never wait on
one another: every exchange happens on the host between launches."""
from __future__ import annotations

import numpy as np
import pytest

import misa_b200 as mb
from misa_b200 import decomp
from scenarios import A0, MASS, make

pytestmark = pytest.mark.gpu


def _buffers(n):
    import torch
    return torch.empty(n, dtype=torch.uint8, device="cuda")


def _copy(dst, src):
    import torch
    dst.copy_(src)
    torch.cuda.synchronize()


@pytest.mark.parametrize("world", [2, 3])
def test_slabs_on_one_device_match_the_whole_lattice_bitwise(world):
    sc = make(cells=(8, 7, 12), temperature=900.0, vacancy=0.01, seed=91, jitter=0.05)
    nsteps = 6
    kw = dict(lattice_const=A0, mass=MASS, dt=1.0, cutoff=sc.cutoff, stencil_skin=sc.skin)
    with mb.Sim(sc.cells, sc.tables, **kw) as whole:
        whole.upload(sc.box)
        whole.run(nsteps, energy_every=1)
        ref, _ = whole.download()
        e_ref = whole.energies()
    ranks = [decomp.SlabRank(sc.cells, sc.tables, r, world, _buffers, **kw) for r in range(world)]
    ring = decomp.LocalRing(_copy)
    try:
        for r in ranks:
            r.upload(sc.box)
        decomp.exchange_codes(ranks, ring)
        for _ in range(nsteps + 1):  # the first step is the priming pass (forces at x_0)
            decomp.step_all(ranks, ring, energy=True)
        got = np.concatenate([r.sim.download()[0] for r in ranks])
        e = sum(r.sim.energies() for r in ranks)
    finally:
        for r in ranks:
            r.close()
    for k in ("type", "x", "v", "f", "rho", "df"):
        assert np.array_equal(got[k], ref[k]), k
    n = int((sc.box["type"] >= 0).sum())
    assert np.array_equal(e[:, 0] / world, e_ref[:, 0])
    assert np.max(np.abs(e[:, 1:] - e_ref[:, 1:])) / n < 1e-12


def test_slab_refuses_whole_lattice_stepping_and_thin_slabs():
    sc = make(cells=(8, 7, 12))
    with mb.Sim(sc.cells, sc.tables, slab=(0, 6)) as s:
        s.upload(decomp.slab_records(sc.box, sc.cells, 0, 6))
        with pytest.raises(mb.MbError, match="slab"):
            s.run(1)
    with pytest.raises(mb.MbError, match="ghost width"):
        mb.Sim(sc.cells, sc.tables, slab=(0, 1))
    with pytest.raises(mb.MbError, match="interstitials"):
        mb.Sim(sc.cells, sc.tables, slab=(0, 6), max_interstitials=4)
