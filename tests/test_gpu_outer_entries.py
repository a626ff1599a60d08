"""The force pass walks only the outer stencil entries (those beyond the cutoff at the
ideal lattice) that the density pass of the same positions found inside the cutoff for
some site of a work item.  A slab whose ghost positions are written again between the
two passes has no valid masks and walks every outer entry; on a strongly disordered
lattice, where many outer pairs come inside the cutoff and many stay out, both must give
bitwise the same trajectory."""
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


def _run(sc, nsteps, full_walk):
    kw = dict(lattice_const=A0, mass=MASS, dt=1.0, cutoff=sc.cutoff, stencil_skin=sc.skin)
    ranks = [decomp.SlabRank(sc.cells, sc.tables, r, 2, _buffers, **kw) for r in range(2)]
    ring = decomp.LocalRing(_copy)
    try:
        for r in ranks:
            r.upload(sc.box)
        decomp.exchange_codes(ranks, ring)
        for _ in range(nsteps + 1):
            halos = [r.pack(decomp.POS) for r in ranks]
            ring.exchange_all(halos)
            for r in ranks:
                r.unpack(decomp.POS)
            for r in ranks:
                r.sim.phase(0, True)
            if full_walk:  # the same ghost positions once more: the density pass's masks are dropped
                for r in ranks:
                    r.unpack(decomp.POS)
            halos = [r.pack(decomp.DF) for r in ranks]
            ring.exchange_all(halos)
            for r in ranks:
                r.unpack(decomp.DF)
            for r in ranks:
                r.sim.phase(1, True)
        out = np.concatenate([r.sim.download()[0] for r in ranks])
        e = sum(r.sim.energies() for r in ranks)
    finally:
        for r in ranks:
            r.close()
    return out, e


def test_masked_outer_walk_equals_the_full_walk_bitwise():
    sc = make(cells=(12, 10, 12), temperature=900.0, vacancy=0.01, seed=23, jitter=0.15)
    masked, e_masked = _run(sc, 4, full_walk=False)
    full, e_full = _run(sc, 4, full_walk=True)
    for k in ("x", "v", "f", "rho", "df"):
        assert np.array_equal(masked[k], full[k]), k
    assert np.array_equal(e_masked, e_full)


@pytest.fixture
def masks_off(monkeypatch):
    def off():
        monkeypatch.setenv("MB_OUTER_MASKS", "0")
    return off


def _sim_run(sc, precision, nsteps):
    with mb.Sim(sc.cells, sc.tables, lattice_const=A0, mass=MASS, dt=1.0, cutoff=sc.cutoff,
                stencil_skin=sc.skin, precision=precision, max_interstitials=max(1, sc.itl.shape[0])) as sim:
        sim.upload(sc.box, sc.itl if sc.itl.shape[0] else None)
        sim.run(nsteps)
        return sim.download()


@pytest.mark.parametrize("precision", [mb.MB_PREC_FP64, mb.MB_PREC_MIXED])
def test_device_resident_steps_with_and_without_masks_are_bitwise_equal(precision, masks_off):
    # 40 cells along x: the mixed path takes its brick walk; interstitials flag sites
    sc = make(cells=(40, 12, 10), temperature=900.0, vacancy=0.01, n_itl=3, seed=29, jitter=0.15)
    b1, i1 = _sim_run(sc, precision, 5)
    masks_off()
    b2, i2 = _sim_run(sc, precision, 5)
    for k in ("x", "v", "f"):
        assert np.array_equal(b1[k], b2[k]), k
        assert np.array_equal(i1[k], i2[k]), k


def test_batched_small_lattices_with_and_without_masks_are_bitwise_equal(masks_off):
    # lattices narrower than 32 cells: the linear walk over every lattice's items
    scs = [make(cells=c, temperature=900.0, vacancy=0.01, seed=40 + k, jitter=0.15)
           for k, c in enumerate([(8, 9, 10), (12, 8, 8), (16, 10, 6)])]
    kw = dict(lattice_const=A0, mass=MASS, dt=1.0, cutoff=scs[0].cutoff, stencil_skin=scs[0].skin)

    def run():
        with mb.Ensemble(scs[0].tables, **kw) as ens:
            slots = [ens.add(sc.cells, sc.box, steps=0) for sc in scs]
            ens.run(5)
            return [ens.download(s)[0] for s in slots]

    a = run()
    masks_off()
    b = run()
    for x, y in zip(a, b):
        assert np.array_equal(x["x"], y["x"]) and np.array_equal(x["f"], y["f"])
