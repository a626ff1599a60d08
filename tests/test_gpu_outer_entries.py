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
