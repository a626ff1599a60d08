"""Half-neighbour (Newton's third law) passes of the oracle, no GPU.

The reference's USE_NEWTONS_THIRD_LOW build walks half stencils and gives each pair's
shares to both atoms, ghosts included (src/kernels/kernel_pairs.hpp:21-32, 39-60); the
host then adds every ghost record to the atom it images.  On one periodic rank that
fold must give back the full-neighbour rho and forces."""
from __future__ import annotations

import numpy as np
import pytest

import misa_b200 as mb
from oracle import oracle as orc
from scenarios import A0, make, rel_err


def _box(ext, sc):
    return mb.lattice.ext_to_box(ext, sc.cells, sc.ghost)


def test_half_stencil_holds_one_of_each_opposite_pair():
    sc = make(cells=(6, 5, 5))
    even, odd = sc.stencil()
    he, ho = orc.half_stencil(even), orc.half_stencil(odd)
    # each pair of sites appears once in the even/odd full stencils per direction and once
    # in the half stencils altogether (cross-parity pairs: o from even, -o from odd)
    assert 2 * (he.size + ho.size) == even.size + odd.size
    # the reverse of an offset is never in a half stencil, whatever the partner's parity
    full = {0: set(even.tolist()), 1: set(odd.tolist())}
    half = {0: set(he.tolist()), 1: set(ho.tolist())}
    for p in (0, 1):
        for o in half[p]:
            assert o > 0 and o in full[p]
            assert -o not in half[0] and -o not in half[1]


@pytest.mark.parametrize("n_types,vac", [(1, 0.02), (3, 0.01)])
def test_half_passes_fold_back_to_full_neighbour_results(n_types, vac):
    sc = make(cells=(6, 5, 7), temperature=900.0, vacancy=vac, n_types=n_types, seed=31, jitter=0.1)
    odom = sc.orc_domain()
    even, odd = sc.stencil()
    he, ho = orc.half_stencil(even), orc.half_stencil(odd)
    pot = sc.orc_pot()
    L = [sc.cells[0] * A0, sc.cells[1] * A0, sc.cells[2] * A0]

    full = sc.ext().view(orc.ATOM)
    orc.rho_pass(pot, odom, full, even, odd, sc.cutoff)
    orc.ghost_fill(odom, full, L, 2)
    orc.force_pass(pot, odom, full, even, odd, sc.cutoff)
    bf = _box(full.view(mb.ATOM_DTYPE), sc)
    live = bf["type"] >= 0

    half = sc.ext().view(orc.ATOM)
    orc.rho_pass_half(pot, odom, half, he, ho, sc.cutoff)
    # ghost records hold shares for their owners; vacant records receive nothing
    assert np.all(half["rho"][half["type"] < 0] == 0.0)
    assert np.abs(half["rho"]).max() > 0
    rho = orc.fold_ghosts(odom, half.view(mb.ATOM_DTYPE), "rho")
    assert rel_err(rho[live], bf["rho"][live]) < 1e-13

    # the host's df pass and ghost refresh, then the half force pass and its fold
    half["rho"] = 0.0
    hb = mb.lattice.ext_to_box(half.view(mb.ATOM_DTYPE), sc.cells, sc.ghost)
    hb["rho"] = rho
    half[:] = mb.lattice.box_to_ext(hb, sc.cells, sc.ghost, A0).view(orc.ATOM)
    orc.df_pass(pot, odom, half)
    orc.ghost_fill(odom, half, L, 2)
    hb = _box(half.view(mb.ATOM_DTYPE), sc)
    assert rel_err(hb["df"][live], bf["df"][live]) < 1e-13
    orc.force_pass_half(pot, odom, half, he, ho, sc.cutoff)
    f = orc.fold_ghosts(odom, half.view(mb.ATOM_DTYPE), "f")
    assert rel_err(f[live], bf["f"][live]) < 1e-12
    # Newton's third law: the shares, ghosts included, sum to zero
    assert np.abs(half["f"].sum(axis=0)).max() < 1e-9 * np.abs(half["f"]).max()
