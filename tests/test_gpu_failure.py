"""Failure detection on the device without a GPU fault.

The persistent ensemble kernel separates its phases with grid barriers whose waits are
bounded.  Here the poll limit is set to 0 (mb_ensemble_set_wait_limit), so the first
CTA that finds a barrier still closed gives up at once: the launch ends early, the host
reads MB_ERR_TIMEOUT, and the context stays usable.  The barrier waits sit between the
tile phases, so no CTA leaves with a tile copy in flight; the tile (mbarrier) waits keep
their default limit."""
from __future__ import annotations

import numpy as np
import pytest

import misa_b200 as mb
from misa_b200 import _abi
from scenarios import make

pytestmark = pytest.mark.gpu


def _ens(sc):
    e = mb.Ensemble(sc.tables, lattice_const=sc.a0, mass=sc.mass, dt=sc.dt, cutoff=sc.cutoff, stencil_skin=sc.skin)
    e.set_mode(1)  # the persistent kernel: the one with grid barriers
    return e


def test_grid_barrier_wait_gives_up_and_the_ensemble_recovers():
    # 16^3 cells: 16 tiles of 512 sites, so the launch has 16 CTAs that meet at barriers
    first = make(cells=(16, 16, 16), temperature=600.0, vacancy=0.01, n_itl=2, seed=31, jitter=0.05)
    second = make(cells=(16, 16, 16), temperature=900.0, vacancy=0.005, n_itl=3, seed=32, jitter=0.05)
    with _ens(first) as ens:
        a = ens.add(first.cells, first.box, first.itl, steps=0)
        ens.run(2)  # the default limit: normal steps
        ens.set_wait_limit(0)
        with pytest.raises(mb.MbError) as err:
            ens.run(3)
        assert err.value.code == _abi.MB_ERR_TIMEOUT
        assert "grid barrier" in str(err.value)
        # the error is reported once; the ensemble takes new work and computes it right
        ens.set_wait_limit(-1)
        ens.remove(a)
        b = ens.add(second.cells, second.box, second.itl, steps=0)
        ens.run(5)
        got_box, got_itl = ens.download(b)
    with _ens(second) as fresh:
        s = fresh.add(second.cells, second.box, second.itl, steps=0)
        fresh.run(5)
        ref_box, ref_itl = fresh.download(s)
    for name in ("x", "v", "f"):
        assert np.array_equal(got_box[name], ref_box[name]), name
        assert np.array_equal(got_itl[name], ref_itl[name]), name
