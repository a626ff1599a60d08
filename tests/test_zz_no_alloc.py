"""The allocation-free rho pass (mb_eam_rho_calc_noalloc), through the C ABI.

It serves hosts that cannot let a plugin call cudaMalloc (device memory already
owned by the host's own pool allocator, or a timestep loop that must not take the
synchronisation an allocation can cause).  Its scratch is a fixed device array
inside the library, so these checks compare it with the allocating
mb_eam_rho_calc on the same inputs, twice in a row with different lattices (the
second call must not see the first call's leftovers), and check that lattices
beyond the fixed scratch are refused.  Collected last on purpose."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import misa_b200 as mb
from misa_b200 import _abi
from scenarios import A0, make, rel_err

pytestmark = pytest.mark.gpu


def _prepare(hooks, sc):
    dom = mb.lattice.domain(sc.cells, sc.ghost)
    hooks.domain_init(dom)
    even, odd = mb.lattice.stencil_linear(A0, sc.reach, dom.ext_size_x, dom.ext_size_y)
    hooks.nei_offset_init(even, odd)
    hooks.pot_init(sc.tables)


def test_noalloc_rho_matches_allocating_rho_twice_in_a_row():
    hooks = mb.Hooks(0)
    lib = _abi.lib()
    for cells, seed, vac in (((6, 6, 6), 1, 0.02), ((7, 5, 6), 2, 0.05)):
        sc = make(cells=cells, temperature=900.0, vacancy=vac, seed=seed, jitter=0.1)
        _prepare(hooks, sc)
        ref = sc.ext()
        got = ref.copy()
        hooks.rho_calc(ref, sc.cutoff)
        _abi.check(lib.mb_eam_rho_calc_noalloc(_abi.ptr(got), sc.cutoff))
        bref = mb.lattice.ext_to_box(ref, sc.cells, sc.ghost)
        bgot = mb.lattice.ext_to_box(got, sc.cells, sc.ghost)
        live = bref["type"] >= 0
        assert rel_err(bgot["rho"][live], bref["rho"][live]) < 1e-12
        assert rel_err(bgot["df"][live], bref["df"][live]) < 1e-12
        # every other byte of the host array is untouched by both
        for name in ("id", "type", "x", "v", "f"):
            assert np.array_equal(got[name], ref[name])
        assert np.array_equal(bgot["rho"][~live], bref["rho"][~live])


def test_noalloc_refuses_types_without_a_potential_table_and_leaves_the_array():
    hooks = mb.Hooks(0)
    sc = make(cells=(6, 6, 6), seed=5)
    _prepare(hooks, sc)
    ext = sc.ext()
    ext["type"][len(ext) // 2] = 2  # the one-type potential has a table for type 0 only
    before = ext.copy()
    rc = _abi.lib().mb_eam_rho_calc_noalloc(_abi.ptr(ext), sc.cutoff)
    assert rc == _abi.MB_ERR_ARG
    assert b"potential table" in _abi.lib().mb_last_error()
    assert ext.tobytes() == before.tobytes()
    # the next call on a valid lattice is not affected by the refused one
    ok = sc.ext()
    ref = ok.copy()
    hooks.rho_calc(ref, sc.cutoff)
    _abi.check(_abi.lib().mb_eam_rho_calc_noalloc(_abi.ptr(ok), sc.cutoff))
    live = ref["type"] >= 0
    assert rel_err(ok["rho"][live], ref["rho"][live]) < 1e-12


def test_noalloc_refuses_lattices_beyond_its_scratch():
    hooks = mb.Hooks(0)
    sc = make(cells=(40, 40, 40), temperature=300.0, seed=3, jitter=0.0)
    _prepare(hooks, sc)
    ext = sc.ext()
    rc = _abi.lib().mb_eam_rho_calc_noalloc(_abi.ptr(ext), sc.cutoff)
    assert rc == _abi.MB_ERR_ARG
    assert b"at most" in _abi.lib().mb_last_error()
