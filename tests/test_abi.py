"""C-ABI checks that need no GPU: the library loads, exports every entry point
include/misa_b200.h declares, and its host-side pieces (spline table build,
stencil generation, argument validation) agree with the oracle."""
from __future__ import annotations

import ctypes as C
import pathlib
import re

import numpy as np
import pytest

import misa_b200 as mb
from misa_b200 import _abi
from oracle import oracle as orc
from scenarios import A0, RC, SKIN

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_functions() -> list[str]:
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*?\**\s*\b(mb_[a-z0-9_]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 30
    lib = _abi.lib()
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_abi.SIGNATURES), set(names) - set(_abi.SIGNATURES)


def test_record_layouts_match_the_reference_structs():
    assert _abi.ATOM_DTYPE.itemsize == 104  # _cuAtomElement
    assert C.sizeof(_abi.MbDeviceDomain) == 9 * 4 + 4 + 3 * 8
    assert _abi.ATOM_DTYPE.fields["x"][1] == 16 and _abi.ATOM_DTYPE.fields["df"][1] == 96


def test_spline_coefficients_match_the_oracle_bitwise():
    t = mb.potential.fe_analytic()
    for row, dx in ((t.f[0], t.dr), (t.F[0], t.drho), (t.phi[0], t.dr)):
        y = np.ascontiguousarray(row)
        ours = np.zeros((y.size, 7))
        _abi.check(_abi.lib().mb_spline_coeffs(_abi.dptr(y), y.size, dx, _abi.dptr(ours)))
        np.testing.assert_array_equal(ours, orc.spline_coeffs(y, dx))


@pytest.mark.parametrize("reach", [RC, RC + SKIN, 7.5])
def test_stencil_matches_the_oracle(reach):
    cells, ghost = (8, 8, 8), (6, 3, 3)
    dom = mb.lattice.domain(cells, ghost)
    e, o = mb.lattice.stencil_linear(A0, reach, dom.ext_size_x, dom.ext_size_y)
    oe, oo = orc.stencil(orc.make_domain(cells, ghost), A0, reach)
    np.testing.assert_array_equal(e, oe)
    np.testing.assert_array_equal(o, oo)


def test_ghost_width_covers_the_stencil():
    assert mb.lattice.ghost_for_reach(A0, RC) == (4, 2, 2)
    assert mb.lattice.ghost_for_reach(A0, RC + SKIN) == (4, 2, 2)


def test_hooks_validate_call_order_and_arguments():
    lib = _abi.lib()
    dom = mb.lattice.domain((4, 4, 4), (3, 2, 2))  # odd doubled ghost: rejected
    assert lib.mb_domain_init(C.byref(dom)) == _abi.MB_ERR_ARG
    assert b"even" in lib.mb_last_error()
    bad = mb.lattice.domain((4, 4, 4), (4, 2, 2))
    bad.ext_size_y += 1
    assert lib.mb_domain_init(C.byref(bad)) == _abi.MB_ERR_ARG
    assert lib.mb_cli_set_batches(0) == _abi.MB_ERR_ARG
    assert lib.mb_cli_set_batches(3) == 0 and lib.mb_cli_batches() == 3
    assert lib.mb_cli_set_batches(1) == 0


def test_host_slab_calls_check_their_arguments():
    lib = _abi.lib()
    n = C.c_int32(-1)
    assert lib.mb_sim_set_host_slabs(None, 4) == _abi.MB_ERR_ARG
    assert lib.mb_sim_host_slabs(None, C.byref(n)) == _abi.MB_ERR_ARG and n.value == -1


def test_stencil_beyond_ghost_is_rejected():
    lib = _abi.lib()
    dom = mb.lattice.domain((6, 6, 6), (2, 1, 1))
    assert lib.mb_domain_init(C.byref(dom)) == 0
    e, o = mb.lattice.stencil_linear(A0, RC, dom.ext_size_x, dom.ext_size_y)
    rc = lib.mb_nei_offset_init(_abi.i64ptr(e), e.size, _abi.i64ptr(o), o.size)
    assert rc == _abi.MB_ERR_ARG and b"ghost" in lib.mb_last_error()


def test_compute_without_device_fails_loudly():
    """No silent CPU path: on a machine without a GPU the library reports CUDA errors."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert _abi.lib().mb_env_init(0) != 0
    with pytest.raises(mb.MbError):
        mb.Sim((5, 5, 5), mb.potential.fe_analytic())
