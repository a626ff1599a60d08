"""setfl / funcfl potential files (host side): layout, pair ordering, r*phi -> phi."""
from __future__ import annotations

import numpy as np
import pytest

import misa_b200 as mb

P = mb.potential

# 2 elements, Nrho = 4, Nr = 5; values laid out three to a line, as files in the wild are
TINY_SETFL = """comment 1
comment 2
comment 3
2 Fe Cu
4 0.5 5 0.25 1.0
26 55.845 2.855 bcc
-0.0 -1.0 -2.0
-3.0
10 9 8 7 6
29 63.546 3.615 fcc
0 -2 -4 -6
20 18 16
14 12
0.0 0.25 0.5 0.75 1.0
0.0 0.5 1.0 1.5 2.0
0.0 1.0 2.0 3.0 4.0
"""


def test_tiny_setfl_layout(tmp_path):
    p = tmp_path / "tiny.setfl"
    p.write_text(TINY_SETFL)
    t, meta = P.read_setfl(p)
    assert meta["elements"] == ["Fe", "Cu"] and meta["numbers"] == [26, 29]
    assert meta["masses"] == [55.845, 63.546] and meta["lattices"] == ["bcc", "fcc"]
    assert (t.n_types, t.nrho, t.nr, t.drho, t.dr, t.cutoff) == (2, 4, 5, 0.5, 0.25, 1.0)
    np.testing.assert_array_equal(t.F, [[0, -1, -2, -3], [0, -2, -4, -6]])
    np.testing.assert_array_equal(t.f, [[10, 9, 8, 7, 6], [20, 18, 16, 14, 12]])
    # file pair order (0,0), (1,0), (1,1) -> packed rows (0,0), (0,1), (1,1); phi = (r phi) / r
    # with r = k * 0.25: row (0,0) r*phi = r -> phi = 1; (1,0): r*phi = 2r -> 2; (1,1): 4r -> 4
    np.testing.assert_allclose(t.phi, [[1.0] * 5, [2.0] * 5, [4.0] * 5], rtol=1e-15)


def test_setfl_round_trip(tmp_path):
    t = P.alloy_analytic(3, nr=800, nrho=700)
    p = tmp_path / "alloy.setfl"
    P.write_setfl(p, t, elements=["Fe", "Cu", "Ni"], numbers=[26, 29, 28])
    t2, meta = P.read_setfl(p)
    assert meta["elements"] == ["Fe", "Cu", "Ni"]
    assert (t2.n_types, t2.nr, t2.nrho) == (3, 800, 700)
    assert t2.dr == t.dr and t2.drho == t.drho and t2.cutoff == t.cutoff
    np.testing.assert_array_equal(t2.f, t.f)
    np.testing.assert_array_equal(t2.F, t.F)
    np.testing.assert_allclose(t2.phi[:, 1:], t.phi[:, 1:], rtol=1e-14)


def test_funcfl(tmp_path):
    p = tmp_path / "x.eam"
    p.write_text("funcfl comment\n26 55.845 2.855 bcc\n3 0.1 4 0.5 1.5\n"
                 "0 -1 -2\n0 1 2 3\n"       # F, then Z(r)
                 "4 3 2 1\n")              # f(r)
    t, meta = P.read_funcfl(p)
    assert t.n_types == 1 and meta["numbers"] == [26]
    np.testing.assert_array_equal(t.F[0], [0, -1, -2])
    np.testing.assert_array_equal(t.f[0], [4, 3, 2, 1])
    r = np.arange(4) * 0.5
    expect = P.HARTREE_BOHR * np.array([0, 1, 2, 3.0]) ** 2 / np.where(r > 0, r, 1)
    np.testing.assert_allclose(t.phi[0, 1:], expect[1:], rtol=1e-15)
    assert t.phi[0, 0] == t.phi[0, 1]


def test_truncated_files_raise(tmp_path):
    p = tmp_path / "bad.setfl"
    p.write_text("\n".join(TINY_SETFL.splitlines()[:-2]) + "\n")
    with pytest.raises(ValueError):
        P.read_setfl(p)
    q = tmp_path / "bad.eam"
    q.write_text("c\n26 55.845 2.855 bcc\n3 0.1 4 0.5 1.5\n0 -1 -2\n0 1 2 3\n4 3 2\n")
    with pytest.raises(ValueError):
        P.read_funcfl(q)


def test_file_tables_feed_the_oracle(tmp_path):
    """Tables read from a file drive the CPU oracle exactly as the tables they came from."""
    from oracle import oracle as orc
    from scenarios import make
    t = P.alloy_analytic(2, nr=1500, nrho=1500)
    p = tmp_path / "fecu.setfl"
    P.write_setfl(p, t, elements=["Fe", "Cu"])
    t2, _ = P.read_setfl(p)
    res = []
    for tab in (t, t2):
        sc = make(cells=(4, 4, 4), temperature=600.0, vacancy=0.02, seed=5, tables=tab, n_types=2)
        odom = sc.orc_domain()
        even, odd = orc.stencil(odom, sc.a0, sc.reach)
        ext = sc.ext().view(orc.ATOM)
        orc.compute_forces(sc.orc_pot(), odom, ext, None, even, odd, sc.md_params())
        res.append(ext)
    live = res[0]["type"] >= 0
    np.testing.assert_allclose(res[1]["f"][live], res[0]["f"][live], rtol=1e-12, atol=1e-12)
