"""Pins of the CPU oracle (no GPU): analytic known answers, finite differences,
momentum and energy conservation, and the committed golden fixture.

The reference ships no tests or golden vectors and cannot be built here, so these
identities are what the oracle is checked against."""
from __future__ import annotations

import pathlib

import numpy as np
import pytest

import misa_b200 as mb
from oracle import oracle as orc
from scenarios import A0, RC, make

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"

# BCC shells inside rc = 5.6 A for a0 = 2.855 A (in units of a0): count, distance
SHELLS = [(8, np.sqrt(3) / 2), (6, 1.0), (12, np.sqrt(2)), (24, np.sqrt(11) / 2), (8, np.sqrt(3))]


def test_spline_reproduces_cubics_in_the_interior():
    n, dx = 64, 0.1
    x = np.arange(n) * dx
    y = 0.3 * x ** 3 - 1.2 * x ** 2 + 0.5 * x + 2.0
    c = orc.spline_coeffs(y, dx)
    # on intervals whose end slopes use the 4th-order formula (2 <= m <= n-4)
    for m in range(2, n - 4):
        for p in (0.0, 0.25, 0.5, 0.9):
            xv = (m + p) * dx
            val = ((c[m, 3] * p + c[m, 2]) * p + c[m, 1]) * p + c[m, 0]
            der = (c[m, 6] * p + c[m, 5]) * p + c[m, 4]
            assert val == pytest.approx(0.3 * xv ** 3 - 1.2 * xv ** 2 + 0.5 * xv + 2.0, rel=1e-12, abs=1e-12)
            assert der == pytest.approx(0.9 * xv ** 2 - 2.4 * xv + 0.5, rel=1e-10, abs=1e-10)


def test_spline_continuity_and_end_rules():
    n, dx = 50, 0.2
    y = np.sin(np.arange(n) * dx)
    c = orc.spline_coeffs(y, dx)
    for m in range(n - 2):  # value and slope continuous across knots
        v1 = c[m, 3] + c[m, 2] + c[m, 1] + c[m, 0]
        d1 = c[m, 6] + c[m, 5] + c[m, 4]
        assert v1 == pytest.approx(c[m + 1, 0], abs=1e-13)
        assert d1 == pytest.approx(c[m + 1, 4], abs=1e-12)
    assert c[0, 1] == pytest.approx(y[1] - y[0])
    assert c[n - 1, 1] == pytest.approx(y[n - 1] - y[n - 2])
    assert c[n - 1, 2] == 0.0 and c[n - 1, 3] == 0.0


def test_embedding_continues_linearly_past_the_table():
    t = mb.potential.fe_analytic()
    pot = orc.Pot.from_tables(t)
    rho_max = (t.nrho - 1) * t.drho
    slope = (t.F[0, -1] - t.F[0, -2]) / t.drho
    for rho in (50.0, 60.0, 174.165):
        assert pot.dF(0, rho) == pytest.approx(slope, rel=1e-12)
        assert pot.F(0, rho) == pytest.approx(t.F[0, -1] + slope * (rho - rho_max), rel=1e-12)
    # inside the table: F' of -sqrt(rho) to interpolation accuracy
    for rho in (10.0, 25.0, 40.0):
        assert pot.dF(0, rho) == pytest.approx(-0.5 / np.sqrt(rho), rel=1e-6)


def _perfect_lattice_known_answers():
    rc, A, B = RC, 0.8, -0.2
    rho = sum(n * (rc - d * A0) ** 2 for n, d in SHELLS)
    pair = 0.5 * sum(n * A * (rc - d * A0) ** 2 * (1 + B * d * A0) for n, d in SHELLS)
    t = mb.potential.fe_analytic()
    slope = (t.F[0, -1] - t.F[0, -2]) / t.drho
    F = t.F[0, -1] + slope * (rho - (t.nrho - 1) * t.drho)
    return rho, slope, F + pair


def test_perfect_lattice_known_answers():
    rho_ka, df_ka, e_ka = _perfect_lattice_known_answers()
    assert rho_ka == pytest.approx(174.165, abs=5e-3)  # sum of (rc - r)^2 over the 58 neighbours
    sc = make(cells=(5, 5, 5), temperature=0.0, jitter=0.0)
    ext = sc.ext().view(orc.ATOM)
    even, odd = orc.stencil(sc.orc_domain(), A0, sc.reach)
    pot = sc.orc_pot()
    pe, ke = orc.compute_forces(pot, sc.orc_domain(), ext, None, even, odd, sc.md_params())
    box = mb.lattice.ext_to_box(ext, sc.cells, sc.ghost)
    assert np.allclose(box["rho"], rho_ka, rtol=1e-12)
    assert np.allclose(box["df"], df_ka, rtol=1e-12)
    assert np.max(np.abs(box["f"])) < 1e-11
    assert pe / box.shape[0] == pytest.approx(e_ka, rel=1e-12)
    assert ke == 0.0


def test_stencil_matches_shell_count():
    sc = make(cells=(5, 5, 5))
    even, odd = orc.stencil(sc.orc_domain(), A0, RC)
    assert even.size == odd.size == 58
    even, odd = orc.stencil(sc.orc_domain(), A0, RC + 0.7)
    assert even.size == 88  # + 6 sites at 2 a0 and 24 at sqrt(19)/2 a0
    assert sorted(even.tolist()) != sorted(odd.tolist())  # parities need their own offsets


def _energy(sc, ext, itl, even, odd, pot):
    pe, _ = orc.compute_forces(pot, sc.orc_domain(), ext, itl, even, odd, sc.md_params())
    return pe


@pytest.mark.parametrize("n_itl", [0, 2])
def test_forces_are_minus_energy_gradient(n_itl):
    sc = make(cells=(5, 5, 5), temperature=300.0, vacancy=0.02, n_itl=n_itl, seed=3, jitter=0.08)
    pot = sc.orc_pot()
    even, odd = orc.stencil(sc.orc_domain(), A0, sc.reach)
    ext = sc.ext().view(orc.ATOM)
    itl = sc.itl.view(orc.ATOM).copy() if n_itl else None
    _energy(sc, ext, itl, even, odd, pot)
    box = mb.lattice.ext_to_box(ext, sc.cells, sc.ghost)
    h = 1e-5
    live = np.flatnonzero(box["type"] >= 0)
    rng = np.random.default_rng(0)
    picks = [("site", k) for k in rng.choice(live, 3, replace=False)] + [("itl", k) for k in range(n_itl)]
    for kind, k in picks:
        for c in range(3):
            grads = []
            for sgn in (+1, -1):
                b2 = box.copy()
                i2 = None if itl is None else itl.copy()
                if kind == "site":
                    b2["x"][k, c] += sgn * h
                else:
                    i2["x"][k, c] += sgn * h
                e2 = mb.lattice.box_to_ext(b2, sc.cells, sc.ghost, A0).view(orc.ATOM)
                grads.append(_energy(sc, e2, i2, even, odd, pot))
            fd = -(grads[0] - grads[1]) / (2 * h)
            f = box["f"][k, c] if kind == "site" else itl["f"][k, c]
            assert f == pytest.approx(fd, rel=1e-5, abs=1e-6), (kind, k, c)


def test_total_force_vanishes_with_interstitials():
    sc = make(cells=(6, 6, 6), temperature=900.0, vacancy=0.01, n_itl=4, seed=5)
    pot = sc.orc_pot()
    even, odd = orc.stencil(sc.orc_domain(), A0, sc.reach)
    ext = sc.ext().view(orc.ATOM)
    itl = sc.itl.view(orc.ATOM).copy()
    orc.compute_forces(pot, sc.orc_domain(), ext, itl, even, odd, sc.md_params())
    box = mb.lattice.ext_to_box(ext, sc.cells, sc.ghost)
    live = box["type"] >= 0
    total = box["f"][live].sum(axis=0) + itl["f"].sum(axis=0)
    assert np.max(np.abs(total)) < 1e-9
    assert np.max(np.abs(itl["f"])) > 1.0  # interstitials at octahedral sites are strongly pushed


def test_nve_energy_is_conserved():
    sc = make(cells=(6, 6, 6), temperature=600.0, vacancy=0.01, n_itl=2, seed=7, jitter=0.0)
    pot = sc.orc_pot()
    even, odd = orc.stencil(sc.orc_domain(), A0, sc.reach)
    ext = sc.ext().view(orc.ATOM)
    itl = sc.itl.view(orc.ATOM).copy()
    e = orc.md_run(pot, sc.orc_domain(), ext, itl, even, odd, sc.md_params(), 200)
    tot = e[:, 0] + e[:, 1]
    n = int((sc.box["type"] >= 0).sum()) + itl.shape[0]
    assert np.max(np.abs(tot - tot[0])) / n < 2e-4  # eV/atom, dt = 1 fs
    assert e[-1, 1] > 0


def recs(a: np.ndarray, dtype) -> np.ndarray:
    return np.ascontiguousarray(a).view(dtype).reshape(-1)


def test_golden_fixture_reproduced():
    g = np.load(GOLDEN / "small_md.npz")
    t = mb.potential.EamTables(1, float(g["dr"]), float(g["drho"]), float(g["cutoff"]), g["f_tab"], g["F_tab"],
                               g["phi_tab"])
    pot = orc.Pot.from_tables(t)
    cells = tuple(int(c) for c in g["cells"])
    ghost = tuple(int(c) for c in g["ghost"])
    dom = orc.make_domain(cells, ghost)
    ext = mb.lattice.box_to_ext(recs(g["box_in"], mb.ATOM_DTYPE), cells, ghost, float(g["a0"])).view(orc.ATOM)
    itl = recs(g["itl_in"], orc.ATOM).copy()
    even, odd = g["even"], g["odd"]
    mp = orc.md_params(float(g["a0"]), float(g["mass"]), float(g["dt"]), float(g["cutoff"]), 1.0)
    e = orc.md_run(pot, dom, ext, itl, even, odd, mp, int(g["nsteps"]))
    box = mb.lattice.ext_to_box(ext, cells, ghost)
    np.testing.assert_allclose(e, g["energies"], rtol=1e-13, atol=1e-12)
    np.testing.assert_allclose(box["x"], recs(g["box_out"], mb.ATOM_DTYPE)["x"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(box["f"], recs(g["box_out"], mb.ATOM_DTYPE)["f"], rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(itl["f"], recs(g["itl_out"], orc.ATOM)["f"], rtol=1e-11, atol=1e-11)


def _analytic_lattice(sc, conventional_F):
    """rho, df, forces and energy per atom of the box from the analytic functions
    f = (rc - r)^2, phi = 0.8 (rc - r)^2 (1 - 0.2 r) and F = -sqrt(rho), by direct pair
    sums (minimum image).  conventional_F: F continues linearly past the table's last
    density with the table's end slope, as the tabulated potential does."""
    box = sc.box
    live = box["type"] >= 0
    x = box["x"][live]
    L = np.array(sc.cells) * A0
    d = x[:, None, :] - x[None, :, :]
    d -= L * np.rint(d / L)
    r = np.linalg.norm(d, axis=-1)
    np.fill_diagonal(r, np.inf)
    m = r < RC
    rs = np.where(m, r, 1.0)
    f = np.where(m, (RC - rs) ** 2, 0.0)
    phi = np.where(m, 0.8 * (RC - rs) ** 2 * (1 - 0.2 * rs), 0.0)
    dfr = np.where(m, -2 * (RC - rs), 0.0)
    dphi = np.where(m, 0.8 * (-2 * (RC - rs) * (1 - 0.2 * rs) - 0.2 * (RC - rs) ** 2), 0.0)
    rho = f.sum(1)
    t = mb.potential.fe_analytic()
    rmax = (t.nrho - 1) * t.drho
    s = (t.F[0, -1] - t.F[0, -2]) / t.drho
    if conventional_F:
        F = np.where(rho <= rmax, -np.sqrt(rho), -np.sqrt(rmax) + s * (rho - rmax))
        dF = np.where(rho <= rmax, -0.5 / np.sqrt(rho), s)
    else:
        F, dF = -np.sqrt(rho), -0.5 / np.sqrt(rho)
    g = dphi + (dF[:, None] + dF[None, :]) * dfr
    force = (-(g * np.where(m, 1.0 / rs, 0.0))[:, :, None] * d).sum(1)
    return live, rho, dF, force, (F.sum() + 0.5 * phi.sum()) / x.shape[0]


def test_tabulated_potential_against_its_analytic_functions():
    """The tabulation error, apart from the parity of oracle and library: the 5000-knot
    tables against the closed forms they sample."""
    from scenarios import rel_err
    t = mb.potential.fe_analytic()
    pot = orc.Pot.from_tables(t)
    dr = t.dr
    # interior intervals reproduce the quadratic f and the cubic phi to rounding
    for r in np.linspace(0.5, RC - 3 * dr, 97):
        assert pot.rho(0, r) == pytest.approx((RC - r) ** 2, abs=1e-12)
        assert pot.drho(0, r) == pytest.approx(-2 * (RC - r), abs=1e-10)
        assert pot.phi(0, 0, r) == pytest.approx(0.8 * (RC - r) ** 2 * (1 - 0.2 * r), abs=1e-12)
    # the last interval (one-sided end slope): small, bounded departures
    r = RC - 0.5 * dr
    assert abs(pot.rho(0, r) - (RC - r) ** 2) < 1e-6
    assert abs(pot.drho(0, r) + 2 * (RC - r)) < 1e-3
    # a disordered lattice (sigma 0.1 A: some pairs cross into the last interval)
    sc = make(cells=(5, 5, 5), temperature=0.0, vacancy=0.02, seed=3, jitter=0.1)
    ext = sc.ext().view(orc.ATOM)
    even, odd = orc.stencil(sc.orc_domain(), A0, sc.reach)
    pe, _ = orc.compute_forces(sc.orc_pot(), sc.orc_domain(), ext, None, even, odd, sc.md_params())
    box = mb.lattice.ext_to_box(ext.view(mb.ATOM_DTYPE), sc.cells, sc.ghost)
    live, rho, dF, force, e = _analytic_lattice(sc, conventional_F=True)
    n = int(live.sum())
    assert rel_err(box["rho"][live], rho) < 1e-8
    assert rel_err(box["df"][live], dF) < 1e-12
    assert rel_err(box["f"][live], force) < 1e-4
    assert abs(pe / n - e) < 1e-8
    # the table-range convention itself (F linear past rho = 50 against -sqrt(rho) at
    # rho ~ 174) is a different potential, not an error: eV/atom and percent-level forces
    live, rho, dF, force, e_pure = _analytic_lattice(sc, conventional_F=False)
    assert 2.0 < abs(pe / n - e_pure) < 3.0
    assert 0.05 < rel_err(box["f"][live], force) < 0.2


def test_perfect_lattice_analytic_energy_known_answer():
    # the known answer of the analytic potential at the perfect BCC Fe lattice (a0 2.855 A,
    # rc 5.6 A): rho = 174.165 and E = -sqrt(rho) + 1/2 sum phi = 13.0355 eV/atom; the tabulated
    # potential (F linear past rho = 50) gives 10.3813 eV/atom there, which the oracle hits
    sc = make(cells=(5, 5, 5), temperature=0.0, jitter=0.0)
    live, rho, _, force, e_pure = _analytic_lattice(sc, conventional_F=False)
    assert np.allclose(rho, 174.165, atol=5e-3)
    assert e_pure == pytest.approx(13.0355, abs=5e-4)
    assert np.abs(force).max() < 1e-11
    _, _, _, _, e_conv = _analytic_lattice(sc, conventional_F=True)
    assert e_conv == pytest.approx(10.3813, abs=5e-4)
    ext = sc.ext().view(orc.ATOM)
    even, odd = orc.stencil(sc.orc_domain(), A0, sc.reach)
    pe, _ = orc.compute_forces(sc.orc_pot(), sc.orc_domain(), ext, None, even, odd, sc.md_params())
    assert pe / int(live.sum()) == pytest.approx(e_conv, rel=1e-10)


@pytest.mark.parametrize("name,cells", [("fe20", (5, 6, 4)), ("fe128", (12, 10, 9))])
def test_oracle_workload_builder_equals_the_package_set_up(name, cells):
    # The CPU reference arm of the benchmark builds its inputs with oracle/workload.py
    # (it must not load the product library); the GPU arm with the package.  Same seeds,
    # same bytes: the two arms time the same workload.
    from oracle import workload as W
    c = W.CONFIGS[name]
    box_o, itl_o = W.config_state(name, cells)
    box = mb.lattice.bcc_box(cells, A0)
    mb.lattice.add_vacancies(box, c["vacancy"], c["seed"])
    n_itl = int(round(c["n_itl"] * np.prod(cells) / float(np.prod(c["cells"]))))
    itl = mb.lattice.octahedral_interstitials(n_itl, cells, A0, c["seed"])
    mb.lattice.maxwell_boltzmann(box, itl, c["temperature"], W.MASS, c["velocity_seed"])
    assert box.tobytes() == box_o.tobytes()
    assert itl.tobytes() == itl_o.tobytes()
    ghost = mb.lattice.ghost_for_reach(A0, W.RC + W.SKIN)
    assert W.ghost_for_reach(A0, W.RC + W.SKIN) == ghost
    assert W.box_to_ext(box_o, cells, ghost).tobytes() == mb.lattice.box_to_ext(box, cells, ghost, A0).tobytes()
    t, to = mb.potential.fe_analytic(), W.fe_tables()
    for k in ("f", "F", "phi"):
        assert np.array_equal(getattr(t, k), getattr(to, k))
    assert (t.dr, t.drho, t.cutoff) == (to.dr, to.drho, to.cutoff)
