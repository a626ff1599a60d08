"""Mixed precision and the batched ensemble on the device.

Bars (from the target of the mixed form): relative force RMS error against the FP64
oracle <= 1e-6 (sqrt(sum |dF|^2) / sqrt(sum |F|^2)); NVE energy drift <= 1e-5
eV/atom; a lattice gives the same result alone and inside a batch (bitwise for
positions and forces, 1e-12 relative for energies)."""
from __future__ import annotations

import numpy as np
import pytest

import misa_b200 as mb
from oracle import oracle as orc
from scenarios import A0, MASS, make

pytestmark = pytest.mark.gpu
F_RMS_TOL = 1e-6


def rms_rel(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2)) / np.sqrt(np.sum(b ** 2)))


def _oracle_forces(sc, box=None, itl=None):
    odom = sc.orc_domain()
    even, odd = orc.stencil(odom, sc.a0, sc.reach)
    b = sc.box if box is None else box
    ext = mb.lattice.box_to_ext(b, sc.cells, sc.ghost, sc.a0).view(orc.ATOM)
    i = None
    if itl is not None and itl.shape[0]:
        i = itl.view(orc.ATOM).copy()
    pe, ke = orc.compute_forces(sc.orc_pot(), odom, ext, i, even, odd, sc.md_params())
    return mb.lattice.ext_to_box(ext, sc.cells, sc.ghost), i, pe


def _ens(sc, **kw):
    return mb.Ensemble(sc.tables, lattice_const=sc.a0, mass=sc.mass, dt=sc.dt, cutoff=sc.cutoff,
                       stencil_skin=sc.skin, **kw)


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("n_itl", [0, 3])
def test_mixed_forces_within_1e6_of_fp64_oracle(n_itl, mode):
    # mode 1: the persistent tile kernel; mode 2: the split density / force kernels
    sc = make(cells=(9, 8, 10), temperature=900.0, vacancy=0.01, n_itl=n_itl, seed=71, jitter=0.1)
    bo, io, pe = _oracle_forces(sc, itl=sc.itl)
    with _ens(sc) as ens:
        ens.set_mode(mode)
        slot = ens.add(sc.cells, sc.box, sc.itl if n_itl else None, steps=0)
        ens.run(0)  # priming launch only: forces at the uploaded positions
        bg, ig = ens.download(slot)
    live = bo["type"] >= 0
    fo = bo["f"][live]
    fg = bg["f"][live]
    if n_itl:
        fo = np.concatenate([fo, io["f"]])
        fg = np.concatenate([fg, ig["f"]])
    err = rms_rel(fg, fo)
    assert err < F_RMS_TOL, err
    assert rms_rel(bg["rho"][live], bo["rho"][live]) < 1e-6
    np.testing.assert_allclose(bg["x"][live], sc.box["x"][live], rtol=0, atol=1e-12)


def test_split_brick_walk_forces_within_1e6_of_fp64_oracle():
    # a lattice 32 cells wide walks bricks (the large-lattice path) instead of linear items
    sc = make(cells=(32, 9, 10), temperature=900.0, vacancy=0.01, n_itl=2, seed=76, jitter=0.1)
    bo, io, pe = _oracle_forces(sc, itl=sc.itl)
    with _ens(sc) as ens:
        ens.set_mode(2)
        slot = ens.add(sc.cells, sc.box, sc.itl, steps=0)
        ens.run(0)
        bg, ig = ens.download(slot)
    live = bo["type"] >= 0
    fo = np.concatenate([bo["f"][live], io["f"]])
    fg = np.concatenate([bg["f"][live], ig["f"]])
    assert rms_rel(fg, fo) < F_RMS_TOL
    assert rms_rel(bg["rho"][live], bo["rho"][live]) < 1e-6


@pytest.mark.parametrize("cells", [(32, 9, 10), (9, 8, 10)])
def test_eight_shell_stencil_forces_within_1e6_of_fp64_oracle(cells):
    # skin 1.3 A: the built-in stencil of BCC shells 1-8 (112 vectors), brick and linear walks
    sc = make(cells=cells, temperature=900.0, vacancy=0.01, n_itl=2, seed=77, jitter=0.15)
    sc.skin = 1.3
    sc.ghost = mb.lattice.ghost_for_reach(A0, sc.cutoff + sc.skin)
    bo, io, pe = _oracle_forces(sc, itl=sc.itl)
    with _ens(sc) as ens:
        ens.set_mode(2)
        slot = ens.add(sc.cells, sc.box, sc.itl, steps=0)
        ens.run(0)
        bg, ig = ens.download(slot)
    live = bo["type"] >= 0
    fo = np.concatenate([bo["f"][live], io["f"]])
    fg = np.concatenate([bg["f"][live], ig["f"]])
    assert rms_rel(fg, fo) < F_RMS_TOL
    assert rms_rel(bg["rho"][live], bo["rho"][live]) < 1e-6


def test_split_kernels_track_persistent_kernel():
    sc = make(cells=(10, 9, 8), temperature=900.0, vacancy=0.005, n_itl=2, seed=74)
    out = {}
    for mode in (1, 2):
        with _ens(sc) as ens:
            ens.set_mode(mode)
            s = ens.add(sc.cells, sc.box, sc.itl, steps=40)
            ens.advance(100, energy_every=10)
            out[mode] = (*ens.download(s), ens.energies(s), ens.status(s)[0])
    (b1, i1, e1, n1), (b2, i2, e2, n2) = out[1], out[2]
    assert n1 == n2 == 40
    live = b1["type"] >= 0
    # same pair arithmetic, different summation order: rounding-level differences only
    assert np.max(np.abs(b1["x"][live] - b2["x"][live])) < 1e-6
    assert np.max(np.abs(i1["x"] - i2["x"])) < 1e-6
    assert np.array_equal(e1[:, 0], e2[:, 0])
    n = int(live.sum()) + 2
    assert np.max(np.abs((e1[:, 1] + e1[:, 2]) - (e2[:, 1] + e2[:, 2]))) / n < 1e-7
    with _ens(sc) as ens:
        with pytest.raises(mb.MbError):
            ens.set_mode(3)


def test_mixed_sim_tracks_fp64_sim():
    sc = make(cells=(8, 8, 8), temperature=900.0, vacancy=0.005, n_itl=2, seed=72)
    out = {}
    for prec in (mb.MB_PREC_FP64, mb.MB_PREC_MIXED):
        with mb.Sim(sc.cells, sc.tables, lattice_const=A0, mass=MASS, dt=1.0, stencil_skin=sc.skin,
                    precision=prec, max_interstitials=4) as sim:
            sim.upload(sc.box, sc.itl)
            sim.run(100, energy_every=10)
            out[prec] = (*sim.download(), sim.energies())
    b64, i64, e64 = out[mb.MB_PREC_FP64]
    b32, i32, e32 = out[mb.MB_PREC_MIXED]
    live = b64["type"] >= 0
    n = int(live.sum()) + 2
    assert np.max(np.abs(b32["x"][live] - b64["x"][live])) < 1e-5
    assert rms_rel(b32["f"][live], b64["f"][live]) < 1e-4  # trajectories separate slowly
    assert np.array_equal(e32[:, 0], e64[:, 0])
    assert np.max(np.abs((e32[:, 1] + e32[:, 2]) - (e64[:, 1] + e64[:, 2]))) / n < 1e-6


def drift_per_atom(e: np.ndarray, n_atoms: int, skip: int = 1) -> float:
    """Systematic energy change over the run: least-squares slope of the total
    energy against the step, times the run length, per atom (the VV fluctuation
    about the shadow energy is not drift)."""
    t = e[skip:, 0]
    tot = e[skip:, 1] + e[skip:, 2]
    slope = np.polyfit(t, tot, 1)[0]
    return abs(slope) * (t[-1] - t[0]) / n_atoms


def test_mixed_nve_drift():
    # vacancies only: every atom stays within the stencil skin of its site, so the
    # dynamics is exactly conservative and what remains is integrator + precision error
    sc = make(cells=(10, 10, 10), temperature=900.0, vacancy=0.005, n_itl=0, seed=73, jitter=0.0)
    out = {}
    for prec in (mb.MB_PREC_FP64, mb.MB_PREC_MIXED):
        with mb.Sim(sc.cells, sc.tables, lattice_const=A0, mass=MASS, dt=1.0, stencil_skin=sc.skin,
                    precision=prec) as sim:
            sim.upload(sc.box)
            sim.run(3000, energy_every=100)
            out[prec] = sim.energies()
    n = int((sc.box["type"] >= 0).sum())
    e = out[mb.MB_PREC_MIXED]
    assert e.shape[0] == 31
    assert drift_per_atom(e, n) < 1e-5
    tot = e[:, 1] + e[:, 2]
    assert np.max(np.abs(tot - tot[0])) / n < 5e-5
    # the mixed run follows the FP64 energy record
    e64 = out[mb.MB_PREC_FP64]
    assert np.max(np.abs(tot - (e64[:, 1] + e64[:, 2]))) / n < 1e-6


@pytest.mark.parametrize("mode", [1, 2])
def test_batched_equals_alone(mode):
    specs = [((8, 9, 10), 0, 0.01), ((12, 8, 8), 2, 0.0), ((9, 9, 9), 1, 0.005), ((16, 10, 8), 0, 0.0)]
    scs = [make(cells=c, temperature=600.0 + 100 * k, vacancy=v, n_itl=n, seed=80 + k)
           for k, (c, n, v) in enumerate(specs)]
    alone = []
    for sc in scs:
        with _ens(sc) as ens:
            ens.set_mode(mode)
            s = ens.add(sc.cells, sc.box, sc.itl if sc.itl.shape[0] else None, steps=25)
            ens.advance(100, energy_every=5)
            alone.append((*ens.download(s), ens.energies(s)))
    with _ens(scs[0]) as ens:
        ens.set_mode(mode)
        slots = [ens.add(sc.cells, sc.box, sc.itl if sc.itl.shape[0] else None, steps=25) for sc in scs]
        ens.advance(100, energy_every=5)
        for k, s in enumerate(slots):
            b, i, e = ens.download(s), None, None
            b, i = b
            e = ens.energies(s)
            ab, ai, ae = alone[k]
            assert np.array_equal(b["x"], ab["x"]), k
            assert np.array_equal(b["f"], ab["f"]), k
            assert np.array_equal(i["x"], ai["x"]), k
            assert np.array_equal(e[:, 0], ae[:, 0])
            np.testing.assert_allclose(e[:, 1:], ae[:, 1:], rtol=1e-12)
            assert ens.status(s)[0] == 25


def test_batched_equals_alone_with_large_planes():
    # lattices with planes of >= 64 x 64 sites are walked by bricks inside a batch (z blocks
    # of 8 cells by 8 chunks; these two end in shorter blocks), small ones plane by plane,
    # and a lattice alone by the single-lattice bricks: the same positions and forces
    specs = [((64, 66, 6), 2, 0.005), ((70, 65, 9), 0, 0.01), ((8, 9, 10), 1, 0.0)]
    scs = [make(cells=c, temperature=700.0 + 100 * k, vacancy=v, n_itl=n, seed=120 + k)
           for k, (c, n, v) in enumerate(specs)]
    alone = []
    for sc in scs:
        with _ens(sc) as ens:
            s = ens.add(sc.cells, sc.box, sc.itl if sc.itl.shape[0] else None, steps=20)
            ens.advance(100, energy_every=5)
            alone.append((*ens.download(s), ens.energies(s)))
    with _ens(scs[0]) as ens:
        slots = [ens.add(sc.cells, sc.box, sc.itl if sc.itl.shape[0] else None, steps=20) for sc in scs]
        ens.advance(100, energy_every=5)
        for k, s in enumerate(slots):
            (b, i), e = ens.download(s), ens.energies(s)
            ab, ai, ae = alone[k]
            assert np.array_equal(b["x"], ab["x"]), k
            assert np.array_equal(b["f"], ab["f"]), k
            assert np.array_equal(i["x"], ai["x"]), k
            np.testing.assert_allclose(e[:, 1:], ae[:, 1:], rtol=1e-12)


def test_uneven_step_targets_and_slot_reuse():
    sc = make(cells=(8, 8, 8), temperature=600.0, seed=91)
    with _ens(sc) as ens:
        a = ens.add(sc.cells, sc.box, steps=5)
        b = ens.add(sc.cells, sc.box, steps=12)
        n = ens.advance(100)
        assert n == 13  # priming launch + 12 steps
        assert ens.status(a)[0] == 5 and ens.status(b)[0] == 12
        ens.remove(a)
        c = ens.add(sc.cells, sc.box, steps=5)
        assert c == a  # freed slot is reused
        ens.advance(100)
        assert ens.status(c)[0] == 5 and ens.status(b)[0] == 12
        # a lattice advanced 5 steps twice from the same start is the same lattice
        with _ens(sc) as ref:
            r = ref.add(sc.cells, sc.box, steps=5)
            ref.advance(100)
            assert np.array_equal(ref.download(r)[0]["x"], ens.download(c)[0]["x"])


def test_hbm_budget_and_slot_limit_refuse_admission():
    sc = make(cells=(8, 8, 8), seed=92)
    one = mb.Ensemble.lattice_bytes(sc.cells, 0)
    with _ens(sc, hbm_budget_bytes=int(2.5 * one)) as ens:
        ens.add(sc.cells, sc.box)
        ens.add(sc.cells, sc.box)
        with pytest.raises(mb.MbError) as ei:
            ens.add(sc.cells, sc.box)
        assert ei.value.code == mb._abi.MB_ERR_NOMEM
    with _ens(sc, max_lattices=1) as ens:
        ens.add(sc.cells, sc.box)
        with pytest.raises(mb.MbError):
            ens.add(sc.cells, sc.box)


def test_autotune_keeps_state_and_results():
    specs = [(8, 8, 8), (17, 9, 8), (10, 20, 9)]
    scs = [make(cells=c, temperature=700.0, seed=95 + k) for k, c in enumerate(specs)]
    with _ens(scs[0]) as ens:
        slots = [ens.add(sc.cells, sc.box, steps=10) for sc in scs]
        pol, ms = ens.autotune(3)
        assert -1 <= pol <= 4 and ms > 0
        assert all(ens.status(s)[0] == 0 for s in slots)  # tuning took no simulation steps
        ens.advance(100)
        tuned = [ens.download(s)[0] for s in slots]
    with _ens(scs[0]) as ens:  # the chosen kernel, set by hand, from the same start
        if pol == 4:
            ens.set_mode(2)
        else:
            ens.set_mode(1)
            ens.set_policy(pol)
        slots = [ens.add(sc.cells, sc.box, steps=10) for sc in scs]
        ens.advance(100)
        plain = [ens.download(s)[0] for s in slots]
    for a, b in zip(tuned, plain):
        assert np.array_equal(a["x"], b["x"])


def test_persistent_tile_policies_share_arithmetic():
    specs = [(8, 8, 8), (17, 9, 8), (10, 20, 9)]
    scs = [make(cells=c, temperature=700.0, seed=95 + k) for k, c in enumerate(specs)]
    res = []
    for pol in (-1, 0, 3):
        with _ens(scs[0]) as ens:
            ens.set_mode(1)
            ens.set_policy(pol)
            slots = [ens.add(sc.cells, sc.box, steps=10) for sc in scs]
            ens.advance(100)
            res.append([ens.download(s)[0] for s in slots])
    for other in res[1:]:  # tile shape changes the schedule, not the per-site arithmetic
        for a, b in zip(res[0], other):
            assert np.array_equal(a["x"], b["x"])
