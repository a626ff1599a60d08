"""FP64 parity of the CUDA path against the CPU oracle, through the C ABI.

Tolerances (the drop-in bar): forces within 1e-10 relative (max |dF| over the
largest |F|), rho / df within 1e-12 relative, energies within 1e-12 eV/atom."""
from __future__ import annotations

import pathlib

import numpy as np
import pytest

import misa_b200 as mb
from oracle import oracle as orc
from scenarios import A0, MASS, make, rel_err

pytestmark = pytest.mark.gpu
GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
F_TOL = 1e-10
E_TOL = 1e-12  # eV / atom


@pytest.fixture(scope="module")
def hooks():
    h = mb.Hooks(0)
    yield h
    mb.Hooks.clean()


def _hook_setup(hooks, sc, reach=None, start=(0, 0, 0)):
    dom = mb.lattice.domain(sc.cells, sc.ghost, start)
    hooks.domain_init(dom)
    even, odd = mb.lattice.stencil_linear(A0, reach or sc.reach, dom.ext_size_x, dom.ext_size_y)
    hooks.nei_offset_init(even, odd)
    hooks.pot_init(sc.tables)
    odom = orc.make_domain(sc.cells, sc.ghost, start)
    return dom, odom, even, odd


def _box(ext, sc):
    return mb.lattice.ext_to_box(ext, sc.cells, sc.ghost)


@pytest.mark.parametrize("n_types,vac,start", [(1, 0.02, (0, 0, 0)), (3, 0.01, (0, 0, 0)), (1, 0.0, (1, 0, 0))])
def test_hook_rho_df_force_match_oracle(hooks, n_types, vac, start):
    sc = make(cells=(7, 6, 5), temperature=900.0, vacancy=vac, n_types=n_types, seed=21, jitter=0.1)
    dom, odom, even, odd = _hook_setup(hooks, sc, start=start)
    ext_gpu = sc.ext()
    ext_orc = ext_gpu.copy().view(orc.ATOM)
    before = ext_gpu.copy()
    pot = sc.orc_pot()
    hooks.rho_calc(ext_gpu, sc.cutoff)
    orc.rho_pass(pot, odom, ext_orc, even, odd, sc.cutoff)
    bg, bo = _box(ext_gpu, sc), _box(ext_orc, sc)
    live = bg["type"] >= 0
    assert rel_err(bg["rho"][live], bo["rho"][live]) < 1e-12
    assert rel_err(bg["df"][live], bo["df"][live]) < 1e-12
    # vacant sites and ghosts are left as they were (the reference writes box sites with type >= 0 only)
    bb = _box(before, sc)
    assert np.array_equal(bg["rho"][~live], bb["rho"][~live])
    hooks.df_calc(ext_gpu, sc.cutoff)  # full-neighbour build: a no-op
    # the host refreshes ghost df before the force pass
    L = [sc.cells[0] * A0, sc.cells[1] * A0, sc.cells[2] * A0]
    orc.ghost_fill(odom, ext_gpu.view(orc.ATOM), L, 2)
    orc.ghost_fill(odom, ext_orc, L, 2)
    hooks.force_calc(ext_gpu, sc.cutoff)
    orc.force_pass(pot, odom, ext_orc, even, odd, sc.cutoff)
    bg, bo = _box(ext_gpu, sc), _box(ext_orc, sc)
    assert rel_err(bg["f"][live], bo["f"][live]) < F_TOL
    assert np.abs(bo["f"][live]).max() > 0.1
    k, c = hooks.last_timing()
    assert k > 0 and c > 0


@pytest.mark.parametrize("batches", [3, 9])
def test_hooks_streamed_in_slabs_match_one_piece_and_oracle(hooks, batches):
    # the reference's -b/--batches z-slab streaming: every slab count gives the same bytes
    sc = make(cells=(7, 6, 9), temperature=900.0, vacancy=0.02, seed=29, jitter=0.1)
    dom, odom, even, odd = _hook_setup(hooks, sc)
    L = [sc.cells[0] * A0, sc.cells[1] * A0, sc.cells[2] * A0]
    out = {}
    try:
        for b in (1, batches):
            hooks.set_batches(b)
            ext = sc.ext()
            hooks.rho_calc(ext, sc.cutoff)
            orc.ghost_fill(odom, ext.view(orc.ATOM), L, 2)
            hooks.force_calc(ext, sc.cutoff)
            out[b] = ext
            k, c = hooks.last_timing()
            assert k > 0 and c > 0
    finally:
        hooks.set_batches(1)
    assert out[1].tobytes() == out[batches].tobytes()
    pot = sc.orc_pot()
    eo = sc.ext().view(orc.ATOM)
    orc.rho_pass(pot, odom, eo, even, odd, sc.cutoff)
    orc.ghost_fill(odom, eo, L, 2)
    orc.force_pass(pot, odom, eo, even, odd, sc.cutoff)
    bg, bo = _box(out[batches], sc), _box(eo, sc)
    live = bg["type"] >= 0
    assert rel_err(bg["rho"][live], bo["rho"][live]) < 1e-12
    assert rel_err(bg["df"][live], bo["df"][live]) < 1e-12
    assert rel_err(bg["f"][live], bo["f"][live]) < F_TOL
    # ghost records come back as they went in
    assert np.array_equal(out[batches]["x"], sc.ext()["x"])


def test_hook_with_setfl_alloy_matches_oracle(hooks, tmp_path):
    # a two-element Fe-Cu table written as a setfl file and read back drives both paths
    t = mb.potential.alloy_analytic(2, nr=3000, nrho=3000)
    path = tmp_path / "fecu.setfl"
    mb.potential.write_setfl(path, t, elements=["Fe", "Cu"], numbers=[26, 29])
    tables, meta = mb.potential.read_setfl(path)
    assert meta["elements"] == ["Fe", "Cu"]
    sc = make(cells=(6, 7, 5), temperature=900.0, vacancy=0.01, seed=23, jitter=0.1, tables=tables, n_types=2)
    dom, odom, even, odd = _hook_setup(hooks, sc)
    ext_gpu = sc.ext()
    ext_orc = ext_gpu.copy().view(orc.ATOM)
    pot = sc.orc_pot()
    hooks.rho_calc(ext_gpu, sc.cutoff)
    orc.rho_pass(pot, odom, ext_orc, even, odd, sc.cutoff)
    L = [sc.cells[0] * A0, sc.cells[1] * A0, sc.cells[2] * A0]
    orc.ghost_fill(odom, ext_gpu.view(orc.ATOM), L, 2)
    orc.ghost_fill(odom, ext_orc, L, 2)
    hooks.force_calc(ext_gpu, sc.cutoff)
    orc.force_pass(pot, odom, ext_orc, even, odd, sc.cutoff)
    bg, bo = _box(ext_gpu, sc), _box(ext_orc, sc)
    live = bg["type"] >= 0
    assert set(np.unique(bg["type"][live])) == {0, 1}
    assert rel_err(bg["rho"][live], bo["rho"][live]) < 1e-12
    assert rel_err(bg["f"][live], bo["f"][live]) < F_TOL


@pytest.mark.parametrize("n_types,start", [(1, (0, 0, 0)), (3, (1, 0, 0))])
def test_half_neighbour_hooks_match_oracle(hooks, n_types, start):
    # the reference's USE_NEWTONS_THIRD_LOW build: half stencils, shares to box and ghost
    # records; the host folds ghost shares into their owners between the passes
    sc = make(cells=(6, 7, 5), temperature=900.0, vacancy=0.02, n_types=n_types, seed=27, jitter=0.1)
    dom = mb.lattice.domain(sc.cells, sc.ghost, start)
    odom = orc.make_domain(sc.cells, sc.ghost, start)
    hooks.domain_init(dom)
    even, odd = mb.lattice.stencil_linear(A0, sc.reach, dom.ext_size_x, dom.ext_size_y)
    he, ho = orc.half_stencil(even), orc.half_stencil(odd)
    hooks.pot_init(sc.tables)
    hooks.set_half_neighbour(True)
    try:
        with pytest.raises(mb.MbError, match="half stencil"):
            hooks.nei_offset_init(even, odd)  # a full stencil holds every pair twice
        hooks.nei_offset_init(he, ho)
        pot = sc.orc_pot()
        L = [sc.cells[0] * A0, sc.cells[1] * A0, sc.cells[2] * A0]
        ext_gpu = sc.ext()
        ext_orc = ext_gpu.copy().view(orc.ATOM)
        hooks.rho_calc(ext_gpu, sc.cutoff)
        orc.rho_pass_half(pot, odom, ext_orc, he, ho, sc.cutoff)
        # every ext record, ghosts included, against the oracle's shares
        assert rel_err(ext_gpu["rho"], ext_orc["rho"]) < 1e-12
        assert np.array_equal(ext_gpu["x"], ext_orc["x"])
        # host: fold ghost shares into owners, df pass, refresh ghost df
        for e in (ext_gpu, ext_orc.view(mb.ATOM_DTYPE)):
            folded = orc.fold_ghosts(odom, e, "rho")
            b = mb.lattice.ext_to_box(e, sc.cells, sc.ghost)
            b["rho"] = folded
            e[:] = mb.lattice.box_to_ext(b, sc.cells, sc.ghost, A0)
        hooks.df_calc(ext_gpu, sc.cutoff)
        orc.df_pass(pot, odom, ext_orc)
        live = _box(ext_gpu, sc)["type"] >= 0
        assert rel_err(_box(ext_gpu, sc)["df"][live], _box(ext_orc, sc)["df"][live]) < 1e-12
        orc.ghost_fill(odom, ext_gpu.view(orc.ATOM), L, 2)
        orc.ghost_fill(odom, ext_orc, L, 2)
        hooks.force_calc(ext_gpu, sc.cutoff)
        orc.force_pass_half(pot, odom, ext_orc, he, ho, sc.cutoff)
        assert rel_err(ext_gpu["f"], ext_orc["f"]) < F_TOL
        # after the fold the forces are the full-neighbour forces
        full = sc.ext().view(orc.ATOM)
        orc.rho_pass(pot, odom, full, even, odd, sc.cutoff)
        orc.ghost_fill(odom, full, L, 2)
        orc.force_pass(pot, odom, full, even, odd, sc.cutoff)
        fg = orc.fold_ghosts(odom, ext_gpu, "f")
        assert rel_err(fg[live], _box(full.view(mb.ATOM_DTYPE), sc)["f"][live]) < F_TOL
        with pytest.raises(mb.MbError, match="full-neighbour"):
            mb.check(mb.lib().mb_eam_rho_calc_noalloc(mb.ptr(ext_gpu), sc.cutoff))
    finally:
        hooks.set_half_neighbour(False)


def test_hook_rejects_types_without_a_potential_table(hooks):
    sc = make(cells=(6, 6, 6), seed=5)
    _hook_setup(hooks, sc)
    ext = sc.ext()
    ext["type"][len(ext) // 2] = 2  # the one-type potential has a table for type 0 only
    with pytest.raises(mb.MbError, match="potential table"):
        hooks.rho_calc(ext, sc.cutoff)


def test_hook_df_from_rho_matches_oracle(hooks):
    sc = make(cells=(6, 6, 6), temperature=600.0, vacancy=0.01, seed=4)
    dom, odom, even, odd = _hook_setup(hooks, sc)
    ext = sc.ext()
    rng = np.random.default_rng(9)
    ext["rho"] = rng.uniform(0.0, 80.0, size=ext.shape[0])  # both inside and past the table
    eo = ext.copy().view(orc.ATOM)
    hooks.df_from_rho(ext)
    orc.df_pass(sc.orc_pot(), odom, eo)
    live = _box(ext, sc)["type"] >= 0
    assert rel_err(_box(ext, sc)["df"][live], _box(eo, sc)["df"][live]) < 1e-13


def test_pinned_host_memory_hook(hooks):
    import ctypes as C
    sc = make(cells=(6, 6, 6), temperature=300.0, seed=8)
    dom, odom, even, odd = _hook_setup(hooks, sc)
    n = dom.ext_size_x * dom.ext_size_y * dom.ext_size_z
    p = C.c_void_p()
    alloc = C.c_int()
    mb.check(mb.lib().mb_create_atoms_mem(C.byref(p), 104, dom.ext_size_x, dom.ext_size_y, dom.ext_size_z,
                                          C.byref(alloc)))
    assert alloc.value == 1
    try:
        buf = np.ctypeslib.as_array((C.c_uint8 * (104 * n)).from_address(p.value)).view(mb.ATOM_DTYPE)
        buf[:] = sc.ext()
        ref = buf.copy().view(orc.ATOM)
        hooks.rho_calc(buf, sc.cutoff)
        orc.rho_pass(sc.orc_pot(), odom, ref, even, odd, sc.cutoff)
        assert rel_err(_box(buf, sc)["rho"], _box(ref, sc)["rho"]) < 1e-12
    finally:
        rel = C.c_int()
        mb.check(mb.lib().mb_release_atoms_mem(p, C.byref(rel)))
        assert rel.value == 1


def _oracle_md(sc, nsteps):
    odom = sc.orc_domain()
    even, odd = orc.stencil(odom, sc.a0, sc.reach)
    ext = sc.ext().view(orc.ATOM)
    itl = sc.itl.view(orc.ATOM).copy() if sc.itl.shape[0] else None
    e = orc.md_run(sc.orc_pot(), odom, ext, itl, even, odd, sc.md_params(), nsteps)
    return _box(ext, sc), itl, e


def _sim(sc, precision=mb.MB_PREC_FP64):
    return mb.Sim(sc.cells, sc.tables, lattice_const=sc.a0, mass=sc.mass, dt=sc.dt, cutoff=sc.cutoff,
                  stencil_skin=sc.skin, precision=precision, max_interstitials=max(8, sc.itl.shape[0]))


def test_wide_reach_interstitial_windows_match_oracle():
    # cutoff + skin = 9.0 A: about 262 sites lie in reach of an interstitial, more than the
    # per-warp list of in-reach window sites holds (256), so the interstitial passes walk
    # every window candidate instead; the results are still the oracle's
    sc = make(cells=(8, 8, 8), temperature=600.0, vacancy=0.01, n_itl=3, seed=53, skin=3.4)
    nsteps = 5
    bo, io, eo = _oracle_md(sc, nsteps)
    with _sim(sc) as sim:
        sim.upload(sc.box, sc.itl)
        sim.run(nsteps, energy_every=1)
        bg, ig = sim.download()
        eg = sim.energies()
    live = bo["type"] >= 0
    n_atoms = int(live.sum()) + 3
    assert np.max(np.abs(bg["x"][live] - bo["x"][live])) < 1e-10
    assert rel_err(bg["f"][live], bo["f"][live]) < F_TOL
    assert rel_err(ig["f"], io["f"]) < F_TOL
    assert np.max(np.abs(ig["x"] - io["x"])) < 1e-10
    assert np.max(np.abs(eg[:, 1:] - eo)) / n_atoms < E_TOL


@pytest.mark.parametrize("n_itl,vac,n_types", [(0, 0.0, 1), (3, 0.01, 1), (2, 0.01, 3)])
def test_device_md_matches_oracle(n_itl, vac, n_types):
    sc = make(cells=(6, 7, 8), temperature=600.0, vacancy=vac, n_itl=n_itl, seed=31, n_types=n_types)
    nsteps = 10
    bo, io, eo = _oracle_md(sc, nsteps)
    n_atoms = int((sc.box["type"] >= 0).sum()) + n_itl
    with _sim(sc) as sim:
        sim.upload(sc.box, sc.itl if n_itl else None)
        sim.run(nsteps, energy_every=1)
        bg, ig = sim.download()
        eg = sim.energies()
    live = bo["type"] >= 0
    assert np.array_equal(bg["type"], bo["type"])
    assert np.max(np.abs(bg["x"][live] - bo["x"][live])) < 1e-10
    assert rel_err(bg["f"][live], bo["f"][live]) < F_TOL
    assert rel_err(bg["v"][live], bo["v"][live]) < 1e-10
    assert rel_err(bg["rho"][live], bo["rho"][live]) < 1e-11
    if n_itl:
        assert rel_err(ig["f"], io["f"]) < F_TOL
        assert np.max(np.abs(ig["x"] - io["x"])) < 1e-10
    assert eg.shape == (nsteps + 1, 3)
    assert np.array_equal(eg[:, 0], np.arange(nsteps + 1))
    assert np.max(np.abs(eg[:, 1] - eo[:, 0])) / n_atoms < E_TOL
    assert np.max(np.abs(eg[:, 2] - eo[:, 1])) / n_atoms < E_TOL


def test_golden_fixture_on_device():
    g = np.load(GOLDEN / "small_md.npz")
    rec = lambda a: np.ascontiguousarray(a).view(mb.ATOM_DTYPE).reshape(-1)  # noqa: E731
    t = mb.potential.EamTables(1, float(g["dr"]), float(g["drho"]), float(g["cutoff"]), g["f_tab"], g["F_tab"],
                               g["phi_tab"])
    cells = tuple(int(c) for c in g["cells"])
    box_in, itl_in = rec(g["box_in"]), rec(g["itl_in"])
    with mb.Sim(cells, t, lattice_const=float(g["a0"]), mass=float(g["mass"]), dt=float(g["dt"]),
                cutoff=float(g["cutoff"]), stencil_skin=float(g["skin"]), max_interstitials=8) as sim:
        sim.upload(box_in, itl_in)
        sim.run(int(g["nsteps"]), energy_every=1)
        bg, ig = sim.download()
        eg = sim.energies()
    bo, io = rec(g["box_out"]), rec(g["itl_out"])
    live = bo["type"] >= 0
    n = int(live.sum()) + io.shape[0]
    assert rel_err(bg["f"][live], bo["f"][live]) < F_TOL
    assert rel_err(ig["f"], io["f"]) < F_TOL
    assert np.max(np.abs(eg[:, 1:] - g["energies"])) / n < E_TOL


def test_host_buffer_step_matches_oracle():
    sc = make(cells=(6, 6, 6), temperature=900.0, vacancy=0.01, n_itl=2, seed=41)
    # forces at the starting positions are part of the host state
    odom = sc.orc_domain()
    even, odd = orc.stencil(odom, sc.a0, sc.reach)
    ext = sc.ext().view(orc.ATOM)
    itl = sc.itl.view(orc.ATOM).copy()
    orc.compute_forces(sc.orc_pot(), odom, ext, itl, even, odd, sc.md_params())
    box = _box(ext, sc).view(mb.ATOM_DTYPE).copy()
    itl_g = itl.view(mb.ATOM_DTYPE).copy()
    orc.md_run(sc.orc_pot(), odom, ext, itl, even, odd, sc.md_params(), 3)
    bo = _box(ext, sc)
    with _sim(sc) as sim:
        for _ in range(3):
            sim.step_host(box, itl_g)
    live = bo["type"] >= 0
    assert rel_err(box["f"][live], bo["f"][live]) < F_TOL
    assert np.max(np.abs(box["x"][live] - bo["x"][live])) < 1e-10
    assert rel_err(itl_g["f"], itl["f"]) < F_TOL


def _host_state(sc):
    """Box records and interstitials with the forces of their starting positions."""
    odom = sc.orc_domain()
    even, odd = orc.stencil(odom, sc.a0, sc.reach)
    ext = sc.ext().view(orc.ATOM)
    itl = sc.itl.view(orc.ATOM).copy()
    orc.compute_forces(sc.orc_pot(), odom, ext, itl, even, odd, sc.md_params())
    return odom, even, odd, ext, itl


def test_host_buffer_step_in_slabs_matches_oracle():
    # 23 layers in z: 4 slabs of 5-6 layers (the stencil and the interstitial windows
    # reach 5), interstitials spread over the box, some near the periodic z faces
    sc = make(cells=(8, 6, 23), temperature=900.0, vacancy=0.01, n_itl=7, seed=43)
    odom, even, odd, ext, itl = _host_state(sc)
    box = _box(ext, sc).view(mb.ATOM_DTYPE).copy()
    itl_g = itl.view(mb.ATOM_DTYPE).copy()
    orc.md_run(sc.orc_pot(), odom, ext, itl, even, odd, sc.md_params(), 3)
    bo = _box(ext, sc)
    with _sim(sc) as sim:
        assert sim.host_slabs() == 1  # automatic: too few records to be worth streaming
        sim.set_host_slabs(4)
        assert sim.host_slabs() == 4
        for _ in range(3):
            sim.step_host(box, itl_g)
    live = bo["type"] >= 0
    assert rel_err(box["f"][live], bo["f"][live]) < F_TOL
    assert np.max(np.abs(box["x"][live] - bo["x"][live])) < 1e-10
    assert np.max(np.abs(box["v"][live] - bo["v"][live])) < 1e-10
    assert rel_err(itl_g["f"], itl["f"]) < F_TOL
    assert np.max(np.abs(itl_g["x"] - itl["x"])) < 1e-10


@pytest.mark.parametrize("cells,n_itl", [((6, 6, 40), 9), ((7, 5, 33), 0)])
def test_host_buffer_slabs_are_bitwise_one_piece(cells, n_itl):
    sc = make(cells=cells, temperature=1200.0, vacancy=0.01, n_itl=n_itl, seed=47)
    _, _, _, ext, itl = _host_state(sc)
    box0 = _box(ext, sc).view(mb.ATOM_DTYPE).copy()
    itl0 = itl.view(mb.ATOM_DTYPE).copy()
    out = {}
    for slabs in (1, 32, 5, 4):
        box, ig = box0.copy(), itl0.copy()
        with _sim(sc) as sim:
            sim.set_host_slabs(slabs)
            out[slabs, "n"] = sim.host_slabs()
            for _ in range(4):
                sim.step_host(box, ig if n_itl else None)
        out[slabs] = (box, ig)
    # as many as the reach allows: slabs of at least ceil((cutoff + skin) / a0) + 1 = 4 layers
    assert out[1, "n"] == 1 and out[32, "n"] == cells[2] // 4 and out[5, "n"] == 5 and out[4, "n"] == 4
    for slabs in (32, 5, 4):
        for a, b in zip(out[1], out[slabs]):
            assert a.tobytes() == b.tobytes(), slabs


def test_graph_replay_is_bitwise_identical_to_direct_launches():
    sc = make(cells=(8, 8, 8), temperature=600.0, vacancy=0.005, n_itl=2, seed=51)
    out = []
    for graphs in (True, False):
        with _sim(sc) as sim:
            sim.set_graphs(graphs)
            sim.upload(sc.box, sc.itl)
            sim.run(20)
            out.append(sim.download())
    assert np.array_equal(out[0][0]["x"], out[1][0]["x"])
    assert np.array_equal(out[0][0]["f"], out[1][0]["f"])
    assert np.array_equal(out[0][1]["x"], out[1][1]["x"])


def test_nve_drift_on_device():
    sc = make(cells=(10, 10, 10), temperature=600.0, vacancy=0.005, n_itl=2, seed=61, jitter=0.0)
    with _sim(sc) as sim:
        sim.upload(sc.box, sc.itl)
        sim.run(2000, energy_every=100)
        e = sim.energies()
    n = int((sc.box["type"] >= 0).sum()) + 2
    tot = e[:, 1] + e[:, 2]
    assert np.max(np.abs(tot - tot[0])) / n < 2e-4


def test_bad_inputs_are_rejected_on_device():
    sc = make(cells=(6, 6, 6))
    with pytest.raises(mb.MbError):
        mb.Sim((2, 2, 2), sc.tables)  # box smaller than two interaction spheres
    with _sim(sc) as sim:
        too_many = mb.lattice.octahedral_interstitials(20, sc.cells, A0, 1)
        with pytest.raises(mb.MbError):
            sim.upload(sc.box, too_many)
        bad = sc.box.copy()
        bad["type"][3] = 99
        with pytest.raises(mb.MbError):
            sim.upload(bad)
        # a type the potential has no table for (one-type potential: only type 0)
        bad["type"][3] = 1
        with pytest.raises(mb.MbError, match="potential table"):
            sim.upload(bad)
        itl = mb.lattice.octahedral_interstitials(1, sc.cells, A0, 2)
        itl["type"] = 2
        with pytest.raises(mb.MbError, match="potential table"):
            sim.upload(sc.box, itl)
