"""Parity at the benchmark configurations themselves, against the CPU oracle.

* fe20: 20^3 BCC Fe cells (16,000 atoms), a0 = 2.855 A, 600 K Maxwell-Boltzmann
  velocities from seed 42 with zero net momentum, dt = 1 fs, 100 velocity-Verlet steps;
  forces, positions and energies compared after every step.
* fe128: 128^3 cells (4,194,304 sites), 0.5% vacancies (seed 7), 200 interstitials at
  random octahedral sites (seed 7), 300 K; the first 10 steps compared with the oracle,
  both through the device-resident run (persistent grids, shared-memory tables, graph
  replay) and through the host-buffer step with its automatic z-slab count.

Tolerances: forces 1e-10 relative (max |dF| / max |F|), positions and velocities 1e-10
absolute (A, A/fs), energies 1e-12 eV/atom."""
from __future__ import annotations

import numpy as np
import pytest

import misa_b200 as mb
from oracle import workload as W
from scenarios import rel_err

pytestmark = pytest.mark.gpu

F_TOL, X_TOL, E_TOL = 1e-10, 1e-10, 1e-12


def _sim(cells, n_itl):
    return mb.Sim(cells, mb.potential.fe_analytic(), lattice_const=W.A0, mass=W.MASS, dt=W.DT, cutoff=W.RC,
                  stencil_skin=W.SKIN, max_interstitials=max(1, n_itl))


def _as_mb(a):
    return np.ascontiguousarray(a).view(mb.ATOM_DTYPE)


def _compare(bg, ig, bo, io, what=("x", "v", "f")):
    live = bo["type"] >= 0
    assert np.array_equal(bg["type"], bo["type"])
    errs = {}
    if "f" in what:
        errs["f"] = rel_err(bg["f"][live], bo["f"][live])
        assert errs["f"] < F_TOL, errs
    for k in ("x", "v"):
        if k in what:
            errs[k] = float(np.max(np.abs(bg[k][live] - bo[k][live])))
            assert errs[k] < X_TOL, errs
    if io is not None and io.shape[0]:
        n = io.shape[0]
        assert rel_err(ig["f"][:n], io["f"]) < F_TOL
        assert np.max(np.abs(ig["x"][:n] - io["x"])) < X_TOL
        assert np.max(np.abs(ig["v"][:n] - io["v"])) < X_TOL
    return errs


def test_fe20_600K_every_step_of_100_matches_oracle():
    cells = W.CONFIGS["fe20"]["cells"]
    box, itl = W.config_state("fe20")
    assert box.shape[0] == 16000 and itl.shape[0] == 0
    ref = W.OracleRun(box, None, cells)
    n = ref.n_atoms
    with _sim(cells, 0) as sim:
        sim.upload(_as_mb(box), None)
        sim.run(0, energy_every=1)  # forces and energies at the start
        e0 = sim.energies()
        bg, _ = sim.download()
        # the start is the perfect lattice: every force vanishes by symmetry (both paths
        # leave rounding noise only), so the relative comparison starts at step 1
        assert np.abs(bg["f"]).max() < 1e-12 and np.abs(ref.box()["f"]).max() < 1e-12
        assert abs(e0[-1, 1] - ref.pe) / n < E_TOL and abs(e0[-1, 2] - ref.ke) / n < E_TOL
        worst = 0.0
        for step in range(1, 101):
            eo = ref.steps(1, record=True)  # (pe, ke) before and after the step
            sim.run(1, energy_every=1)
            eg = sim.energies()
            assert int(eg[-1, 0]) == step
            de = max(abs(eg[-1, 1] - eo[-1, 0]), abs(eg[-1, 2] - eo[-1, 1])) / n
            assert de < E_TOL, (step, de)
            bg, _ = sim.download()
            errs = _compare(bg, None, ref.box(), None)
            worst = max(worst, errs["f"])
    print(f"fe20: 100 steps, worst force rel err {worst:.2e}")


@pytest.fixture(scope="module")
def fe128():
    """The fe128 state with the forces of its starting positions, and the oracle after
    10 steps with the energies of every step."""
    cells = W.CONFIGS["fe128"]["cells"]
    box, itl = W.config_state("fe128")
    assert box.shape[0] == 4194304 and itl.shape[0] == 200
    ref = W.OracleRun(box, itl, cells)
    box0, itl0 = ref.box().copy(), ref.itl.copy()  # with the forces at step 0
    energies = ref.steps(10, record=True)
    return dict(cells=cells, box0=box0, itl0=itl0, box10=ref.box(), itl10=ref.itl, energies=energies,
                n=ref.n_atoms)


def test_fe128_first_10_steps_on_device_match_oracle(fe128):
    cells, n = fe128["cells"], fe128["n"]
    with _sim(cells, 200) as sim:
        sim.upload(_as_mb(fe128["box0"]), _as_mb(fe128["itl0"]))
        sim.run(10, energy_every=1)
        bg, ig = sim.download()
        eg = sim.energies()
    errs = _compare(bg, ig, fe128["box10"], fe128["itl10"])
    live = fe128["box10"]["type"] >= 0
    assert rel_err(bg["rho"][live], fe128["box10"]["rho"][live]) < 1e-11
    eo = fe128["energies"]
    assert np.array_equal(eg[:, 0], np.arange(11))
    de = max(np.max(np.abs(eg[:, 1] - eo[:, 0])), np.max(np.abs(eg[:, 2] - eo[:, 1]))) / n
    assert de < E_TOL, de
    print(f"fe128 device-resident: force {errs['f']:.2e}, x {errs['x']:.2e}, v {errs['v']:.2e}, energy {de:.2e} eV/atom")


def test_fe128_first_10_steps_through_host_buffers_match_oracle(fe128):
    cells = fe128["cells"]
    box = _as_mb(fe128["box0"]).copy()
    itl = _as_mb(fe128["itl0"]).copy()
    with _sim(cells, 200) as sim:
        slabs = sim.host_slabs()
        assert slabs > 4  # the automatic count streams this lattice in many z-slabs
        for _ in range(10):
            sim.step_host(box, itl)
    errs = _compare(box, itl, fe128["box10"], fe128["itl10"])
    print(f"fe128 host buffers in {slabs} z-slabs: force {errs['f']:.2e}, x {errs['x']:.2e}, v {errs['v']:.2e}")
