"""The mixed-precision and batched configurations at their own sizes.

* 128^3 and 200^3 cells (4.2 M and 16 M atoms, 0.5% vacancies, 200 / 763 octahedral
  interstitials, 300 K / 900 K), thermally disordered by FP64 steps: the mixed forces at
  the read-back state against the FP64 forces at the same state, relative force RMS
  within 1e-6 (the FP64 path is pinned to the oracle by tests/test_gpu_configs.py).
* The 512-lattice ensemble (edges uniform in [8, 40] cells, seed 11, 300-1200 K, 0-1%
  vacancies): after 5 batched steps, a lattice's positions and forces are bitwise those
  of the same lattice advanced alone."""
from __future__ import annotations

import numpy as np
import pytest

import misa_b200 as mb
from oracle import workload as W

pytestmark = pytest.mark.gpu

F_RMS_TOL = 1e-6


def _sim(cells, n_itl, precision):
    return mb.Sim(cells, mb.potential.fe_analytic(), lattice_const=W.A0, mass=W.MASS, dt=W.DT, cutoff=W.RC,
                  stencil_skin=W.SKIN, precision=precision, max_interstitials=max(1, n_itl))


def _forces(cells, n_itl, box, itl, precision):
    with _sim(cells, n_itl, precision) as s:
        s.upload(box, itl)
        s.run(0)
        b, i = s.download()
    return np.concatenate([b["f"][b["type"] >= 0], i["f"]])


@pytest.mark.parametrize("name,thermal_steps", [("fe128", 100), ("fe200", 30)])
def test_mixed_forces_at_the_configuration_size_within_1e6_of_fp64(name, thermal_steps):
    box, itl = W.config_state(name)
    cells = W.CONFIGS[name]["cells"]
    box, itl = np.ascontiguousarray(box).view(mb.ATOM_DTYPE), np.ascontiguousarray(itl).view(mb.ATOM_DTYPE)
    n = itl.shape[0]
    with _sim(cells, n, mb.MB_PREC_FP64) as s:  # a thermally disordered state
        s.upload(box, itl)
        s.run(thermal_steps)
        tbox, titl = s.download()
    f64 = _forces(cells, n, tbox, titl, mb.MB_PREC_FP64)
    f32 = _forces(cells, n, tbox, titl, mb.MB_PREC_MIXED)
    err = float(np.sqrt(np.sum((f32 - f64) ** 2) / np.sum(f64 ** 2)))
    print(f"{name}: mixed force RMS rel err {err:.2e} after {thermal_steps} FP64 steps")
    assert err < F_RMS_TOL, err


def test_ensemble_of_512_lattices_batched_equals_alone():
    rng = np.random.default_rng(11)
    edges = rng.integers(8, 41, size=(512, 3))
    temps = rng.uniform(300.0, 1200.0, size=512)
    vacs = rng.uniform(0.0, 0.01, size=512)
    kw = dict(lattice_const=W.A0, mass=W.MASS, dt=W.DT, cutoff=W.RC, stencil_skin=W.SKIN)
    boxes = []
    for k in range(512):
        cells = tuple(int(e) for e in edges[k])
        box = mb.lattice.bcc_box(cells, W.A0)
        mb.lattice.add_vacancies(box, float(vacs[k]), 1000 + k)
        mb.lattice.maxwell_boltzmann(box, None, float(temps[k]), W.MASS, 5000 + k)
        boxes.append((cells, box))
    sizes = [np.prod(c) for c, _ in boxes]
    picks = [int(np.argmin(sizes)), int(np.argmax(sizes)), 255]
    with mb.Ensemble(mb.potential.fe_analytic(), **kw) as ens:
        slots = [ens.add(c, b, steps=0) for c, b in boxes]
        ens.run(5)
        batched = {k: ens.download(slots[k])[0] for k in picks}
    for k in picks:
        cells, box = boxes[k]
        with mb.Ensemble(mb.potential.fe_analytic(), **kw) as one:
            s = one.add(cells, box, steps=0)
            one.run(5)
            alone = one.download(s)[0]
        assert np.array_equal(batched[k]["x"], alone["x"]), k
        assert np.array_equal(batched[k]["f"], alone["f"]), k
