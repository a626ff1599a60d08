"""Serving loop: request stream, validation, continuous batching, cancellation."""
from __future__ import annotations

import threading

import numpy as np
import pytest

import misa_b200 as mb
from misa_b200 import serve


def test_poisson_stream_statistics():
    reqs = serve.poisson_stream(2000, rate=50.0, seed=13)
    gaps = np.diff([0.0] + [r.arrival for r in reqs])
    assert abs(gaps.mean() - 1 / 50.0) < 0.002
    sizes = np.array([r.n_atoms for r in reqs])
    assert sizes.min() >= 2 * 6 ** 3 and sizes.max() <= 2.3e6
    assert abs(np.median(np.log(sizes)) - 0.5 * (np.log(1e3) + np.log(2e6))) < 0.3
    steps = np.array([r.steps for r in reqs])
    assert steps.min() >= 100 and steps.max() <= 5000
    assert all(300 <= r.temperature <= 1200 and 0 <= r.vacancy <= 0.01 for r in reqs)


def test_request_validation_without_a_device():
    budget = 64 << 20
    ok = serve.Request(0, 0.0, (8, 8, 8), 10, 300.0, 0.0, 1)
    assert serve.validate_request(ok, budget) == ""
    assert "edges" in serve.validate_request(serve.Request(1, 0.0, (3, 8, 8), 10, 300.0, 0.0, 1), budget)
    assert "steps" in serve.validate_request(serve.Request(2, 0.0, (8, 8, 8), 0, 300.0, 0.0, 1), budget)
    assert "vacancy" in serve.validate_request(serve.Request(3, 0.0, (8, 8, 8), 5, 300.0, 0.9, 1), budget)
    assert "budget" in serve.validate_request(serve.Request(4, 0.0, (200, 200, 200), 5, 300.0, 0.0, 1), budget)


def test_shortest_work_first_order_without_a_device():
    a = serve.Request(0, 0.0, (10, 10, 10), 1000, 300.0, 0.0, 1)  # 2,000 sites x 1,000 steps
    b = serve.Request(1, 0.1, (10, 10, 10), 100, 300.0, 0.0, 1)  # less work, arrived later
    c = serve.Request(2, 0.2, (40, 40, 40), 100, 300.0, 0.0, 1)  # 128,000 sites x 100 steps
    d = serve.Request(3, 0.3, (20, 20, 20), 5000, 300.0, 0.0, 1)
    d.snapshot, d.steps_before = np.zeros(1), 4000  # resumed from a checkpoint: first
    assert [r.rid for r in sorted([a, b, c, d], key=serve.admission_key)] == [3, 1, 0, 2]
    assert serve.lattice_sites(c) == 128000
    with pytest.raises(ValueError):
        serve.Server.__init__(object.__new__(serve.Server), order="random")


def _small_stream(n, seed=5):
    return serve.poisson_stream(n, rate=200.0, seed=seed, atoms=(1e3, 2e4), steps=(10, 40))


def _alone(req):
    with mb.Ensemble(mb.potential.fe_analytic(), lattice_const=serve.A0, mass=serve.MASS) as ens:
        s = ens.add(req.cells, serve.build_lattice(req), steps=req.steps)
        ens.advance(10 * req.steps + 10)
        return ens.download(s)[0]


@pytest.mark.gpu
def test_continuous_batching_results_match_alone_runs():
    reqs = _small_stream(10)
    srv = serve.Server(chunk=7, keep_results=True)
    stats = srv.serve(reqs, realtime=True)
    srv.close()
    assert stats["completed"] == 10 and stats["rejected"] == 0
    assert stats["atom_steps_per_s"] > 0 and stats["latency_p99_s"] >= stats["latency_p50_s"] > 0
    # arrivals overlapped with running work: some request was admitted while others ran
    assert any(r.admitted > min(q.admitted for q in reqs) for r in reqs)
    for r in reqs[:4]:
        assert np.array_equal(r.result["x"], _alone(r)["x"])


@pytest.mark.gpu
def test_budget_queues_and_faults_are_contained():
    reqs = _small_stream(8, seed=9)
    one = max(mb.Ensemble.lattice_bytes(r.cells, 0) for r in reqs)
    srv = serve.Server(hbm_budget_bytes=int(1.6 * one), chunk=5, keep_results=True)
    bad = serve.Request(100, 0.0, (2, 2, 2), 10, 300.0, 0.0, 1)
    huge = serve.Request(101, 0.0, (300, 300, 300), 10, 300.0, 0.0, 1)
    peak = []
    victim = reqs[3]

    def tick(s):
        peak.append(len(s.running))
        if victim.status == "running" and len(peak) == 2:
            s.cancel(victim)

    stats = srv.serve(reqs + [bad, huge], realtime=False, on_tick=tick)
    srv.close()
    assert bad.status == "rejected" and huge.status == "rejected"
    assert max(peak) < len(reqs)  # the budget made later requests wait for memory
    waited = [r for r in reqs if r.status == "done" and r.admitted > min(q.finished for q in reqs if q.status == "done")]
    assert waited
    finished = [r for r in reqs if r.status == "done"]
    assert len(finished) + (victim.status == "cancelled") == len(reqs)
    for r in finished[:3]:
        assert np.array_equal(r.result["x"], _alone(r)["x"])


@pytest.mark.gpu
def test_large_admission_is_prepared_off_the_loop_thread(monkeypatch):
    # small lattices run for many steps while a 2 M-atom request arrives: its lattice is
    # built on a worker thread while the device advances the others, and the loop thread
    # only uploads it between chunks, so the request joins while the others still run
    built_on = {}
    build = serve.build_lattice

    def recording_build(req):
        built_on[req.rid] = threading.get_ident()
        return build(req)

    monkeypatch.setattr(serve, "build_lattice", recording_build)
    small = serve.poisson_stream(3, rate=1000.0, seed=21, atoms=(2e4, 5e4), steps=(40000, 40000))
    big = serve.Request(50, 0.05, serve.cells_for_atoms(2e6), 20, 600.0, 0.005, 77)
    srv = serve.Server(chunk=20)
    stats = srv.serve(small + [big], realtime=True)
    srv.close()
    assert stats["completed"] == 4
    assert built_on[big.rid] != threading.get_ident()  # not on the loop thread
    assert big.rid in dict(srv.admit_stall)
    assert big.admitted < max(r.finished for r in small)  # it joined while the others ran


@pytest.mark.gpu
@pytest.mark.parametrize("order", ["shortest", "fifo"])
def test_admission_order_under_a_batch_target(order):
    # three requests at once, a batch target of one lattice: shortest-first runs the two
    # short requests before the long one, first-come-first-served the long one first
    long_ = serve.Request(0, 0.0, (12, 12, 12), 400, 300.0, 0.0, 1)
    short = [serve.Request(k, 0.0, (10, 10, 10), 40, 300.0, 0.0, k) for k in (1, 2)]
    srv = serve.Server(chunk=10, order=order, batch_atoms=serve.lattice_sites(long_))
    peak = []
    stats = srv.serve([long_] + short, realtime=False, on_tick=lambda s: peak.append(len(s.running)))
    srv.close()
    assert stats["completed"] == 3 and max(peak) == 1
    first = short[0].finished < short[1].finished < long_.finished
    assert first if order == "shortest" else long_.finished < short[0].finished
    everything = serve.Server(chunk=10, batch_atoms=0)  # no target: all three at once
    peak = []
    everything.serve([serve.Request(k, 0.0, (10, 10, 10), 40, 300.0, 0.0, k) for k in range(3)], realtime=False,
                     on_tick=lambda s: peak.append(len(s.running)))
    everything.close()
    assert max(peak) == 3


@pytest.mark.gpu
def test_preempted_request_resumes_from_its_checkpoint():
    req = serve.Request(0, 0.0, (10, 10, 10), 300, 900.0, 0.005, 5)
    alone = _alone(serve.Request(0, 0.0, (10, 10, 10), 300, 900.0, 0.005, 5))
    srv = serve.Server(chunk=25, keep_results=True)
    hit = []

    def tick(s):
        if not hit and req.status == "running":
            box, done = s.checkpoint(req)
            assert box.shape[0] == 2 * 10 ** 3
            if done >= 100:
                s.preempt(req)
                hit.append(req.steps_before)

    stats = srv.serve([req], realtime=False, on_tick=tick)
    srv.close()
    assert stats["completed"] == 1 and req.status == "done"
    assert hit and 100 <= hit[0] < 300
    # resumed from positions, velocities and forces read back mid-run: the same
    # trajectory up to the rounding of the read-back state (the FP32 displacements the
    # mixed pair terms use are re-derived from it; measured 7.8e-8 A after 200 steps at
    # 900 K)
    assert np.max(np.abs(req.result["x"] - alone["x"])) < 1e-6
    assert np.max(np.abs(req.result["v"] - alone["v"])) < 1e-8
