"""Continuous-batching MD server on one GPU.

Requests (one periodic BCC lattice each, with its own size, temperature, vacancy
fraction and number of steps) are admitted into slots of an ``Ensemble`` whenever
their device memory fits the HBM budget; all admitted lattices advance together,
one persistent kernel launch per timestep, each stopping at its own step target.
Between chunks of launches the loop retires finished lattices (download + free)
and admits queued requests, so work arriving while others run joins the batch as
soon as memory frees up.  Per-request completion latency and aggregate
atom-steps/s are reported.

Request preparation (building the lattice records on the host) runs on worker threads
as soon as a request is queued, while the device advances the running lattices: the
loop thread only uploads a prepared lattice, so a large arrival does not hold up the
launches of the others.  The time the loop thread spends admitting requests between
chunks is recorded (``admit_stall_s``).

Admission order: by default the queued request with the least remaining work (sites x
steps) goes first, requests resumed from a checkpoint ahead of all, and new lattices
join only while the atoms in flight stay under a batch target (``batch_atoms``; 4 M by
default, enough to fill the GPU; a request is always admitted when nothing runs).  With
every request in one batch each step costs the whole batch's time, so even the shortest
request waits as long as a step of everything; shortest-first under a target lets short
requests finish within a few seconds while the batch still saturates the device (the same
work, so about the same makespan and throughput).  ``order="fifo"`` and
``batch_atoms=0`` give first-come, first-served admission of everything that fits the
budget.

Host-side failure handling: malformed requests are rejected at submission; a
request larger than the whole budget is rejected instead of queued forever; a
request can be cancelled while queued or in flight (its slot is freed, the other
lattices are untouched).

Checkpoint / resume: ``checkpoint(req)`` reads a running request's state (positions,
velocities, forces of its lattice at its current step) back to the host;
``preempt(req)`` does that, frees its slot and puts it back at the head of the queue,
so that it resumes from the saved state with its remaining steps when memory allows
(e.g. to make room for a more urgent lattice).
"""
from __future__ import annotations

import concurrent.futures as cf
import dataclasses
import heapq
import time

import numpy as np

from . import Ensemble, lattice, potential
from ._abi import MB_ERR_NOMEM, MbError

A0 = 2.855
MASS = 55.845


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float          # s after the stream start
    cells: tuple
    steps: int
    temperature: float
    vacancy: float
    seed: int
    n_atoms: int = 0
    # filled by the server
    status: str = "new"     # new, queued, running, done, rejected, cancelled
    slot: int = -1
    admitted: float = float("nan")
    finished: float = float("nan")
    reason: str = ""
    result: np.ndarray | None = None
    energies: np.ndarray | None = None
    # checkpoint / resume
    snapshot: np.ndarray | None = None  # box records of the last checkpoint
    steps_before: int = 0               # steps done before the current admission

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def cells_for_atoms(n_atoms: float, min_cells: int = 6) -> tuple:
    """Near-cubic BCC box (2 sites per cell) with about n_atoms sites."""
    c = max(min_cells, int(round((n_atoms / 2.0) ** (1.0 / 3.0))))
    rest = n_atoms / (2.0 * c)
    cy = max(min_cells, int(round(np.sqrt(rest))))
    cz = max(min_cells, int(round(rest / cy)))
    return (c, cy, cz)


def poisson_stream(n: int, rate: float = 50.0, seed: int = 13, atoms=(1e3, 2e6), steps=(100, 5000),
                   temperature=(300.0, 1200.0), vacancy=(0.0, 0.01)) -> list[Request]:
    """Poisson arrivals (mean `rate` per s); atoms log-uniform, steps, temperature and
    vacancy fraction uniform over the given ranges."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    out = []
    for k in range(n):
        na = float(np.exp(rng.uniform(np.log(atoms[0]), np.log(atoms[1]))))
        cells = cells_for_atoms(na)
        out.append(Request(rid=k, arrival=float(t[k]), cells=cells,
                           steps=int(rng.integers(steps[0], steps[1] + 1)),
                           temperature=float(rng.uniform(*temperature)), vacancy=float(rng.uniform(*vacancy)),
                           seed=int(rng.integers(1 << 30)), n_atoms=2 * cells[0] * cells[1] * cells[2]))
    return out


def build_lattice(req: Request) -> np.ndarray:
    box = lattice.bcc_box(req.cells, A0)
    lattice.add_vacancies(box, req.vacancy, req.seed)
    lattice.maxwell_boltzmann(box, None, req.temperature, MASS, req.seed + 1)
    req.n_atoms = int((box["type"] >= 0).sum())
    return box


def lattice_sites(req: Request) -> int:
    """Sites of a request's lattice (2 per BCC cell; its atoms, up to the vacancies)."""
    return 2 * int(req.cells[0]) * int(req.cells[1]) * int(req.cells[2])


def admission_key(req: Request) -> tuple:
    """Sort key of the shortest-work-first queue: requests resumed from a checkpoint
    first, then the least remaining work (sites x steps left), then arrival."""
    resumed = 0 if req.snapshot is not None else 1
    return (resumed, lattice_sites(req) * (req.steps - req.steps_before), req.arrival, req.rid)


def validate_request(req: Request, budget: int) -> str:
    """Why a request cannot be served at all ("" when it can)."""
    if len(req.cells) != 3 or min(req.cells) < 6:
        return "lattice edges must be >= 6 cells"
    if req.steps < 1:
        return "steps must be >= 1"
    if not (0.0 <= req.vacancy < 0.5) or not (req.temperature >= 0.0):
        return "bad vacancy fraction or temperature"
    if Ensemble.lattice_bytes(req.cells, 0) > budget:
        return "lattice larger than the whole HBM budget"
    return ""


class Server:
    def __init__(self, tables: potential.EamTables | None = None, hbm_budget_bytes: int = 160 << 30,
                 chunk: int = 50, energy_every: int = 0, keep_results: bool = False, prep_workers: int = 2,
                 prep_ahead: int = 4, order: str = "shortest", batch_atoms: float = 4e6):
        """prep_workers threads build the lattices of up to prep_ahead queued requests
        ahead of their admission (0 workers: built on the loop thread at admission).
        order: "shortest" (least remaining work first) or "fifo"; batch_atoms: sites in
        flight beyond which queued requests wait for running ones to finish (0: no
        target, only the HBM budget)."""
        if order not in ("shortest", "fifo"):
            raise ValueError("order must be 'shortest' or 'fifo'")
        self.order = order
        self.batch_atoms = float(batch_atoms)
        self.tables = tables or potential.fe_analytic()
        self.budget = int(hbm_budget_bytes)
        self.ens = Ensemble(self.tables, lattice_const=A0, mass=MASS, hbm_budget_bytes=self.budget)
        self.chunk = chunk
        self.energy_every = energy_every
        self.keep_results = keep_results
        self.queue: list[Request] = []
        self.running: dict[int, Request] = {}
        self.done: list[Request] = []
        self.rejected: list[Request] = []
        self.t0 = None
        self.launches = 0
        self.prep_ahead = max(1, prep_ahead)
        self.pool = cf.ThreadPoolExecutor(max_workers=prep_workers) if prep_workers > 0 else None
        self.prepared: dict[int, cf.Future] = {}
        self.admit_stall: list[tuple[int, float]] = []  # (rid, seconds the loop thread spent admitting it)

    def close(self):
        if self.pool is not None:
            self.pool.shutdown(wait=True, cancel_futures=True)
        self.ens.close()

    def now(self) -> float:
        return time.perf_counter() - self.t0

    # ------------------------------------------------------------ requests
    def submit(self, req: Request) -> bool:
        why = validate_request(req, self.budget)
        if why:
            req.status, req.reason = "rejected", why
            self.rejected.append(req)
            return False
        req.status = "queued"
        self.queue.append(req)
        self._order_queue()
        self._prefetch()
        return True

    def _order_queue(self) -> None:
        if self.order == "shortest":
            self.queue.sort(key=admission_key)

    def running_sites(self) -> int:
        return sum(lattice_sites(r) for r in self.running.values())

    def _prefetch(self) -> None:
        if self.pool is None:
            return
        for req in self.queue[:self.prep_ahead]:
            if req.rid not in self.prepared and req.snapshot is None:
                self.prepared[req.rid] = self.pool.submit(build_lattice, req)

    def checkpoint(self, req: Request) -> tuple[np.ndarray, int]:
        """A running request's lattice at its current step and the steps it has done."""
        if req.status != "running":
            raise ValueError("only a running request can be checkpointed")
        done, _, _ = self.ens.status(req.slot)
        box = self.ens.download(req.slot)[0]
        return box, req.steps_before + int(done)

    def preempt(self, req: Request) -> None:
        """Checkpoint a running request, free its slot and queue it first: it resumes
        from the checkpoint with its remaining steps."""
        box, done = self.checkpoint(req)
        self.ens.remove(req.slot)
        del self.running[req.slot]
        req.slot = -1
        req.snapshot, req.steps_before = box, done
        req.status = "queued"
        self.queue.insert(0, req)
        self._order_queue()  # resumed requests stay at the head

    def cancel(self, req: Request) -> None:
        if req.status == "queued":
            self.queue.remove(req)
            fut = self.prepared.pop(req.rid, None)
            if fut is not None:
                fut.cancel()
        elif req.status == "running":
            self.ens.remove(req.slot)
            del self.running[req.slot]
        req.status = "cancelled"

    def _admit(self) -> None:
        # in queue order (see _order_queue): a head request whose lattice is still being
        # built waits (the running lattices keep advancing) unless nothing else runs
        while self.queue:
            req = self.queue[0]
            if self.running and self.batch_atoms > 0 and \
                    self.running_sites() + lattice_sites(req) > self.batch_atoms:
                return  # the batch is full: wait for a running lattice to finish
            t_in = time.perf_counter()
            fut = self.prepared.get(req.rid)
            if req.snapshot is not None:
                box = req.snapshot  # resuming from a checkpoint
            elif fut is None:
                box = build_lattice(req)
            elif fut.done() or not self.running:
                box = fut.result()
            else:
                self._prefetch()
                return
            try:
                req.slot = self.ens.add(req.cells, box, steps=req.steps - req.steps_before)
            except MbError as e:
                if e.code == MB_ERR_NOMEM and self.running:
                    return  # wait for memory to free up (the prepared lattice is kept)
                self.queue.pop(0)
                self.prepared.pop(req.rid, None)
                req.status, req.reason = "rejected", str(e)
                self.rejected.append(req)
                continue
            self.queue.pop(0)
            self.prepared.pop(req.rid, None)
            req.snapshot = None
            req.status = "running"
            req.admitted = self.now()
            self.running[req.slot] = req
            self.admit_stall.append((req.rid, time.perf_counter() - t_in))
            self._prefetch()

    def _retire(self) -> None:
        for slot, req in list(self.running.items()):
            done, target, _ = self.ens.status(slot)
            if done >= target:
                if self.keep_results:
                    req.result = self.ens.download(slot)[0]
                    req.energies = self.ens.energies(slot)
                self.ens.remove(slot)
                del self.running[slot]
                req.status = "done"
                req.finished = self.now()
                self.done.append(req)

    # ------------------------------------------------------------ event loop
    def serve(self, requests: list[Request], realtime: bool = True, max_seconds: float = 1e9,
              on_tick=None) -> dict:
        """Runs until every request is done, rejected or cancelled.  With realtime the
        arrivals happen on the wall clock; otherwise all arrive at once."""
        pending = [(r.arrival if realtime else 0.0, r.rid, r) for r in requests]
        heapq.heapify(pending)
        self.t0 = time.perf_counter()
        work = 0
        while pending or self.queue or self.running:
            t = self.now()
            if t > max_seconds:
                break
            while pending and pending[0][0] <= t:
                self.submit(heapq.heappop(pending)[2])
            self._admit()
            if not self.running:
                if pending:
                    time.sleep(max(0.0, min(0.05, pending[0][0] - self.now())))
                continue
            self.launches += self.ens.advance(self.chunk, self.energy_every)
            self._retire()
            if on_tick:
                on_tick(self)
        makespan = self.now()
        self.ens.sync()
        for r in self.done:
            work += r.n_atoms * r.steps
        lat = np.array([r.latency for r in self.done]) if self.done else np.zeros(1)
        stall = np.array([s for _, s in self.admit_stall]) if self.admit_stall else np.zeros(1)
        return {"completed": len(self.done), "rejected": len(self.rejected), "makespan_s": makespan,
                "atom_steps": work, "atom_steps_per_s": work / makespan if makespan > 0 else 0.0,
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "launches": self.launches, "admit_stall_s": {"max": float(stall.max()), "mean": float(stall.mean())},
                "unfinished": len(self.queue) + len(self.running)}
