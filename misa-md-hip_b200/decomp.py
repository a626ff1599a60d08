"""One periodic lattice decomposed into z-slabs, one slab per rank (one GPU each).

MISA-MD's host decomposes its lattice over MPI ranks and exchanges ghost layers around
the plugin's passes (the plugin's buffers hold "the lattice atoms array in current MPI
process (including ghost regions)", src/double-buffer/rho_double_buffer_imp.h:38-39;
the per-pass schedule is src/hip_arch_acc_imp.cpp:163-225).  Here each rank keeps its
slab resident on its GPU (``Sim(..., slab=(z_first, z_count))``) and a timestep is

    positions of the gz lowest / highest box layers -> neighbours' ghost layers
    rho / df of the slab                               (phase 0)
    df of the gz lowest / highest box layers         -> neighbours' ghost layers
    forces, velocity-Verlet, drift                     (phase 1)

The messages are device buffers; ``TorchExchange`` moves them with torch.distributed
point-to-point operations (NCCL between GPUs; gloo on CPU tensors for the plumbing
tests), ``LocalRing`` hands them over inside one process (several slabs on one device,
each launch finished before the next: nothing waits on another rank inside a kernel).
x and y stay whole and periodic on every rank; z is periodic across the ring of ranks
(the last slab's top layers are the first slab's bottom ghost, shifted by -L_z).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import ATOM_DTYPE, MB_PREC_FP64, Sim

POS, DF, CODE = 1, 2, 3  # halo fields (mb_sim_halo_*)


def partition(cells_z: int, world: int, min_cells: int) -> list[tuple[int, int]]:
    """Even split of cells_z unit cells over `world` ranks: [(z_first, z_count)], the
    first cells_z % world ranks one cell thicker.  Every slab must be at least
    min_cells thick (the stencil's z reach), else ValueError."""
    if world < 1 or cells_z < 1:
        raise ValueError("need world >= 1 and cells_z >= 1")
    base, extra = divmod(cells_z, world)
    out, z = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        if world > 1 and n < min_cells:
            raise ValueError(f"{cells_z} cells over {world} ranks leaves a slab of {n} < {min_cells} cells "
                             "(the ghost width)")
        out.append((z, n))
        z += n
    return out


def neighbours(rank: int, world: int) -> tuple[int, int]:
    """(below, above) on the periodic ring of ranks."""
    return (rank - 1) % world, (rank + 1) % world


def slab_records(box: np.ndarray, cells, z_first: int, z_count: int) -> np.ndarray:
    """The box-order records of unit cells [z_first, z_first + z_count) (z is slowest)."""
    per = 2 * cells[0] * cells[1]
    return np.ascontiguousarray(box[z_first * per:(z_first + z_count) * per])


@dataclasses.dataclass
class Halo:
    """One rank's four messages of a field: what it sends down / up and what it
    receives from below / above (device buffers of equal size)."""
    send_down: object
    send_up: object
    recv_below: object
    recv_above: object


class TorchExchange:
    """Ghost-layer exchange over torch.distributed point-to-point operations (NCCL for
    CUDA tensors).  The four operations of a rank are issued as one batch in a fixed
    order (send down, send up, receive from above, receive from below), so with two
    ranks, where both neighbours are the same peer, the sends and receives pair up in
    order: my down message is the other rank's message from above."""

    def __init__(self, dist, rank: int, world: int, group=None):
        self.dist, self.rank, self.world, self.group = dist, rank, world, group
        self.below, self.above = neighbours(rank, world)

    def exchange_all(self, halos: list[Halo]) -> None:
        assert len(halos) == 1, "one slab per process"
        self.exchange(halos[0])

    def exchange(self, h: Halo) -> None:
        d = self.dist
        ops = [d.P2POp(d.isend, h.send_down, self.below, self.group),
               d.P2POp(d.isend, h.send_up, self.above, self.group),
               d.P2POp(d.irecv, h.recv_above, self.above, self.group),
               d.P2POp(d.irecv, h.recv_below, self.below, self.group)]
        for w in d.batch_isend_irecv(ops):
            w.wait()


def _ptr(buf) -> int:
    return int(buf.data_ptr())


class SlabRank:
    """One rank's slab of a z-decomposed periodic lattice (FP64, no interstitials).

    buffers(nbytes) -> a device buffer object with .data_ptr() (a CUDA tensor when the
    exchange is NCCL).  With world == 1 the slab is the whole lattice and no exchange
    happens (its z ghosts are periodic images written on the device)."""

    def __init__(self, cells, tables, rank: int, world: int, buffers, lattice_const: float = 2.855,
                 mass: float = 55.845, dt: float = 1.0, cutoff: float | None = None, stencil_skin: float = 0.7,
                 ghost_z: int = 2):
        self.cells = tuple(int(c) for c in cells)
        self.rank, self.world = rank, world
        self.parts = partition(self.cells[2], world, ghost_z)
        self.z_first, self.z_count = self.parts[rank]
        kw = dict(lattice_const=lattice_const, mass=mass, dt=dt, cutoff=cutoff, stencil_skin=stencil_skin,
                  precision=MB_PREC_FP64, max_interstitials=0)
        self.sim = Sim(self.cells, tables, slab=None if world == 1 else (self.z_first, self.z_count), **kw)
        self.Lz = self.cells[2] * lattice_const
        self.halos = {}
        if world > 1:
            for what in (POS, DF, CODE):
                n = self.sim.halo_bytes(what)
                self.halos[what] = Halo(buffers(n), buffers(n), buffers(n), buffers(n))
        # across the periodic wrap: rank 0's bottom ghost comes from the top of the last
        # slab (z - L_z), the last rank's top ghost from the bottom of the first (z + L_z)
        self.shift_below = -self.Lz if rank == 0 else 0.0
        self.shift_above = self.Lz if rank == world - 1 else 0.0

    def close(self) -> None:
        self.sim.close()

    # the three steps of one exchange; between pack and unpack the host moves the buffers
    def pack(self, what: int) -> Halo:
        h = self.halos[what]
        self.sim.halo_pack(what, 0, _ptr(h.send_down))
        self.sim.halo_pack(what, 1, _ptr(h.send_up))
        return h

    def unpack(self, what: int) -> None:
        h = self.halos[what]
        self.sim.halo_unpack(what, 0, _ptr(h.recv_below), self.shift_below)
        self.sim.halo_unpack(what, 1, _ptr(h.recv_above), self.shift_above)

    def upload(self, box: np.ndarray) -> None:
        """box: the whole lattice's box-order records; this rank takes its layers."""
        assert box.dtype == ATOM_DTYPE
        self.sim.upload(slab_records(box, self.cells, self.z_first, self.z_count) if self.world > 1 else box)


def step_all(ranks: list[SlabRank], exchange, energy: bool = False, sync=None) -> None:
    """One timestep of every slab this process drives (one per GPU under torchrun, or
    several on one device with a LocalRing).  sync() runs between the packs and the
    message transfer and again before the unpacks (a stream synchronisation for NCCL)."""
    for what, phase in ((POS, 0), (DF, 1)):
        if ranks[0].world > 1:
            halos = [r.pack(what) for r in ranks]
            if sync:
                sync()
            exchange.exchange_all(halos)
            if sync:
                sync()
            for r in ranks:
                r.unpack(what)
        for r in ranks:
            r.sim.phase(phase, energy)


def exchange_codes(ranks: list[SlabRank], exchange, sync=None) -> None:
    """After an upload: the site codes (vacancies) of the ghost layers, once."""
    if ranks[0].world == 1:
        return
    halos = [r.pack(CODE) for r in ranks]
    if sync:
        sync()
    exchange.exchange_all(halos)
    if sync:
        sync()
    for r in ranks:
        r.unpack(CODE)


class LocalRing:
    """All slabs in this process, on one device: every rank's receive buffers are filled
    from its neighbours' send buffers with device-to-device copies."""

    def __init__(self, copy):
        self.copy = copy  # copy(dst_buffer, src_buffer)

    def exchange_all(self, halos: list[Halo]) -> None:
        world = len(halos)
        for r, h in enumerate(halos):
            below, above = neighbours(r, world)
            self.copy(h.recv_below, halos[below].send_up)
            self.copy(h.recv_above, halos[above].send_down)
