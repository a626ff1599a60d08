"""Host plumbing of the z-slab decomposition (misa-md-hip_b200/decomp.py) on CPU:
the partition of the lattice over ranks, and the ghost-layer exchange between gloo
ranks on 127.0.0.1 (two ranks, where both neighbours are the same peer, and three)."""
from __future__ import annotations

import socket

import numpy as np
import pytest

import misa_b200 as mb
from misa_b200 import decomp


def test_partition_and_neighbours():
    assert decomp.partition(12, 1, 2) == [(0, 12)]
    assert decomp.partition(12, 3, 2) == [(0, 4), (4, 4), (8, 4)]
    assert decomp.partition(11, 3, 2) == [(0, 4), (4, 4), (8, 3)]
    assert sum(n for _, n in decomp.partition(128, 8, 2)) == 128
    with pytest.raises(ValueError, match="ghost"):
        decomp.partition(5, 3, 2)
    assert decomp.neighbours(0, 3) == (2, 1) and decomp.neighbours(2, 3) == (1, 0)
    assert decomp.neighbours(0, 2) == (1, 1)


def test_slab_records_are_the_slab_layers():
    cells = (3, 4, 6)
    box = mb.lattice.bcc_box(cells, 2.855)
    parts = decomp.partition(cells[2], 3, 2)
    got = np.concatenate([decomp.slab_records(box, cells, z0, n) for z0, n in parts])
    assert got.tobytes() == box.tobytes()
    z = decomp.slab_records(box, cells, *parts[1])["x"][:, 2]
    h = 0.5 * 2.855
    assert z.min() == 2 * 2.855 and z.max() == 3 * 2.855 + h  # cells 2..3, body centres included


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_exchange_ghost_layers_with_their_neighbours(world):
    import torch.multiprocessing as mp

    import _decomp_child

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_decomp_child.rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=90) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    for rank, below, above in res:
        b, a = decomp.neighbours(rank, world)
        # my bottom ghost is the top (send_up) of the rank below; my top ghost the bottom
        # (send_down) of the rank above
        assert below == 10 * b + 2 and above == 10 * a + 1
