"""Child-process body of the gloo exchange test (tests/test_decomp.py): importable
without pytest, it loads the package the way tests/conftest.py does."""
from __future__ import annotations

import datetime
import os


def rank_main(rank: int, world: int, port: int, q) -> None:
    import conftest  # noqa: F401  (makes the package importable as misa_b200)
    import torch
    import torch.distributed as dist
    from misa_b200 import decomp

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n = 5
        mk = lambda v: torch.full((n,), float(v), dtype=torch.float64)  # noqa: E731
        h = decomp.Halo(mk(10 * rank + 1), mk(10 * rank + 2), mk(-1), mk(-1))
        decomp.TorchExchange(dist, rank, world).exchange_all([h])
        q.put((rank, float(h.recv_below[0]), float(h.recv_above[0])))
    finally:
        dist.destroy_process_group()
