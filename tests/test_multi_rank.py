"""The N > 1 plumbing of bench.py on CPU: two `gloo` ranks on 127.0.0.1.

`bench.py --gpus N` runs N independent replicas (the hot path does not shard: no
collective on the data path); the ranks only meet in a barrier around the timed region
and in the max-over-ranks of the measured time.  These tests run that plumbing with two
CPU processes, and the reference arm under torchrun, where rank 0 alone measures and
prints."""
from __future__ import annotations

import json
import os
import pathlib
import socket
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench

    world, r, local, pg = bench.dist_setup()
    try:
        bench.barrier(pg)
        t = bench.reduce_max(pg, 1.5 + rank)  # each rank's own time; the job's is the slowest
        bench.barrier(pg)
        out.put((r, world, local, pg.get_backend(), t))
    finally:
        pg.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [(r, w, l, b) for r, w, l, b, _ in res] == [(0, 2, 0, "gloo"), (1, 2, 1, "gloo")]
    assert all(t == 2.5 for *_, t in res)


def test_reference_arm_under_torchrun_prints_one_line_from_rank_zero():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--config", "small", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=240, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(s) for s in r.stdout.splitlines() if s.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_loads_the_oracle_and_not_the_product():
    # The CPU reference arm builds its workload with oracle/workload.py and times the C
    # oracle: the product library must not be mapped into its process.
    code = ("import json, sys; sys.argv = ['bench.py', '--impl', 'reference', '--config', 'small', '--steps', '1', "
            "'--warmup', '0']; import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'product': 'libmisa_b200' in maps, 'oracle': 'liboracle' in maps, "
            "'pkg': 'misa_b200' in sys.modules}))")
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=240, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(s) for s in r.stdout.splitlines() if s.startswith("{")]
    assert lines[0]["impl"] == "reference" and lines[0]["value"] > 0
    assert lines[1] == {"product": False, "oracle": True, "pkg": False}


if __name__ == "__main__":
    pytest.main([__file__, "-q"])
