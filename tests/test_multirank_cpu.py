"""The N > 1 plumbing of bench.py on host processes (gloo, world size 2):
max over ranks and the barrier agree on every rank, and the reference arm
runs on rank 0 alone (other ranks exit 0 without output)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        m = bench.max_over_ranks(float(rank + 1) * 1.5, world)
        bench.barrier(world)
        q.put((rank, m))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_barrier_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert all(p.exitcode == 0 for p in ps)
    assert got == [(0, 3.0), (1, 3.0)]


def test_reference_arm_only_on_rank_zero():
    if not (os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libszp_ref.so")) or
            os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so"))):
        pytest.skip("oracle not built")
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--side", "64", "--steps", "1",
           "--warmup", "1"]
    outs = []
    for rank in (1, 0):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(r.stdout.strip())
    assert outs[0] == ""
    line = json.loads(outs[1].splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
