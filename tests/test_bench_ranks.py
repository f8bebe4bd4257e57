"""bench.py's multi-rank logic on CPU: two gloo ranks agree on the slowest rank's time and on the
whole-job rate (independent replicas, weak scaling), and under a two-rank launch the reference
arm prints one line from rank 0 and nothing from rank 1."""
import datetime
import json
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        local = [3.0, 5.0][rank]
        m1 = bench.max_over_ranks(local, dist, torch.device("cpu"))
        m2 = bench.max_over_ranks(10.0 - local, dist, torch.device("cpu"))  # the other rank is slower here
        rate = bench.job_rate(world, 1000, 0.5)
        dist.barrier()
        q.put((rank, m1, m2, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted(q.get(timeout=180) for _ in range(2))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [g[0] for g in got] == [0, 1]
    assert all(g[1] == 5.0 and g[2] == 7.0 for g in got)  # every rank sees the maximum
    assert all(g[3] == 4000.0 for g in got)                # 2 replicas x 1000 cells / 0.5 s
    assert all(p.exitcode == 0 for p in procs)


def test_single_rank_max_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(2.5, None, torch.device("cpu")) == 2.5
    assert bench.job_rate(1, 512 ** 3, 2.0e-3) == 512 ** 3 / 2.0e-3


@pytest.mark.parametrize("rank", [1, 0])
def test_reference_arm_under_two_ranks(rank):
    env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0", "--n", "64"],
                       env=env, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    if rank == 1:
        assert lines == []
    else:
        assert len(lines) == 1
        d = json.loads(lines[0])
        assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
        assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
