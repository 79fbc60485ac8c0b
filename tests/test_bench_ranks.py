"""bench.py's multi-rank plumbing on CPU (gloo, world size 2): the reductions
that turn per-rank times and counts into whole-job numbers, and the reference
arm, which only rank 0 runs."""
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


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    ranks = bench.Ranks(world)
    ranks.barrier()
    res = {"max": ranks.max(1.5 + rank), "sum": ranks.sum(10 * (rank + 1)), "world": ranks.world,
           "rank": ranks.rank, "backend": ranks.backend}
    ranks.close()
    out.put(res)


def test_ranks_reduce_over_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted([q.get(timeout=10) for _ in procs], key=lambda r: r["rank"])
    assert [r["rank"] for r in res] == [0, 1]
    for r in res:
        assert r["world"] == 2 and r["backend"] == "gloo"
        assert r["max"] == 2.5          # max over ranks of the device times
        assert r["sum"] == 30.0         # whole-job totals


@pytest.mark.timeout(300)
def test_reference_arm_prints_once_under_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--edges", "400"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=280, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(l) for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1                      # rank 0 alone runs and prints
    line = lines[0]
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "port"
