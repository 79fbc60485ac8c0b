"""bench.py's multi-rank plumbing on CPU (gloo, world size 2): the reductions
that turn per-rank times and counts into whole-job numbers, and the reference
arm, which only rank 0 runs."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
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


# ---- graph sharding of the batched and served workloads (device calls stubbed)
class _FakeInfo:
    def __init__(self, samples):
        self.samples = samples


class _FakeGpu:
    """Stands in for bundling_thingy_b200.Gpu: a graph's 'samples' are a
    function of its control points, and its records encode them."""

    seen = []

    def __init__(self, options=None):
        self.n = 0
        self.tag = 0

    def upload(self, graph):
        xy, starts = graph
        self.n = int(starts.size) * 3 + int(xy.shape[0])
        self.tag = int(round(float(np.asarray(xy, np.float64).sum()) * 1e3)) & 0xFFFFFFFF
        _FakeGpu.seen.append(self.tag)
        return self.n

    def iterate(self, n=1):
        pass

    def info(self):
        return _FakeInfo(self.n)

    def read_records(self, out):
        out = out.reshape(-1).view(np.uint8)[: 12 * self.n]
        out[:4] = np.frombuffer(np.uint32(self.tag).tobytes(), np.uint8)
        return out

    def close(self):
        pass


class _FakeBatch:
    def __init__(self, device=0):
        self.slots = []

    @staticmethod
    def autotune(jobs, iterations=3, device=0):
        return {"mean_tile": 128, "mean_ctas_per_sm": 0}, 1.0

    def set_shape(self, mean_tile=128, mean_ctas_per_sm=0):
        pass

    def add_many(self, items):
        out = []
        for o, xy, starts in items:
            g = _FakeGpu(o)
            g.upload((xy, starts))
            _FakeGpu.seen.pop()          # batch uploads are not plain-loop work
            self.slots.append(g)
            out.append((len(self.slots) - 1, g.n))
        return out

    def iterate(self, n=1):
        pass

    def iterate_timed(self, n=1):
        return 1.0

    def slot(self, s):
        return self.slots[s]

    def close(self):
        pass


def _shard_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import bundling_thingy_b200 as bt

    _FakeGpu.seen = []
    bt.Gpu, bt.Batch = _FakeGpu, _FakeBatch
    bench.pinned_buffer = lambda nbytes: np.zeros(nbytes, np.uint8)
    ranks = bench.Ranks(world)
    args = bench.parse_args(["--graphs", "24", "--gpus", str(world)])
    res = bench.batched_measure(args, ranks)
    sb = bench.ServedBench(args, ranks, 6)
    served_sizes = [int(j.starts.size) for j in sb.jobs]
    total = sb.rate(10.0, 2.0 + rank)   # whole-job rate: requests of every rank over the slowest span
    ranks.close()
    out.put({"rank": rank, "seen": list(_FakeGpu.seen), "graphs": res["graphs"], "samples": res["samples"],
             "exact": res["bit_exact_vs_plain"], "served_seed": bench.served_seed(rank),
             "served_sizes": served_sizes, "served_rate": total})


def _run_ranks(world):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    return sorted(res, key=lambda r: r["rank"])


@pytest.mark.timeout(300)
def test_batched_and_served_shards_partition_the_work_over_gloo():
    one = _run_ranks(1)[0]
    two = _run_ranks(2)
    # Every graph of the batched workload is bundled by exactly one rank (the
    # plain loop also warms up on each grid class's largest graph).
    seen = [set(r["seen"]) for r in two]
    assert len(set(one["seen"])) == 24
    assert seen[0] | seen[1] == set(one["seen"])
    assert not seen[0] & seen[1]
    # Whole-job totals reduce to the single-rank run's.
    for r in two:
        assert r["graphs"] == one["graphs"] == 24
        assert r["samples"] == one["samples"]
        assert r["exact"]
    # Each rank serves its own arrival stream; rank 0 replays the workload's seed.
    assert two[0]["served_seed"] == one["served_seed"] != two[1]["served_seed"]
    assert two[0]["served_sizes"] == one["served_sizes"] != two[1]["served_sizes"]
    assert two[0]["served_rate"] == two[1]["served_rate"] == 2 * 10.0 / 3.0
