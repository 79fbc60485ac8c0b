"""Seeded synthetic trail graphs standing in for the reference's datasets.

The reference's ``data/*.trl`` files are Git-LFS pointer stubs, so every
workload here is generated from a seed. Seeds are 1234 + the workload's index
(small=0, mid=1, large=2, batched=3, served=4).

* ``mixture_graph``: nodes from a 2-D Gaussian mixture in [0,1]^2, straight
  edges between distinct node pairs drawn with probability proportional to
  exp(-d/0.3) without replacement (small: 235 nodes / 8 components / 2,101
  edges; mid: 1,715 / 20 / 9,780).
* ``polyline_graph``: random-walk polylines with 2..8 control points, start
  uniform in [0.08,0.92]^2 (so the fitted extent stays about the unit square), total length U(0.02, 0.08), heading jitter +-30 degrees
  per bend (large: 100,000 polylines, about 5 million samples at spacing 1/1000).

``write_trl`` emits the reference's trail format (one edge per line, a leading
id token, then x y pairs; src/graph.rs:42-59).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

SEED_BASE = 1234


@dataclass
class Workload:
    """One bundling job: control points, CSR starts and its parameters."""

    name: str
    xy: np.ndarray          # float32 [P, 2]
    starts: np.ndarray      # uint32 [E + 1]
    width: int
    height: int
    radius: int
    sigma: float
    shrink: float
    spacing: float          # fraction of the canvas; 0 = one texel (reference)
    iterations: int
    seed: int
    meta: dict = field(default_factory=dict)

    @property
    def edges(self) -> int:
        return int(self.starts.size - 1)


def _mixture_nodes(rng, n_nodes, n_components, sd=0.05):
    centres = rng.uniform(0.15, 0.85, size=(n_components, 2))
    comp = rng.integers(0, n_components, size=n_nodes)
    pts = centres[comp] + rng.normal(0.0, sd, size=(n_nodes, 2))
    return np.clip(pts, 0.0, 1.0)


def _weighted_pairs(rng, nodes, n_edges, scale=0.3):
    """Distinct undirected pairs, p ~ exp(-d/scale), drawn without replacement
    by sequential rejection (equivalent to successive weighted draws)."""
    n = len(nodes)
    if n * (n - 1) // 2 < n_edges:
        raise ValueError("not enough node pairs")
    keys = np.zeros(0, np.int64)   # accepted pairs as lo * n + hi, draw order
    while True:
        m = max(4 * (n_edges - keys.size), 1024)
        i = rng.integers(0, n, size=m)
        j = rng.integers(0, n, size=m)
        u = rng.random(size=m)
        d = np.hypot(*(nodes[i] - nodes[j]).T)
        ok = (i != j) & (u < np.exp(-d / scale))
        lo, hi = np.minimum(i[ok], j[ok]), np.maximum(i[ok], j[ok])
        keys = np.concatenate([keys, lo.astype(np.int64) * n + hi])
        # Keep each pair's first draw, in draw order.
        _, first = np.unique(keys, return_index=True)
        keys = keys[np.sort(first)]
        if keys.size >= n_edges:
            keys = keys[:n_edges]
            break
    return np.stack([keys // n, keys % n], axis=1)


def mixture_graph(n_nodes, n_components, n_edges, seed):
    rng = np.random.default_rng(seed)
    nodes = _mixture_nodes(rng, n_nodes, n_components)
    pairs = _weighted_pairs(rng, nodes, n_edges)
    xy = nodes[pairs.reshape(-1)].astype(np.float32)
    starts = (np.arange(n_edges + 1, dtype=np.uint32) * 2).astype(np.uint32)
    return xy, starts


def polyline_graph(n_edges, seed, k_min=2, k_max=8, length=(0.02, 0.08), jitter_deg=30.0, inset=0.08):
    rng = np.random.default_rng(seed)
    k = rng.integers(k_min, k_max + 1, size=n_edges)
    total = rng.uniform(*length, size=n_edges)
    # Starts are inset by the longest walk so the bounding box stays near
    # [0,1]^2 and the 95% fit keeps lengths in canvas units.
    start = rng.uniform(inset, 1.0 - inset, size=(n_edges, 2))
    heading0 = rng.uniform(0.0, 2.0 * np.pi, size=n_edges)
    starts = np.zeros(n_edges + 1, np.int64)
    starts[1:] = np.cumsum(k)
    P = int(starts[-1])
    xy = np.empty((P, 2), np.float64)
    segs = k - 1
    jit = np.deg2rad(jitter_deg)
    # Per-edge random walk: equal segment lengths, heading jitter per bend.
    seg_len = total / segs
    turn = rng.uniform(-jit, jit, size=P)
    for e_chunk in np.array_split(np.arange(n_edges), max(1, n_edges // 20000)):
        for e in e_chunk:
            s = starts[e]
            h = heading0[e]
            x, y = start[e]
            xy[s] = (x, y)
            for t in range(1, k[e]):
                h += turn[s + t]
                x += seg_len[e] * np.cos(h)
                y += seg_len[e] * np.sin(h)
                xy[s + t] = (x, y)
    return xy.astype(np.float32), starts.astype(np.uint32)


def small(seed_offset: int = 0) -> Workload:
    """235 nodes, 8 components, 2,101 straight edges; 256^2, sigma 8 px,
    10 iterations with kernel shrink 0.75, neighbour radius 2 texels,
    spacing 1/200 of the canvas."""
    seed = SEED_BASE + 0 + seed_offset
    xy, starts = mixture_graph(235, 8, 2101, seed)
    return Workload("small", xy, starts, 256, 256, 2, 8.0, 0.75, 1.0 / 200, 10, seed)


def mid(seed_offset: int = 0) -> Workload:
    """1,715 nodes, 20 components, 9,780 edges; 1024^2, sigma 12 px,
    30 iterations, radius 8 texels, spacing 1/400."""
    seed = SEED_BASE + 1 + seed_offset
    xy, starts = mixture_graph(1715, 20, 9780, seed)
    return Workload("mid", xy, starts, 1024, 1024, 8, 12.0, 1.0, 1.0 / 400, 30, seed)


def large(n_edges: int = 100_000, seed_offset: int = 0) -> Workload:
    """100,000 random-walk polylines (2..8 control points), about 5M samples at
    spacing 1/1000; 2048^2, sigma 16 px, 30 iterations, radius 16 texels."""
    seed = SEED_BASE + 2 + seed_offset
    xy, starts = polyline_graph(n_edges, seed)
    return Workload("large", xy, starts, 2048, 2048, 16, 16.0, 1.0, 1.0 / 1000, 30, seed)


def batched_jobs(n_graphs: int = 256, seed: int = SEED_BASE + 3, iterations: int = 10):
    """Independent graphs: edges log-uniform in [200, 20000], grid in
    {256, 512, 1024}^2, radius grid/128 texels, sigma grid/128 px."""
    rng = np.random.default_rng(seed)
    jobs = []
    for g in range(n_graphs):
        edges = int(np.exp(rng.uniform(np.log(200), np.log(20000))))
        size = int(rng.choice([256, 512, 1024]))
        nodes = max(16, edges // 6)
        xy, starts = mixture_graph(nodes, int(rng.integers(4, 21)), edges, seed * 1000 + g)
        radius = max(1, size // 128)
        jobs.append(Workload(f"batched-{g}", xy, starts, size, size, radius, size / 128.0, 1.0,
                             1.0 / (size // 2), iterations, seed * 1000 + g))
    return jobs


def served_jobs(n_requests: int, rate: float = 200.0, seed: int = SEED_BASE + 4, iterations: int = 10):
    """Poisson arrivals at `rate`/s; edges log-uniform in [500, 50000]; grid in
    {512, 1024, 2048}^2. Returns (arrival_seconds, workloads)."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_requests))
    jobs = []
    for g in range(n_requests):
        edges = int(np.exp(rng.uniform(np.log(500), np.log(50000))))
        size = int(rng.choice([512, 1024, 2048]))
        nodes = max(16, edges // 6)
        xy, starts = mixture_graph(nodes, int(rng.integers(4, 21)), edges, seed * 1000 + g)
        radius = max(1, size // 128)
        jobs.append(Workload(f"served-{g}", xy, starts, size, size, radius, size / 128.0, 1.0,
                             1.0 / (size // 2), iterations, seed * 1000 + g))
    return arrivals, jobs


def write_trl(path_or_file, xy: np.ndarray, starts: np.ndarray) -> None:
    """Write a trail file: '<id> x0 y0 x1 y1 ...' per edge, float32 round-trip
    precision."""
    lines = []
    for e in range(starts.size - 1):
        s, t = int(starts[e]), int(starts[e + 1])
        coords = " ".join(f"{float(v):.9g}" for v in xy[s:t].reshape(-1))
        lines.append(f"{e} {coords}")
    text = "\n".join(lines) + "\n"
    if hasattr(path_or_file, "write"):
        path_or_file.write(text)
    else:
        with open(path_or_file, "w") as f:
            f.write(text)
