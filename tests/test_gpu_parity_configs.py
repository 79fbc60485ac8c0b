"""Parity on the configurations the metric is quoted on, through the C ABI.

* Large workload (100k polylines, 4.95M samples, 2048^2, sigma 16, radius
  16), the configuration the bench times: at iterations 1, 6, 15 and 30 the
  GPU's positions of the previous iteration go through the oracle's
  neighbour mean (src/shaders/neighbor_mean.wgsl:163-203 with the exact sum)
  for a contiguous block of 250k samples, and its splat, blur and
  normalisation for the whole map; the GPU's next iteration must equal both
  bit for bit (positions, neighbour counts, splat counts, blurred and
  normalised density).
* Mid workload (9,780 edges, 1024^2, sigma 12, radius 8): every one of its
  30 iterations against the oracle's own chained run.
* The canonical fixed-point mean against the reference's f32 running sum
  (`displacement += delta`, neighbor_mean.wgsl:196-197, cells row-major and
  samples by ascending index): the largest per-step gap on both workloads
  must stay within the positional tolerance (1e-4 of the canvas extent =
  2e-4 clip units). The measured gaps are printed.
"""
import numpy as np
import pytest

import bundling_thingy_b200 as bt
from bundling_thingy_b200 import synthetic

from conftest import oracle_config

pytestmark = pytest.mark.gpu

POS_TOL = 2e-4          # 1e-4 of the canvas extent (2 clip units)
DENSITY_RTOL = 1e-5
BLOCK = 250_000


def opts_for(w: synthetic.Workload) -> bt.Options:
    return bt.Options(width=w.width, height=w.height, neighbor_radius=w.radius, sample_spacing=w.spacing,
                      blur_sigma=w.sigma, blur_shrink=w.shrink, record_neighbors=True)


def test_large_config_steps_at_iterations_1_6_15_30(oracle):
    w = synthetic.large()
    gpu = bt.Gpu(opts_for(w))
    n = gpu.upload((w.xy, w.starts))
    assert 4_500_000 < n < 5_500_000
    mv = oracle.movable_mask(gpu.read_paths(), n)
    taps = oracle.blur_weights(float(np.float32(w.sigma)))
    done = 0
    gaps = {}
    for k in (1, 6, 15, 30):
        if k - 1 > done:
            gpu.iterate(k - 1 - done)
        prev, ids = gpu.read_points()
        gpu.iterate(1)
        done = k
        xy, ids_k = gpu.read_points()
        np.testing.assert_array_equal(ids_k, ids)
        nb = gpu.read_neighbors()
        # A contiguous block of whole paths, somewhere else at each iteration.
        b0 = (k * 1_000_003) % (n - BLOCK)
        b1 = b0 + BLOCK
        mask = np.zeros(n, np.uint8)
        mask[b0:b1] = mv[b0:b1]
        oxy, onb = oracle.neighbor_mean(prev, mask, w.width, w.height, w.radius, mode=0)
        assert np.abs(xy[b0:b1] - oxy[b0:b1]).max() <= POS_TOL
        np.testing.assert_array_equal(xy[b0:b1], oxy[b0:b1])
        np.testing.assert_array_equal(nb[b0:b1], onb[b0:b1])
        assert onb[b0:b1][mask[b0:b1] == 1].min() >= 1
        # The reference's own f32 running sum on the same block.
        fxy, fnb = oracle.neighbor_mean(prev, mask, w.width, w.height, w.radius, mode=1)
        np.testing.assert_array_equal(fnb, onb)
        gaps[k] = float(np.abs(fxy[b0:b1] - oxy[b0:b1]).max())
        assert gaps[k] <= POS_TOL, (k, gaps[k])
        # Density of iteration k from the GPU's own positions, whole map.
        counts = oracle.splat(xy, w.width, w.height)
        np.testing.assert_array_equal(gpu.read_counts(), counts)
        _, vt, peak = oracle.blur(counts, w.width, w.height, taps)
        raw, gpeak = gpu.read_density_raw()
        assert gpeak == peak
        np.testing.assert_allclose(raw, vt, rtol=DENSITY_RTOL, atol=DENSITY_RTOL * peak)
        np.testing.assert_array_equal(raw, vt)
        np.testing.assert_array_equal(gpu.read_density(), oracle.normalize(vt, peak))
    print(f"[f32 running-sum gap, large, radius 16] max |fixed - f32| per step (clip units): {gaps}")
    gpu.close()


def test_mid_config_all_thirty_iterations(oracle):
    w = synthetic.mid()
    o = opts_for(w)
    gpu = bt.Gpu(o)
    ora = oracle.Pipeline(oracle_config(oracle, o))
    n = gpu.upload((w.xy, w.starts))
    assert ora.upload(w.xy, w.starts) == n
    mv = oracle.movable_mask(ora.paths(), n)
    gaps = {}
    for it in range(1, w.iterations + 1):
        prev, _ = ora.points()
        gpu.iterate(1)
        ora.iterate(1)
        gxy, gid = gpu.read_points()
        oxy, oid = ora.points()
        np.testing.assert_array_equal(gid, oid)
        assert np.abs(gxy - oxy).max() <= POS_TOL
        np.testing.assert_array_equal(gxy, oxy)
        np.testing.assert_array_equal(gpu.read_neighbors(), ora.neighbors())
        if it in (1, 10, 20, 30):
            np.testing.assert_array_equal(gpu.read_counts(), ora.counts())
            raw, gpeak = gpu.read_density_raw()
            _, overt, opeak = ora.blurred()
            assert gpeak == opeak
            np.testing.assert_array_equal(raw, overt)
            np.testing.assert_array_equal(gpu.read_density(), ora.normalized())
            fxy, _ = oracle.neighbor_mean(prev, mv, w.width, w.height, w.radius, mode=1)
            gaps[it] = float(np.abs(fxy - oxy).max())
            assert gaps[it] <= POS_TOL, (it, gaps[it])
    assert gpu.info().iterations == w.iterations
    print(f"[f32 running-sum gap, mid, radius 8] max |fixed - f32| per step (clip units): {gaps}")
    gpu.close()
